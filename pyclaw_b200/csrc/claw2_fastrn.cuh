// claw2_fastrn.cuh -- round-to-nearest double division and square root
// without slow-path branches, for the FP64-latency-bound Riemann solvers and
// limiter.
//
// IEEE division and square root on the GPU end every result with a range
// test and a branch to a slow path; each one becomes its own basic block, so
// the compiler cannot overlap the ~20-40 independent-ish divisions and roots
// of one Riemann solve.  FastRn computes each result with straight-line code
// and proves, also with straight-line code, that it is the correctly rounded
// one; a solve runs with FastRn and is redone with IeeeRn only when some proof
// failed, so its results are those of IEEE arithmetic in every case.  The
// solve keeps one FastRn object and reads its `ok` flag at the end (the step
// kernel: once per tile, then redoes the whole tile with IeeeRn if any proof
// failed).
//
// Division a/b.  Reciprocal approximation y0 of b (PTX rcp.approx.ftz.f64),
// one Newton-Raphson step y = y0 + y0*(1 - b*y0), q0 = a*y and one correction
// q = q0 + y*(a - b*q0) (Markstein, "Computation of elementary functions on the
// IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990), all FMAs.
// Proof that q = RN(a/b): rr = a - b*q computed with one FMA.  When q is
// within an ulp of a/b, rr is exactly representable (an integer multiple of
// ulp(b)*ulp(q) smaller than |b|*ulp(q)), so |a/b - q| = |rr|/|b|.  A quotient
// of two doubles is never the midpoint of two consecutive doubles, so
// q = RN(a/b) exactly when |a/b - q| is less than half the gap from q to its
// neighbour on the side of a/b: ulp(q)/2, or ulp(q)/4 below a power of two.
// The test is |rr| < |b|*ulp(q)/2, with ulp(q)/4 whenever q is a power of two
// (conservative above it); the bound is a product by a power of two, hence
// exact.  When q is not within an ulp, |a - b*q| >= |b|*ulp(q)/2 and the
// rounded rr cannot pass.  Range: |b|, |q| in [2^-480, 2^544) keep every step
// free of overflow and underflow (|a| >= 2^-961, so the remainder's units are
// representable); zero, subnormal, infinite or NaN divisors and huge or tiny
// quotients fail the proof.  A zero dividend with an in-range divisor gives
// a*y, the zero of the IEEE sign.
//
// Square root of x.  Reciprocal square-root approximation y0 (PTX
// rsqrt.approx.ftz.f64), then the coupled Newton-Raphson iteration for
// g ~ sqrt(x) and h ~ 1/(2 sqrt(x)) (g0 = x*y0, h0 = y0/2, e = 1/2 - g0*h0,
// g1 = g0 + g0*e, h1 = h0 + h0*e) and one correction s = g1 + h1*(x - g1*g1)
// (the same reference; also Muller et al., Handbook of Floating-Point
// Arithmetic, square root by Newton-Raphson iteration with an FMA).  Proof
// that s = RN(sqrt(x)): with U = ulp(s), x and s*s are integer multiples of
// U*U, so r = x - s*s = k*U*U with an integer k, and r is exact (one FMA)
// whenever |k| < 2^53.  The square root of a double is never a midpoint, and
// with s = S*U (S the integer significand) s = RN(sqrt(x)) exactly when
// (s - U/2)^2 < x < (s + U/2)^2, i.e. -S + 1/4 < k < S + 1/4, i.e.
// -s*U < r <= s*U (no multiple of U*U lies strictly between s*U and
// s*U + U*U/4).  Below a power of two the gap is U/2; there the test uses
// s*U/2 on both sides (conservative).  When |k| >= 2^53 > S the rounded r is
// at least 2^53*U*U in magnitude and fails.  Range: x in [2^-960, 2^1024),
// finite and positive, so that U*U is representable and nothing overflows;
// zero, negative, subnormal, infinite and NaN arguments fail the proof.
#pragma once

#if defined(__CUDACC__)

namespace claw2 {

struct FastRn {
    bool ok = true;

    // a / b
    __device__ __forceinline__ double operator()(double a, double b)
    {
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
        y = fma(y, fma(-b, y, 1.0), y);
        const double q0 = a * y;
        const double q = fma(fma(-b, q0, a), y, q0);
        // proof of correct rounding
        const double rr = fma(-b, q, a);
        const int qh = __double2hiint(q), ql = __double2loint(q), bh = __double2hiint(b);
        const unsigned qe = (unsigned)qh & 0x7ff00000u, be = (unsigned)bh & 0x7ff00000u;
        // biased exponents in [1023-480, 1023-480+1024): |b|, |q| in [2^-480, 2^544)
        const bool range = (((qe - (543u << 20)) | (be - (543u << 20))) >> 20) < 1024u;
        const bool pow2 = ((qh & 0x000fffff) | ql) == 0;
        const double half_ulp = __hiloint2double((int)(qe - ((pow2 ? 54u : 53u) << 20)), 0);
        const bool zero = a == 0.0;
        ok = ok && (zero ? ((be - (543u << 20)) >> 20) < 1024u : (range && fabs(rr) < fabs(b) * half_ulp));
        return zero ? a * y : q;
    }

    // sqrt(x)
    __device__ __forceinline__ double sqrt(double x)
    {
        double y;
        asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
        const double g0 = x * y, h0 = 0.5 * y;
        const double e = fma(-g0, h0, 0.5);
        const double g = fma(g0, e, g0), h = fma(h0, e, h0);
        const double s = fma(fma(-g, g, x), h, g);
        // proof of correct rounding
        const double r = fma(-s, s, x);
        const int sh = __double2hiint(s), sl = __double2loint(s), xh = __double2hiint(x);
        // x positive with biased exponent in [63, 2047): x in [2^-960, 2^1024)
        const bool range = (unsigned)xh - (63u << 20) < ((2047u - 63u) << 20);
        const bool pow2 = ((sh & 0x000fffff) | sl) == 0;
        // s*ulp(s), or s*ulp(s)/2 at a power of two
        const double su = s * __hiloint2double((int)(((unsigned)sh & 0x7ff00000u) - ((pow2 ? 53u : 52u) << 20)), 0);
        ok = ok && range && r <= su && r > -su;
        return s;
    }
};

}  // namespace claw2

#endif

namespace claw2 {
// IEEE division and square root: the path that redoes a tile whose FastRn
// proofs did not all pass
struct IeeeRn {
    static constexpr bool ok = true;
#if defined(__CUDACC__)
    __host__ __device__
#endif
    inline double operator()(double a, double b) const { return a / b; }
#if defined(__CUDACC__)
    __host__ __device__
#endif
    inline double sqrt(double x) const { return ::sqrt(x); }
};
}  // namespace claw2
