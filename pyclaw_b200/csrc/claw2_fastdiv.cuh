// claw2_fastdiv.cuh -- round-to-nearest double division without a slow-path
// branch, for the FP64-latency-bound Riemann solvers and limiter.
//
// IEEE division on the GPU ends every quotient with a range test and a branch
// to a slow path; each division becomes its own basic block, so the compiler
// cannot overlap the ~15-30 independent-ish divisions of one Riemann solve.
// fdiv() computes the quotient with straight-line code and proves, also with
// straight-line code, that it is the correctly rounded quotient; a solve runs
// with fdiv() and is redone with IEEE division only when some proof failed, so
// its results are those of IEEE division in every case.  The solve keeps one
// FastDiv object and reads its `ok` flag at the end (the step kernel: once per
// tile, then redoes the whole tile with IeeeDiv if any proof failed).
//
// Quotient: reciprocal approximation y0 of b (PTX rcp.approx.ftz.f64), one
// Newton-Raphson step y = y0 + y0*(1 - b*y0), q0 = a*y, and one correction
// q = q0 + y*(a - b*q0) (Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990), all FMAs.
//
// Proof that q = RN(a/b): let rr = a - b*q, computed with one FMA.  When q is
// within an ulp of a/b, rr is exactly representable (it is an integer multiple
// of ulp(b)*ulp(q) smaller than |b|*ulp(q)), so the FMA gives it exactly and
// |a/b - q| = |rr|/|b|.  A quotient of two doubles is never the midpoint of
// two consecutive doubles, so q = RN(a/b) exactly when |a/b - q| is less than
// half the gap from q to its neighbour on the side of a/b: ulp(q)/2, or
// ulp(q)/4 below a power of two.  The test used is |rr| < |b|*ulp(q)/2, with
// ulp(q)/4 whenever q is a power of two (conservative on its upper side); the
// bound is a product by a power of two, hence exact.  When q is not within an
// ulp, |a - b*q| >= |b|*ulp(q)/2 and the rounded rr cannot pass the test.
// Range: |b| and |q| in [2^-480, 2^544) keep every step above free of
// overflow and underflow (|a| >= 2^-961, so the remainder's units are normal
// or exactly representable subnormals); anything else -- zero, subnormal,
// infinite or NaN divisors, huge or tiny quotients -- fails the proof.  A zero
// dividend with an in-range divisor gives a*y, the zero of the right sign.
#pragma once

#if defined(__CUDACC__)

namespace claw2 {

struct FastDiv {
    bool ok = true;

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
};

}  // namespace claw2

#endif

namespace claw2 {
// IEEE division: the path that redoes a tile whose FastDiv proofs did not all pass
struct IeeeDiv {
    static constexpr bool ok = true;
#if defined(__CUDACC__)
    __host__ __device__
#endif
    inline double operator()(double a, double b) const { return a / b; }
};
}  // namespace claw2
