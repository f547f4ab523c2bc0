// claw2_riemann.cuh -- per-interface Riemann solvers for the sm_100a step.
//
// The reference calls rpn2/rpt2 once per 1D slice through Fortran callbacks
// (src/pyclaw/classic/flux2.f90:104-105, :184-198) and passes Roe averages
// from rpn2 to rpt2 through a COMMON block.  On the GPU each thread owns one
// interface, so a solver here is a struct of device functions working on
// register arrays for that interface; the Roe averages stay in registers
// between the normal and the transverse solve.
//
// Every expression keeps the reference's evaluation order (left to right,
// parentheses as written, no FMA contraction: this file is compiled with
// --fmad=false), so results agree bit for bit with the CPU oracle except for
// the sign of exact zeros where a structurally zero term is skipped.
//
// Indexing: qL is the cell left of the interface (Fortran qr(:,i-1)), qR the
// cell right of it (Fortran ql(:,i)).  IXY = 1 for x slices, 2 for y slices;
// MU/MV are the 0-based normal / transverse momentum components.
#pragma once

#if defined(__CUDACC__)
#define CLAW2_DEV __device__ __forceinline__
#else
#include <cmath>
#define CLAW2_DEV inline
#endif

namespace claw2 {

template <int IXY> struct Dir {
    static constexpr int MU = IXY == 1 ? 1 : 2;
    static constexpr int MV = IXY == 1 ? 2 : 1;
};

// ---------------------------------------------------------------------------
// Euler equations, Roe solver with Harten-Hyman entropy fix
// development/rp_approaches/rpn2_euler_5wave.f:87-298 and
// rpt2_euler_5wave.f:47-95.  TRACER selects the 5-equation form.
// ---------------------------------------------------------------------------
template <bool TRACER> struct RpEuler {
    static constexpr int MEQN = TRACER ? 5 : 4;
    static constexpr int MW = TRACER ? 5 : 4;
    static constexpr int MAUX = 0;
    static constexpr int NROE = 7;   // u, v, a, enth, u2v2, g1a2, euv

    // What rpn2 computes from one cell alone, for either of the cell's two
    // interfaces along a slice: sqrt(rho), the pressure, the three Roe-average
    // numerators (rhou/sqrt(rho), rhov/sqrt(rho), (E+p)/sqrt(rho)) and, for the
    // entropy fix, the normal velocity rhou/rho and the sound speed
    // sqrt(gamma*p/rho).  The lean tile body computes them once per cell and
    // hands them to the neighbouring interface by warp shuffle.
    struct Cell {
        double sq, p, U, V, H, un, c;
        template <class F> CLAW2_DEV Cell map(F f) const { return Cell{f(sq), f(p), f(U), f(V), f(H), f(un), f(c)}; }
    };
    template <int IXY>
    static CLAW2_DEV Cell cell(const double (&q)[MEQN], const double* prm)
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double gamma = prm[0], gamma1 = prm[1];
        Cell c;
        c.sq = sqrt(q[0]);
        c.p = gamma1 * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
        c.U = q[mu] / c.sq;
        c.V = q[mv] / c.sq;
        c.H = (q[3] + c.p) / c.sq;
        c.un = q[mu] / q[0];
        c.c = sqrt(gamma * c.p / q[0]);
        return c;
    }

    template <int IXY>
    static CLAW2_DEV void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const double* auxL, const double* auxR, const double* prm,
                                                double (&wave)[MW][MEQN], double (&s)[MW],
                                                double (&amdq)[MEQN], double (&apdq)[MEQN],
                                                double (&roe)[NROE])
    {
        rpn2c<IXY>(qL, qR, cell<IXY>(qL, prm), cell<IXY>(qR, prm), prm, wave, s, amdq, apdq, roe);
    }

    // rpn2 with the two cells' quantities given (Cell, same expressions)
    template <int IXY>
    static CLAW2_DEV void rpn2c(const double (&qL)[MEQN], const double (&qR)[MEQN], const Cell& L, const Cell& R,
                                const double* prm, double (&wave)[MW][MEQN], double (&s)[MW],
                                double (&amdq)[MEQN], double (&apdq)[MEQN], double (&roe)[NROE])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double gamma = prm[0], gamma1 = prm[1];
        // Roe averages, :87-104: u = (qL(mu)/sqrt(rhoL) + qR(mu)/sqrt(rhoR))/(sqrt(rhoL)+sqrt(rhoR)), ...
        const double rhsqrtl = L.sq;
        const double rhsqrtr = R.sq;
        const double rhsq2 = rhsqrtl + rhsqrtr;
        const double u = (L.U + R.U) / rhsq2;
        const double v = (L.V + R.V) / rhsq2;
        const double enth = (L.H + R.H) / rhsq2;
        const double u2v2 = u * u + v * v;
        const double asq = gamma1 * (enth - .5 * u2v2);
        const double a = sqrt(asq);
        const double g1a2 = gamma1 / asq;
        const double euv = enth - u2v2;
        roe[0] = u; roe[1] = v; roe[2] = a; roe[3] = enth; roe[4] = u2v2; roe[5] = g1a2; roe[6] = euv;

        // wave strengths and waves, :110-165
        const double d0 = qR[0] - qL[0];
        const double d1 = qR[mu] - qL[mu];
        const double d2 = qR[mv] - qL[mv];
        const double d3 = qR[3] - qL[3];
        bool same = d0 == 0.0 && d1 == 0.0 && d2 == 0.0 && d3 == 0.0;
        if constexpr (TRACER) same = same && qR[4] - qL[4] == 0.0;
        if (same) {
            // Equal states: every strength is zero, so every wave and, through
            // the entropy fix (whose s1 equals s0 here, so no transonic split)
            // and apdq = sum s*wave - amdq, both fluctuations are zero; only the
            // sign of a zero can differ from computing them.  The speeds still
            // count in the CFL number.
#pragma unroll
            for (int p = 0; p < MW; p++) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) wave[p][m] = 0.0;
            }
            s[0] = u - a; s[1] = u; s[2] = u; s[3] = u + a;
            if constexpr (TRACER) s[4] = u;
#pragma unroll
            for (int m = 0; m < MEQN; m++) { amdq[m] = 0.0; apdq[m] = 0.0; }
            return;
        }
        const double a3 = g1a2 * (euv * d0 + u * d1 + v * d2 - d3);
        const double a2 = d2 - v * d0;
        const double a4 = (d1 + (a - u) * d0 - a * a3) / (2.0 * a);
        const double a1 = d0 - a3 - a4;
        wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; wave[0][3] = a1 * (enth - u * a);
        s[0] = u - a;
        wave[1][0] = 0.0; wave[1][mu] = 0.0; wave[1][mv] = a2; wave[1][3] = a2 * v;
        s[1] = u;
        wave[2][0] = a3; wave[2][mu] = a3 * u; wave[2][mv] = a3 * v; wave[2][3] = a3 * 0.5 * u2v2;
        s[2] = u;
        wave[3][0] = a4; wave[3][mu] = a4 * (u + a); wave[3][mv] = a4 * v; wave[3][3] = a4 * (enth + u * a);
        s[3] = u + a;
        if constexpr (TRACER) {
            wave[0][4] = 0.0; wave[1][4] = 0.0; wave[2][4] = 0.0; wave[3][4] = 0.0;
            wave[4][0] = 0.0; wave[4][1] = 0.0; wave[4][2] = 0.0; wave[4][3] = 0.0;
            wave[4][4] = qR[4] - qL[4];
            s[4] = u;
        }

        // entropy fix, :205-286
        {
            // cim1 = sqrt(gamma*pim1/rhoim1) and qr(mu,i-1)/rhoim1 of the left cell;
            // gamma1*(qr(4,i-1) - 0.5*(qr(mu,i-1)**2 + qr(mv,i-1)**2)/rhoim1) is its
            // pressure bit for bit: the two squares are the same and IEEE addition commutes
            const double cim1 = L.c;
            const double s0 = L.un - cim1;
            if (s0 >= 0.0 && s[0] > 0.0) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) amdq[m] = 0.0;
            } else {
                const double rho1 = qL[0] + wave[0][0];
                const double rhou1 = qL[mu] + wave[0][mu];
                const double rhov1 = qL[mv] + wave[0][mv];
                const double en1 = qL[3] + wave[0][3];
                const double p1 = gamma1 * (en1 - 0.5 * (rhou1 * rhou1 + rhov1 * rhov1) / rho1);
                const double c1 = sqrt(gamma * p1 / rho1);
                const double s1 = rhou1 / rho1 - c1;
                double sfract;
                if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
                else if (s[0] < 0.0) sfract = s[0];
                else sfract = 0.0;
#pragma unroll
                for (int m = 0; m < MEQN; m++) amdq[m] = sfract * wave[0][m];
                if (s[1] < 0.0) {
                    // shear and entropy (and tracer) waves; wave 2's first and
                    // normal-momentum entries are structural zeros
                    amdq[0] = amdq[0] + s[2] * wave[2][0];
                    amdq[mu] = amdq[mu] + s[2] * wave[2][mu];
                    amdq[mv] = amdq[mv] + s[1] * wave[1][mv];
                    amdq[mv] = amdq[mv] + s[2] * wave[2][mv];
                    amdq[3] = amdq[3] + s[1] * wave[1][3];
                    amdq[3] = amdq[3] + s[2] * wave[2][3];
                    if constexpr (TRACER) amdq[4] = amdq[4] + s[4] * wave[4][4];
                    const double ci = R.c;              // the right cell's, as cim1
                    const double s3 = R.un + ci;
                    const double rho2 = qR[0] - wave[3][0];
                    const double rhou2 = qR[mu] - wave[3][mu];
                    const double rhov2 = qR[mv] - wave[3][mv];
                    const double en2 = qR[3] - wave[3][3];
                    const double p2 = gamma1 * (en2 - 0.5 * (rhou2 * rhou2 + rhov2 * rhov2) / rho2);
                    const double c2 = sqrt(gamma * p2 / rho2);
                    const double s2 = rhou2 / rho2 + c2;
                    bool add4 = true;
                    if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s[3]) / (s3 - s2);
                    else if (s[3] < 0.0) sfract = s[3];
                    else add4 = false;
                    if (add4) {
#pragma unroll
                        for (int m = 0; m < 4; m++) amdq[m] = amdq[m] + sfract * wave[3][m];
                    }
                }
            }
        }
        // apdq = sum s*wave - amdq, :291-298 (structural zeros skipped)
        {
            double df0 = s[0] * wave[0][0];
            df0 = df0 + s[2] * wave[2][0];
            df0 = df0 + s[3] * wave[3][0];
            double dfu = s[0] * wave[0][mu];
            dfu = dfu + s[2] * wave[2][mu];
            dfu = dfu + s[3] * wave[3][mu];
            double dfv = s[0] * wave[0][mv];
            dfv = dfv + s[1] * wave[1][mv];
            dfv = dfv + s[2] * wave[2][mv];
            dfv = dfv + s[3] * wave[3][mv];
            double dfe = s[0] * wave[0][3];
            dfe = dfe + s[1] * wave[1][3];
            dfe = dfe + s[2] * wave[2][3];
            dfe = dfe + s[3] * wave[3][3];
            apdq[0] = df0 - amdq[0];
            apdq[mu] = dfu - amdq[mu];
            apdq[mv] = dfv - amdq[mv];
            apdq[3] = dfe - amdq[3];
            if constexpr (TRACER) apdq[4] = s[4] * wave[4][4] - amdq[4];
        }
    }

    // The lean tile body keeps an interface's waves as their strengths alpha[p]
    // and rebuilds wave p from alpha[p] and the Roe averages with rpn2c's own
    // expressions (same operands, same operations: the same bits), which holds
    // 4-5 doubles per interface instead of 16-25 through the limiter.
    static constexpr int NROE_WAVE = 5;          // u, v, a, enth, u2v2 build the waves
    template <int IXY, int P>
    static CLAW2_DEV void wave_of(double al, const double (&roe)[NROE], double (&w)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double u = roe[0], v = roe[1], a = roe[2], enth = roe[3], u2v2 = roe[4];
        if constexpr (P == 0) { w[0] = al; w[mu] = al * (u - a); w[mv] = al * v; w[3] = al * (enth - u * a); }
        else if constexpr (P == 1) { w[0] = 0.0; w[mu] = 0.0; w[mv] = al; w[3] = al * v; }
        else if constexpr (P == 2) { w[0] = al; w[mu] = al * u; w[mv] = al * v; w[3] = al * 0.5 * u2v2; }
        else if constexpr (P == 3) { w[0] = al; w[mu] = al * (u + a); w[mv] = al * v; w[3] = al * (enth + u * a); }
        else { w[0] = 0.0; w[1] = 0.0; w[2] = 0.0; w[3] = 0.0; }
        if constexpr (TRACER) w[4] = P == 4 ? al : 0.0;
    }
    // speed of wave P (rpn2c's s[P])
    template <int P>
    static CLAW2_DEV double speed(const double (&roe)[NROE])
    {
        if constexpr (P == 0) return roe[0] - roe[2];
        else if constexpr (P == 3) return roe[0] + roe[2];
        else return roe[0];
    }
    // Between two equal states, speed of wave P of the other direction's
    // solve from this direction's Roe averages: that solve's normal average
    // is this one's transverse average v (the same operands and operations),
    // and its sound speed is this one's a (the pressure and enthalpy do not
    // depend on the direction, and u*u + v*v == v*v + u*u exactly).
    template <int P>
    static CLAW2_DEV double speed_other(const double (&roe)[NROE])
    {
        if constexpr (P == 0) return roe[1] - roe[2];
        else if constexpr (P == 3) return roe[1] + roe[2];
        else return roe[1];
    }
    // rpn2c returning the wave strengths instead of the waves and speeds
    template <int IXY>
    static CLAW2_DEV void rpn2a(const double (&qL)[MEQN], const double (&qR)[MEQN], const Cell& L, const Cell& R,
                                const double* prm, double (&alpha)[MW], double (&amdq)[MEQN], double (&apdq)[MEQN],
                                double (&roe)[NROE])
    {
        constexpr int mv = Dir<IXY>::MV;
        double wave[MW][MEQN], s[MW];
        rpn2c<IXY>(qL, qR, L, R, prm, wave, s, amdq, apdq, roe);
        alpha[0] = wave[0][0];
        alpha[1] = wave[1][mv];
        alpha[2] = wave[2][0];
        alpha[3] = wave[3][0];
        if constexpr (TRACER) alpha[4] = wave[4][4];
    }

    // rpt2_euler_5wave.f:47-95.  The split uses this interface's Roe averages.
    template <int IXY>
    static CLAW2_DEV void rpt2(int, const double (&asdq)[MEQN], const double (&roe)[NROE],
                                                const double*, const double*, const double*,
                                                const double*, double (&bm)[MEQN], double (&bp)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double u = roe[0], v = roe[1], a = roe[2], enth = roe[3], u2v2 = roe[4], g1a2 = roe[5], euv = roe[6];
        const double a3 = g1a2 * (euv * asdq[0] + u * asdq[mu] + v * asdq[mv] - asdq[3]);
        const double a2 = asdq[mu] - u * asdq[0];
        const double a4 = (asdq[mv] + (a - v) * asdq[0] - a * a3) / (2.0 * a);
        const double a1 = asdq[0] - a3 - a4;
        double wb[3][4];
        wb[0][0] = a1; wb[0][mu] = a1 * u; wb[0][mv] = a1 * (v - a); wb[0][3] = a1 * (enth - v * a);
        wb[1][0] = a3; wb[1][mu] = a3 * u + a2; wb[1][mv] = a3 * v; wb[1][3] = a3 * 0.5 * u2v2 + a2 * u;
        wb[2][0] = a4; wb[2][mu] = a4 * u; wb[2][mv] = a4 * (v + a); wb[2][3] = a4 * (enth + v * a);
        const double sb0 = v - a, sb1 = v, sb2 = v + a;
        const double mn0 = fmin(sb0, 0.0), mn1 = fmin(sb1, 0.0), mn2 = fmin(sb2, 0.0);
        const double mx0 = fmax(sb0, 0.0), mx1 = fmax(sb1, 0.0), mx2 = fmax(sb2, 0.0);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            double b = mn0 * wb[0][m];
            b = b + mn1 * wb[1][m];
            bm[m] = b + mn2 * wb[2][m];
            double c = mx0 * wb[0][m];
            c = c + mx1 * wb[1][m];
            bp[m] = c + mx2 * wb[2][m];
        }
        if constexpr (TRACER) {
            bm[4] = fmin(v, 0.0) * asdq[4];
            bp[4] = fmax(v, 0.0) * asdq[4];
        }
    }
};

// ---------------------------------------------------------------------------
// Constant-coefficient acoustics, q = (p,u,v); params rho, bulk, cc, zz.
// Eigenvectors (-Z,1,0) with speed -c and (Z,1,0) with speed +c; transverse
// split with (-Z,0,1) and (Z,0,1).  Same formulas as the oracle.
// ---------------------------------------------------------------------------
struct RpAcoustics {
    static constexpr int MEQN = 3, MW = 2, MAUX = 0, NROE = 1;

    template <int IXY>
    static CLAW2_DEV void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const double*, const double*, const double* prm,
                                                double (&wave)[MW][MEQN], double (&s)[MW],
                                                double (&amdq)[MEQN], double (&apdq)[MEQN],
                                                double (&)[NROE])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double cc = prm[2], zz = prm[3];
        const double delta1 = qR[0] - qL[0];
        const double delta2 = qR[mu] - qL[mu];
        const double a1 = (-delta1 + zz * delta2) / (2.0 * zz);
        const double a2 = (delta1 + zz * delta2) / (2.0 * zz);
        wave[0][0] = -a1 * zz; wave[0][mu] = a1; wave[0][mv] = 0.0; s[0] = -cc;
        wave[1][0] = a2 * zz;  wave[1][mu] = a2; wave[1][mv] = 0.0; s[1] = cc;
        amdq[0] = s[0] * wave[0][0]; amdq[mu] = s[0] * wave[0][mu]; amdq[mv] = 0.0;
        apdq[0] = s[1] * wave[1][0]; apdq[mu] = s[1] * wave[1][mu]; apdq[mv] = 0.0;
    }

    template <int IXY>
    static CLAW2_DEV void rpt2(int, const double (&asdq)[MEQN], const double (&)[NROE],
                                                const double*, const double*, const double*,
                                                const double* prm, double (&bm)[MEQN], double (&bp)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double cc = prm[2], zz = prm[3];
        const double a1 = (-asdq[0] + zz * asdq[mv]) / (2.0 * zz);
        const double a2 = (asdq[0] + zz * asdq[mv]) / (2.0 * zz);
        bm[0] = cc * a1 * zz; bm[mu] = 0.0; bm[mv] = -cc * a1;
        bp[0] = cc * a2 * zz; bp[mu] = 0.0; bp[mv] = cc * a2;
    }
};

// ---------------------------------------------------------------------------
// Variable-coefficient acoustics, aux = (rho, c).  Left-going wave in the
// left cell's material, right-going in the right cell's; the transverse split
// of a fluctuation sitting in cell i1 uses the materials below/above it.
// ---------------------------------------------------------------------------
struct RpVcAcoustics {
    static constexpr int MEQN = 3, MW = 2, MAUX = 2, NROE = 1;

    template <int IXY>
    static CLAW2_DEV void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const double* auxL, const double* auxR, const double*,
                                                double (&wave)[MW][MEQN], double (&s)[MW],
                                                double (&amdq)[MEQN], double (&apdq)[MEQN],
                                                double (&)[NROE])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double zi = auxR[0] * auxR[1];
        const double zim = auxL[0] * auxL[1];
        const double delta1 = qR[0] - qL[0];
        const double delta2 = qR[mu] - qL[mu];
        const double a1 = (-delta1 + zi * delta2) / (zim + zi);
        const double a2 = (delta1 + zim * delta2) / (zim + zi);
        wave[0][0] = -a1 * zim; wave[0][mu] = a1; wave[0][mv] = 0.0; s[0] = -auxL[1];
        wave[1][0] = a2 * zi;   wave[1][mu] = a2; wave[1][mv] = 0.0; s[1] = auxR[1];
        amdq[0] = s[0] * wave[0][0]; amdq[mu] = s[0] * wave[0][mu]; amdq[mv] = 0.0;
        apdq[0] = s[1] * wave[1][0]; apdq[mu] = s[1] * wave[1][mu]; apdq[mv] = 0.0;
    }

    // a1/a2/a3: aux of cell i1 in the slice below, in the slice, and above.
    template <int IXY>
    static CLAW2_DEV void rpt2(int, const double (&asdq)[MEQN], const double (&)[NROE],
                                                const double* a1p, const double* a2p, const double* a3p,
                                                const double*, double (&bm)[MEQN], double (&bp)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double cm = a1p[1], cp = a3p[1];
        const double zm = a1p[0] * a1p[1];
        const double zz = a2p[0] * a2p[1];
        const double zp = a3p[0] * a3p[1];
        const double b1 = (-asdq[0] + zz * asdq[mv]) / (zm + zz);
        const double b2 = (asdq[0] + zz * asdq[mv]) / (zz + zp);
        bm[0] = cm * b1 * zm; bm[mu] = 0.0; bm[mv] = -cm * b1;
        bp[0] = cp * b2 * zp; bp[mu] = 0.0; bp[mv] = cp * b2;
    }
};

// ---------------------------------------------------------------------------
// Shallow water, Roe solver with Harten-Hyman transonic fix; params grav.
// ---------------------------------------------------------------------------
struct RpShallow {
    static constexpr int MEQN = 3, MW = 3, MAUX = 0, NROE = 3;   // ubar, vbar, cbar

    // What rpn2 computes from one cell alone (see RpEuler::Cell): sqrt(h),
    // the Roe-average numerators hu/sqrt(h), hv/sqrt(h), and for the
    // transonic fix the normal velocity hu/h and the wave speed sqrt(g h).
    struct Cell {
        double sq, U, V, un, c;
        template <class F> CLAW2_DEV Cell map(F f) const { return Cell{f(sq), f(U), f(V), f(un), f(c)}; }
    };
    template <int IXY>
    static CLAW2_DEV Cell cell(const double (&q)[MEQN], const double* prm)
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double grav = prm[0];
        Cell c;
        c.sq = sqrt(q[0]);
        c.U = q[mu] / c.sq;
        c.V = q[mv] / c.sq;
        c.un = q[mu] / q[0];
        c.c = sqrt(grav * q[0]);
        return c;
    }

    template <int IXY>
    static CLAW2_DEV void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const double*, const double*, const double* prm,
                                                double (&wave)[MW][MEQN], double (&s)[MW],
                                                double (&amdq)[MEQN], double (&apdq)[MEQN],
                                                double (&roe)[NROE])
    {
        rpn2c<IXY>(qL, qR, cell<IXY>(qL, prm), cell<IXY>(qR, prm), prm, wave, s, amdq, apdq, roe);
    }

    // rpn2 with the two cells' quantities given (Cell, same expressions)
    template <int IXY>
    static CLAW2_DEV void rpn2c(const double (&qL)[MEQN], const double (&qR)[MEQN], const Cell& L, const Cell& R,
                                const double* prm, double (&wave)[MW][MEQN], double (&s)[MW],
                                double (&amdq)[MEQN], double (&apdq)[MEQN], double (&roe)[NROE])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double grav = prm[0];
        const double hl = qL[0], hr = qR[0];
        const double hsqrtl = L.sq, hsqrtr = R.sq;
        const double hsq2 = hsqrtl + hsqrtr;
        const double ubar = (L.U + R.U) / hsq2;
        const double vbar = (L.V + R.V) / hsq2;
        const double hbar = 0.5 * (hl + hr);
        const double cbar = sqrt(grav * hbar);
        const double delta1 = hr - hl;
        const double delta2 = qR[mu] - qL[mu];
        const double delta3 = qR[mv] - qL[mv];
        roe[0] = ubar; roe[1] = vbar; roe[2] = cbar;
        if (delta1 == 0.0 && delta2 == 0.0 && delta3 == 0.0) {
            // equal states: zero waves and fluctuations (see RpEuler::rpn2c);
            // the speeds still count in the CFL number
#pragma unroll
            for (int p = 0; p < MW; p++) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) wave[p][m] = 0.0;
            }
            s[0] = ubar - cbar; s[1] = ubar; s[2] = ubar + cbar;
#pragma unroll
            for (int m = 0; m < MEQN; m++) { amdq[m] = 0.0; apdq[m] = 0.0; }
            return;
        }
        const double a1 = ((ubar + cbar) * delta1 - delta2) / (2.0 * cbar);
        const double a2 = delta3 - vbar * delta1;
        const double a3 = (delta2 - (ubar - cbar) * delta1) / (2.0 * cbar);
        wave[0][0] = a1; wave[0][mu] = a1 * (ubar - cbar); wave[0][mv] = a1 * vbar; s[0] = ubar - cbar;
        wave[1][0] = 0.0; wave[1][mu] = 0.0; wave[1][mv] = a2; s[1] = ubar;
        wave[2][0] = a3; wave[2][mu] = a3 * (ubar + cbar); wave[2][mv] = a3 * vbar; s[2] = ubar + cbar;

        const double s0 = L.un - L.c;          // qL(mu)/hl - sqrt(grav*hl)
        if (s0 >= 0.0 && s[0] > 0.0) {
            amdq[0] = 0.0; amdq[1] = 0.0; amdq[2] = 0.0;
        } else {
            const double h1 = hl + wave[0][0];
            const double hu1 = qL[mu] + wave[0][mu];
            const double s1 = hu1 / h1 - sqrt(grav * h1);
            double sfract;
            if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
            else if (s[0] < 0.0) sfract = s[0];
            else sfract = 0.0;
#pragma unroll
            for (int m = 0; m < MEQN; m++) amdq[m] = sfract * wave[0][m];
            if (s[1] < 0.0) {
                amdq[mv] = amdq[mv] + s[1] * wave[1][mv];
                const double s3 = R.un + R.c;  // qR(mu)/hr + sqrt(grav*hr)
                const double h2 = hr - wave[2][0];
                const double hu2 = qR[mu] - wave[2][mu];
                const double s2 = hu2 / h2 + sqrt(grav * h2);
                bool add3 = true;
                if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s[2]) / (s3 - s2);
                else if (s[2] < 0.0) sfract = s[2];
                else add3 = false;
                if (add3) {
#pragma unroll
                    for (int m = 0; m < MEQN; m++) amdq[m] = amdq[m] + sfract * wave[2][m];
                }
            }
        }
        double df0 = s[0] * wave[0][0];
        df0 = df0 + s[2] * wave[2][0];
        double dfu = s[0] * wave[0][mu];
        dfu = dfu + s[2] * wave[2][mu];
        double dfv = s[0] * wave[0][mv];
        dfv = dfv + s[1] * wave[1][mv];
        dfv = dfv + s[2] * wave[2][mv];
        apdq[0] = df0 - amdq[0];
        apdq[mu] = dfu - amdq[mu];
        apdq[mv] = dfv - amdq[mv];
    }

    // waves as strengths times rpn2c's eigenvectors (see RpEuler::wave_of)
    static constexpr int NROE_WAVE = 3;          // ubar, vbar, cbar
    template <int IXY, int P>
    static CLAW2_DEV void wave_of(double al, const double (&roe)[NROE], double (&w)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double ubar = roe[0], vbar = roe[1], cbar = roe[2];
        if constexpr (P == 0) { w[0] = al; w[mu] = al * (ubar - cbar); w[mv] = al * vbar; }
        else if constexpr (P == 1) { w[0] = 0.0; w[mu] = 0.0; w[mv] = al; }
        else { w[0] = al; w[mu] = al * (ubar + cbar); w[mv] = al * vbar; }
    }
    template <int P>
    static CLAW2_DEV double speed(const double (&roe)[NROE])
    {
        if constexpr (P == 0) return roe[0] - roe[2];
        else if constexpr (P == 2) return roe[0] + roe[2];
        else return roe[0];
    }
    // Between two equal states, speed of wave P of the other direction's
    // solve from this direction's Roe averages (see RpEuler::speed_other;
    // cbar depends on the depths alone).
    template <int P>
    static CLAW2_DEV double speed_other(const double (&roe)[NROE])
    {
        if constexpr (P == 0) return roe[1] - roe[2];
        else if constexpr (P == 2) return roe[1] + roe[2];
        else return roe[1];
    }
    template <int IXY>
    static CLAW2_DEV void rpn2a(const double (&qL)[MEQN], const double (&qR)[MEQN], const Cell& L, const Cell& R,
                                const double* prm, double (&alpha)[MW], double (&amdq)[MEQN], double (&apdq)[MEQN],
                                double (&roe)[NROE])
    {
        constexpr int mv = Dir<IXY>::MV;
        double wave[MW][MEQN], s[MW];
        rpn2c<IXY>(qL, qR, L, R, prm, wave, s, amdq, apdq, roe);
        alpha[0] = wave[0][0];
        alpha[1] = wave[1][mv];
        alpha[2] = wave[2][0];
    }

    template <int IXY>
    static CLAW2_DEV void rpt2(int, const double (&asdq)[MEQN], const double (&roe)[NROE],
                                                const double*, const double*, const double*,
                                                const double*, double (&bm)[MEQN], double (&bp)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        const double u = roe[0], v = roe[1], c = roe[2];
        const double a1 = ((v + c) * asdq[0] - asdq[mv]) / (2.0 * c);
        const double a2 = asdq[mu] - u * asdq[0];
        const double a3 = (asdq[mv] - (v - c) * asdq[0]) / (2.0 * c);
        double wb[3][3];
        wb[0][0] = a1; wb[0][mu] = a1 * u; wb[0][mv] = a1 * (v - c);
        wb[1][0] = 0.0; wb[1][mu] = a2; wb[1][mv] = 0.0;
        wb[2][0] = a3; wb[2][mu] = a3 * u; wb[2][mv] = a3 * (v + c);
        const double mn0 = fmin(v - c, 0.0), mn1 = fmin(v, 0.0), mn2 = fmin(v + c, 0.0);
        const double mx0 = fmax(v - c, 0.0), mx1 = fmax(v, 0.0), mx2 = fmax(v + c, 0.0);
        bm[0] = mn0 * wb[0][0] + mn2 * wb[2][0];
        bp[0] = mx0 * wb[0][0] + mx2 * wb[2][0];
        {
            double b = mn0 * wb[0][mu];
            b = b + mn1 * wb[1][mu];
            bm[mu] = b + mn2 * wb[2][mu];
            double c2 = mx0 * wb[0][mu];
            c2 = c2 + mx1 * wb[1][mu];
            bp[mu] = c2 + mx2 * wb[2][mu];
        }
        bm[mv] = mn0 * wb[0][mv] + mn2 * wb[2][mv];
        bp[mv] = mx0 * wb[0][mv] + mx2 * wb[2][mv];
    }
};

// ---------------------------------------------------------------------------
// Two-dimensional p-system with f-waves (nonlinear elasticity in layered
// media, apps/psystem_2d/psystem.py): q = (eps, rho u, rho v), aux = (rho, K,
// linearity, eps of the cell before the step); sigma = K eps (linearity 1) or
// exp(K eps) - 1 (linearity 2), c = sqrt(sigma_eps / rho), Z = rho c.  The
// normal solve splits the flux jump of f = (-u, -sigma, 0) on (1, Z_left) with
// speed -c_left and (1, -Z_right) with speed c_right; the transverse solve
// splits a fluctuation on (1, Z_below) going down with -c_below and
// (1, -Z_above) going up with c_above.  Same formulas as the oracle.
// ---------------------------------------------------------------------------
struct RpPsystem {
    static constexpr int MEQN = 3, MW = 2, MAUX = 4, NROE = 1;

    static CLAW2_DEV void cell(const double* aux, double eps, double& sigma, double& c, double& z)
    {
        const double rho = aux[0], K = aux[1];
        double se;
        if (aux[2] == 1.0) { sigma = K * eps; se = K; }
        else { const double e = exp(K * eps); sigma = e - 1.0; se = K * e; }
        c = sqrt(se / rho);
        z = rho * c;
    }

    template <int IXY>
    static CLAW2_DEV void rpn2(const double (&qL)[MEQN], const double (&qR)[MEQN],
                                                const double* auxL, const double* auxR, const double*,
                                                double (&wave)[MW][MEQN], double (&s)[MW],
                                                double (&amdq)[MEQN], double (&apdq)[MEQN],
                                                double (&)[NROE])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        double sgl, cl, zl, sgr, cr, zr;
        cell(auxL, qL[0], sgl, cl, zl);
        cell(auxR, qR[0], sgr, cr, zr);
        const double ul = qL[mu] / auxL[0];
        const double ur = qR[mu] / auxR[0];
        const double df1 = (-ur) - (-ul);
        const double df2 = (-sgr) - (-sgl);
        const double b1 = (zr * df1 + df2) / (zl + zr);
        const double b2 = (zl * df1 - df2) / (zl + zr);
        wave[0][0] = b1; wave[0][mu] = b1 * zl; wave[0][mv] = 0.0; s[0] = -cl;
        wave[1][0] = b2; wave[1][mu] = -b2 * zr; wave[1][mv] = 0.0; s[1] = cr;
#pragma unroll
        for (int m = 0; m < MEQN; m++) { amdq[m] = wave[0][m]; apdq[m] = wave[1][m]; }
    }

    // a1p/a3p: aux of the cells below and above the one the fluctuation sits in
    template <int IXY>
    static CLAW2_DEV void rpt2(int, const double (&asdq)[MEQN], const double (&)[NROE],
                                                const double* a1p, const double*, const double* a3p,
                                                const double*, double (&bm)[MEQN], double (&bp)[MEQN])
    {
        constexpr int mu = Dir<IXY>::MU, mv = Dir<IXY>::MV;
        double sgb, cb, zb, sga, ca, za;
        cell(a1p, a1p[3], sgb, cb, zb);
        cell(a3p, a3p[3], sga, ca, za);
        const double gb = (za * asdq[0] + asdq[mv]) / (zb + za);
        const double ga = (zb * asdq[0] - asdq[mv]) / (zb + za);
        bm[0] = -cb * gb; bm[mu] = 0.0; bm[mv] = -cb * gb * zb;
        bp[0] = ca * ga; bp[mu] = 0.0; bp[mv] = -ca * ga * za;
    }
};

}  // namespace claw2
