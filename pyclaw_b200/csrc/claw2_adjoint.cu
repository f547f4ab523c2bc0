// claw2_adjoint.cu -- multi-shot variable-coefficient acoustics and the
// hand-written adjoint of its unsplit step (include/claw2_adjoint.h).
//
// Forward.  A shot is one wavefield; all shots share aux = (rho, c) and dt.
// claw2_shots_step runs the fused tile step (the light body of
// claw2_light.cuh) with the shot as the third grid dimension.
//
// Adjoint.  One step of the reference's unsplit method (step2.f90:92-248,
// flux2.f90:104-206, limiter.f90:34-58, philim.f90:18-55) with the vc-acoustics
// Riemann solvers, per slice line and interface k (between cells k-1, k):
//   rpn2:    a1 = (-dp + zR du)/(zL+zR),  a2 = (dp + zL du)/(zL+zR),  z = rho c
//            W1 = a1 (-zL, 1), s1 = -cL;  W2 = a2 (zR, 1), s2 = cR
//            amdq = s1 W1, apdq = s2 W2
//   limiter: L_p = phi(r_p) W_p, r_p = W_p(k).W_p(k -+ 1) / |W_p(k)|^2
//   cqxx  = sum_p |s_p| (1 - |s_p| dt/dx) L_p,  fadd = cqxx/2
//   rpt2:    A = amdq + cqxx in cell k-1, P = apdq - cqxx in cell k, each split
//            into bm = c- b1 (z-, 0, -1)... with the aux of the cell and its two
//            neighbours across the slice
//   update:  q(k) += -dtdx (apdq(k) + amdq(k+1)) - dtdx (fadd(k+1) - fadd(k))
//               - dtdy (g2 - g1) on the own slice, +dtdy g2 / -dtdy g1 on the
//               slices above / below.
// The adjoint transposes that map with the limiter branches frozen.  It is
// organised like the forward: one CTA per AT x AT tile (and shot), one warp
// per slice line, one lane per interface.  Each CTA recomputes the forward
// values of every interface its cells depend on and gathers the adjoint into
// its own cells only, so no two CTAs write the same cell and the result is
// deterministic.  A cell's state enters only its own row's x-slice and its own
// column's y-slice, so the lines of a tile are its own rows/columns plus one
// line on each side whose transverse splits read the tile's aux.
#include <cuda_runtime.h>

#include <cstring>

#define CLAW2_EXPORT __attribute__((visibility("default")))
#include "../../include/claw2.h"
#include "../../include/claw2_adjoint.h"
#include "claw2_devattr.h"
#include "claw2_kernels.cuh"
#include "claw2_light.cuh"

namespace claw2 {
namespace adj {

constexpr int AT = 27;        // cells per tile side: 32 lanes = interfaces i0-2 .. i0+AT+2
constexpr int ANT = 256;      // 8 warps
constexpr int AR = AT + 4;    // shared accumulators: the tile plus a two-cell ghost ring
constexpr int FT = 29;        // forward tile (the plain step's unsplit tile)
#ifndef CLAW2_ADJ_MINB
#define CLAW2_ADJ_MINB 2      // resident CTAs per SM the register budget is sized for
#endif

struct AdjArgs {
    const double* q;          // state at the start of the step, shot 0
    const double* aux;        // (rho, c)
    const double* lam_in;     // adjoint of the step's output, shot 0
    double* lam_out;          // adjoint of the step's input (unfolded), shot 0
    double* gaux;             // aux gradient accumulator, shot 0
    long long ld, plane, qstride, gstride;
    int mx, my;
    double dtdx, dtdy;
    int order, trans;
    int mthlim[2];
};

__device__ __forceinline__ long long cell(const AdjArgs& a, int i, int j)
{
    return (long long)(j + CLAW2_NUM_GHOST) * a.ld + (i + CLAW2_NUM_GHOST);
}

// philim.f90:18-55 as a function of r, with the derivative of the branch the
// comparisons select (the same comparisons as philim in claw2_kernels.cuh).
__device__ __forceinline__ double philim_branch(double r, int meth, double& d)
{
    double t, dt, u, du;
    switch (meth) {
    case 2:                                            // superbee
        if (1.0 < 2.0 * r) { t = 1.0; dt = 0.0; } else { t = 2.0 * r; dt = 2.0; }
        if (2.0 < r) { u = 2.0; du = 0.0; } else { u = r; du = 1.0; }
        if (!(t > u)) { t = u; dt = du; }
        if (0.0 > t) { d = 0.0; return 0.0; }
        d = dt;
        return t;
    case 3: {                                          // van Leer
        const double ar = fabs(r);
        const double sg = r > 0.0 ? 1.0 : (r < 0.0 ? -1.0 : 0.0);
        const double den = 1.0 + ar;
        d = ((1.0 + sg) * den - (r + ar) * sg) / (den * den);
        return (r + ar) / den;
    }
    case 4: {                                          // MC
        const double c = (1.0 + r) / 2.0;
        if (c < 2.0) { t = c; dt = 0.5; } else { t = 2.0; dt = 0.0; }
        if (!(t < 2.0 * r)) { t = 2.0 * r; dt = 2.0; }
        if (0.0 > t) { d = 0.0; return 0.0; }
        d = dt;
        return t;
    }
    case 5:
        d = 1.0;
        return r;
    default:                                           // minmod (and ids outside 1..5)
        if (1.0 < r) { t = 1.0; dt = 0.0; } else { t = r; dt = 1.0; }
        if (0.0 > t) { d = 0.0; return 0.0; }
        d = dt;
        return t;
    }
}

// What one lane hands to the cell it owns on its line (cell k, right of its
// interface): the state adjoint (pressure, normal velocity) and the aux
// gradient of cell k on the line itself, on the line below and above.
struct LineOut {
    double dq_p, dq_n;
    double ga_own[2], ga_dn[2], ga_up[2];
};

// Transposed transverse split of a fluctuation with pressure component `asdq`
// sitting in a cell whose (rho, c) on the lines below/at/above are
// (r0,c0)/(r1,c1)/(r2,c2) and whose impedance-sum reciprocals are iD1 =
// 1/(z0+z1), iD2 = 1/(z1+z2).  bm_*, bp_*: adjoints of bmasdq/bpasdq
// (pressure and transverse components).  Returns d/d asdq; g_*: aux gradient.
__device__ __forceinline__ double split_T(double asdq, double bm_p, double bm_t, double bp_p, double bp_t, double r0,
                                          double c0, double r1, double c1, double r2, double c2, double iD1,
                                          double iD2, double& gr0, double& gc0, double& gr1, double& gc1,
                                          double& gr2, double& gc2)
{
    const double zm = r0 * c0, zp = r2 * c2;
    const double b1 = -asdq * iD1, b2 = asdq * iD2;
    const double db1 = c0 * zm * bm_p - c0 * bm_t;
    const double db2 = c2 * zp * bp_p + c2 * bp_t;
    const double dcm = b1 * zm * bm_p - b1 * bm_t;
    const double dcp = b2 * zp * bp_p + b2 * bp_t;
    const double dD1 = -b1 * db1 * iD1, dD2 = -b2 * db2 * iD2;
    const double dzm = c0 * b1 * bm_p + dD1;
    const double dzp = c2 * b2 * bp_p + dD2;
    const double dzz = dD1 + dD2;
    gr0 = c0 * dzm; gc0 = r0 * dzm + dcm;
    gr1 = c1 * dzz; gc1 = r1 * dzz;
    gr2 = c2 * dzp; gc2 = r2 * dzp + dcp;
    return -db1 * iD1 + db2 * iD2;
}

// One slice line of the adjoint.  full = false for a line whose cells the
// tile does not own: only its transverse splits' aux gradients on the
// neighbouring lines (ga_dn, ga_up) are needed.
// y lines read their inputs from a staged copy (adj_stage_y): field f, row r
// (the lane's left cell k-1 at r = lane), column c (the line at c = sc)
constexpr int YR = 33;                 // rows j0-3 .. j0+AT+2
constexpr int YP = ANT / 32 + 3;       // columns c0-1 .. c0+8, padded to an odd pitch
constexpr int YF = 7;                  // p, v, rho, c, lambda_p, lambda_u, lambda_v

template <int IXY>
__device__ __forceinline__ void adj_line(const AdjArgs& a, const double* __restrict__ q,
                                         const double* __restrict__ lin, const double* __restrict__ STG, int sc,
                                         int i0, int j0, int line, bool lineok, bool full, LineOut& o)
{
    constexpr int MN = IXY == 1 ? 1 : 2;     // normal velocity component
    constexpr int MT = IXY == 1 ? 2 : 1;     // transverse velocity component
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int len = IXY == 1 ? a.mx : a.my;
    const int k = (IXY == 1 ? i0 : j0) - 2 + lane;
    const long long P = a.plane;
    const long long along = IXY == 1 ? 1 : a.ld, across = IXY == 1 ? a.ld : 1;
    const double dtn = IXY == 1 ? a.dtdx : a.dtdy, dtt = IXY == 1 ? a.dtdy : a.dtdx;
    const double* __restrict__ aux = a.aux;
    // the forward solves interfaces -1..len+1 of slices -1..len_other and limits 0..len
    const bool ex = lineok && k >= -1 && k <= len + 1;
    const bool lim = ex && a.order == 2 && k >= 0 && k <= len && lane >= 1 && lane <= 30;
    const bool trans = a.trans > 0;
    const long long oR = IXY == 1 ? cell(a, k, line) : cell(a, line, k);
    const long long oL = oR - along;
    // side 0: cell k-1, side 1: cell k; dl: the line below (-1), on (0), above (+1)
    auto Gq = [&](int m, int side) -> double {          // m 0: pressure, 1: normal velocity
        if constexpr (IXY == 2) return STG[(m * YR + lane + side) * YP + sc];
        else return q[(side ? oR : oL) + (m ? MN * P : 0)];
    };
    auto Ga = [&](int f, int side, int dl) -> double {  // f 0: rho, 1: c
        if constexpr (IXY == 2) return STG[((2 + f) * YR + lane + side) * YP + sc + dl];
        else return aux[(side ? oR : oL) + dl * across + f * P];
    };
    auto Gl = [&](int m, int side, int dl) -> double {  // m 0: pressure, 1: transverse, 2: normal
        if constexpr (IXY == 2) return STG[((4 + m) * YR + lane + side) * YP + sc + dl];
        else return lin[(side ? oR : oL) + dl * across + (m == 0 ? 0 : (m == 1 ? MT : MN)) * P];
    };

    // ---------------- forward recompute: normal solve (RpVcAcoustics::rpn2) ----------------
    double rhoL = 0.0, cL = 0.0, rhoR = 0.0, cR = 0.0, zL = 0.0, zR = 0.0, d2 = 0.0, den = 1.0, a1 = 0.0, a2 = 0.0;
    if (ex) {
        rhoL = Ga(0, 0, 0); cL = Ga(1, 0, 0);
        rhoR = Ga(0, 1, 0); cR = Ga(1, 1, 0);
        zR = rhoR * cR;
        zL = rhoL * cL;
        const double d1 = Gq(0, 1) - Gq(0, 0);
        d2 = Gq(1, 1) - Gq(1, 0);
        den = zL + zR;
        a1 = (-d1 + zR * d2) / den;
        a2 = (d1 + zL * d2) / den;
    }
    const double w1p = -a1 * zL, w1n = a1, w2p = a2 * zR, w2n = a2;
    const double s1 = -cL, s2 = cR;
    const double w1p_l = __shfl_up_sync(FULL, w1p, 1), w1n_l = __shfl_up_sync(FULL, w1n, 1);
    const double w2p_l = __shfl_up_sync(FULL, w2p, 1), w2n_l = __shfl_up_sync(FULL, w2n, 1);
    const double w1p_r = __shfl_down_sync(FULL, w1p, 1), w1n_r = __shfl_down_sync(FULL, w1n, 1);
    const double w2p_r = __shfl_down_sync(FULL, w2p, 1), w2n_r = __shfl_down_sync(FULL, w2n, 1);

    // ---------------- forward recompute: limiter and corrections ----------------
    bool l1 = false, l2 = false;
    double phi1 = 1.0, phi2 = 1.0, dphi1 = 0.0, dphi2 = 0.0, r1 = 0.0, r2 = 0.0, wn1 = 1.0, wn2 = 1.0;
    double nb1p = 0.0, nb1n = 0.0, nb2p = 0.0, nb2n = 0.0;
    if (lim && a.mthlim[0] != 0) {
        const double wn = w1p * w1p + w1n * w1n;
        if (wn != 0.0) {
            l1 = true;
            wn1 = wn;
            nb1p = s1 > 0.0 ? w1p_l : w1p_r;
            nb1n = s1 > 0.0 ? w1n_l : w1n_r;
            r1 = (w1p * nb1p + w1n * nb1n) / wn;
            phi1 = philim_branch(r1, a.mthlim[0], dphi1);
        }
    }
    if (lim && a.mthlim[1] != 0) {
        const double wn = w2p * w2p + w2n * w2n;
        if (wn != 0.0) {
            l2 = true;
            wn2 = wn;
            nb2p = s2 > 0.0 ? w2p_l : w2p_r;
            nb2n = s2 > 0.0 ? w2n_l : w2n_r;
            r2 = (w2p * nb2p + w2n * nb2n) / wn;
            phi2 = philim_branch(r2, a.mthlim[1], dphi2);
        }
    }
    const bool second = a.order == 2;
    const bool cor = second && a.trans == 2;
    const double dtave = 0.5 * (dtn + dtn);
    const double as1 = fabs(s1), as2 = fabs(s2);
    const double f1 = as1 * (1.0 - as1 * dtave), f2 = as2 * (1.0 - as2 * dtave);
    const double cqp = second ? f1 * (phi1 * w1p) + f2 * (phi2 * w2p) : 0.0;

    // ---------------- transverse splits, transposed ----------------
    // this lane's cell k on the lines below/above, and the impedance-sum
    // reciprocals of cell k (cell k-1's come from the lane to the left)
    double rB0 = 0.0, cB0 = 0.0, rB2 = 0.0, cB2 = 0.0, iB1 = 0.0, iB2 = 0.0;
    if (ex && trans) {
        rB0 = Ga(0, 1, -1); cB0 = Ga(1, 1, -1);
        rB2 = Ga(0, 1, 1); cB2 = Ga(1, 1, 1);
        iB1 = 1.0 / (rB0 * cB0 + zR);
        iB2 = 1.0 / (zR + rB2 * cB2);
    }
    const double iA1 = __shfl_up_sync(FULL, iB1, 1), iA2 = __shfl_up_sync(FULL, iB2, 1);
    double gA_r0 = 0, gA_c0 = 0, gA_r1 = 0, gA_c1 = 0, gA_r2 = 0, gA_c2 = 0;
    double gB_r0 = 0, gB_c0 = 0, gB_r1 = 0, gB_c1 = 0, gB_r2 = 0, gB_c2 = 0;
    double gApd = 0.0, gPpd = 0.0;                                // d/d asdq(1) of A and P
    if (ex && trans) {
        const double h = 0.5 * dtn;
        const double LAp0 = Gl(0, 0, -1), LAt0 = Gl(1, 0, -1);
        const double LAp1 = Gl(0, 0, 0), LAt1 = Gl(1, 0, 0);
        const double LAp2 = Gl(0, 0, 1), LAt2 = Gl(1, 0, 1);
        const double LBp0 = Gl(0, 1, -1), LBt0 = Gl(1, 1, -1);
        const double LBp1 = Gl(0, 1, 0), LBt1 = Gl(1, 1, 0);
        const double LBp2 = Gl(0, 1, 1), LBt2 = Gl(1, 1, 1);
        const double Ap = s1 * w1p + (cor ? cqp : 0.0);
        const double Pp = s2 * w2p - (cor ? cqp : 0.0);
        const double rA0 = Ga(0, 0, -1), cA0 = Ga(1, 0, -1);
        const double rA2 = Ga(0, 0, 1), cA2 = Ga(1, 0, 1);
        // g1(c) = dtt (lam(c) - lam(c, below)), g2(c) = dtt (lam(c, above) - lam(c)); d/d bm = -h g1, d/d bp = -h g2
        gApd = split_T(Ap, -h * (dtt * (LAp1 - LAp0)), -h * (dtt * (LAt1 - LAt0)), -h * (dtt * (LAp2 - LAp1)),
                       -h * (dtt * (LAt2 - LAt1)), rA0, cA0, rhoL, cL, rA2, cA2, iA1, iA2, gA_r0, gA_c0, gA_r1, gA_c1,
                       gA_r2, gA_c2);
        gPpd = split_T(Pp, -h * (dtt * (LBp1 - LBp0)), -h * (dtt * (LBt1 - LBt0)), -h * (dtt * (LBp2 - LBp1)),
                       -h * (dtt * (LBt2 - LBt1)), rB0, cB0, rhoR, cR, rB2, cB2, iB1, iB2, gB_r0, gB_c0, gB_r1, gB_c1,
                       gB_r2, gB_c2);
    }

    // ---------------- correction fluxes and limiter, transposed ----------------
    double gW1p = 0, gW1n = 0, gW2p = 0, gW2n = 0, gs1 = 0, gs2 = 0;
    double send1p = 0.0, send1n = 0.0, send2p = 0.0, send2n = 0.0;   // to the upwind neighbour's wave
    if (full && ex) {
        const double LAp1 = Gl(0, 0, 0), LAn1 = Gl(2, 0, 0);
        const double LBp1 = Gl(0, 1, 0), LBn1 = Gl(2, 1, 0);
        const double gAm_p = -dtn * LAp1 + gApd, gAm_n = -dtn * LAn1;   // d/d amdq
        const double gAp_p = -dtn * LBp1 + gPpd, gAp_n = -dtn * LBn1;   // d/d apdq
        gW1p = s1 * gAm_p; gW1n = s1 * gAm_n; gW2p = s2 * gAp_p; gW2n = s2 * gAp_n;
        gs1 = w1p * gAm_p + w1n * gAm_n;
        gs2 = w2p * gAp_p + w2n * gAp_n;
        if (second) {
            const double gcq_p = 0.5 * (-dtn * (LAp1 - LBp1)) + (cor ? gApd - gPpd : 0.0);
            const double gcq_n = 0.5 * (-dtn * (LAn1 - LBn1));
            const double gL1p = f1 * gcq_p, gL1n = f1 * gcq_n, gL2p = f2 * gcq_p, gL2n = f2 * gcq_n;
            const double gf1 = phi1 * (w1p * gcq_p + w1n * gcq_n), gf2 = phi2 * (w2p * gcq_p + w2n * gcq_n);
            const double sg1 = s1 > 0.0 ? 1.0 : (s1 < 0.0 ? -1.0 : 0.0);
            const double sg2 = s2 > 0.0 ? 1.0 : (s2 < 0.0 ? -1.0 : 0.0);
            gs1 += sg1 * (1.0 - 2.0 * as1 * dtave) * gf1;
            gs2 += sg2 * (1.0 - 2.0 * as2 * dtave) * gf2;
            gW1p += phi1 * gL1p; gW1n += phi1 * gL1n;
            gW2p += phi2 * gL2p; gW2n += phi2 * gL2n;
            if (l1) {
                const double gr = dphi1 * (w1p * gL1p + w1n * gL1n);
                const double gdot = gr / wn1, gwn = -r1 * gdot;   // a reciprocal of a subnormal wn would overflow
                gW1p += 2.0 * gwn * w1p + gdot * nb1p;
                gW1n += 2.0 * gwn * w1n + gdot * nb1n;
                send1p = gdot * w1p; send1n = gdot * w1n;
            }
            if (l2) {
                const double gr = dphi2 * (w2p * gL2p + w2n * gL2n);
                const double gdot = gr / wn2, gwn = -r2 * gdot;
                gW2p += 2.0 * gwn * w2p + gdot * nb2p;
                gW2n += 2.0 * gwn * w2n + gdot * nb2n;
                send2p = gdot * w2p; send2n = gdot * w2n;
            }
        }
    }
    double gqR_p = 0, gqR_n = 0, gqL_p = 0, gqL_n = 0, grL = 0, gcL = 0, grR = 0, gcR = 0;
    if (full) {                                   // warp-uniform
        // a wave with s > 0 read its left neighbour, otherwise its right one
        const bool left1 = s1 > 0.0, left2 = s2 > 0.0;
        const double fr1p = __shfl_down_sync(FULL, left1 ? send1p : 0.0, 1);
        const double fr1n = __shfl_down_sync(FULL, left1 ? send1n : 0.0, 1);
        const double fr2p = __shfl_down_sync(FULL, left2 ? send2p : 0.0, 1);
        const double fr2n = __shfl_down_sync(FULL, left2 ? send2n : 0.0, 1);
        const double fl1p = __shfl_up_sync(FULL, left1 ? 0.0 : send1p, 1);
        const double fl1n = __shfl_up_sync(FULL, left1 ? 0.0 : send1n, 1);
        const double fl2p = __shfl_up_sync(FULL, left2 ? 0.0 : send2p, 1);
        const double fl2n = __shfl_up_sync(FULL, left2 ? 0.0 : send2n, 1);
        if (lane < 31) { gW1p += fr1p; gW1n += fr1n; gW2p += fr2p; gW2n += fr2n; }
        if (lane > 0) { gW1p += fl1p; gW1n += fl1n; gW2p += fl2p; gW2n += fl2n; }
        // ---------------- normal solve, transposed ----------------
        if (ex) {
            const double ga1 = -zL * gW1p + gW1n;
            const double ga2 = zR * gW2p + gW2n;
            const double inv = 1.0 / den;
            const double gd1 = (ga2 - ga1) * inv;
            const double gd2 = (zR * ga1 + zL * ga2) * inv;
            const double gden = -(a1 * ga1 + a2 * ga2) * inv;
            const double gzL = -a1 * gW1p + d2 * ga2 * inv + gden;
            const double gzR = a2 * gW2p + d2 * ga1 * inv + gden;
            gqR_p = gd1; gqL_p = -gd1;
            gqR_n = gd2; gqL_n = -gd2;
            grL = cL * gzL; gcL = -gs1 + rhoL * gzL;
            grR = cR * gzR; gcR = gs2 + rhoR * gzR;
        }
    }

    // ---------------- gather onto cell k (this lane) from interfaces k and k+1 ----------------
    o.dq_p = gqR_p + __shfl_down_sync(FULL, gqL_p, 1);
    o.dq_n = gqR_n + __shfl_down_sync(FULL, gqL_n, 1);
    o.ga_own[0] = (grR + gB_r1) + __shfl_down_sync(FULL, grL + gA_r1, 1);
    o.ga_own[1] = (gcR + gB_c1) + __shfl_down_sync(FULL, gcL + gA_c1, 1);
    o.ga_dn[0] = gB_r0 + __shfl_down_sync(FULL, gA_r0, 1);
    o.ga_dn[1] = gB_c0 + __shfl_down_sync(FULL, gA_c0, 1);
    o.ga_up[0] = gB_r2 + __shfl_down_sync(FULL, gA_r2, 1);
    o.ga_up[1] = gB_c2 + __shfl_down_sync(FULL, gA_c2, 1);
}

// Copy what the y lines c0 .. c0+7 read (state, material and adjoint of their
// columns and of the two next to them, rows j0-3 .. j0+AT+2) into STG with
// row-wise loads; a y line's lanes then read down a column of STG (odd pitch:
// no bank conflicts) instead of with a row-pitch stride from global memory.
// Cells outside the ghosted array are set to 0 (no lane reads them).
__device__ __forceinline__ void adj_stage_y(const AdjArgs& a, const double* __restrict__ q,
                                            const double* __restrict__ lin, double* STG, int c0, int j0)
{
    constexpr int NC = ANT / 32 + 2, NPOS = YR * NC, FS = YR * YP;
    const long long P = a.plane;
    for (int t = threadIdx.x; t < NPOS; t += ANT) {      // positions once, then every field
        const int r = t / NC, c = t - r * NC;
        const int col = c0 - 1 + c, row = j0 - 3 + r;
        const bool in = col >= -CLAW2_NUM_GHOST && col < a.mx + CLAW2_NUM_GHOST && row >= -CLAW2_NUM_GHOST &&
                        row < a.my + CLAW2_NUM_GHOST;
        const long long o = in ? cell(a, col, row) : 0;
        double* d = STG + r * YP + c;
        d[0 * FS] = in ? q[o] : 0.0;
        d[1 * FS] = in ? q[o + 2 * P] : 0.0;
        d[2 * FS] = in ? a.aux[o] : 0.0;
        d[3 * FS] = in ? a.aux[o + P] : 0.0;
        d[4 * FS] = in ? lin[o] : 0.0;
        d[5 * FS] = in ? lin[o + P] : 0.0;
        d[6 * FS] = in ? lin[o + 2 * P] : 0.0;
    }
}

// One sweep direction of a tile: lines first..last in chunks of 8 (one per
// warp).  Each chunk stages its lines' aux gradients for the neighbouring
// lines (up, dn) in one half of XS, passes one barrier, and then every line
// adds to its own row: its own terms, up from the line below and dn from the
// line above; the chunk's first line also adds its dn to the row below the
// chunk and its last line its up to the row above (those rows belong to the
// neighbouring chunks, whose writes the barriers order).
template <int IXY>
__device__ __forceinline__ void adj_sweep(const AdjArgs& a, const double* __restrict__ q,
                                          const double* __restrict__ lin, int i0, int j0, int ilo, int ihi, int jlo,
                                          int jhi, double* GQ, double* GA, double* XS, double* STG, int& chunk)
{
    constexpr int MN = IXY == 1 ? 1 : 2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int o0 = IXY == 1 ? j0 : i0;                 // lines run across the tile
    const int olen = IXY == 1 ? a.my : a.mx;
    const int llo = IXY == 1 ? jlo : ilo, lhi = IXY == 1 ? jhi : ihi;    // own lines
    const int clo = IXY == 1 ? ilo : jlo, chi = IXY == 1 ? ihi : jhi;    // own cells along a line
    const int first = o0 - 1 > -1 ? o0 - 1 : -1;
    const int last = o0 + AT < olen ? o0 + AT : olen;
    auto sidx = [&](int c, int l) {
        return IXY == 1 ? (l - j0 + 2) * AR + (c - i0 + 2) : (c - j0 + 2) * AR + (l - i0 + 2);
    };
    for (int c0 = first; c0 <= last; c0 += ANT / 32, chunk++) {
        const int line = c0 + warp;
        const int clast = c0 + ANT / 32 - 1 < last ? c0 + ANT / 32 - 1 : last;
        const bool ok = line <= last;
        const bool own = ok && line >= llo && line < lhi;
        if constexpr (IXY == 2) {
            // the previous chunk's barrier has passed: no lane still reads STG
            adj_stage_y(a, q, lin, STG, c0, j0);
            __syncthreads();
        }
        LineOut o;
        adj_line<IXY>(a, q, lin, STG, line - c0 + 1, i0, j0, line, ok, own, o);
        const int c = (IXY == 1 ? i0 : j0) - 2 + lane;
        const bool cown = ok && c >= clo && c < chi;
        double* X = XS + (chunk & 1) * 4 * ANT;
        X[0 * ANT + tid] = o.ga_up[0];
        X[1 * ANT + tid] = o.ga_up[1];
        X[2 * ANT + tid] = o.ga_dn[0];
        X[3 * ANT + tid] = o.ga_dn[1];
        if (cown && own) {
            const int s = sidx(c, line);
            GQ[s] += o.dq_p;
            GQ[MN * AR * AR + s] += o.dq_n;
        }
        __syncthreads();
        if (cown) {
            if (own) {
                double g0 = o.ga_own[0], g1 = o.ga_own[1];
                if (line > c0) { g0 += X[0 * ANT + tid - 32]; g1 += X[1 * ANT + tid - 32]; }
                if (line < clast) { g0 += X[2 * ANT + tid + 32]; g1 += X[3 * ANT + tid + 32]; }
                const int s = sidx(c, line);
                GA[s] += g0;
                GA[AR * AR + s] += g1;
            }
            if (line == c0 && line - 1 >= llo && line - 1 < lhi) {
                const int s = sidx(c, line - 1);
                GA[s] += o.ga_dn[0];
                GA[AR * AR + s] += o.ga_dn[1];
            }
            if (line == clast && line + 1 >= llo && line + 1 < lhi) {
                const int s = sidx(c, line + 1);
                GA[s] += o.ga_up[0];
                GA[AR * AR + s] += o.ga_up[1];
            }
        }
    }
}

__global__ void __launch_bounds__(ANT, CLAW2_ADJ_MINB) adjoint_kernel(AdjArgs a)
{
    extern __shared__ double adj_smem[];
    double* GQ = adj_smem;                    // 3 x AR x AR state adjoint
    double* GA = GQ + 3 * AR * AR;            // 2 x AR x AR aux gradient
    double* XS = GA + 2 * AR * AR;            // 2 x 4 x ANT cross-line exchange
    double* STG = XS + 2 * 4 * ANT;           // YF x YR x YP staged inputs of a chunk of y lines
    const int shot = blockIdx.z;
    const double* __restrict__ q = a.q + shot * a.qstride;
    const double* __restrict__ lin = a.lam_in + shot * a.qstride;
    double* lout = a.lam_out + shot * a.qstride;
    double* gaux = a.gaux + shot * a.gstride;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * AT, j0 = blockIdx.y * AT;
    // cells this CTA owns: its tile, plus the ghost ring on domain sides
    const int ilo = i0 == 0 ? -2 : i0, ihi = i0 + AT >= a.mx ? a.mx + 2 : i0 + AT;
    const int jlo = j0 == 0 ? -2 : j0, jhi = j0 + AT >= a.my ? a.my + 2 : j0 + AT;
    const long long P = a.plane;
    {
        // the lines this tile sweeps reach one cell beyond its ghost ring
        const DevCtx ctx{nullptr};
        prefetch_box<ANT>(ctx, q, 3, P, a.ld, a.mx, a.my, j0 - 3, j0 + AT + 2, i0 - 3, i0 + AT + 2);
        prefetch_box<ANT>(ctx, a.aux, 2, P, a.ld, a.mx, a.my, j0 - 3, j0 + AT + 2, i0 - 3, i0 + AT + 2);
        prefetch_box<ANT>(ctx, lin, 3, P, a.ld, a.mx, a.my, j0 - 3, j0 + AT + 2, i0 - 3, i0 + AT + 2);
    }

    for (int t = tid; t < AR * AR; t += ANT) {
        const int i = i0 - 2 + t % AR, j = j0 - 2 + t / AR;
        const bool interior = i >= 0 && i < a.mx && j >= 0 && j < a.my && i < ihi && j < jhi;
        const long long o = cell(a, i, j);
#pragma unroll
        for (int m = 0; m < 3; m++) GQ[m * AR * AR + t] = interior ? lin[o + m * P] : 0.0;   // identity term
        GA[t] = 0.0;
        GA[AR * AR + t] = 0.0;
    }
    __syncthreads();
    int chunk = 0;
    adj_sweep<1>(a, q, lin, i0, j0, ilo, ihi, jlo, jhi, GQ, GA, XS, STG, chunk);     // x-slices: rows
    adj_sweep<2>(a, q, lin, i0, j0, ilo, ihi, jlo, jhi, GQ, GA, XS, STG, chunk);     // y-slices: columns
    __syncthreads();

    for (int t = tid; t < AR * AR; t += ANT) {
        const int i = i0 - 2 + t % AR, j = j0 - 2 + t / AR;
        if (i < ilo || i >= ihi || j < jlo || j >= jhi) continue;
        const long long o = cell(a, i, j);
#pragma unroll
        for (int m = 0; m < 3; m++) lout[o + m * P] = GQ[m * AR * AR + t];
        gaux[o] += GA[t];
        gaux[o + P] += GA[AR * AR + t];
    }
}

// ---------------------------------------------------------------------------
// forward: the plain tile step with the shot as third grid dimension
// ---------------------------------------------------------------------------
#ifndef CLAW2_LIGHT_MINB
#define CLAW2_LIGHT_MINB 3
#endif
__global__ void __launch_bounds__(256, CLAW2_LIGHT_MINB) shots_step_kernel(StepArgs common, long long qstride)
{
    extern __shared__ double smem_dyn[];
    DevCtx ctx{smem_dyn};
    const int shot = blockIdx.z;
    StepArgs a = common;
    a.qin += shot * qstride;
    a.qout += shot * qstride;
    a.partials += (long long)shot * gridDim.x * gridDim.y;
    a.ticket += shot;
    a.cfl_out += shot;
    const TileId t{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x, (int)gridDim.y,
                   (int)(blockIdx.y * gridDim.x + blockIdx.x), (int)(gridDim.x * gridDim.y)};
    light_tile_at<RpVcAcoustics, FT, FT, 256>(a, ctx, t);
}

struct ShotIO {
    double* q;
    long long ld, plane, qstride;
    int mx, my, nrec;
    int bcl[2], bcu[2];
    const int32_t* src;
    const double* amp;
    const int32_t* rec;
    double* traces;
};

// one CTA per shot: the source, its ghost images, then the receivers
__global__ void inject_record_kernel(ShotIO s)
{
    const int shot = blockIdx.x;
    double* p = s.q + shot * s.qstride;          // pressure plane of this shot
    auto off = [&](int i, int j) { return (long long)(j + CLAW2_NUM_GHOST) * s.ld + (i + CLAW2_NUM_GHOST); };
    const int ncell = s.mx * s.my;
    if (threadIdx.x == 0 && s.amp && s.src[shot] >= 0 && s.src[shot] < ncell) {
        const int i = s.src[shot] % s.mx, j = s.src[shot] / s.mx;
        const double v = p[off(i, j)] + s.amp[shot];
        p[off(i, j)] = v;
        int gx[2], gy[2];
        bool nx[2], ny[2];
        const int kx = ghost_images(i, s.mx, s.bcl[0], s.bcu[0], gx, nx);
        const int ky = ghost_images(j, s.my, s.bcl[1], s.bcu[1], gy, ny);
        for (int u = 0; u < kx; u++) p[off(gx[u], j)] = v;
        for (int w = 0; w < ky; w++) p[off(i, gy[w])] = v;
        for (int u = 0; u < kx; u++)
            for (int w = 0; w < ky; w++) p[off(gx[u], gy[w])] = v;
    }
    __syncthreads();
    if (s.traces)
        for (int r = threadIdx.x; r < s.nrec; r += blockDim.x) {
            const int c = s.rec[r];
            s.traces[(long long)shot * s.nrec + r] = (c >= 0 && c < ncell) ? p[off(c % s.mx, c / s.mx)] : 0.0;
        }
}

struct FoldArgs {
    double* x;
    long long ld, plane, stride;
    int mx, my, ncomp;
    int bcl[2], bcu[2];
    int negate;                 // 1: walls negate the normal velocity (state); 0: aux
    int nrec;
    const int32_t* rec;
    const double* gtrace;
};

// Transpose of one side's ghost fill along one axis (fill_body in claw2_capi.cu):
// the adjoint of each ghost cell goes back to its source cell, then is zeroed.
template <int AXIS>
__device__ __forceinline__ void fold_axis(const FoldArgs& f, double* x)
{
    const int n = AXIS == 0 ? f.mx : f.my;
    // along the other axis: y-fold covers all columns (ghosts too), x-fold the interior rows
    const int olo = AXIS == 1 ? -CLAW2_NUM_GHOST : 0;
    const int ohi = AXIS == 1 ? f.mx + CLAW2_NUM_GHOST : f.my;
    const int nother = ohi - olo;
    const int total = f.ncomp * nother * 2;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int o = olo + t % nother;
        const int side = (t / nother) % 2;
        const int m = t / (2 * nother);
        const int bc = side == 0 ? f.bcl[AXIS] : f.bcu[AXIS];
        auto off = [&](int along) {
            const int i = AXIS == 0 ? along : o, j = AXIS == 0 ? o : along;
            return (long long)m * f.plane + (long long)(j + CLAW2_NUM_GHOST) * f.ld + (i + CLAW2_NUM_GHOST);
        };
        for (int g = 0; g < CLAW2_NUM_GHOST; g++) {
            int dst, src;
            if (side == 0) {
                dst = -1 - g;
                src = bc == CLAW2_BC_EXTRAP ? 0 : (bc == CLAW2_BC_PERIODIC ? n - 1 - g : g);
            } else {
                dst = n + g;
                src = bc == CLAW2_BC_EXTRAP ? n - 1 : (bc == CLAW2_BC_PERIODIC ? g : n - 1 - g);
            }
            double v = x[off(dst)];
            if (bc == CLAW2_BC_WALL && f.negate && m == AXIS + 1) v = -v;
            x[off(src)] += v;
            x[off(dst)] = 0.0;
        }
    }
}

// one CTA per shot
__global__ void fold_kernel(FoldArgs f)
{
    double* x = f.x + blockIdx.x * f.stride;
    fold_axis<1>(f, x);         // the y fill ran last, so its transpose runs first
    __syncthreads();
    fold_axis<0>(f, x);
    __syncthreads();
    if (f.gtrace && threadIdx.x == 0)
        for (int r = 0; r < f.nrec; r++) {
            const int c = f.rec[r];
            if (c < 0 || c >= f.mx * f.my) continue;
            x[(long long)(c / f.mx + CLAW2_NUM_GHOST) * f.ld + (c % f.mx + CLAW2_NUM_GHOST)] +=
                f.gtrace[(long long)blockIdx.x * f.nrec + r];
        }
}

}  // namespace adj
}  // namespace claw2

using namespace claw2;
using namespace claw2::adj;

namespace {

int shots_check(const claw2_problem* p, int nshots)
{
    if (!p || nshots < 1) return CLAW2_ERR_INVALID;
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (p->rp != CLAW2_RP_VC_ACOUSTICS || p->transverse < 0 || p->index_capa >= 0 || p->use_fwave)
        return CLAW2_ERR_UNSUPPORTED;
    if (p->mx < 4 || p->my < 4) return CLAW2_ERR_UNSUPPORTED;
    for (int d = 0; d < 2; d++) {
        if (p->bc_lower[d] == CLAW2_BC_CUSTOM || p->bc_upper[d] == CLAW2_BC_CUSTOM) return CLAW2_ERR_UNSUPPORTED;
        if (p->aux_bc_lower[d] == CLAW2_BC_CUSTOM || p->aux_bc_upper[d] == CLAW2_BC_CUSTOM) return CLAW2_ERR_UNSUPPORTED;
        if ((p->aux_bc_lower[d] == CLAW2_BC_PERIODIC) != (p->aux_bc_upper[d] == CLAW2_BC_PERIODIC))
            return CLAW2_ERR_UNSUPPORTED;
    }
    return CLAW2_OK;
}

int ftiles(const claw2_problem* p, int* nbx, int* nby)
{
    *nbx = (p->mx + FT - 1) / FT;
    *nby = (p->my + FT - 1) / FT;
    return *nbx * *nby;
}

inline cudaStream_t Sx(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

size_t claw2_shots_scratch_bytes(const claw2_problem* p, int nshots)
{
    if (!p || nshots < 1 || p->mx < 1 || p->my < 1) return 0;
    int nbx, nby;
    const size_t nt = (size_t)ftiles(p, &nbx, &nby);
    const size_t tickets = ((size_t)nshots * sizeof(unsigned int) + 255) / 256 * 256;
    return tickets + sizeof(double) * nt * (size_t)nshots;
}

int claw2_shots_step(const claw2_problem* p, int nshots, long long shot_stride, const double* q_in, double* q_out,
                     const double* aux, double dt, void* scratch, double* cfl_dev, void* stream)
{
    int rc = shots_check(p, nshots);
    if (rc) return rc;
    if (!q_in || !q_out || !aux || !scratch || !cfl_dev || q_in == q_out) return CLAW2_ERR_INVALID;
    claw2_layout L;
    claw2_get_layout(p, &L);
    if (shot_stride < L.q_elems && nshots > 1) return CLAW2_ERR_INVALID;
    StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.qin = q_in; a.qout = q_out; a.aux = aux; a.dt = dt;
    a.ld = L.ld; a.plane = L.plane; a.mx = p->mx; a.my = p->my; a.dx = p->dx; a.dy = p->dy;
    a.order = p->order; a.trans = p->transverse; a.capa = -1; a.fwave = 0;
    for (int w = 0; w < 2; w++) {
        a.mthlim[w] = p->mthlim[w];
        if (p->mthlim[w] > 0) a.limit_any = 1;
    }
    a.ghost_fused = 1;
    for (int d = 0; d < 2; d++) { a.bcl[d] = p->bc_lower[d]; a.bcu[d] = p->bc_upper[d]; }
    const size_t tickets = ((size_t)nshots * sizeof(unsigned int) + 255) / 256 * 256;
    a.ticket = static_cast<unsigned int*>(scratch);
    a.partials = reinterpret_cast<double*>(static_cast<char*>(scratch) + tickets);
    a.cfl_out = cfl_dev;
    using SM = LightSmem<FT, FT, 256>;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, shots_step_kernel, SM::bytes) != cudaSuccess) return CLAW2_ERR_CUDA;
    int nbx, nby;
    ftiles(p, &nbx, &nby);
    shots_step_kernel<<<dim3(nbx, nby, nshots), 256, SM::bytes, Sx(stream)>>>(a, shot_stride);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

int claw2_shots_inject_record(const claw2_problem* p, int nshots, long long shot_stride, double* q,
                              const int32_t* src_cell, const double* src_amp, int nrec, const int32_t* rec_cell,
                              double* traces, void* stream)
{
    int rc = shots_check(p, nshots);
    if (rc) return rc;
    if (!q || nrec < 0 || (src_amp && !src_cell) || (traces && nrec > 0 && !rec_cell)) return CLAW2_ERR_INVALID;
    claw2_layout L;
    claw2_get_layout(p, &L);
    ShotIO s;
    s.q = q; s.ld = L.ld; s.plane = L.plane; s.qstride = shot_stride; s.mx = p->mx; s.my = p->my; s.nrec = nrec;
    for (int d = 0; d < 2; d++) { s.bcl[d] = p->bc_lower[d]; s.bcu[d] = p->bc_upper[d]; }
    s.src = src_cell; s.amp = src_amp; s.rec = rec_cell; s.traces = nrec > 0 ? traces : nullptr;
    inject_record_kernel<<<nshots, 128, 0, Sx(stream)>>>(s);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

int claw2_shots_adjoint_step(const claw2_problem* p, int nshots, long long shot_stride, const double* q,
                             const double* aux, double dt, const double* lam_in, double* lam_out, double* gaux,
                             long long gaux_stride, void* stream)
{
    int rc = shots_check(p, nshots);
    if (rc) return rc;
    if (!q || !aux || !lam_in || !lam_out || !gaux || lam_in == lam_out) return CLAW2_ERR_INVALID;
    claw2_layout L;
    claw2_get_layout(p, &L);
    if (nshots > 1 && (shot_stride < L.q_elems || gaux_stride < 2 * L.plane)) return CLAW2_ERR_INVALID;
    AdjArgs a;
    a.q = q; a.aux = aux; a.lam_in = lam_in; a.lam_out = lam_out; a.gaux = gaux;
    a.ld = L.ld; a.plane = L.plane; a.qstride = shot_stride; a.gstride = gaux_stride;
    a.mx = p->mx; a.my = p->my;
    a.dtdx = dt / p->dx; a.dtdy = dt / p->dy;
    a.order = p->order; a.trans = p->transverse;
    a.mthlim[0] = p->mthlim[0]; a.mthlim[1] = p->mthlim[1];
    constexpr int smem = (5 * AR * AR + 2 * 4 * ANT + YF * YR * YP) * 8;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, adjoint_kernel, smem) != cudaSuccess) return CLAW2_ERR_CUDA;
    const dim3 grid((p->mx + AT - 1) / AT, (p->my + AT - 1) / AT, nshots);
    adjoint_kernel<<<grid, ANT, smem, Sx(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

static int fold_launch(const claw2_problem* p, int nshots, long long stride, double* x, int ncomp, const int* bl,
                       const int* bu, int negate, int nrec, const int32_t* rec, const double* gtrace, void* stream)
{
    claw2_layout L;
    claw2_get_layout(p, &L);
    FoldArgs f;
    f.x = x; f.ld = L.ld; f.plane = L.plane; f.stride = stride; f.mx = p->mx; f.my = p->my; f.ncomp = ncomp;
    for (int d = 0; d < 2; d++) { f.bcl[d] = bl[d]; f.bcu[d] = bu[d]; }
    f.negate = negate; f.nrec = nrec; f.rec = rec; f.gtrace = gtrace;
    fold_kernel<<<nshots, 256, 0, Sx(stream)>>>(f);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

int claw2_shots_adjoint_fold(const claw2_problem* p, int nshots, long long shot_stride, double* lam, int nrec,
                             const int32_t* rec_cell, const double* gtrace, void* stream)
{
    int rc = shots_check(p, nshots);
    if (rc) return rc;
    if (!lam || nrec < 0 || (gtrace && nrec > 0 && !rec_cell)) return CLAW2_ERR_INVALID;
    return fold_launch(p, nshots, shot_stride, lam, 3, p->bc_lower, p->bc_upper, 1, nrec, rec_cell,
                       nrec > 0 ? gtrace : nullptr, stream);
}

int claw2_shots_fold_aux(const claw2_problem* p, int nshots, long long gaux_stride, double* gaux, void* stream)
{
    int rc = shots_check(p, nshots);
    if (rc) return rc;
    if (!gaux) return CLAW2_ERR_INVALID;
    return fold_launch(p, nshots, gaux_stride, gaux, 2, p->aux_bc_lower, p->aux_bc_upper, 0, 0, nullptr, nullptr,
                       stream);
}

}  // extern "C"
