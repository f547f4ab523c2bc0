// claw2_light.cuh -- a leaner tile body for the two-wave acoustics solvers.
//
// Constant- and variable-coefficient acoustics (3 equations, 2 waves) have
// waves, fluctuations and transverse splits whose transverse-velocity (resp.
// normal-velocity) components are structural zeros.  This body computes the
// same unsplit step as step_tile_at (step2.f90:92-248 / flux2.f90:104-206)
// with the same operations on every non-zero component and skips the terms
// that only add an exact zero, so the results are the same values (only the
// sign of an exact zero can differ).  Tile, lanes and chunking are those of
// step_tile_at: one warp per slice line, one lane per interface k = i0-1+slot.
// Neighbouring interfaces exchange waves and left-cell fluxes by warp shuffles
// instead of shared memory; the own-line contributions of a cell stay in
// registers, and only the two cross-line terms (C0 to the line above, C4 to the
// line below) go through a double-buffered shared array, so one block barrier
// per chunk of lines suffices.
#pragma once

#include "claw2_kernels.cuh"

namespace claw2 {

// Normal and transverse solves of the two acoustics solvers on scalars:
// (p, normal velocity) of the two cells -> the two waves (pressure and normal
// components) and speeds; a fluctuation's pressure component -> bmasdq/bpasdq
// (pressure and transverse components).  Same operations as
// RpAcoustics/RpVcAcoustics in claw2_riemann.cuh.
struct LightAcoustics {
    static constexpr bool VC = false;
    CLAW2_HD static void rpn2(double pL, double nL, double pR, double nR, const double*, const double*,
                              const double* prm, double& w1p, double& w1n, double& s1, double& w2p, double& w2n,
                              double& s2)
    {
        const double cc = prm[2], zz = prm[3];
        const double delta1 = pR - pL, delta2 = nR - nL;
        const double a1 = (-delta1 + zz * delta2) / (2.0 * zz);
        const double a2 = (delta1 + zz * delta2) / (2.0 * zz);
        w1p = -a1 * zz; w1n = a1; s1 = -cc;
        w2p = a2 * zz; w2n = a2; s2 = cc;
    }
    // asdq(mv) is a structural zero: (-A + zz*0)/(2zz) has the value -A/(2zz)
    CLAW2_HD static void rpt2(double A, const double*, const double*, const double*, const double* prm,
                              double& bmp, double& bmt, double& bpp, double& bpt)
    {
        const double cc = prm[2], zz = prm[3];
        const double a1 = -A / (2.0 * zz);
        const double a2 = A / (2.0 * zz);
        bmp = cc * a1 * zz; bmt = -cc * a1;
        bpp = cc * a2 * zz; bpt = cc * a2;
    }
};

struct LightVcAcoustics {
    static constexpr bool VC = true;
    CLAW2_HD static void rpn2(double pL, double nL, double pR, double nR, const double* auxL, const double* auxR,
                              const double*, double& w1p, double& w1n, double& s1, double& w2p, double& w2n,
                              double& s2)
    {
        const double zi = auxR[0] * auxR[1];
        const double zim = auxL[0] * auxL[1];
        const double delta1 = pR - pL, delta2 = nR - nL;
        const double a1 = (-delta1 + zi * delta2) / (zim + zi);
        const double a2 = (delta1 + zim * delta2) / (zim + zi);
        w1p = -a1 * zim; w1n = a1; s1 = -auxL[1];
        w2p = a2 * zi; w2n = a2; s2 = auxR[1];
    }
    // a1p/a2p/a3p: (rho, c) of the cell below, the cell, the cell above
    CLAW2_HD static void rpt2(double A, const double* a1p, const double* a2p, const double* a3p, const double*,
                              double& bmp, double& bmt, double& bpp, double& bpt)
    {
        const double cm = a1p[1], cp = a3p[1];
        const double zm = a1p[0] * a1p[1];
        const double zz = a2p[0] * a2p[1];
        const double zp = a3p[0] * a3p[1];
        const double b1 = -A / (zm + zz);
        const double b2 = A / (zz + zp);
        bmp = cm * b1 * zm; bmt = -cm * b1;
        bpp = cp * b2 * zp; bpt = cp * b2;
    }
};

template <class RP> struct LightOf;
template <> struct LightOf<RpAcoustics> { using type = LightAcoustics; };
template <> struct LightOf<RpVcAcoustics> { using type = LightVcAcoustics; };

// shared memory of the light body (doubles): the tile state, the cross-line
// exchange (2 buffers x 4 values x NT), the reduction scratch and the staged
// inputs of one chunk of y lines (4 fields x YR rows x YP columns)
template <int TX, int TY, int NT> struct LightSmem {
    static constexpr int QX = 3 * TX * TY;
    static constexpr int CX = 2 * 4 * NT;
    static constexpr int YR = TY + 4;            // rows j0-2 .. j0+TY+1 read by the lanes
    static constexpr int YP = NT / 32 + 3;       // columns c0-1 .. c0+LPC, padded to an odd pitch
    static constexpr int YS = 4 * YR * YP;
    static constexpr int total = QX + CX + NT + YS;
    static constexpr int bytes = total * 8;
};

// Copy what the y lines c0 .. c0+LPC-1 read (pressure and y-velocity of their
// columns, (rho, c) of those columns and the two next to them) into STG with
// row-wise (coalesced) loads.  Each lane of a y line reads down a column, which
// in global memory is a row-pitch stride per lane; in STG the pitch YP is odd,
// so those reads are free of bank conflicts.  Cells outside the ghosted array
// are set to 0 (no lane reads them).
template <int TY, int NT, bool VC, class Ctx>
CLAW2_HD void light_stage_y(const StepArgs& a, Ctx& ctx, const double* __restrict__ qin, double* STG, int c0, int j0)
{
    constexpr int YR = TY + 4, YP = NT / 32 + 3, NC = NT / 32 + 2, NPOS = YR * NC, FS = YR * YP;
    const long long P = a.plane;
    for (int t = ctx.tid(); t < NPOS; t += NT) {          // positions once, then every field
        const int r = t / NC, c = t - r * NC;
        const int col = c0 - 1 + c, row = j0 - 2 + r;
        const bool in = col >= -CLAW2_NUM_GHOST && col < a.mx + CLAW2_NUM_GHOST && row >= -CLAW2_NUM_GHOST &&
                        row < a.my + CLAW2_NUM_GHOST;
        const long long o = in ? qoff(a, 0, col, row) : 0;
        double* d = STG + r * YP + c;
        d[0 * FS] = in ? qin[o] : 0.0;
        d[1 * FS] = in ? qin[o + 2 * P] : 0.0;
        if (VC) {
            d[2 * FS] = in ? a.aux[o] : 0.0;
            d[3 * FS] = in ? a.aux[o + P] : 0.0;
        }
    }
}

// One chunk of one sweep direction (see sweep_chunk for the meaning of the
// arguments).  buf selects the half of the exchange array this chunk uses.
template <class LRP, int IXY, int TX, int TY, int NT, class Ctx>
CLAW2_HD void light_chunk(const StepArgs& a, Ctx& ctx, const double* __restrict__ qin, double* Qx, double* CXb,
                          const double* STG, int i0, int j0, int line, int cfirst, int clast, bool lineok,
                          double dtn, double dtt, double& cflm)
{
    // y lines read their inputs from the staged copy: field f, row r (= the
    // lane's left cell k-1 at r = slot), column c (= line at c = line-cfirst+1)
    constexpr int YR = TY + 4, YP = NT / 32 + 3;
    auto stg = [&](int f, int r, int c) -> double { return STG[(f * YR + r) * YP + c]; };
    constexpr int MU = IXY == 1 ? 1 : 2, MV = IXY == 1 ? 2 : 1;
    constexpr int NCELL = IXY == 1 ? TX : TY;
    constexpr int NSLOT = NCELL + 3;
    const int tid = ctx.tid();
    const int slot = tid & 31;
    const int len = IXY == 1 ? a.mx : a.my;
    const int k = (IXY == 1 ? i0 : j0) - 1 + slot;
    const bool ifok = lineok && slot < NSLOT && k <= len + 1;
    const bool lim = ifok && slot >= 1 && slot <= NSLOT - 2 && k >= 0 && k <= len;
    const long long P = a.plane;
    const long long along = IXY == 1 ? 1 : a.ld, across = IXY == 1 ? a.ld : 1;
    const long long oL = IXY == 1 ? qoff(a, 0, k - 1, line) : qoff(a, 0, line, k - 1);
    const long long oR = oL + along;

    // ---------------- normal solve ----------------
    double w1p = 0.0, w1n = 0.0, s1 = 0.0, w2p = 0.0, w2n = 0.0, s2 = 0.0;
    const int sc = line - cfirst + 1;                 // this line's column in STG (y lines)
    if (ifok) {
        double auxL[2] = {0.0, 0.0}, auxR[2] = {0.0, 0.0};
        if constexpr (IXY == 2) {
            if (LRP::VC) {
                auxL[0] = stg(2, slot, sc); auxL[1] = stg(3, slot, sc);
                auxR[0] = stg(2, slot + 1, sc); auxR[1] = stg(3, slot + 1, sc);
            }
            LRP::rpn2(stg(0, slot, sc), stg(1, slot, sc), stg(0, slot + 1, sc), stg(1, slot + 1, sc), auxL, auxR,
                      a.prm, w1p, w1n, s1, w2p, w2n, s2);
        } else {
            if (LRP::VC) {
                auxL[0] = a.aux[oL]; auxL[1] = a.aux[oL + P];
                auxR[0] = a.aux[oR]; auxR[1] = a.aux[oR + P];
            }
            LRP::rpn2(qin[oL], qin[oL + MU * P], qin[oR], qin[oR + MU * P], auxL, auxR, a.prm, w1p, w1n, s1, w2p,
                      w2n, s2);
        }
    }
    const double l1p = ctx.shfl_up(w1p), l1n = ctx.shfl_up(w1n), l2p = ctx.shfl_up(w2p), l2n = ctx.shfl_up(w2n);
    const double r1p = ctx.shfl_down(w1p), r1n = ctx.shfl_down(w1n);
    const double r2p = ctx.shfl_down(w2p), r2n = ctx.shfl_down(w2n);

    // ---------------- CFL, limiter, corrections, transverse ----------------
    double apdq_p = 0.0, apdq_n = 0.0, fadd_p = 0.0, fadd_n = 0.0;
    double bmR_p = 0.0, bmR_t = 0.0, bpR_p = 0.0, bpR_t = 0.0;
    double x0 = 0.0, x1 = 0.0, x2 = 0.0, x3 = 0.0, x4 = 0.0, x5 = 0.0, x6 = 0.0, x7 = 0.0;   // for the cell left
    if (lim) {
        {
            const double c1 = dtn * s1, c2 = -dtn * s1;
            cflm = cflm > c1 ? cflm : c1;
            cflm = cflm > c2 ? cflm : c2;
            const double c3 = dtn * s2, c4 = -dtn * s2;
            cflm = cflm > c3 ? cflm : c3;
            cflm = cflm > c4 ? cflm : c4;
        }
        const double amdq_p = s1 * w1p, amdq_n = s1 * w1n;
        apdq_p = s2 * w2p;
        apdq_n = s2 * w2n;
        double cq_p = 0.0, cq_n = 0.0;
        if (a.order == 2) {
            const double dtdxave = 0.5 * (dtn + dtn);
            double L1p = w1p, L1n = w1n, L2p = w2p, L2n = w2n;
            if (a.limit_any && a.mthlim[0] != 0) {
                const double wn = w1p * w1p + w1n * w1n;
                if (wn != 0.0) {
                    const double dot = s1 > 0.0 ? w1p * l1p + w1n * l1n : w1p * r1p + w1n * r1n;
                    const double phi = philim(wn, dot, a.mthlim[0]);
                    L1p = phi * w1p;
                    L1n = phi * w1n;
                }
            }
            if (a.limit_any && a.mthlim[1] != 0) {
                const double wn = w2p * w2p + w2n * w2n;
                if (wn != 0.0) {
                    const double dot = s2 > 0.0 ? w2p * l2p + w2n * l2n : w2p * r2p + w2n * r2n;
                    const double phi = philim(wn, dot, a.mthlim[1]);
                    L2p = phi * w2p;
                    L2n = phi * w2n;
                }
            }
            const double as1 = fabs(s1), as2 = fabs(s2);
            const double f1 = as1 * (1.0 - as1 * dtdxave), f2 = as2 * (1.0 - as2 * dtdxave);
            cq_p = f1 * L1p;
            cq_n = f1 * L1n;
            cq_p = cq_p + f2 * L2p;
            cq_n = cq_n + f2 * L2n;
            fadd_p = 0.5 * cq_p;
            fadd_n = 0.5 * cq_n;
        }
        double bmL_p = 0.0, bmL_t = 0.0, bpL_p = 0.0, bpL_t = 0.0;
        if (a.trans > 0) {
            const bool cor = a.order == 2 && a.trans == 2;
            const double A = cor ? amdq_p + cq_p : amdq_p;
            const double Pf = cor ? apdq_p - cq_p : apdq_p;
            double ax1[2] = {0.0, 0.0}, ax2[2] = {0.0, 0.0}, ax3[2] = {0.0, 0.0};
            if (LRP::VC) {
                if constexpr (IXY == 2) {
                    ax1[0] = stg(2, slot, sc - 1); ax1[1] = stg(3, slot, sc - 1);
                    ax2[0] = stg(2, slot, sc); ax2[1] = stg(3, slot, sc);
                    ax3[0] = stg(2, slot, sc + 1); ax3[1] = stg(3, slot, sc + 1);
                } else {
                    ax1[0] = a.aux[oL - across]; ax1[1] = a.aux[oL - across + P];
                    ax2[0] = a.aux[oL]; ax2[1] = a.aux[oL + P];
                    ax3[0] = a.aux[oL + across]; ax3[1] = a.aux[oL + across + P];
                }
            }
            LRP::rpt2(A, ax1, ax2, ax3, a.prm, bmL_p, bmL_t, bpL_p, bpL_t);
            if (LRP::VC) {
                if constexpr (IXY == 2) {
                    ax1[0] = stg(2, slot + 1, sc - 1); ax1[1] = stg(3, slot + 1, sc - 1);
                    ax2[0] = stg(2, slot + 1, sc); ax2[1] = stg(3, slot + 1, sc);
                    ax3[0] = stg(2, slot + 1, sc + 1); ax3[1] = stg(3, slot + 1, sc + 1);
                } else {
                    ax1[0] = a.aux[oR - across]; ax1[1] = a.aux[oR - across + P];
                    ax2[0] = a.aux[oR]; ax2[1] = a.aux[oR + P];
                    ax3[0] = a.aux[oR + across]; ax3[1] = a.aux[oR + across + P];
                }
            }
            LRP::rpt2(Pf, ax1, ax2, ax3, a.prm, bmR_p, bmR_t, bpR_p, bpR_t);
        }
        const double hl = 0.5 * dtn;
        x0 = dtn * amdq_p; x1 = dtn * amdq_n;
        x2 = fadd_p; x3 = fadd_n;
        x4 = hl * bmL_p; x5 = hl * bmL_t;
        x6 = hl * bpL_p; x7 = hl * bpL_t;
    }
    // what the right neighbour (interface k+1) hands to this lane's cell k
    const double y0 = ctx.shfl_down(x0), y1 = ctx.shfl_down(x1), y2 = ctx.shfl_down(x2), y3 = ctx.shfl_down(x3);
    const double y4 = ctx.shfl_down(x4), y5 = ctx.shfl_down(x5), y6 = ctx.shfl_down(x6), y7 = ctx.shfl_down(x7);

    // ---------------- the slice's contributions to cell k ----------------
    const bool cellok = lim && slot <= NCELL && k < len;
    const bool trans = a.trans > 0;
    double C0p = 0.0, C0t = 0.0, C1p = 0.0, C1n = 0.0, C2p = 0.0, C2n = 0.0, C3p = 0.0, C3t = 0.0, C4p = 0.0,
           C4t = 0.0;
    if (cellok) {
        const double hr = 0.5 * dtn;
        const double qadd_p = (0.0 - dtn * apdq_p) - y0, qadd_n = (0.0 - dtn * apdq_n) - y1;
        const double dF_p = y2 - fadd_p, dF_n = y3 - fadd_n;
        const double g1p = (0.0 - y4) - hr * bmR_p, g1t = (0.0 - y5) - hr * bmR_t;
        const double g2p = (0.0 - y6) - hr * bpR_p, g2t = (0.0 - y7) - hr * bpR_t;
        C0p = dtt * g2p; C0t = dtt * g2t;
        C1p = qadd_p; C1n = qadd_n;
        C2p = dtn * dF_p; C2n = dtn * dF_n;
        C3p = dtt * (g2p - g1p); C3t = dtt * (g2t - g1t);
        C4p = dtt * g1p; C4t = dtt * g1t;
    }
    const int warp = tid >> 5;
    CXb[0 * NT + tid] = C0p;
    CXb[1 * NT + tid] = C0t;
    CXb[2 * NT + tid] = C4p;
    CXb[3 * NT + tid] = C4t;
    ctx.sync();

    // ---------------- combine slices line-1, line, line+1 per cell ----------------
    if (cellok) {
        auto qx = [&](int m, int kk, int ll) -> double& {
            const int ci = IXY == 1 ? kk : ll, cj = IXY == 1 ? ll : kk;
            return Qx[(m * TY + (cj - j0)) * TX + (ci - i0)];
        };
        auto qi = [&](int m, int kk, int ll) -> double {
            return IXY == 1 ? qin[qoff(a, m, kk, ll)] : qx(m, kk, ll);
        };
        auto in_tile_line = [&](int ll) {
            return IXY == 1 ? (ll >= j0 && ll < j0 + TY && ll < a.my) : (ll >= i0 && ll < i0 + TX && ll < a.mx);
        };
        const int up = tid - 32, dn = tid + 32;     // the lanes of lines line-1 and line+1
        if (in_tile_line(line)) {
            double vp, vn, vt;
            if (line == cfirst) {
                vp = qx(0, k, line); vn = qx(MU, k, line); vt = qx(MV, k, line);
            } else {
                vp = qi(0, k, line); vn = qi(MU, k, line); vt = qi(MV, k, line);
                if (trans) {
                    vp = vp + CXb[0 * NT + up];
                    vt = vt + CXb[1 * NT + up];
                }
            }
            if (IXY == 1) {
                vp = vp + C1p - C2p;
                vn = vn + C1n - C2n;
                if (trans) {
                    vp = vp - C3p;
                    vt = vt - C3t;
                }
            } else if (trans) {
                vp = vp + (C1p - C2p - C3p);
                vn = vn + (C1n - C2n);
                vt = vt - C3t;
            } else {
                vp = vp + (C1p - C2p);
                vn = vn + (C1n - C2n);
            }
            if (trans && line != clast) {
                vp = vp - CXb[2 * NT + dn];
                vt = vt - CXb[3 * NT + dn];
            }
            qx(0, k, line) = vp; qx(MU, k, line) = vn; qx(MV, k, line) = vt;
        }
        if (line == clast && in_tile_line(line + 1)) {
            double vp = qi(0, k, line + 1), vn = qi(MU, k, line + 1), vt = qi(MV, k, line + 1);
            if (trans) {
                vp = vp + C0p;
                vt = vt + C0t;
            }
            qx(0, k, line + 1) = vp; qx(MU, k, line + 1) = vn; qx(MV, k, line + 1) = vt;
        }
        if (trans && line == cfirst && in_tile_line(line - 1)) {
            qx(0, k, line - 1) = qx(0, k, line - 1) - C4p;
            qx(MV, k, line - 1) = qx(MV, k, line - 1) - C4t;
        }
    }
    (void)warp;
}

// Whole-tile unsplit step with the light body (capacity and f-waves are not
// used by these solvers' configurations; the caller checks a.capa < 0 and
// !a.fwave).
template <class RP, int TX, int TY, int NT, class Ctx>
CLAW2_HD void light_tile_at(const StepArgs& a, Ctx& ctx, const TileId& tile)
{
    using LRP = typename LightOf<RP>::type;
    using SM = LightSmem<TX, TY, NT>;
    constexpr int LPC = NT / 32;
    static_assert(TX + 3 <= 32 && TY + 3 <= 32, "tile too wide for one 32-lane line");
    double* Qx = ctx.smem();
    double* CX = Qx + SM::QX;
    double* red = CX + SM::CX;
    double* STG = red + NT;
    const int tid = ctx.tid();
    const int warp = tid >> 5;
    const int i0 = tile.bx * TX, j0 = tile.by * TY;
    const double* qin = a.qin;
    double* qout = a.qout;
    double dt = a.dt;
    if (a.ctrl) {
        if (a.ctrl->done) return;
        dt = a.ctrl->dt;
        const int cur = a.ctrl->cur;
        qin = cur ? a.q1 : a.q0;
        qout = cur ? a.q0 : a.q1;
    }
    const double dtdx = dt / a.dx, dtdy = dt / a.dy;
    double cflm = 0.0;
    int chunk = 0;
    {
        const int first = j0 - 1;
        const int last = (j0 + TY < a.my) ? j0 + TY : a.my;
        for (int c0 = first; c0 <= last; c0 += LPC, chunk++) {
            const int line = c0 + warp;
            const int clast = (c0 + LPC - 1 < last) ? c0 + LPC - 1 : last;
            light_chunk<LRP, 1, TX, TY, NT>(a, ctx, qin, Qx, CX + (chunk & 1) * 4 * NT, nullptr, i0, j0, line, c0,
                                            clast, line <= last, dtdx, dtdy, cflm);
        }
    }
    {
        const int first = i0 - 1;
        const int last = (i0 + TX < a.mx) ? i0 + TX : a.mx;
        for (int c0 = first; c0 <= last; c0 += LPC, chunk++) {
            const int line = c0 + warp;
            const int clast = (c0 + LPC - 1 < last) ? c0 + LPC - 1 : last;
            // the previous chunk's barrier has passed: no lane still reads STG
            light_stage_y<TY, NT, LRP::VC>(a, ctx, qin, STG, c0, j0);
            ctx.sync();
            light_chunk<LRP, 2, TX, TY, NT>(a, ctx, qin, Qx, CX + (chunk & 1) * 4 * NT, STG, i0, j0, line, c0,
                                            clast, line <= last, dtdy, dtdx, cflm);
        }
    }
    ctx.sync();
    finish_tile<3, TX, TY, NT>(a, ctx, tile, Qx, TX * TY, red, qout, i0, j0, cflm, dt);
}

}  // namespace claw2
