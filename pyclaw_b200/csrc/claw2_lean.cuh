// claw2_lean.cuh -- a leaner unsplit tile body for the solvers with dense
// waves and no aux arrays (Euler 4- and 5-wave Roe, shallow-water Roe).
//
// Same step as step_tile_at (step2.f90:92-248 / flux2.f90:104-206) with the
// same operations in the same order, so the results are the same values; only
// the data movement differs, as in the acoustics body of claw2_light.cuh:
//  - each lane computes the quantities of one cell that the normal solve
//    needs (RP::Cell: square roots, pressures, Roe-average numerators) and
//    takes those of the cell right of its interface from the next lane, so
//    each cell's are computed once per line instead of once per interface;
//    with TX = 28 the 32 lanes hold the 32 cells i0-2 .. i0+29 of the line's
//    31 interfaces;
//  - the normal solve stays in registers; for the limiter each lane takes its
//    right neighbour's wave by warp shuffle and forms dotr = wave(k).wave(k+1);
//    dotl of lane k is dotr of lane k-1 (one more shuffle), the same products
//    summed in the same component order (a*b == b*a exactly);
//  - what the cell left of an interface needs from it (dtdx*amdq, fadd and
//    the two transverse splits) moves one lane by shuffle;
//  - a cell's own-line contributions stay in registers; only the two
//    cross-line terms (to the line above and below) go through a
//    double-buffered shared array: one block barrier per chunk of lines;
//  - the tile's whole input halo (rows j0-2..j0+TY+1, columns i0-2..i0+TX+1)
//    is staged in shared memory once by the tensor memory accelerator (two
//    boxes of 16 columns x 32 rows x MEQN fields, 128-byte swizzle; see
//    claw2_tma.cuh) while the threads wait on an mbarrier; x lines read rows
//    of it and y lines read down its columns;
//  - a tile whose staged halo holds one state skips both sweeps: every
//    interface would join two equal states, so its cells keep their values
//    and its CFL number comes from one Riemann solve (uniform_cfl).
#pragma once

#include "claw2_kernels.cuh"
#include "claw2_tma.cuh"

namespace claw2 {

// Shared memory of the lean body (doubles): the staged input halo (2 boxes x
// MEQN fields x TR rows x 16 columns, at a 1024-byte boundary for the
// swizzle), the tile state, the cross-line exchange (2 buffers x 2 terms x
// MEQN x NT) and the reduction scratch; `bytes` includes up to 1 KB of
// alignment padding in front of the halo.
template <class RP, int TX, int TY, int NT> struct LeanSmem {
    static constexpr int MEQN = RP::MEQN;
    static constexpr int QP = TX | 1;            // row pitch of the tile state: odd, so that
                                                 // y lines walking down a column avoid bank conflicts
    static constexpr int QX = MEQN * TY * QP;
    static constexpr int CX = 2 * 2 * MEQN * NT;
    static constexpr int TR = TY + 4;            // rows j0-2 .. j0+TY+1
    static constexpr int BOX = MEQN * TR * 16;   // one box: columns 16b .. 16b+15 of the halo
    static constexpr int HS = 2 * BOX;
    static constexpr int total = HS + QX + CX + NT;
    static constexpr int bytes = total * 8 + 1024;
    static_assert(TX + 4 == 32 && TR == 32, "the halo is two 16 x 32 boxes");
    static_assert((BOX * 8) % 1024 == 0, "each box starts on a 1024-byte boundary");
};

// The staged input of halo row r, column c, field m: H holds q(m, i0-2+c, j0-2+r).
template <int MEQN, int TR>
__device__ __forceinline__ int lean_hidx(int m, int r, int c)
{
    return (c >> 4) * (MEQN * TR * 16) + m * (TR * 16) + swz128(r, c & 15);
}

// One chunk of one sweep direction (arguments as in sweep_chunk); CXb is the
// half of the exchange array this chunk uses.
template <class RP, int IXY, int TX, int TY, int NT, class Ctx>
CLAW2_HD void lean_chunk(const StepArgs& a, Ctx& ctx, const double* H, double* Qx, double* CXb, int i0, int j0,
                         int line, int cfirst, int clast, bool lineok, double dtn, double dtt, double& cflm)
{
    constexpr int MEQN = RP::MEQN, MW = RP::MW, NROE = RP::NROE;
    using SM = LeanSmem<RP, TX, TY, NT>;
    constexpr int TR = SM::TR;
    // the staged input of cell (kk along the slice, ll across it)
    auto hq = [&](int m, int kk, int ll) -> double {
        return IXY == 1 ? H[lean_hidx<MEQN, TR>(m, ll - j0 + 2, kk - i0 + 2)]
                        : H[lean_hidx<MEQN, TR>(m, kk - j0 + 2, ll - i0 + 2)];
    };
    constexpr int NCELL = IXY == 1 ? TX : TY;
    constexpr int NSLOT = NCELL + 3;
    const int tid = ctx.tid();
    const int slot = tid & 31;
    const int len = IXY == 1 ? a.mx : a.my;
    const int k = (IXY == 1 ? i0 : j0) - 1 + slot;
    const bool ifok = lineok && slot < NSLOT && k <= len + 1;
    const bool lim = ifok && slot >= 1 && slot <= NSLOT - 2 && k >= 0 && k <= len;

    // ---------------- normal solve ----------------
    // the waves are kept as their strengths: wave p is alpha[p] times rpn2c's
    // eigenvector of the Roe averages, rebuilt with the same operations where
    // it is needed (RP::wave_of), and s[p] is RP::speed<p>(roe)
    double alpha[MW], amdq[MEQN], apdq[MEQN], roe[NROE];
#pragma unroll
    for (int p = 0; p < MW; p++) alpha[p] = 0.0;
#pragma unroll
    for (int m = 0; m < MEQN; m++) { amdq[m] = 0.0; apdq[m] = 0.0; }
#pragma unroll
    for (int r = 0; r < NROE; r++) roe[r] = 0.0;
    {
        // this lane's cell k-1, and cell k from the next lane
        typename RP::Cell L{};
        double qL[MEQN];
        const bool cellok = lineok && k - 1 <= len + 1;
#pragma unroll
        for (int m = 0; m < MEQN; m++) qL[m] = cellok ? hq(m, k - 1, line) : 0.0;
        if (cellok) L = RP::template cell<IXY>(qL, a.prm);
        const typename RP::Cell R = L.map([&](double v) { return ctx.shfl_down(v); });
        if (ifok) {
            double qR[MEQN];
#pragma unroll
            for (int m = 0; m < MEQN; m++) qR[m] = hq(m, k, line);
            RP::template rpn2a<IXY>(qL, qR, L, R, a.prm, alpha, amdq, apdq, roe);
        }
    }

    // ---------------- CFL, limiter, second-order corrections ----------------
    if (lim) {
        static_for<MW>([&](auto P) {
            const double sp = RP::template speed<decltype(P)::value>(roe);
            const double c1 = dtn * sp, c2 = -dtn * sp;
            cflm = cflm > c1 ? cflm : c1;
            cflm = cflm > c2 ? cflm : c2;
        });
    }
    double cqxx[MEQN], fadd[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) { cqxx[m] = 0.0; fadd[m] = 0.0; }
    if (a.order == 2) {                       // uniform: every lane takes part in the shuffles
        const double dtdxave = 0.5 * (dtn + dtn);
        // the right neighbour's strengths and the Roe averages its waves use
        double alr[MW], roer[NROE];
#pragma unroll
        for (int p = 0; p < MW; p++) alr[p] = ctx.shfl_down(alpha[p]);
#pragma unroll
        for (int r = 0; r < NROE; r++) roer[r] = r < RP::NROE_WAVE ? ctx.shfl_down(roe[r]) : 0.0;
        static_for<MW>([&](auto P) {
            constexpr int p = decltype(P)::value;
            double wv[MEQN], wn[MEQN];
            RP::template wave_of<IXY, p>(alpha[p], roe, wv);
            RP::template wave_of<IXY, p>(alr[p], roer, wn);
            // dotr = wave(k).wave(k+1); dotl of lane k is dotr of lane k-1
            double dotr = 0.0;
#pragma unroll
            for (int m = 0; m < MEQN; m++) dotr = dotr + wv[m] * wn[m];
            const double dotl = ctx.shfl_up(dotr);
            const double sp = RP::template speed<p>(roe);
            if (lim) {
                const int meth = a.mthlim[p];
                if (a.limit_any && meth != 0) {
                    double wnorm2 = 0.0;
#pragma unroll
                    for (int m = 0; m < MEQN; m++) wnorm2 = wnorm2 + wv[m] * wv[m];
                    if (wnorm2 != 0.0) {
                        const double phi = philim(wnorm2, sp > 0.0 ? dotl : dotr, meth);
#pragma unroll
                        for (int m = 0; m < MEQN; m++) wv[m] = phi * wv[m];
                    }
                }
                const double as = fabs(sp);
                const double f = as * (1.0 - as * dtdxave);
#pragma unroll
                for (int m = 0; m < MEQN; m++) cqxx[m] = (p == 0) ? f * wv[m] : cqxx[m] + f * wv[m];
            }
        });
#pragma unroll
        for (int m = 0; m < MEQN; m++) fadd[m] = 0.5 * cqxx[m];
    }

    // ---------------- transverse splits ----------------
    double bmL[MEQN], bpL[MEQN], bmR[MEQN], bpR[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) { bmL[m] = 0.0; bpL[m] = 0.0; bmR[m] = 0.0; bpR[m] = 0.0; }
    if (lim && a.trans > 0) {
        const bool cor = a.order == 2 && a.trans == 2;
        double A[MEQN], Pf[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            A[m] = cor ? amdq[m] + cqxx[m] : amdq[m];
            Pf[m] = cor ? apdq[m] - cqxx[m] : apdq[m];
        }
        const double noaux[1] = {0.0};
        // a zero fluctuation splits into zeros (up to the sign of zero), so
        // its transverse solve is skipped
        bool nzA = false, nzP = false;
#pragma unroll
        for (int m = 0; m < MEQN; m++) { nzA = nzA || A[m] != 0.0; nzP = nzP || Pf[m] != 0.0; }
        if (nzA) RP::template rpt2<IXY>(1, A, roe, noaux, noaux, noaux, a.prm, bmL, bpL);
        if (nzP) RP::template rpt2<IXY>(2, Pf, roe, noaux, noaux, noaux, a.prm, bmR, bpR);
    }

    // ---------------- the slice's contributions to cell k ----------------
    // what interface k+1 hands to its left cell (this lane's cell k)
    const double hl = 0.5 * dtn;
    double y0[MEQN], y1[MEQN], y2[MEQN], y3[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) {
        // a cell-owning lane (cellok) takes these from lane k+1, which is
        // always a limited interface (lim), so no lane needs them zeroed
        y0[m] = ctx.shfl_down(dtn * amdq[m]);
        y1[m] = ctx.shfl_down(fadd[m]);
        y2[m] = ctx.shfl_down(hl * bmL[m]);
        y3[m] = ctx.shfl_down(hl * bpL[m]);
    }
    const bool cellok = lim && slot <= NCELL && k < len;
    const bool trans = a.trans > 0;
    double C0[MEQN], C1[MEQN], C2[MEQN], C3[MEQN], C4[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) {
        C0[m] = 0.0; C1[m] = 0.0; C2[m] = 0.0; C3[m] = 0.0; C4[m] = 0.0;
    }
    if (cellok) {
        const double hr = 0.5 * dtn;
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            const double qadd = (0.0 - dtn * apdq[m]) - y0[m];
            const double dF = y1[m] - fadd[m];
            const double g1 = (0.0 - y2[m]) - hr * bmR[m];
            const double g2 = (0.0 - y3[m]) - hr * bpR[m];
            C0[m] = dtt * g2;
            C1[m] = qadd;
            C2[m] = dtn * dF;
            C3[m] = dtt * (g2 - g1);
            C4[m] = dtt * g1;
        }
    }
#pragma unroll
    for (int m = 0; m < MEQN; m++) {
        CXb[m * NT + tid] = C0[m];
        CXb[(MEQN + m) * NT + tid] = C4[m];
    }
    ctx.sync();

    // ---------------- combine slices line-1, line, line+1 per cell ----------------
    if (cellok) {
        auto qx = [&](int m, int kk, int ll) -> double& {
            const int ci = IXY == 1 ? kk : ll, cj = IXY == 1 ? ll : kk;
            return Qx[(m * TY + (cj - j0)) * SM::QP + (ci - i0)];
        };
        auto qi = [&](int m, int kk, int ll) -> double { return IXY == 1 ? hq(m, kk, ll) : qx(m, kk, ll); };
        auto in_tile_line = [&](int ll) {
            return IXY == 1 ? (ll >= j0 && ll < j0 + TY && ll < a.my) : (ll >= i0 && ll < i0 + TX && ll < a.mx);
        };
        const int up = tid - 32, dn = tid + 32;     // the lanes of lines line-1 and line+1
        if (in_tile_line(line)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double v;
                if (line == cfirst) v = qx(m, k, line);                 // has up(line-1) already
                else {
                    v = qi(m, k, line);
                    if (trans) v = v + CXb[m * NT + up];
                }
                if (IXY == 1) {
                    v = v + C1[m] - C2[m];
                    if (trans) v = v - C3[m];
                } else {
                    v = v + (trans ? (C1[m] - C2[m] - C3[m]) : (C1[m] - C2[m]));
                }
                if (trans && line != clast) v = v - CXb[(MEQN + m) * NT + dn];
                qx(m, k, line) = v;
            }
        }
        if (line == clast && in_tile_line(line + 1)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double v = qi(m, k, line + 1);
                if (trans) v = v + C0[m];
                qx(m, k, line + 1) = v;
            }
        }
        if (trans && line == cfirst && in_tile_line(line - 1)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) qx(m, k, line - 1) = qx(m, k, line - 1) - C4[m];
        }
    }
}

// True in every thread when the tile's input halo (rows j0-2..j0+TY+1,
// columns i0-2..i0+TX+1, clipped to the ghosted array: every cell either sweep
// reads) holds one state.  A NaN never compares equal, so a non-finite halo
// is never uniform.
template <class RP, int TX, int TY, int TR>
__device__ __forceinline__ bool lean_uniform_halo(const StepArgs& a, const double* H, int i0, int j0, int tid, int nt)
{
    constexpr int MEQN = RP::MEQN;
    const int rmax = a.my + 3 - j0, cmax = a.mx + 3 - i0;   // last halo row / column inside the array
    double q0[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) q0[m] = H[lean_hidx<MEQN, TR>(m, 0, 0)];
    bool same = true;
    // columns c, c+1 (c even) sit side by side in the swizzled box: one
    // 16-byte load per pair
    for (int e = tid; e < TR * 16; e += nt) {
        const int r = e >> 4, c = (e & 15) * 2;
        if (r <= rmax && c <= cmax) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                const double2 v = *reinterpret_cast<const double2*>(H + lean_hidx<MEQN, TR>(m, r, c));
                same = same && v.x == q0[m] && (c + 1 > cmax || v.y == q0[m]);
            }
        }
    }
    return __syncthreads_and(same);
}

// The two sweeps of the full tile step over the staged halo H; returns this
// thread's running CFL maximum.
template <class RP, int TX, int TY, int NT, class Ctx>
__device__ __forceinline__ double lean_tile_sweeps(const StepArgs& a, Ctx& ctx, const double* H, double* Qx, double* CX,
                                                   int i0, int j0, double dtdx, double dtdy)
{
    constexpr int MEQN = RP::MEQN;
    constexpr int LPC = NT / 32;
    const int warp = ctx.tid() >> 5;
    double cflm = 0.0;
    int chunk = 0;
    {
        const int first = j0 - 1;
        const int last = (j0 + TY < a.my) ? j0 + TY : a.my;
        for (int c0 = first; c0 <= last; c0 += LPC, chunk++) {
            const int line = c0 + warp;
            const int clast = (c0 + LPC - 1 < last) ? c0 + LPC - 1 : last;
            lean_chunk<RP, 1, TX, TY, NT>(a, ctx, H, Qx, CX + (chunk & 1) * 2 * MEQN * NT, i0, j0, line, c0, clast,
                                          line <= last, dtdx, dtdy, cflm);
        }
    }
    {
        const int first = i0 - 1;
        const int last = (i0 + TX < a.mx) ? i0 + TX : a.mx;
        for (int c0 = first; c0 <= last; c0 += LPC, chunk++) {
            const int line = c0 + warp;
            const int clast = (c0 + LPC - 1 < last) ? c0 + LPC - 1 : last;
            lean_chunk<RP, 2, TX, TY, NT>(a, ctx, H, Qx, CX + (chunk & 1) * 2 * MEQN * NT, i0, j0, line, c0, clast,
                                          line <= last, dtdy, dtdx, cflm);
        }
    }
    return cflm;
}

// Whole-tile unsplit step with the lean body (the caller checks that the
// problem has no capacity function and no f-waves).  tm0 / tm1: tensor maps
// of the input state (uncontrolled mode: both of a.qin; controlled mode: of
// a.q0 and a.q1) over the ghosted planes (mx+4 x my+4 x MEQN, row pitch ld,
// 16 x 32 x MEQN boxes, 128-byte swizzle); bar: an mbarrier in shared memory.
// The halo copy is waited for at most about a second (clock64 cycles); a
// tile whose copy does not arrive reports a timeout instead of a result.
constexpr long long kTmaWaitCycles = 2000000000LL;

template <class RP, int TX, int TY, int NT, class Ctx>
__device__ __forceinline__ void lean_tile_at(const StepArgs& a, Ctx& ctx, const TileId& tile, const CUtensorMap* tm0,
                                             const CUtensorMap* tm1, uint64_t* bar)
{
    constexpr int MEQN = RP::MEQN;
    using SM = LeanSmem<RP, TX, TY, NT>;
    static_assert(TX + 4 <= 32 && TY + 4 <= 32, "a line's cells i0-2 .. i0+TX+1 must fit its 32 lanes");
    static_assert(RP::MAUX == 0, "the lean body serves the solvers without aux arrays");
    double* H = ctx.smem();
    {
        const uint32_t s0 = smem_addr(H);
        H += ((1024u - (s0 & 1023u)) & 1023u) / 8;       // 1024-byte boundary for the swizzled boxes
    }
    double* Qx = H + SM::HS;
    double* CX = Qx + SM::QX;
    double* red = CX + SM::CX;
    const int tid = ctx.tid();
    const int i0 = tile.bx * TX, j0 = tile.by * TY;
    double* qout = a.qout;
    double dt = a.dt;
    const CUtensorMap* tm = tm0;
    if (a.ctrl) {
        if (a.ctrl->done) return;                  // uniform across the grid
        dt = a.ctrl->dt;
        const int cur = a.ctrl->cur;
        tm = cur ? tm1 : tm0;
        qout = cur ? a.q0 : a.q1;
    }
    // stage the halo: rows j0-2.., columns i0-2.. are ghosted-array indices
    // j0, i0 (x = i0 is even, so the box starts on a 16-byte boundary)
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_arrive_expect_tx(bar, (uint32_t)(SM::HS * 8 + a.halo_shortfall));
        tma_load_3d(H, tm, bar, i0, j0, 0);
        tma_load_3d(H + SM::BOX, tm, bar, i0 + 16, j0, 0);
    }
    const double dtdx = dt / a.dx, dtdy = dt / a.dy;
    double cflm = 0.0;
    ctx.sync();                                    // the barrier is initialised
    // the whole CTA takes the same path
    const bool fault = __syncthreads_or(!mbar_wait_bounded(bar, 0, kTmaWaitCycles));
    bool keep = false;                             // the tile's cells keep their values
    if (fault) {
        mbar_wait_bounded(bar, 0, kTmaWaitCycles);  // let a late copy land before the CTA moves on
    } else if (lean_uniform_halo<RP, TX, TY, SM::TR>(a, H, i0, j0, tid, NT)) {
        // A tile whose input halo holds one state has zero waves and
        // fluctuations at every interface: its cells keep their values (the
        // full step adds only zeros) and only its CFL number is computed.
        double q0[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) q0[m] = H[lean_hidx<MEQN, SM::TR>(m, 0, 0)];
        bool finite = true;
        const double cu = uniform_cfl<RP>(q0, a.prm, dtdx, dtdy, finite);
        if (finite) {                              // the same in every thread
            for (int e = tid; e < TY * SM::QP; e += NT) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) Qx[m * TY * SM::QP + e] = q0[m];
            }
            cflm = cu;
            keep = true;
        }
    }
    if (!fault && !keep) cflm = lean_tile_sweeps<RP, TX, TY, NT>(a, ctx, H, Qx, CX, i0, j0, dtdx, dtdy);
    ctx.sync();
    finish_tile<MEQN, TX, TY, NT, SM::QP>(a, ctx, tile, Qx, TY * SM::QP, red, qout, i0, j0, cflm, dt, fault);
}

}  // namespace claw2
