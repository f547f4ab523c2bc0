// claw2_kernels.cuh -- the fused tile kernels of the 2D wave-propagation step.
//
// One CTA owns a TX x TY tile of output cells and computes everything the
// reference's step2 (src/pyclaw/classic/step2.f90:92-248) or step2ds
// (step2ds.f90:96-252) does for those cells: the normal Riemann solves on
// every interface the tile depends on, the wave limiter (limiter.f90:34-58),
// the second-order correction fluxes and transverse splits (flux2.f90:104-206),
// the conservative update, the CFL number, and the ghost cells the next step
// needs.  q is read from global memory (L1/L2 resident tile); the x-swept
// intermediate state of the tile lives in shared memory.
//
// Order of floating-point operations.  In the reference, slice j writes its
// contributions into rows j-1, j, j+1 of qnew in slice order, so every cell
// receives, left to right: the +dtdy*gadd(2) of slice j-1, the main update of
// slice j, the -dtdy*gadd(1) of slice j+1; then the same from the y slices
// i-1, i, i+1.  A CTA processes its slices in chunks of LPC slices at once;
// inside a chunk the three kinds of contribution are applied in three passes
// separated by barriers (pass a: "from the slice below", b: "own slice",
// c: "from the slice above"), which reproduces that order exactly for every
// cell, whichever chunk its neighbouring slices fall in.
//
// The body is written against a small execution context (thread/block index,
// barrier, atomics) so that the same source builds as a CUDA kernel and, for
// development only, as host code.
#pragma once

#include "claw2_riemann.cuh"

#if defined(__CUDACC__)
#define CLAW2_HD __host__ __device__ __forceinline__
#else
#define CLAW2_HD inline
#include <cmath>
using std::sqrt; using std::fabs; using std::fmin; using std::fmax; using std::copysign; using std::isfinite;
#endif

namespace claw2 {

struct StepArgs {
    const double* qin;     // current state (device layout, ghosts filled)
    double* qout;          // next state
    const double* aux;     // aux (device layout, ghosts filled) or null
    double* q0;            // controlled mode: the two state buffers
    double* q1;
    claw2_control* ctrl;   // controlled mode when non-null
    double* partials;      // one double per CTA
    unsigned int* ticket;  // block-arrival counter, zero between launches
    double* cfl_out;       // uncontrolled mode: CFL number (NaN if the state went non-finite)
    long long ld, plane;
    int mx, my;
    double dx, dy, dt;
    int order, trans, capa, fwave, limit_any;
    int mthlim[CLAW2_MAX_WAVES];
    double prm[CLAW2_MAX_PARAMS];
    int ghost_fused;
    int bcl[2], bcu[2];
    int src, src_aux;      // source term fused into the final write (claw2_source)
    int ctrl_readonly;     // controlled mode that reports the CFL (cfl_out, +inf if
                           // non-finite) instead of updating ctrl (domain decomposition)
    int halo_shortfall;    // bytes more than its halo copies deliver that a lean-body CTA
                           // waits for (0; set only to test the bounded wait)
};

template <int IXY> struct Phase;

// Solvers whose rpn2 splits into per-cell quantities (RP::Cell, RP::cell,
// RP::rpn2c): the Euler and shallow-water Roe solvers.
template <class RP> struct HasCell { static constexpr bool value = false; };
template <bool T> struct HasCell<RpEuler<T>> { static constexpr bool value = true; };
template <> struct HasCell<RpShallow> { static constexpr bool value = true; };

CLAW2_HD long long qoff(const StepArgs& a, int m, int i, int j)
{
    return (long long)m * a.plane + (long long)(j + CLAW2_NUM_GHOST) * a.ld + (i + CLAW2_NUM_GHOST);
}

// philim.f90:18-55; ids outside 1..5 fall through to minmod like the computed GOTO
CLAW2_HD double philim(double a, double b, int meth)
{
    const double r = b / a;
    double t, u;
    switch (meth) {
    case 2:
        t = 1.0 < 2.0 * r ? 1.0 : 2.0 * r;
        u = 2.0 < r ? 2.0 : r;
        t = t > u ? t : u;
        return 0.0 > t ? 0.0 : t;
    case 3:
        return (r + fabs(r)) / (1.0 + fabs(r));
    case 4: {
        const double c = (1.0 + r) / 2.0;
        t = c < 2.0 ? c : 2.0;
        t = t < 2.0 * r ? t : 2.0 * r;
        return 0.0 > t ? 0.0 : t;
    }
    case 5:
        return r;
    default:
        t = 1.0 < r ? 1.0 : r;
        return 0.0 > t ? 0.0 : t;
    }
}

// One iteration of Solver.evolve_to_time after the step (src/pyclaw/solver.py:650-691)
// followed by the clamp at the top of the next iteration (:637-641).
CLAW2_HD void control_update(claw2_control* c, double cfl, int nonfinite)
{
    c->cfl = cfl;
    if (nonfinite) {                     // 1: non-finite state, 2: a tile's input never arrived
        c->error = nonfinite == 2 ? CLAW2_ERR_TIMEOUT : CLAW2_ERR_NONFINITE;
        c->done = 1;
        c->iter++;
        return;
    }
    if (cfl <= c->cfl_max) {
        c->status_cflmax = (c->status_cflmax > cfl) ? c->status_cflmax : cfl;
        if (c->dt_variable) c->t += c->dt;
        else c->t = c->tstart + (double)(c->iter + 1) * c->dt;
        c->numsteps++;
        c->cur ^= 1;
    } else {
        c->rejected++;
        if (!c->dt_variable) {
            c->status_cflmax = (cfl > c->status_cflmax) ? cfl : c->status_cflmax;
            c->error = CLAW2_ERR_CFL;
            c->done = 1;
            c->iter++;
            return;
        }
    }
    if (c->dt_variable) {
        if (cfl > 0.0) {
            const double cand = c->dt * c->cfl_desired / cfl;
            c->dt = (cand < c->dt_max) ? cand : c->dt_max;
            c->status_dtmin = (c->dt < c->status_dtmin) ? c->dt : c->status_dtmin;
            c->status_dtmax = (c->dt > c->status_dtmax) ? c->dt : c->status_dtmax;
        } else {
            c->dt = c->dt_max;
        }
    }
    c->iter++;
    if (c->t >= c->tend || c->take_one_step) { c->done = 1; return; }
    if (c->iter >= c->max_steps) {
        c->done = 1;
        if (c->dt_variable && c->t < c->tend && c->numsteps == c->max_steps) c->error = CLAW2_ERR_MAX_STEPS;
        return;
    }
    if (c->t + c->dt > c->tend && c->tstart < c->tend) c->dt = c->tend - c->t;
    if (c->tend - c->t - c->dt < 1.e-14 * c->t) c->dt = c->tend - c->t;
}

// Ghost images of interior index i along one axis (solver.py:386-432):
// returns how many ghost indices map to i, their indices and whether the
// normal component is negated (walls).  The caller guarantees n >= 4 and that
// a periodic side is matched by a periodic opposite side, so the lower images
// (i in {0,1}, or {n-2,n-1} when periodic) and the upper ones never meet and
// no cell has more than two images.
CLAW2_HD int ghost_images(int i, int n, int bl, int bu, int (&g)[2], bool (&neg)[2])
{
    int k = 0;
    if (bl == CLAW2_BC_EXTRAP && i == 0) { g[0] = -1; neg[0] = false; g[1] = -2; neg[1] = false; k = 2; }
    else if (bl == CLAW2_BC_PERIODIC && i >= n - 2) { g[k] = i - n; neg[k++] = false; }
    else if (bl == CLAW2_BC_WALL && i <= 1) { g[k] = -1 - i; neg[k++] = true; }
    if (bu == CLAW2_BC_EXTRAP && i == n - 1) { g[0] = n; neg[0] = false; g[1] = n + 1; neg[1] = false; k = 2; }
    else if (bu == CLAW2_BC_PERIODIC && i <= 1) { g[k] = n + i; neg[k++] = false; }
    else if (bu == CLAW2_BC_WALL && i >= n - 2) { g[k] = 2 * n - 1 - i; neg[k++] = true; }
    return k;
}

// Write the ghost cells that are images of final cell (i, j) with value v
// (ghost fill fused into the step).
template <int MEQN>
CLAW2_HD void write_ghosts(const StepArgs& a, double* qo, int i, int j, const double (&v)[MEQN])
{
    int gx[2], gy[2];
    bool nx[2], ny[2];
    const int kx = ghost_images(i, a.mx, a.bcl[0], a.bcu[0], gx, nx);
    const int ky = ghost_images(j, a.my, a.bcl[1], a.bcu[1], gy, ny);
    for (int p = 0; p < kx; p++)
#pragma unroll
        for (int m = 0; m < MEQN; m++) qo[qoff(a, m, gx[p], j)] = (m == 1 && nx[p]) ? -v[m] : v[m];
    for (int r = 0; r < ky; r++)
#pragma unroll
        for (int m = 0; m < MEQN; m++) qo[qoff(a, m, i, gy[r])] = (m == 2 && ny[r]) ? -v[m] : v[m];
    for (int p = 0; p < kx; p++)
        for (int r = 0; r < ky; r++)
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double w = v[m];
                if (m == 1 && nx[p]) w = -w;
                if (m == 2 && ny[r]) w = -w;
                qo[qoff(a, m, gx[p], gy[r])] = w;
            }
}

template <int A, int B> struct CMax { static constexpr int value = A > B ? A : B; };

// Shared-memory footprint of the tile kernels (doubles).
//   Qx   the tile's state after the x sweep (then the final state)
//   WB   per interface slot: waves and speeds (read by the neighbouring
//        slots of the same warp); after the limiter the slot is reused for
//        the five per-cell contribution products of the slice (see S3)
//   B2   per interface slot: amdq, apdq and Roe averages from the normal
//        solve; overwritten by the same thread with what the cell to the left
//        of the interface needs (dtdx*amdq, fadd, dtdx/2*B^-A^-dq, dtdx/2*B^+A^-dq)
template <class RP, int TX, int TY, int NT, bool SPLIT> struct TileSmem {
    static constexpr int MEQN = RP::MEQN, MW = RP::MW, NROE = RP::NROE;
    static constexpr int QROWS = SPLIT ? TY + 4 : TY;
    static constexpr int WBSZ = CMax<MW * MEQN + MW, 5 * MEQN>::value;
    static constexpr int B2SZ = CMax<2 * MEQN + NROE, 4 * MEQN>::value;
    static constexpr int QP = TX | 1;    // row pitch of Qx: odd, so that y lines down a column avoid bank conflicts
    static constexpr int QX = MEQN * QROWS * QP;
    static constexpr int total = QX + (WBSZ + B2SZ) * NT + NT;      // + reduction scratch
    static constexpr int bytes = total * 8;
};

// ---------------------------------------------------------------------------
// One chunk of one sweep direction: LPC = NT/32 slice lines, one warp per
// line, one interface per lane.  IXY = 1: lines are x slices (rows) and the
// interface index runs along x; IXY = 2: lines are y slices (columns).
//   line : slice index (0-based; row for IXY=1, column for IXY=2)
//   k    : interface between cells k-1 and k along the slice
// Lines first..first+nlines-1 are processed in chunks in increasing order.
// S1 (normal solve) -> warp barrier -> S2 (limiter, corrections, transverse
// solves) -> warp barrier -> S3 (per-cell contributions of the slice) ->
// block barrier -> S4 (combine the contributions of slices line-1, line,
// line+1 into each cell, in the reference's order) -> block barrier.
// SPLIT = dimensional splitting (no transverse terms; each cell gets exactly
// one contribution per sweep, so S4 is skipped).
// ---------------------------------------------------------------------------
template <class RP, int IXY, bool SPLIT, int TX, int TY, int NT, class Ctx>
CLAW2_HD void sweep_chunk(const StepArgs& a, Ctx& ctx, const double* qin, double* Qx, double* WB, double* B2,
                          int i0, int j0, int line, int cfirst, int clast, bool lineok, bool cflonly,
                          double dtn, double dtt, double& cflm)
{
    constexpr int MEQN = RP::MEQN, MW = RP::MW, MAUX = RP::MAUX, NROE = RP::NROE;
    constexpr int QROWS = SPLIT ? TY + 4 : TY;
    constexpr int QP = TX | 1;                 // row pitch of Qx (TileSmem::QP)
    constexpr int QROW0 = SPLIT ? -2 : 0;      // tile row of Qx row 0, relative to j0
    constexpr int AUXN = MAUX > 0 ? MAUX : 1;
    constexpr int NCELL = IXY == 1 ? TX : TY;  // cells of the tile along the slice
    constexpr int NSLOT = NCELL + 3;           // interfaces needed along the slice
    const int tid = ctx.tid();
    const int slot = tid & 31;
    const int len = IXY == 1 ? a.mx : a.my;
    const int k = (IXY == 1 ? i0 : j0) - 1 + slot;   // this lane's interface
    const bool ifok = lineok && slot < NSLOT && k <= len + 1;
    // interfaces whose fluxes the tile uses: slots 1..NSLOT-2
    const bool cflok = ifok && slot >= 1 && slot <= NSLOT - 2 && k >= 0 && k <= len;
    const bool lim = cflok && !cflonly;

    auto cell_i = [&](int kk) { return IXY == 1 ? kk : line; };
    auto cell_j = [&](int kk) { return IXY == 1 ? line : kk; };
    auto W = [&](int p, int m, int t) -> double& { return WB[(p * MEQN + m) * NT + t]; };
    auto S = [&](int p, int t) -> double& { return WB[(MW * MEQN + p) * NT + t]; };
    auto X = [&](int d, int t) -> double& { return B2[d * NT + t]; };
    auto C = [&](int d, int m, int t) -> double& { return WB[(d * MEQN + m) * NT + t]; };

    double dtl = dtn, dtr = dtn;
    // ---------------- S1: normal Riemann solve ----------------
    // A line's 32 lanes hold its cells k-1 = i0-2 .. when NCELL + 4 <= 32: then
    // the solvers with per-cell quantities (RP::Cell) compute them once per
    // cell and take the right cell's from the next lane (as the lean body).
    constexpr bool PERCELL = HasCell<RP>::value && NCELL + 4 <= 32;
    const bool fromQx = SPLIT && IXY == 2 && !cflonly;   // split y sweep: the x-swept tile state
    auto load = [&](double (&q)[MEQN], int kk) {
        const int ci = cell_i(kk), cj = cell_j(kk);
        if (fromQx) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) q[m] = Qx[(m * QROWS + (cj - j0 - QROW0)) * QP + (ci - i0)];
        } else {
            const long long o = qoff(a, 0, ci, cj);
#pragma unroll
            for (int m = 0; m < MEQN; m++) q[m] = qin[o + m * a.plane];
        }
    };
    auto publish = [&](const double (&wave)[MW][MEQN], const double (&s)[MW], const double (&amdq)[MEQN],
                       const double (&apdq)[MEQN], const double (&roe)[NROE]) {
#pragma unroll
        for (int p = 0; p < MW; p++) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) W(p, m, tid) = wave[p][m];
            S(p, tid) = s[p];
        }
#pragma unroll
        for (int m = 0; m < MEQN; m++) { X(m, tid) = amdq[m]; X(MEQN + m, tid) = apdq[m]; }
#pragma unroll
        for (int r = 0; r < NROE; r++) X(2 * MEQN + r, tid) = roe[r];
        if (a.capa >= 0) {
            const long long oL = qoff(a, 0, cell_i(k - 1), cell_j(k - 1));
            const long long oR = oL + (IXY == 1 ? 1 : a.ld);
            dtl = dtn / a.aux[oL + a.capa * a.plane];
            dtr = dtn / a.aux[oR + a.capa * a.plane];
        }
    };
    if constexpr (PERCELL) {
        double qL[MEQN];
        typename RP::Cell L{};
        if (lineok && k - 1 <= len + 1) {
            load(qL, k - 1);
            L = RP::template cell<IXY>(qL, a.prm);
        }
        const typename RP::Cell R = L.map([&](double v) { return ctx.shfl_down(v); });
        if (ifok) {
            double qR[MEQN], wave[MW][MEQN], s[MW], amdq[MEQN], apdq[MEQN], roe[NROE];
            load(qR, k);
            RP::template rpn2c<IXY>(qL, qR, L, R, a.prm, wave, s, amdq, apdq, roe);
            publish(wave, s, amdq, apdq, roe);
        }
    } else if (ifok) {
        double qL[MEQN], qR[MEQN], auxL[AUXN], auxR[AUXN];
        double wave[MW][MEQN], s[MW], amdq[MEQN], apdq[MEQN], roe[NROE];
        load(qL, k - 1);
        load(qR, k);
        const long long oL = qoff(a, 0, cell_i(k - 1), cell_j(k - 1));
        const long long oR = oL + (IXY == 1 ? 1 : a.ld);      // cell k: one step along the slice
#pragma unroll
        for (int m = 0; m < MAUX; m++) {
            auxL[m] = a.aux[oL + m * a.plane];
            auxR[m] = a.aux[oR + m * a.plane];
        }
        RP::template rpn2<IXY>(qL, qR, auxL, auxR, a.prm, wave, s, amdq, apdq, roe);
        publish(wave, s, amdq, apdq, roe);
    }
    ctx.syncwarp();

    // ---------------- S2: CFL, limiter, corrections, transverse ----------------
    // kept for S3: this interface's right-going parts (for the cell right of it)
    double apdq[MEQN], fadd[MEQN], bmR[MEQN], bpR[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) { apdq[m] = 0.0; fadd[m] = 0.0; bmR[m] = 0.0; bpR[m] = 0.0; }
    if (cflok) {
#pragma unroll
        for (int p = 0; p < MW; p++) {
            const double sp = S(p, tid);
            const double c1 = dtr * sp, c2 = -dtl * sp;
            cflm = cflm > c1 ? cflm : c1;
            cflm = cflm > c2 ? cflm : c2;
        }
    }
    double cqxx[MEQN], amdq[MEQN];
    if (lim) {
#pragma unroll
        for (int m = 0; m < MEQN; m++) { amdq[m] = X(m, tid); apdq[m] = X(MEQN + m, tid); cqxx[m] = 0.0; }
        if (a.order == 2) {
            const double dtdxave = 0.5 * (dtl + dtr);
#pragma unroll
            for (int p = 0; p < MW; p++) {
                double wv[MEQN];
#pragma unroll
                for (int m = 0; m < MEQN; m++) wv[m] = W(p, m, tid);
                const double sp = S(p, tid);
                const int meth = a.mthlim[p];
                if (a.limit_any && meth != 0) {
                    double wnorm2 = 0.0;
#pragma unroll
                    for (int m = 0; m < MEQN; m++) wnorm2 = wnorm2 + wv[m] * wv[m];
                    if (wnorm2 != 0.0) {
                        // dotl = wave(k-1).wave(k) when s > 0, else dotr = wave(k).wave(k+1)
                        const int nb = sp > 0.0 ? tid - 1 : tid + 1;
                        double dot = 0.0;
#pragma unroll
                        for (int m = 0; m < MEQN; m++) dot = dot + wv[m] * W(p, m, nb);
                        const double phi = philim(wnorm2, dot, meth);
#pragma unroll
                        for (int m = 0; m < MEQN; m++) wv[m] = phi * wv[m];
                    }
                }
                const double as = fabs(sp);
                const double f = (a.fwave ? copysign(1.0, sp) : as) * (1.0 - as * dtdxave);
#pragma unroll
                for (int m = 0; m < MEQN; m++) cqxx[m] = (p == 0) ? f * wv[m] : cqxx[m] + f * wv[m];
            }
#pragma unroll
            for (int m = 0; m < MEQN; m++) fadd[m] = 0.5 * cqxx[m];
        }
    }
    if (lim) {
        double bmL[MEQN], bpL[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) { bmL[m] = 0.0; bpL[m] = 0.0; }
        if (!SPLIT && a.trans > 0) {
            double roe[NROE], A[MEQN], P[MEQN];
#pragma unroll
            for (int r = 0; r < NROE; r++) roe[r] = X(2 * MEQN + r, tid);
            const bool cor = a.order == 2 && a.trans == 2;
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                A[m] = cor ? amdq[m] + cqxx[m] : amdq[m];
                P[m] = cor ? apdq[m] - cqxx[m] : apdq[m];
            }
            double ax1[AUXN], ax2[AUXN], ax3[AUXN];
            // the fluctuation split with ilr = 1 sits in cell k-1, with ilr = 2
            // in cell k; aux of that cell and of its neighbours across the slice
            const long long o1 = qoff(a, 0, cell_i(k - 1), cell_j(k - 1));
            const long long along = IXY == 1 ? 1 : a.ld, across = IXY == 1 ? a.ld : 1;
            {
#pragma unroll
                for (int m = 0; m < MAUX; m++) {
                    ax1[m] = a.aux[o1 - across + m * a.plane];
                    ax2[m] = a.aux[o1 + m * a.plane];
                    ax3[m] = a.aux[o1 + across + m * a.plane];
                }
                RP::template rpt2<IXY>(1, A, roe, ax1, ax2, ax3, a.prm, bmL, bpL);
            }
            {
                const long long o2 = o1 + along;
#pragma unroll
                for (int m = 0; m < MAUX; m++) {
                    ax1[m] = a.aux[o2 - across + m * a.plane];
                    ax2[m] = a.aux[o2 + m * a.plane];
                    ax3[m] = a.aux[o2 + across + m * a.plane];
                }
                RP::template rpt2<IXY>(2, P, roe, ax1, ax2, ax3, a.prm, bmR, bpR);
            }
        }
        // publish what the cell left of the interface needs (own slot only)
        const double hl = 0.5 * dtl;
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            X(0 * MEQN + m, tid) = dtl * amdq[m];
            X(1 * MEQN + m, tid) = fadd[m];
            X(2 * MEQN + m, tid) = hl * bmL[m];
            X(3 * MEQN + m, tid) = hl * bpL[m];
        }
    }
    ctx.syncwarp();     // neighbours' waves and B2 slots are complete

    // ---------------- S3: the slice's contributions to its cells ----------------
    // this lane's cell is k (right of its interface); lanes 1..NCELL
    const bool cellok = lim && slot <= NCELL && k < len;
    const bool trans = !SPLIT && a.trans > 0;
    auto qx = [&](int m, int kk, int ll) -> double& {
        const int ci = IXY == 1 ? kk : ll, cj = IXY == 1 ? ll : kk;
        return Qx[(m * QROWS + (cj - j0 - QROW0)) * QP + (ci - i0)];
    };
    auto capa_of = [&](int kk, int ll) {
        return a.aux[qoff(a, a.capa, IXY == 1 ? kk : ll, IXY == 1 ? ll : kk)];
    };
    auto in_tile_line = [&](int ll) {
        // is slice line ll a row/column of cells whose final value this tile owns?
        return IXY == 1 ? (ll >= j0 + QROW0 && ll < j0 + QROW0 + QROWS && ll < a.my + (SPLIT ? 2 : 0))
                        : (ll >= i0 && ll < i0 + TX && ll < a.mx);
    };
    if (cellok) {
        const double hr = 0.5 * dtr;
        const int nb = tid + 1;
        double qadd[MEQN], dF[MEQN], g1[MEQN], g2[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            qadd[m] = (0.0 - dtr * apdq[m]) - X(0 * MEQN + m, nb);
            dF[m] = X(1 * MEQN + m, nb) - fadd[m];
            g1[m] = (0.0 - X(2 * MEQN + m, nb)) - hr * bmR[m];
            g2[m] = (0.0 - X(3 * MEQN + m, nb)) - hr * bpR[m];
        }
        if (SPLIT) {
            if (in_tile_line(line)) {
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    const double q0 = IXY == 1 ? qin[qoff(a, m, k, line)] : qx(m, k, line);
                    if (a.capa < 0) qx(m, k, line) = q0 + qadd[m] - dtn * dF[m];
                    else qx(m, k, line) = q0 + qadd[m] - dtn * dF[m] / capa_of(k, line);
                }
            }
        } else {
            // contribution products: 0 up = dtt*g2 (to line+1), 1 qadd, 2 dtn*dF,
            // 3 dtt*(g2-g1) (own cell), 4 dn = dtt*g1 (to line-1)
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                C(0, m, tid) = dtt * g2[m];
                C(1, m, tid) = qadd[m];
                C(2, m, tid) = dtn * dF[m];
                C(3, m, tid) = dtt * (g2[m] - g1[m]);
                C(4, m, tid) = dtt * g1[m];
            }
        }
    }
    if (SPLIT) return;      // caller places the block barrier
    ctx.sync();

    // ---------------- S4: combine slices line-1, line, line+1 per cell ------------
    // Lines of this chunk: cfirst..clast.  A cell of line l receives, in this
    // order: up(l-1), main(l), dn(l+1).  Contributions from a slice outside
    // the chunk were applied (up) or will be applied (dn) by that chunk.
    if (cellok) {
        auto from = [&](int d, int m, int dw) -> double { return C(d, m, tid + 32 * dw); };
        // (a) this line's own cells
        if (in_tile_line(line)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double v;
                if (line == cfirst) v = qx(m, k, line);                 // has up(line-1) already
                else {
                    // x sweep: start from q; y sweep: from the x-swept value
                    v = IXY == 1 ? qin[qoff(a, m, k, line)] : qx(m, k, line);
                    if (trans) {
                        if (a.capa < 0) v = v + from(0, m, -1);
                        else v = v + from(0, m, -1) / capa_of(k, line);
                    }
                }
                if (a.capa >= 0) {
                    const double tt = trans ? from(3, m, 0) : 0.0;
                    v = v + from(1, m, 0) - (from(2, m, 0) + tt) / capa_of(k, line);
                } else if (IXY == 1) {
                    v = v + from(1, m, 0) - from(2, m, 0);
                    if (trans) v = v - from(3, m, 0);
                } else {
                    v = v + (trans ? (from(1, m, 0) - from(2, m, 0) - from(3, m, 0)) : (from(1, m, 0) - from(2, m, 0)));
                }
                if (trans && line != clast) {
                    if (a.capa < 0) v = v - from(4, m, 1);
                    else v = v - from(4, m, 1) / capa_of(k, line);
                }
                qx(m, k, line) = v;
            }
        }
        // (b) first contribution to the line after the chunk
        if (line == clast && in_tile_line(line + 1)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double v = IXY == 1 ? qin[qoff(a, m, k, line + 1)] : qx(m, k, line + 1);
                if (trans) {
                    if (a.capa < 0) v = v + from(0, m, 0);
                    else v = v + from(0, m, 0) / capa_of(k, line + 1);
                }
                qx(m, k, line + 1) = v;
            }
        }
        // (c) last contribution to the line before the chunk
        if (trans && line == cfirst && in_tile_line(line - 1)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double& q = qx(m, k, line - 1);
                if (a.capa < 0) q = q - from(4, m, 0);
                else q = q - from(4, m, 0) / capa_of(k, line - 1);
            }
        }
    }
    ctx.sync();
}

// Ask L2 for rows r0..r1 and columns c0..c1 (cell indices, clipped here to
// the ghosted array) of nf planes of a device-layout array, one prefetch per
// 128-byte line spread over the CTA's threads: a tile's x lines then find
// their cells in L2 instead of waiting for DRAM chunk after chunk.  Only a
// hint; no result depends on it.
template <int NT, class Ctx>
CLAW2_HD void prefetch_box(Ctx& ctx, const double* base, int nf, long long P, long long ld, int mx, int my, int r0,
                           int r1, int c0, int c1)
{
    r0 = r0 > -CLAW2_NUM_GHOST ? r0 : -CLAW2_NUM_GHOST;
    r1 = r1 < my + CLAW2_NUM_GHOST - 1 ? r1 : my + CLAW2_NUM_GHOST - 1;
    c0 = c0 > -CLAW2_NUM_GHOST ? c0 : -CLAW2_NUM_GHOST;
    c1 = c1 < mx + CLAW2_NUM_GHOST - 1 ? c1 : mx + CLAW2_NUM_GHOST - 1;
    if (r1 < r0 || c1 < c0) return;
    const long long b0 = (long long)(c0 + CLAW2_NUM_GHOST) * 8, b1 = (long long)(c1 + CLAW2_NUM_GHOST) * 8 + 8;
    const int l0 = (int)(b0 >> 7), nl = (int)((b1 + 127) >> 7) - l0;
    const int nrow = r1 - r0 + 1;
    // one (field, row) per thread, its 128-byte lines in turn
    for (int rf = ctx.tid(); rf < nf * nrow; rf += NT) {
        const int r = rf % nrow, f = rf / nrow;
        const char* row = (const char*)(base + f * P) + (long long)(r0 + r + CLAW2_NUM_GHOST) * ld * 8 +
                          ((long long)l0 << 7);
        for (int line = 0; line < nl; line++) ctx.prefetch_l2(row + (line << 7));
    }
}

// ---------------------------------------------------------------------------
// Whole-tile step: x sweeps then y sweeps, LPC = NT/32 lines per chunk.
// ---------------------------------------------------------------------------
// Tile coordinates of one CTA's work item: tile (bx, by) of an nbx x nby grid
// of tiles; `part` is this tile's slot in a.partials and `ntiles` the number of
// tiles that report to the same arrival counter (a.ticket).
struct TileId {
    int bx, by, nbx, nby, part, ntiles;
};

// Final values of the tile's cells (Qx: row stride TX, component stride QSTR,
// row 0 = tile row j0) and their ghost images, then the block CFL max and the
// last-arriving CTA's reduction over all CTAs (and, in controlled mode, the
// device-side time-step controller).
// Geometric source of the Euler equations with radial symmetry (2D, so the
// factor ndim-1 is 1), two-stage second-order Runge-Kutta step of the
// reference app (apps/euler_2d/shockbubble.py:89-124), with its operation
// order; rad = the cell's radial coordinate.
template <int MEQN>
CLAW2_HD void euler_radial_source(double (&v)[MEQN], double rad, double gamma1, double dt)
{
    if constexpr (MEQN >= 4) {
        const double dt2 = dt / 2.0;
        double rho = v[0];
        double u = v[1] / rho;
        double w = v[2] / rho;
        double press = gamma1 * (v[3] - 0.5 * rho * (u * u + w * w));
        const double h = dt2 * 1.0 / rad;
        const double s0 = v[0] - h * v[2];
        const double s1 = v[1] - h * rho * u * w;
        const double s2 = v[2] - h * rho * w * w;
        const double s3 = v[3] - h * w * (v[3] + press);
        rho = s0;
        u = s1 / rho;
        w = s2 / rho;
        press = gamma1 * (s3 - 0.5 * rho * (u * u + w * w));
        const double f = dt * 1.0 / rad;
        v[0] = v[0] - f * s2;
        v[1] = v[1] - f * rho * u * w;
        v[2] = v[2] - f * rho * w * w;
        v[3] = v[3] - f * w * (s3 + press);
    }
}

// QP: row pitch of Qx in doubles (TX unless the body pads its rows).
// fault: the tile could not be computed (its input never arrived): nothing is
// written and the step reports CLAW2_ERR_TIMEOUT (controlled mode) or a NaN
// CFL number.
template <int MEQN, int TX, int TY, int NT, int QP = TX, class Ctx>
CLAW2_HD void finish_tile(const StepArgs& a, Ctx& ctx, const TileId& tile, const double* Qx, int QSTR, double* red,
                          double* qout, int i0, int j0, double cflm, double dt, bool fault = false)
{
    const int tid = ctx.tid();
    int bad = 0;
    // the tile's final values: one unrolled pass of plain stores (the loads
    // of all its cells issue together), then, on tiles within two cells of
    // a side, a second pass writing the ghost cells that are images of them
    constexpr int NIT = (TX * TY + NT - 1) / NT;
    auto cell_value = [&](int ci, int cj, int i, int j, double (&v)[MEQN]) {
#pragma unroll
        for (int m = 0; m < MEQN; m++) v[m] = Qx[m * QSTR + cj * QP + ci];
        if (a.src == CLAW2_SRC_EULER_RADIAL)
            euler_radial_source<MEQN>(v, a.aux[qoff(a, a.src_aux, i, j)], a.prm[1], dt);
    };
    if (!fault) {
#pragma unroll
        for (int k = 0; k < NIT; k++) {
            const int idx = tid + k * NT;
            const int ci = idx % TX, cj = idx / TX;
            const int i = i0 + ci, j = j0 + cj;
            if (idx < TX * TY && i < a.mx && j < a.my) {
                double v[MEQN];
                cell_value(ci, cj, i, j, v);
#pragma unroll
                for (int m = 0; m < MEQN; m++) {
                    if (!isfinite(v[m])) bad = 1;
                    qout[qoff(a, m, i, j)] = v[m];
                }
            }
        }
        const bool edge = i0 <= 1 || i0 + TX >= a.mx - 2 || j0 <= 1 || j0 + TY >= a.my - 2;
        if (a.ghost_fused && edge) {
            for (int idx = tid; idx < TX * TY; idx += NT) {
                const int ci = idx % TX, cj = idx / TX;
                const int i = i0 + ci, j = j0 + cj;
                if (i >= a.mx || j >= a.my) continue;
                if (i > 1 && i < a.mx - 2 && j > 1 && j < a.my - 2) continue;   // no images
                double v[MEQN];
                cell_value(ci, cj, i, j, v);
                write_ghosts<MEQN>(a, qout, i, j, v);
            }
        }
    }

    // ---- block CFL max (deterministic: max is exact) and last-block epilogue:
    // warp max by shuffles, then one value per warp.  CFL numbers are >= 0; a
    // NaN one counts as a non-finite state, and -1 flags a warp that saw one;
    // a tile that could not be computed reports -2.
    {
        const bool nfw = ctx.warp_any(bad != 0 || cflm != cflm);
        const double mw = ctx.warp_max(cflm);
        if ((tid & 31) == 0) red[tid >> 5] = nfw ? -1.0 : mw;
    }
    ctx.sync();
    constexpr int NW = NT / 32;
    if (tid == 0) {
        double mxv = 0.0;
        int nf = 0;
        for (int t = 0; t < NW; t++) {
            if (red[t] < 0.0) nf = 1;
            else mxv = mxv > red[t] ? mxv : red[t];
        }
        a.partials[tile.part] = fault ? -2.0 : (nf ? -1.0 : mxv);
        ctx.fence();
        const unsigned int prev = ctx.atomic_inc(a.ticket);
        red[NW] = prev == (unsigned int)(tile.ntiles - 1) ? 1.0 : 0.0;     // this CTA arrived last
    }
    ctx.sync();
    if (red[NW] != 0.0) {
        // the last CTA reduces every CTA's partial with all its threads
        ctx.fence();
        double cfl = 0.0;
        bool nonfinite = false, lost = false;
        for (int b = tid; b < tile.ntiles; b += NT) {
            const double v = ctx.load_volatile(&a.partials[b]);
            if (v < 0.0) nonfinite = true;
            else cfl = cfl > v ? cfl : v;
            if (v == -2.0) lost = true;
        }
        const bool nfw = ctx.warp_any(nonfinite);
        const bool lw = ctx.warp_any(lost);
        const double mw = ctx.warp_max(cfl);
        if ((tid & 31) == 0) red[tid >> 5] = lw ? -2.0 : (nfw ? -1.0 : mw);
        ctx.sync();
        if (tid == 0) {
            cfl = 0.0;
            int nf = 0;
            for (int t = 0; t < NW; t++) {
                if (red[t] == -2.0) nf = 2;
                else if (red[t] < 0.0 && nf == 0) nf = 1;
                else if (red[t] >= 0.0) cfl = cfl > red[t] ? cfl : red[t];
            }
            if (a.ctrl && !a.ctrl_readonly) control_update(a.ctrl, cfl, nf);
            else if (a.ctrl_readonly) *a.cfl_out = nf ? 1.0 / 0.0 : cfl;
            else *a.cfl_out = nf ? ctx.nan() : cfl;
            *a.ticket = 0u;
            ctx.fence();
        }
    }
}

// f(IntC<0>{}), ..., f(IntC<N-1>{}): a loop whose index is a compile-time constant
template <int N> struct IntC { static constexpr int value = N; };
template <int N, int I = 0, class F>
__device__ __forceinline__ void static_for(F&& f)
{
    if constexpr (I < N) {
        f(IntC<I>{});
        static_for<N, I + 1>(f);
    }
}

// The CFL number of a tile whose whole input halo holds the one state q.
// Every interface of both sweeps then joins two equal states: rpn2a returns
// zero strengths and fluctuations and the speeds of q's Roe average with
// itself, which are the same for every interface of a direction, so the
// lanes' running maxima of dtn*s and -dtn*s are those of one solve per
// direction; the y solve's speeds follow from the x solve's Roe averages
// (RP::speed_other).  `finite` is cleared when a speed is not finite (the
// full tile step then runs, with its own handling of a non-physical state).
// Not inlined: it runs once per tile and stays out of the body's
// instruction stream.
template <class RP>
__device__ __noinline__ double uniform_cfl(const double (&q)[RP::MEQN], const double* prm, double dtdx, double dtdy,
                                           bool& finite)
{
    constexpr int MEQN = RP::MEQN, MW = RP::MW, NROE = RP::NROE;
    double alpha[MW], amdq[MEQN], apdq[MEQN], roe[NROE];
#pragma unroll
    for (int p = 0; p < MW; p++) alpha[p] = 0.0;
#pragma unroll
    for (int r = 0; r < NROE; r++) roe[r] = 0.0;
    const typename RP::Cell L = RP::template cell<1>(q, prm);
    RP::template rpn2a<1>(q, q, L, L, prm, alpha, amdq, apdq, roe);
    double cflm = 0.0;
    static_for<MW>([&](auto P) {
        const double sp = RP::template speed<decltype(P)::value>(roe);
        finite = finite && isfinite(sp);
        const double c1 = dtdx * sp, c2 = -dtdx * sp;
        cflm = cflm > c1 ? cflm : c1;
        cflm = cflm > c2 ? cflm : c2;
    });
    static_for<MW>([&](auto P) {
        const double sp = RP::template speed_other<decltype(P)::value>(roe);
        finite = finite && isfinite(sp);
        const double c1 = dtdy * sp, c2 = -dtdy * sp;
        cflm = cflm > c1 ? cflm : c1;
        cflm = cflm > c2 ? cflm : c2;
    });
    return cflm;
}

template <class RP, int TX, int TY, int NT, bool SPLIT, class Ctx>
CLAW2_HD void step_tile_at(const StepArgs& a, Ctx& ctx, const TileId& tile)
{
    constexpr int MEQN = RP::MEQN;
    constexpr int LPC = NT / 32;
    static_assert(NT % 32 == 0, "NT must be a multiple of 32");
    static_assert(TX + 3 <= 32 && TY + 3 <= 32, "tile too wide for one 32-lane line");
    using SM = TileSmem<RP, TX, TY, NT, SPLIT>;
    constexpr int QROWS = SM::QROWS;
    constexpr int QROW0 = SPLIT ? -2 : 0;
    double* Qx = ctx.smem();
    double* WB = Qx + SM::QX;
    double* B2 = WB + SM::WBSZ * NT;
    double* red = B2 + SM::B2SZ * NT;
    const int tid = ctx.tid();
    const int warp = tid >> 5;
    const int i0 = tile.bx * TX, j0 = tile.by * TY;

    const double* qin = a.qin;
    double* qout = a.qout;
    double dt = a.dt;
    if (a.ctrl) {
        if (a.ctrl->done) return;                  // uniform across the grid
        dt = a.ctrl->dt;
        const int cur = a.ctrl->cur;
        qin = cur ? a.q1 : a.q0;
        qout = cur ? a.q0 : a.q1;
    }
    const double dtdx = dt / a.dx, dtdy = dt / a.dy;
    double cflm = 0.0;

    // ---- x sweeps: unsplit slices j0-1..j0+TY (rows -1..my); split rows j0-2..j0+TY+1
    {
        const int nlines = SPLIT ? TY + 4 : TY + 2;
        const int first = SPLIT ? j0 - 2 : j0 - 1;
        const int hi = SPLIT ? a.my + 1 : a.my;
        const int last = (first + nlines - 1 < hi) ? first + nlines - 1 : hi;
        for (int c0 = first; c0 <= last; c0 += LPC) {
            const int line = c0 + warp;
            const int clast = (c0 + LPC - 1 < last) ? c0 + LPC - 1 : last;
            sweep_chunk<RP, 1, SPLIT, TX, TY, NT>(a, ctx, qin, Qx, WB, B2, i0, j0, line, c0, clast,
                                                  line <= last, false, dtdx, dtdy, cflm);
            // split: a line reads and writes only its own row of Qx and its own
            // warp's slots of WB/B2, so chunks need no block barrier, only a
            // warp barrier before the next chunk reuses the slots
            if (SPLIT) ctx.syncwarp();
        }
        if (SPLIT) ctx.sync();          // the y sweep reads the whole x-swept tile
    }
    // ---- y sweeps: unsplit columns i0-1..i0+TX (cols -1..mx); split the tile's
    //      columns, plus ghost columns -2,-1 / mx,mx+1 (CFL only, step2ds.f90:177)
    {
        const bool left = i0 == 0, right = i0 + TX >= a.mx;
        const int ninner = SPLIT ? (a.mx - i0 < TX ? a.mx - i0 : TX) : 0;
        if (!SPLIT) {
            const int first = i0 - 1;
            const int last = (i0 + TX < a.mx) ? i0 + TX : a.mx;
            for (int c0 = first; c0 <= last; c0 += LPC) {
                const int line = c0 + warp;
                const int clast = (c0 + LPC - 1 < last) ? c0 + LPC - 1 : last;
                sweep_chunk<RP, 2, SPLIT, TX, TY, NT>(a, ctx, qin, Qx, WB, B2, i0, j0, line, c0, clast,
                                                      line <= last, false, dtdy, dtdx, cflm);
            }
        } else {
            const int nlines = ninner + (left ? 2 : 0) + (right ? 2 : 0);
            for (int c0 = 0; c0 < nlines; c0 += LPC) {
                const int l = c0 + warp;
                int line;
                bool cflonly = false;
                if (left && l < 2) { line = l - 2; cflonly = true; }
                else {
                    const int r = l - (left ? 2 : 0);
                    if (r < ninner) line = i0 + r;
                    else { line = a.mx + (r - ninner); cflonly = true; }
                }
                sweep_chunk<RP, 2, SPLIT, TX, TY, NT>(a, ctx, qin, Qx, WB, B2, i0, j0, line, 0, 0,
                                                      l < nlines, cflonly, dtdy, dtdx, cflm);
                ctx.syncwarp();         // a y line touches only its own column of Qx
            }
            ctx.sync();
        }
    }

    finish_tile<MEQN, TX, TY, NT, SM::QP>(a, ctx, tile, Qx + (-QROW0) * SM::QP, QROWS * SM::QP, red, qout, i0, j0,
                                         cflm, dt);
}

template <class RP, int TX, int TY, int NT, bool SPLIT, class Ctx>
CLAW2_HD void step_tile(const StepArgs& a, Ctx& ctx)
{
    const TileId t{ctx.bx(), ctx.by(), ctx.nbx(), ctx.nby(), ctx.by() * ctx.nbx() + ctx.bx(), ctx.nbx() * ctx.nby()};
    step_tile_at<RP, TX, TY, NT, SPLIT>(a, ctx, t);
}

#if defined(__CUDACC__)
// ---------------------------------------------------------------------------
// device execution context for step_tile (CUDA builds)
// ---------------------------------------------------------------------------
struct DevCtx {
    double* sm;
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ int bx() const { return blockIdx.x; }
    __device__ __forceinline__ int by() const { return blockIdx.y; }
    __device__ __forceinline__ int nbx() const { return gridDim.x; }
    __device__ __forceinline__ int nby() const { return gridDim.y; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ void syncwarp() const { __syncwarp(); }
    __device__ __forceinline__ void fence() const { __threadfence(); }
    __device__ __forceinline__ unsigned atomic_inc(unsigned* p) const { return atomicAdd(p, 1u); }
    __device__ __forceinline__ double load_volatile(const double* p) const { return *(volatile const double*)p; }
    __device__ __forceinline__ double nan() const { return __longlong_as_double(0x7ff8000000000000ULL); }
    __device__ __forceinline__ double* smem() const { return sm; }
    // value of the lane below / above in the warp (own value at the ends)
    __device__ __forceinline__ double shfl_up(double v) const { return __shfl_up_sync(0xffffffffu, v, 1); }
    __device__ __forceinline__ double shfl_down(double v) const { return __shfl_down_sync(0xffffffffu, v, 1); }
    // max over the warp (all lanes get it) and any-lane predicate
    __device__ __forceinline__ double warp_max(double v) const
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, v, o);
            v = v > w ? v : w;
        }
        return v;
    }
    __device__ __forceinline__ bool warp_any(bool p) const { return __any_sync(0xffffffffu, p) != 0; }
    __device__ __forceinline__ void prefetch_l2(const void* p) const { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
};
#endif

}  // namespace claw2
