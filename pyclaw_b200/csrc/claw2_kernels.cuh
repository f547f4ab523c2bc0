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
};

template <int IXY> struct Phase;

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
    if (nonfinite) {
        c->error = CLAW2_ERR_NONFINITE;
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

// Write one final cell value and all ghost cells that are images of it.
template <int MEQN>
CLAW2_HD void write_cell(const StepArgs& a, double* qo, int i, int j, const double (&v)[MEQN])
{
#pragma unroll
    for (int m = 0; m < MEQN; m++) qo[qoff(a, m, i, j)] = v[m];
    if (!a.ghost_fused) return;
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
template <class RP, int TX, int TY, int NT, bool SPLIT> struct TileSmem {
    static constexpr int MEQN = RP::MEQN, MW = RP::MW;
    static constexpr int QROWS = SPLIT ? TY + 4 : TY;
    static constexpr int IFSZ = CMax<MW * MEQN + MW, 4 * MEQN>::value;
    static constexpr int QX = MEQN * QROWS * TX;
    static constexpr int total = QX + IFSZ * NT + NT;      // + reduction scratch
    static constexpr int bytes = total * 8;
};

// ---------------------------------------------------------------------------
// One chunk of one sweep direction.  IXY = 1: lines are x slices (rows), the
// interface index runs along x; IXY = 2: lines are y slices (columns).
//   line : slice index (0-based; row for IXY=1, column for IXY=2)
//   k    : interface between cells k-1 and k along the slice
// Mode: SPLIT = dimensional splitting (no transverse terms, one update pass).
// ---------------------------------------------------------------------------
template <class RP, int IXY, bool SPLIT, int TX, int TY, int NT, class Ctx>
CLAW2_HD void sweep_chunk(const StepArgs& a, Ctx& ctx, const double* qin, double* Qx, double* IFB,
                          int i0, int j0, int line, bool lineok, bool cflonly, int slot, int delta,
                          int nslots, double dtn, double dtt, double& cflm)
{
    constexpr int MEQN = RP::MEQN, MW = RP::MW, MAUX = RP::MAUX, NROE = RP::NROE;
    constexpr int QROWS = SPLIT ? TY + 4 : TY;
    constexpr int QROW0 = SPLIT ? -2 : 0;      // tile row of Qx row 0, relative to j0
    constexpr int AUXN = MAUX > 0 ? MAUX : 1;
    const int tid = ctx.tid();
    const int len = IXY == 1 ? a.mx : a.my;
    const int s0 = (IXY == 1 ? i0 : j0) - 1;   // first interface of the line
    const int k = s0 + slot;
    const bool ifok = lineok && slot < nslots && k <= len + 1;
    // interfaces whose fluxes the tile uses: slots 1..nslots-2
    const bool lim = ifok && !cflonly && slot >= 1 && slot <= nslots - 2 && k >= 0 && k <= len;
    const bool cflok = ifok && slot >= 1 && slot <= nslots - 2 && k >= 0 && k <= len;

    auto cell_i = [&](int kk) { return IXY == 1 ? kk : line; };
    auto cell_j = [&](int kk) { return IXY == 1 ? line : kk; };

    double wave[MW][MEQN], s[MW], amdq[MEQN], apdq[MEQN], roe[NROE];
    double dtl = dtn, dtr = dtn;
    // ---------------- S1: normal Riemann solve ----------------
    if (ifok) {
        double qL[MEQN], qR[MEQN], auxL[AUXN], auxR[AUXN];
        const int iL = cell_i(k - 1), jL = cell_j(k - 1), iR = cell_i(k), jR = cell_j(k);
        if (SPLIT && IXY == 2 && !cflonly) {
            // y sweep of the split step reads the x-swept tile state
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                qL[m] = Qx[(m * QROWS + (jL - j0 - QROW0)) * TX + (iL - i0)];
                qR[m] = Qx[(m * QROWS + (jR - j0 - QROW0)) * TX + (iR - i0)];
            }
        } else {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                qL[m] = qin[qoff(a, m, iL, jL)];
                qR[m] = qin[qoff(a, m, iR, jR)];
            }
        }
#pragma unroll
        for (int m = 0; m < MAUX; m++) {
            auxL[m] = a.aux[qoff(a, m, iL, jL)];
            auxR[m] = a.aux[qoff(a, m, iR, jR)];
        }
        if (a.capa >= 0) {
            dtl = dtn / a.aux[qoff(a, a.capa, iL, jL)];
            dtr = dtn / a.aux[qoff(a, a.capa, iR, jR)];
        }
        RP::template rpn2<IXY>(qL, qR, auxL, auxR, a.prm, wave, s, amdq, apdq, roe);
#pragma unroll
        for (int p = 0; p < MW; p++) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) IFB[(p * MEQN + m) * NT + tid] = wave[p][m];
            IFB[(MW * MEQN + p) * NT + tid] = s[p];
        }
    }
    ctx.sync();

    // ---------------- S2: CFL, limiter, corrections, transverse ----------------
    double fadd[MEQN], bmL[MEQN], bpL[MEQN], bmR[MEQN], bpR[MEQN];
#pragma unroll
    for (int m = 0; m < MEQN; m++) { fadd[m] = 0.0; bmL[m] = 0.0; bpL[m] = 0.0; bmR[m] = 0.0; bpR[m] = 0.0; }
    if (cflok) {
#pragma unroll
        for (int p = 0; p < MW; p++) {
            const double c1 = dtr * s[p], c2 = -dtl * s[p];
            cflm = cflm > c1 ? cflm : c1;
            cflm = cflm > c2 ? cflm : c2;
        }
    }
    if (lim) {
        double cqxx[MEQN];
        if (a.order == 2) {
            if (a.limit_any) {
#pragma unroll
                for (int p = 0; p < MW; p++) {
                    const int meth = a.mthlim[p];
                    if (meth == 0) continue;
                    double wnorm2 = 0.0;
#pragma unroll
                    for (int m = 0; m < MEQN; m++) wnorm2 = wnorm2 + wave[p][m] * wave[p][m];
                    if (wnorm2 == 0.0) continue;
                    // dotl = wave(k-1).wave(k) when s > 0, else dotr = wave(k).wave(k+1)
                    const int nb = s[p] > 0.0 ? tid - delta : tid + delta;
                    double dot = 0.0;
#pragma unroll
                    for (int m = 0; m < MEQN; m++) dot = dot + wave[p][m] * IFB[(p * MEQN + m) * NT + nb];
                    const double phi = philim(wnorm2, dot, meth);
#pragma unroll
                    for (int m = 0; m < MEQN; m++) wave[p][m] = phi * wave[p][m];
                }
            }
            const double dtdxave = 0.5 * (dtl + dtr);
            double f[MW];
#pragma unroll
            for (int p = 0; p < MW; p++) {
                const double as = fabs(s[p]);
                f[p] = (a.fwave ? copysign(1.0, s[p]) : as) * (1.0 - as * dtdxave);
            }
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                double c = 0.0;
#pragma unroll
                for (int p = 0; p < MW; p++) c = c + f[p] * wave[p][m];
                cqxx[m] = c;
                fadd[m] = 0.5 * c;
            }
        } else {
#pragma unroll
            for (int m = 0; m < MEQN; m++) cqxx[m] = 0.0;
        }
        if (!SPLIT && a.trans > 0) {
            double A[MEQN], P[MEQN];
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                if (a.order == 2 && a.trans == 2) { A[m] = amdq[m] + cqxx[m]; P[m] = apdq[m] - cqxx[m]; }
                else { A[m] = amdq[m]; P[m] = apdq[m]; }
            }
            double ax1[AUXN], ax2[AUXN], ax3[AUXN];
            // ilr = 1: the left-going fluctuation sits in cell k-1
            {
                const int ci = cell_i(k - 1), cj = cell_j(k - 1);
#pragma unroll
                for (int m = 0; m < MAUX; m++) {
                    ax1[m] = a.aux[qoff(a, m, IXY == 1 ? ci : ci - 1, IXY == 1 ? cj - 1 : cj)];
                    ax2[m] = a.aux[qoff(a, m, ci, cj)];
                    ax3[m] = a.aux[qoff(a, m, IXY == 1 ? ci : ci + 1, IXY == 1 ? cj + 1 : cj)];
                }
                RP::template rpt2<IXY>(1, A, roe, ax1, ax2, ax3, a.prm, bmL, bpL);
            }
            // ilr = 2: the right-going fluctuation sits in cell k
            {
                const int ci = cell_i(k), cj = cell_j(k);
#pragma unroll
                for (int m = 0; m < MAUX; m++) {
                    ax1[m] = a.aux[qoff(a, m, IXY == 1 ? ci : ci - 1, IXY == 1 ? cj - 1 : cj)];
                    ax2[m] = a.aux[qoff(a, m, ci, cj)];
                    ax3[m] = a.aux[qoff(a, m, IXY == 1 ? ci : ci + 1, IXY == 1 ? cj + 1 : cj)];
                }
                RP::template rpt2<IXY>(2, P, roe, ax1, ax2, ax3, a.prm, bmR, bpR);
            }
        }
    }
    ctx.sync();
    // ---------------- S2b: publish what the cell left of the interface needs -------
    if (lim) {
        const double hl = 0.5 * dtl;
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            IFB[(0 * MEQN + m) * NT + tid] = dtl * amdq[m];
            IFB[(1 * MEQN + m) * NT + tid] = fadd[m];
            IFB[(2 * MEQN + m) * NT + tid] = hl * bmL[m];
            IFB[(3 * MEQN + m) * NT + tid] = hl * bpL[m];
        }
    }
    ctx.sync();

    // ---------------- S3: per-cell increments, applied in reference order --------
    // this thread's cell is k (right of its interface); slots 1..nslots-3
    const int ncell = (IXY == 1 ? TX : TY);
    const bool cellok = lim && slot <= ncell && k < len;
    double qadd[MEQN], dF[MEQN], g1[MEQN], g2[MEQN];
    if (cellok) {
        const double hr = 0.5 * dtr;
        const int nb = tid + delta;
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            qadd[m] = (0.0 - dtr * apdq[m]) - IFB[(0 * MEQN + m) * NT + nb];
            dF[m] = IFB[(1 * MEQN + m) * NT + nb] - fadd[m];
            g1[m] = (0.0 - IFB[(2 * MEQN + m) * NT + nb]) - hr * bmR[m];
            g2[m] = (0.0 - IFB[(3 * MEQN + m) * NT + nb]) - hr * bpR[m];
        }
    }
    const bool trans = !SPLIT && a.trans > 0;
    // tile-cell test for a cell (kk along the slice, ll = line)
    auto in_tile = [&](int kk, int ll) {
        const int ci = IXY == 1 ? kk : ll, cj = IXY == 1 ? ll : kk;
        return ci >= i0 && ci < i0 + TX && ci < a.mx && cj >= j0 + QROW0 && cj < j0 + QROW0 + QROWS && cj < a.my + (SPLIT ? 2 : 0);
    };
    auto qx = [&](int m, int kk, int ll) -> double& {
        const int ci = IXY == 1 ? kk : ll, cj = IXY == 1 ? ll : kk;
        return Qx[(m * QROWS + (cj - j0 - QROW0)) * TX + (ci - i0)];
    };
    auto capa_of = [&](int kk, int ll) {
        return a.aux[qoff(a, a.capa, IXY == 1 ? kk : ll, IXY == 1 ? ll : kk)];
    };
    if (SPLIT) {
        if (cellok && in_tile(k, line)) {
#pragma unroll
            for (int m = 0; m < MEQN; m++) {
                const double q0 = IXY == 1 ? qin[qoff(a, m, k, line)] : qx(m, k, line);
                if (a.capa < 0) qx(m, k, line) = q0 + qadd[m] - dtn * dF[m];
                else qx(m, k, line) = q0 + qadd[m] - dtn * dF[m] / capa_of(k, line);
            }
        }
        ctx.sync();
        return;
    }
    // pass a: contribution of this slice to the slice above (first for x: initialise)
    if (cellok && in_tile(k, line + 1)) {
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            const double q0 = IXY == 1 ? qin[qoff(a, m, k, line + 1)] : qx(m, k, line + 1);
            if (!trans) qx(m, k, line + 1) = q0;
            else if (a.capa < 0) qx(m, k, line + 1) = q0 + dtt * g2[m];
            else qx(m, k, line + 1) = q0 + dtt * g2[m] / capa_of(k, line + 1);
        }
    }
    ctx.sync();
    // pass b: the slice's own cells
    if (cellok && in_tile(k, line)) {
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            double& q = qx(m, k, line);
            if (a.capa >= 0) {
                const double tt = trans ? dtt * (g2[m] - g1[m]) : 0.0;
                q = q + qadd[m] - (dtn * dF[m] + tt) / capa_of(k, line);
            } else if (IXY == 1) {
                q = q + qadd[m] - dtn * dF[m];
                if (trans) q = q - dtt * (g2[m] - g1[m]);
            } else {
                q = q + (trans ? (qadd[m] - dtn * dF[m] - dtt * (g2[m] - g1[m])) : (qadd[m] - dtn * dF[m]));
            }
        }
    }
    ctx.sync();
    // pass c: contribution to the slice below
    if (trans && cellok && in_tile(k, line - 1)) {
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            double& q = qx(m, k, line - 1);
            if (a.capa < 0) q = q - dtt * g1[m];
            else q = q - dtt * g1[m] / capa_of(k, line - 1);
        }
    }
    ctx.sync();
}

// ---------------------------------------------------------------------------
// Whole-tile step.  Lines per chunk LPC = NT/32; a line holds up to 32
// interfaces (TX+3 <= 32 and TY+3 <= 32).
// ---------------------------------------------------------------------------
template <class RP, int TX, int TY, int NT, bool SPLIT, class Ctx>
CLAW2_HD void step_tile(const StepArgs& a, Ctx& ctx)
{
    constexpr int MEQN = RP::MEQN;
    constexpr int SW = 32, LPC = NT / SW;
    static_assert(NT % SW == 0, "NT must be a multiple of 32");
    static_assert(TX + 3 <= SW && TY + 3 <= SW, "tile too wide for one 32-slot line");
    using SM = TileSmem<RP, TX, TY, NT, SPLIT>;
    constexpr int QROWS = SM::QROWS;
    constexpr int QROW0 = SPLIT ? -2 : 0;
    double* Qx = ctx.smem();
    double* IFB = Qx + SM::QX;
    double* red = IFB + SM::IFSZ * NT;
    const int tid = ctx.tid();
    const int i0 = ctx.bx() * TX, j0 = ctx.by() * TY;

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
        const int lo = SPLIT ? -2 : -1, hi = SPLIT ? a.my + 1 : a.my;
        for (int c0 = 0; c0 < nlines; c0 += LPC) {
            const int li = tid / SW, slot = tid % SW;
            const int line = first + c0 + li;
            const bool lineok = (c0 + li < nlines) && line >= lo && line <= hi;
            sweep_chunk<RP, 1, SPLIT, TX, TY, NT>(a, ctx, qin, Qx, IFB, i0, j0, line, lineok, false,
                                                  slot, 1, TX + 3, dtdx, dtdy, cflm);
        }
    }
    // ---- y sweeps: unsplit columns i0-1..i0+TX (cols -1..mx); split the tile's
    //      columns, plus ghost columns -2,-1 / mx,mx+1 (CFL only, step2ds.f90:177)
    {
        const bool left = i0 == 0, right = i0 + TX >= a.mx;
        const int ninner = SPLIT ? (a.mx - i0 < TX ? a.mx - i0 : TX) : TX + 2;
        const int nlines = SPLIT ? ninner + (left ? 2 : 0) + (right ? 2 : 0) : TX + 2;
        for (int c0 = 0; c0 < nlines; c0 += LPC) {
            const int li = tid % LPC, slot = tid / LPC;
            const int l = c0 + li;
            int line;
            bool cflonly = false;
            if (!SPLIT) line = i0 - 1 + l;
            else if (left && l < 2) { line = l - 2; cflonly = true; }
            else {
                const int r = l - (left ? 2 : 0);
                if (r < ninner) line = i0 + r;
                else { line = a.mx + (r - ninner); cflonly = true; }
            }
            const bool lineok = l < nlines && line >= (SPLIT ? -2 : -1) && line <= (SPLIT ? a.mx + 1 : a.mx);
            sweep_chunk<RP, 2, SPLIT, TX, TY, NT>(a, ctx, qin, Qx, IFB, i0, j0, line, lineok, cflonly,
                                                  slot, LPC, TY + 3, dtdy, dtdx, cflm);
        }
    }

    // ---- final values of the tile's cells and their ghost images
    int bad = 0;
    for (int idx = tid; idx < TX * TY; idx += NT) {
        const int ci = idx % TX, cj = idx / TX;
        const int i = i0 + ci, j = j0 + cj;
        if (i >= a.mx || j >= a.my) continue;
        double v[MEQN];
#pragma unroll
        for (int m = 0; m < MEQN; m++) {
            v[m] = Qx[(m * QROWS + (cj - QROW0)) * TX + ci];
            if (!isfinite(v[m])) bad = 1;
        }
        write_cell<MEQN>(a, qout, i, j, v);
    }

    // ---- block CFL max (deterministic: max is exact) and last-block epilogue
    red[tid] = bad ? -1.0 : cflm;        // CFL numbers are >= 0; -1 flags a non-finite cell
    ctx.sync();
    if (tid == 0) {
        double mxv = 0.0;
        int nf = 0;
        for (int t = 0; t < NT; t++) {
            if (red[t] < 0.0) nf = 1;
            else mxv = mxv > red[t] ? mxv : red[t];
        }
        const int nblocks = ctx.nbx() * ctx.nby();
        const int bid = ctx.by() * ctx.nbx() + ctx.bx();
        a.partials[bid] = nf ? -1.0 : mxv;
        ctx.fence();
        const unsigned int prev = ctx.atomic_inc(a.ticket);
        if (prev == (unsigned int)(nblocks - 1)) {
            ctx.fence();
            double cfl = 0.0;
            int nonfinite = 0;
            for (int b = 0; b < nblocks; b++) {
                const double v = ctx.load_volatile(&a.partials[b]);
                if (v < 0.0) nonfinite = 1;
                else cfl = cfl > v ? cfl : v;
            }
            if (a.ctrl) control_update(a.ctrl, cfl, nonfinite);
            else *a.cfl_out = nonfinite ? ctx.nan() : cfl;
            *a.ticket = 0u;
            ctx.fence();
        }
    }
}

}  // namespace claw2
