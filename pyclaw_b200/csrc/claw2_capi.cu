// claw2_capi.cu -- CUDA kernels and the extern "C" ABI declared in include/claw2.h.
//
// Built for sm_100a with --fmad=false (no FMA contraction, so the step
// reproduces the reference's operation-by-operation rounding).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>

#define CLAW2_EXPORT __attribute__((visibility("default")))
#include "../../include/claw2.h"
#include "claw2_devattr.h"
#include "claw2_kernels.cuh"
#include "claw2_light.cuh"
#include "claw2_lean.cuh"

namespace claw2 {

#ifndef CLAW2_MINB
#define CLAW2_MINB 2        // resident CTAs per SM the register budget is sized for
#endif

// Chained steps (launch_step with chained set): once every CTA of this step
// has started, the next step's CTAs may start on the SMs this step frees;
// each waits here until the step before it has completed and its writes are
// visible.  In a kernel launched without the attribute both instructions
// return at once.
__device__ __forceinline__ void chain_wait()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launch kern, as a programmatic dependent of the previous kernel in the
// stream when chained is set (the kernel calls chain_wait before it reads
// anything).
template <class... KArgs, class... Args>
int launch_kernel(void (*kern)(KArgs...), dim3 grid, int threads, int smem, cudaStream_t st, bool chained,
                  Args... args)
{
    if (!chained) {
        kern<<<grid, threads, smem, st>>>(args...);
        return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...) == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

template <class RP, int TX, int TY, int NT, bool SPLIT>
__global__ void __launch_bounds__(NT, CLAW2_MINB) step_kernel(StepArgs a)
{
    chain_wait();
    extern __shared__ double smem_dyn[];
    DevCtx ctx{smem_dyn};
    step_tile<RP, TX, TY, NT, SPLIT>(a, ctx);
}

// The two-wave acoustics solvers have a leaner unsplit body (claw2_light.cuh)
// that needs fewer registers and less shared memory, so more CTAs fit per SM.
template <class RP> struct HasLight { static constexpr bool value = false; };
template <> struct HasLight<RpAcoustics> { static constexpr bool value = true; };
template <> struct HasLight<RpVcAcoustics> { static constexpr bool value = true; };

#ifndef CLAW2_LIGHT_MINB
#define CLAW2_LIGHT_MINB 3
#endif

// Grids with fewer 29x29 tiles than a B200 has SMs leave most of the GPU idle
// for the whole step; they run the light body on 13x13 tiles instead (4 to 5
// times the CTAs; a line still has 32 lanes, of which 16 are used).
constexpr int LIGHT_SMALL_TILE = 13, LIGHT_SMALL_GRID_TILES = 148;

CLAW2_HD bool light_small_grid(int mx, int my)
{
    return (long long)((mx + 28) / 29) * (long long)((my + 28) / 29) < LIGHT_SMALL_GRID_TILES;
}

template <class RP, int T>
__global__ void __launch_bounds__(256, CLAW2_LIGHT_MINB) light_step_kernel(StepArgs a)
{
    chain_wait();
    extern __shared__ double smem_dyn[];
    DevCtx ctx{smem_dyn};
    const TileId t{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x, (int)gridDim.y,
                   (int)(blockIdx.y * gridDim.x + blockIdx.x), (int)(gridDim.x * gridDim.y)};
    light_tile_at<RP, T, T, 256>(a, ctx, t);
}

// The dense-wave solvers without aux arrays (Euler, shallow water) have the
// same data movement in a lean unsplit body (claw2_lean.cuh): shuffles
// instead of shared-memory exchange, one block barrier per chunk.
template <class RP> struct HasLean { static constexpr bool value = false; };
template <> struct HasLean<RpEuler<false>> { static constexpr bool value = true; };
template <> struct HasLean<RpEuler<true>> { static constexpr bool value = true; };
template <> struct HasLean<RpShallow> { static constexpr bool value = true; };

// lean tiles: 28 x 28 cells, so that a line's 32 lanes hold its 32 cells.
// Two block sizes, one line of a chunk per warp: 512 threads (one CTA per SM,
// 16 lines per chunk) halve a tile's latency, which decides the step when the
// grid has few tiles per SM (a launch of a few waves ends with a partial
// one); 256 threads (two CTAs per SM) let one CTA's waits (its halo copy, its
// barriers, the launch of the next CTA) overlap the other's work, which
// decides it when the grid has many tiles, most of them cheap.
constexpr int LTX = 28, LTY = 28;
constexpr int LEAN_BIG_BLOCK_TILES = 8 * 148;   // grids of at most 8 tiles per SM of a B200 use 512 threads

// tm0 / tm1: tensor maps of the input state (see lean_tile_at), passed as
// __grid_constant__ parameters so the TMA unit can read them in place.
template <class RP, int NT>
__global__ void __launch_bounds__(NT, 512 / NT)
lean_step_kernel(StepArgs a, const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1)
{
    extern __shared__ double smem_dyn[];
    __shared__ __align__(8) uint64_t halo_bar;
    chain_wait();
    DevCtx ctx{smem_dyn};
    const TileId t{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x, (int)gridDim.y,
                   (int)(blockIdx.y * gridDim.x + blockIdx.x), (int)(gridDim.x * gridDim.y)};
    lean_tile_at<RP, LTX, LTY, NT>(a, ctx, t, &tm0, &tm1, &halo_bar);
}

// Instance of tile t: the last one with tile_begin <= t (binary search).
// With tb (the instances' tile_begin copied into shared memory by the
// kernel) the search reads shared memory instead of walking the descriptors
// in global memory, a chain of dependent L2 loads per tile.
__device__ __forceinline__ int batch_instance_of(const claw2_batch_instance* __restrict__ inst, int ninst, int t,
                                                 const int* tb = nullptr)
{
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((tb ? tb[mid] : __ldg(&inst[mid].tile_begin)) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// batches of at most this many instances keep their tile_begin table in
// shared memory (4 bytes each)
constexpr int kBatchTableMax = 4096;

// Instance of tile t + 1 given k, the instance of tile t: tile_begin is
// non-decreasing, so it is the last instance at or after k whose tile_begin is
// <= t + 1 (the same one or, crossing an instance's last tile, the next one
// with tiles).
__device__ __forceinline__ int batch_instance_after(const claw2_batch_instance* __restrict__ inst, int ninst, int k,
                                                    int t, const int* tb)
{
    while (k + 1 < ninst && (tb ? tb[k + 1] : __ldg(&inst[k + 1].tile_begin)) <= t + 1) k++;
    return k;
}

// Ask L2 for the input halo of tile t (instance k; rows j0-2..j0+TY+1 and
// columns i0-2..i0+TX+1, clipped to the ghosted arrays, of the current state
// and of aux) while the CTA works on the tile before it: an instance's data is
// read once per step, from HBM, so the tile's first loads would otherwise wait
// for DRAM.  One prefetch per 128-byte line, spread over the CTA's threads.
// The addresses stay inside the instance's arrays; results do not depend on
// it.
template <int MEQN, int MAUX, int TX, int TY, int NT>
__device__ __forceinline__ void batch_prefetch_tile(const claw2_batch_instance* __restrict__ inst, int k, int t)
{
    const claw2_batch_instance& I = inst[k];
    const claw2_control* c = I.ctrl;
    if (c->done) return;
    const double* q = c->cur ? I.q1 : I.q0;
    const int lt = t - I.tile_begin;
    const int i0 = (lt % I.nbx) * TX, j0 = (lt / I.nbx) * TY;
    const int rlo = j0 - 2, rhi = (j0 + TY + 1 < I.my + 1) ? j0 + TY + 1 : I.my + 1;
    const int clo = i0 - 2, chi = (i0 + TX + 1 < I.mx + 1) ? i0 + TX + 1 : I.mx + 1;
    // byte range of one row segment, in whole 128-byte lines
    const long long b0 = (long long)(clo + CLAW2_NUM_GHOST) * 8, b1 = (long long)(chi + CLAW2_NUM_GHOST) * 8 + 8;
    const int l0 = (int)(b0 >> 7), nl = (int)((b1 + 127) >> 7) - l0;
    const int nrow = rhi - rlo + 1;
    // one (field, row) per thread, its 128-byte lines in turn
    for (int rf = threadIdx.x; rf < (MEQN + MAUX) * nrow; rf += NT) {
        const int r = rf % nrow, f = rf / nrow;
        const char* base = f < MEQN ? (const char*)(q + f * I.plane) : (const char*)(I.aux + (f - MEQN) * I.plane);
        const char* row = base + (long long)(rlo + r + CLAW2_NUM_GHOST) * I.ld * 8 + ((long long)l0 << 7);
        for (int line = 0; line < nl; line++) asm volatile("prefetch.global.L2 [%0];" ::"l"(row + (line << 7)));
    }
}

// Batched step: a persistent grid walks the concatenated tile list of all
// instances; each tile (T x T cells) is one tile-body call with that
// instance's buffers, with an L2 prefetch of the CTA's next tile issued first.
// body_doubles: the tile body's shared memory; with `table` set the
// instances' tile_begin table follows it.
template <class RP, int NT, int MINB, bool LIGHT, int T>
__global__ void __launch_bounds__(NT, MINB)
batch_kernel(const claw2_batch_instance* __restrict__ inst, int ninst, int ntiles, StepArgs common, int body_doubles,
             int table)
{
    static_assert(LIGHT || T == 29, "the generic body runs 29x29 tiles in the batch");
    extern __shared__ double smem_dyn[];
    DevCtx ctx{smem_dyn};
    int* tb = nullptr;
    if (table) {
        tb = reinterpret_cast<int*>(smem_dyn + body_doubles);
        for (int i = threadIdx.x; i < ninst; i += NT) tb[i] = __ldg(&inst[i].tile_begin);
        __syncthreads();
    }
    // each CTA takes a contiguous run of tiles: consecutive tiles mostly
    // belong to the same instance (its descriptor and controller stay in L1)
    // and share halo lines with the tile before them
    const int tbeg = (int)((long long)ntiles * blockIdx.x / gridDim.x);
    const int tend = (int)((long long)ntiles * (blockIdx.x + 1) / gridDim.x);
    // the run's first instance by binary search, then one step at a time
    int lo = tbeg < tend ? batch_instance_of(inst, ninst, tbeg, tb) : 0;
    for (int t = tbeg; t < tend; t++) {
        const int nxt = t + 1 < tend ? batch_instance_after(inst, ninst, lo, t, tb) : lo;
        if (t + 1 < tend) batch_prefetch_tile<RP::MEQN, RP::MAUX, T, T, NT>(inst, nxt, t + 1);
        const claw2_batch_instance& I = inst[lo];
        StepArgs a = common;
        a.q0 = I.q0; a.q1 = I.q1; a.aux = I.aux; a.ctrl = I.ctrl;
        a.partials = I.partials; a.ticket = I.ticket;
        a.ld = I.ld; a.plane = I.plane; a.mx = I.mx; a.my = I.my; a.dx = I.dx; a.dy = I.dy;
        a.ghost_fused = (I.mx >= 4 && I.my >= 4) ? common.ghost_fused : 0;
        const int lt = t - I.tile_begin;
        const TileId tile{lt % I.nbx, lt / I.nbx, I.nbx, I.nby, lt, I.nbx * I.nby};
        if constexpr (LIGHT) light_tile_at<RP, T, T, NT>(a, ctx, tile);
        else step_tile_at<RP, 29, 29, NT, false>(a, ctx, tile);
        __syncthreads();                            // shared memory is reused by the next tile
        lo = nxt;
    }
}

// Batched step with one CTA per tile (grid = all tiles of all instances):
// the hardware hands tiles to SMs as slots free up, so uneven tiles balance
// themselves, and no loop state stays live across the tile body.  The tile's
// instance comes from the caller's tile -> instance map when there is one,
// else from a binary search over the descriptors (a chain of dependent L2
// loads at the CTA's start); there is no L2 prefetch of a next tile, the
// other resident CTAs cover the first loads.
template <class RP, int NT, int MINB, bool LIGHT, int T>
__global__ void __launch_bounds__(NT, MINB)
batch_tile_kernel(const claw2_batch_instance* __restrict__ inst, int ninst, StepArgs common,
                  const int32_t* __restrict__ tile_inst)
{
    static_assert(LIGHT || T == 29, "the generic body runs 29x29 tiles in the batch");
    extern __shared__ double smem_dyn[];
    DevCtx ctx{smem_dyn};
    const int t = (int)blockIdx.x;
    int k = tile_inst ? __ldg(&tile_inst[t]) : -1;  // the caller's map: one load
    if (k < 0 || k >= ninst || t < inst[k].tile_begin || t - inst[k].tile_begin >= inst[k].nbx * inst[k].nby)
        k = batch_instance_of(inst, ninst, t);      // no map, or an entry that does not hold tile t
    const claw2_batch_instance& I = inst[k];
    StepArgs a = common;
    a.q0 = I.q0; a.q1 = I.q1; a.aux = I.aux; a.ctrl = I.ctrl;
    a.partials = I.partials; a.ticket = I.ticket;
    a.ld = I.ld; a.plane = I.plane; a.mx = I.mx; a.my = I.my; a.dx = I.dx; a.dy = I.dy;
    a.ghost_fused = (I.mx >= 4 && I.my >= 4) ? common.ghost_fused : 0;
    const int lt = t - I.tile_begin;
    const TileId tile{lt % I.nbx, lt / I.nbx, I.nbx, I.nby, lt, I.nbx * I.nby};
    if constexpr (LIGHT) light_tile_at<RP, T, T, NT>(a, ctx, tile);
    else step_tile_at<RP, 29, 29, NT, false>(a, ctx, tile);
}

// Tile shapes: a line of a chunk has 32 interface slots, so TX+3, TY+3 <= 32.
#ifndef CLAW2_UNT
#define CLAW2_UNT 256
#endif
constexpr int UTX = 29, UTY = 29, UNT = CLAW2_UNT;   // unsplit
constexpr int STX = 28, STY = 28, SNT = 256;   // dimensional splitting

// ---------------------------------------------------------------------------
// ghost fill (device layout): Solver.apply_q_bcs, x sides then y sides
// ---------------------------------------------------------------------------
struct FillArgs {
    double* q;
    long long ld, plane;
    int mx, my, ncomp;
    int bl, bu;        // this axis' lower/upper BC
    int negate;        // 0-based component negated at walls (-1 none)
};

// axis 0 fills ghost columns over all rows (incl. ghost rows); axis 1 fills ghost
// rows over all columns.  One thread per (component, position along the other
// axis, ghost layer, side).
template <int AXIS>
__device__ __forceinline__ void fill_body(const FillArgs& f)
{
    const int other = (AXIS == 0 ? f.my : f.mx) + 2 * CLAW2_NUM_GHOST;
    const int n = AXIS == 0 ? f.mx : f.my;
    const long long total = (long long)f.ncomp * other * 2 * CLAW2_NUM_GHOST;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int o = (int)(t % other) - CLAW2_NUM_GHOST;
        long long r = t / other;
        const int g = (int)(r % CLAW2_NUM_GHOST);
        r /= CLAW2_NUM_GHOST;
        const int side = (int)(r % 2);
        const int m = (int)(r / 2);
        const int bc = side == 0 ? f.bl : f.bu;
        int dst, src;
        if (side == 0) {
            dst = -1 - g;
            if (bc == CLAW2_BC_EXTRAP) src = 0;
            else if (bc == CLAW2_BC_PERIODIC) src = n - 1 - g;
            else if (bc == CLAW2_BC_WALL) src = g;
            else continue;
        } else {
            dst = n + g;
            if (bc == CLAW2_BC_EXTRAP) src = n - 1;
            else if (bc == CLAW2_BC_PERIODIC) src = g;
            else if (bc == CLAW2_BC_WALL) src = n - 1 - g;
            else continue;
        }
        auto off = [&](int along) {
            const int i = AXIS == 0 ? along : o, j = AXIS == 0 ? o : along;
            return (long long)m * f.plane + (long long)(j + CLAW2_NUM_GHOST) * f.ld + (i + CLAW2_NUM_GHOST);
        };
        double v = f.q[off(src)];
        if (bc == CLAW2_BC_WALL && m == f.negate) v = -v;
        f.q[off(dst)] = v;
    }
}

template <int AXIS>
__global__ void fill_kernel(FillArgs f)
{
    fill_body<AXIS>(f);
}

// Fill the ghost cells of q[ctrl->cur] (used after controlled steps when the
// step kernel cannot write ghost images itself).
template <int AXIS>
__global__ void fill_kernel_ctrl(FillArgs f, double* q0, double* q1, const claw2_control* c)
{
    f.q = c->cur ? q1 : q0;
    fill_body<AXIS>(f);
}

// ---------------------------------------------------------------------------
// layout conversion: reference (m fastest, Fortran) <-> device (planes)
// ---------------------------------------------------------------------------
__global__ void ref_to_dev_kernel(const double* ref, double* dev, int nc, int nx, int ny, long long ld,
                                  long long plane, int ghosts_in_ref)
{
    const long long total = (long long)nc * nx * ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(t % nc);
        const long long r = t / nc;
        const int i = (int)(r % nx), j = (int)(r / nx);
        const int off = ghosts_in_ref ? 0 : CLAW2_NUM_GHOST;
        dev[(long long)m * plane + (long long)(j + off) * ld + (i + off)] = ref[t];
    }
}

__global__ void dev_to_ref_kernel(const double* dev, double* ref, int nc, int nx, int ny, long long ld,
                                  long long plane, int ghosts_in_ref)
{
    const long long total = (long long)nc * nx * ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(t % nc);
        const long long r = t / nc;
        const int i = (int)(r % nx), j = (int)(r / nx);
        const int off = ghosts_in_ref ? 0 : CLAW2_NUM_GHOST;
        ref[t] = dev[(long long)m * plane + (long long)(j + off) * ld + (i + off)];
    }
}

// domain decomposition helpers: controller update from a given CFL number,
// and the two halo rows of q[cur] to/from a contiguous buffer
__global__ void control_apply_kernel(claw2_control* c, const double* cfl)
{
    const double v = *cfl;
    const bool nonfinite = !(v < 1.0 / 0.0);          // +inf or NaN
    if (!c->done) control_update(c, nonfinite ? 0.0 : v, nonfinite ? 1 : 0);
}

__global__ void halo_kernel(double* q0, double* q1, const claw2_control* c, double* buf, long long ld,
                            long long plane, int mx, int my, int ncomp, int upper, int unpack)
{
    double* q = c->cur ? q1 : q0;
    const int w = mx + 2 * CLAW2_NUM_GHOST;
    const int total = ncomp * 2 * w;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int i = t % w - CLAW2_NUM_GHOST, r = (t / w) % 2, m = t / (2 * w);
        int row;
        if (!unpack) row = upper ? my - 2 + r : r;
        else row = upper ? my + r : -2 + r;
        const long long o = (long long)m * plane + (long long)(row + CLAW2_NUM_GHOST) * ld + (i + CLAW2_NUM_GHOST);
        if (unpack) q[o] = buf[t];
        else buf[t] = q[o];
    }
}

// Before-step copy of plane `from` of q[cur] (ghost cells included) into
// plane `to` of aux (claw2_hooks.aux_from_q).
__global__ void aux_from_q_kernel(double* aux, const double* q0, const double* q1, const claw2_control* c,
                                  long long plane, int from, int to)
{
    if (c->done) return;
    const double* q = (c->cur ? q1 : q0) + (long long)from * plane;
    double* d = aux + (long long)to * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < plane; t += (long long)gridDim.x * blockDim.x)
        d[t] = q[t];
}

// Gauge samples after a step (claw2_gauges): one block; nothing happens
// unless the controller accepted a step since the last row.
__global__ void gauge_record_kernel(claw2_gauges g, const double* q0, const double* q1, const claw2_control* c,
                                    int meqn, long long ld, long long plane, int mx, int my)
{
    __shared__ int row;
    if (threadIdx.x == 0) {
        row = -1;
        if (c->numsteps != g.state[1]) {
            if (g.state[0] < g.capacity) row = (int)g.state[0];
            else g.state[2] = 1;
        }
    }
    __syncthreads();
    if (row < 0) return;
    const double* q = c->cur ? q1 : q0;
    const int w = 1 + meqn;
    for (int idx = threadIdx.x; idx < g.ngauges * w; idx += blockDim.x) {
        const int k = idx / w, m = idx - k * w;
        double v;
        if (m == 0) v = c->t;
        else {
            const int ix = g.cells[2 * k], iy = g.cells[2 * k + 1];
            if (ix < 0 || ix >= mx || iy < 0 || iy >= my) v = __longlong_as_double(0x7ff8000000000000ULL);
            else v = q[(long long)(m - 1) * plane + (long long)(iy + CLAW2_NUM_GHOST) * ld + ix + CLAW2_NUM_GHOST];
        }
        g.record[((long long)row * g.ngauges + k) * w + m] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        g.state[0] = row + 1;
        g.state[1] = c->numsteps;
    }
}

}  // namespace claw2

using namespace claw2;

// ===========================================================================
// host helpers
// ===========================================================================
namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int solver_shape(int rp, int* meqn, int* mw, int* maux)
{
    switch (rp) {
    case CLAW2_RP_ACOUSTICS: *meqn = 3; *mw = 2; *maux = 0; return 0;
    case CLAW2_RP_VC_ACOUSTICS: *meqn = 3; *mw = 2; *maux = 2; return 0;
    case CLAW2_RP_EULER_4WAVE: *meqn = 4; *mw = 4; *maux = 0; return 0;
    case CLAW2_RP_EULER_5WAVE: *meqn = 5; *mw = 5; *maux = 0; return 0;
    case CLAW2_RP_SHALLOW_ROE: *meqn = 3; *mw = 3; *maux = 0; return 0;
    case CLAW2_RP_PSYSTEM: *meqn = 3; *mw = 2; *maux = 4; return 0;
    default: return -1;
    }
}

bool periodic_ok(int bl, int bu) { return (bl == CLAW2_BC_PERIODIC) == (bu == CLAW2_BC_PERIODIC); }

bool fused_ghosts(const claw2_problem* p)
{
    for (int d = 0; d < 2; d++) {
        if (p->bc_lower[d] == CLAW2_BC_CUSTOM || p->bc_upper[d] == CLAW2_BC_CUSTOM) return false;
        if (!periodic_ok(p->bc_lower[d], p->bc_upper[d])) return false;
    }
    return p->mx >= 4 && p->my >= 4;
}

// Problems stepped by the lean body (launch_step_t): unsplit Euler and
// shallow water without capacity or f-waves.
bool lean_body(const claw2_problem* p)
{
    return p->transverse >= 0 && p->index_capa < 0 && !p->use_fwave &&
           (p->rp == CLAW2_RP_EULER_4WAVE || p->rp == CLAW2_RP_EULER_5WAVE || p->rp == CLAW2_RP_SHALLOW_ROE);
}

void tiles(const claw2_problem* p, int* nbx, int* nby)
{
    const bool split = p->transverse < 0;
    int tx = split ? STX : UTX, ty = split ? STY : UTY;
    // the light body's choice for small grids (launch_light)
    const bool light = !split && p->index_capa < 0 && !p->use_fwave &&
                       (p->rp == CLAW2_RP_ACOUSTICS || p->rp == CLAW2_RP_VC_ACOUSTICS);
    if (light && light_small_grid(p->mx, p->my)) tx = ty = LIGHT_SMALL_TILE;
    // the lean body's tiles (launch_step_t)
    if (lean_body(p)) { tx = LTX; ty = LTY; }
    *nbx = (p->mx + tx - 1) / tx;
    *nby = (p->my + ty - 1) / ty;
}

// The scratch of a step: the 64-byte header (the arrival counter) and one
// CFL partial per tile.
size_t scratch_bytes(const claw2_problem* p)
{
    int nbx, nby;
    tiles(p, &nbx, &nby);
    return 64 + sizeof(double) * (size_t)nbx * (size_t)nby;
}

// Point a's arrival counter and partials into scratch.
void set_scratch(void* scratch, StepArgs& a)
{
    a.ticket = static_cast<unsigned int*>(scratch);
    a.partials = reinterpret_cast<double*>(static_cast<char*>(scratch) + 64);
}

void fill_args(const claw2_problem* p, double* q, StepArgs& a)
{
    claw2_layout L;
    claw2_get_layout(p, &L);
    std::memset(&a, 0, sizeof a);
    a.ld = L.ld; a.plane = L.plane;
    a.mx = p->mx; a.my = p->my;
    a.dx = p->dx; a.dy = p->dy;
    a.order = p->order; a.trans = p->transverse; a.capa = p->index_capa; a.fwave = p->use_fwave;
    a.limit_any = 0;
    for (int w = 0; w < CLAW2_MAX_WAVES; w++) {
        a.mthlim[w] = w < p->num_waves ? p->mthlim[w] : 0;
        if (w < p->num_waves && p->mthlim[w] > 0) a.limit_any = 1;
    }
    for (int k = 0; k < CLAW2_MAX_PARAMS; k++) a.prm[k] = p->params[k];
    a.ghost_fused = fused_ghosts(p) ? 1 : 0;
    for (int d = 0; d < 2; d++) { a.bcl[d] = p->bc_lower[d]; a.bcu[d] = p->bc_upper[d]; }
    (void)q;
}

template <class RP, int T>
int launch_light_t(const StepArgs& a, int nbx, int nby, cudaStream_t st, bool chained)
{
    using SM = LightSmem<T, T, 256>;
    auto kern = light_step_kernel<RP, T>;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, kern, SM::bytes) != cudaSuccess) return CLAW2_ERR_CUDA;
    return launch_kernel(kern, dim3(nbx, nby), 256, SM::bytes, st, chained, a);
}

// nbx x nby come from tiles(), which makes the same choice
template <class RP>
int launch_light(const StepArgs& a, int nbx, int nby, cudaStream_t st, bool chained)
{
    if (light_small_grid(a.mx, a.my)) return launch_light_t<RP, LIGHT_SMALL_TILE>(a, nbx, nby, st, chained);
    return launch_light_t<RP, 29>(a, nbx, nby, st, chained);
}

// cuTensorMapEncodeTiled from the driver, found through the runtime (no link
// against libcuda, so the library still loads on a machine without a GPU)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static std::atomic<void*> fn{nullptr};
    void* f = fn.load(std::memory_order_acquire);
    if (!f) {
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !f)
            return nullptr;
        fn.store(f, std::memory_order_release);
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
}

// Tensor map of one state buffer for the lean body's halo boxes: the ghosted
// planes (mx+4 columns, my+4 rows, meqn fields; rows ld doubles apart, planes
// `plane` doubles apart), boxes of 16 x 32 x meqn, 128-byte swizzle, zeros
// outside the ghosted array.
int halo_tensor_map(CUtensorMap* m, const double* q, const StepArgs& a, int meqn)
{
    auto encode = tensor_map_encoder();
    if (!encode) return CLAW2_ERR_CUDA;
    if ((reinterpret_cast<uintptr_t>(q) & 15u) != 0) return CLAW2_ERR_INVALID;
    const cuuint64_t dims[3] = {(cuuint64_t)(a.mx + 2 * CLAW2_NUM_GHOST), (cuuint64_t)(a.my + 2 * CLAW2_NUM_GHOST),
                                (cuuint64_t)meqn};
    const cuuint64_t strides[2] = {(cuuint64_t)a.ld * sizeof(double), (cuuint64_t)a.plane * sizeof(double)};
    const cuuint32_t box[3] = {16, 32, (cuuint32_t)meqn};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(q), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CLAW2_OK : CLAW2_ERR_CUDA;
}

// bytes of halo that lean-body CTAs wait for in vain (claw2_debug_halo_shortfall)
std::atomic<int> g_halo_shortfall{0};

// chained: the previous operation in the stream is a step kernel of the same
// device loop (launch_kernel).
template <class RP, int NT>
int launch_lean_t(const StepArgs& a0, int nbx, int nby, cudaStream_t st, bool chained)
{
    StepArgs a = a0;
    a.halo_shortfall = g_halo_shortfall.load(std::memory_order_relaxed);
    using SM = LeanSmem<RP, LTX, LTY, NT>;
    auto kern = lean_step_kernel<RP, NT>;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, kern, SM::bytes) != cudaSuccess) return CLAW2_ERR_CUDA;
    CUtensorMap tm0, tm1;
    int rc = halo_tensor_map(&tm0, a.ctrl ? a.q0 : a.qin, a, RP::MEQN);
    if (!rc) rc = a.ctrl ? halo_tensor_map(&tm1, a.q1, a, RP::MEQN) : (tm1 = tm0, CLAW2_OK);
    if (rc) return rc;
    return launch_kernel(kern, dim3(nbx, nby), NT, SM::bytes, st, chained, a, tm0, tm1);
}

template <class RP>
int launch_lean(const StepArgs& a, int nbx, int nby, cudaStream_t st, bool chained)
{
    if ((long long)nbx * nby <= LEAN_BIG_BLOCK_TILES) return launch_lean_t<RP, 512>(a, nbx, nby, st, chained);
    return launch_lean_t<RP, 256>(a, nbx, nby, st, chained);
}

template <class RP, bool SPLIT>
int launch_step_t(const StepArgs& a, int nbx, int nby, cudaStream_t st, bool chained)
{
    if constexpr (!SPLIT && HasLight<RP>::value)
        if (a.capa < 0 && !a.fwave) return launch_light<RP>(a, nbx, nby, st, chained);
    if constexpr (!SPLIT && HasLean<RP>::value)
        if (a.capa < 0 && !a.fwave) return launch_lean<RP>(a, nbx, nby, st, chained);
    constexpr int TX = SPLIT ? STX : UTX, TY = SPLIT ? STY : UTY, NT = SPLIT ? SNT : UNT;
    using SM = TileSmem<RP, TX, TY, NT, SPLIT>;
    auto kern = step_kernel<RP, TX, TY, NT, SPLIT>;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, kern, SM::bytes) != cudaSuccess) return CLAW2_ERR_CUDA;
    return launch_kernel(kern, dim3(nbx, nby), NT, SM::bytes, st, chained, a);
}

// chained: the previous operation in the stream is a step kernel of the same
// device loop, so this step may overlap its end (launch_kernel).
int launch_step(const claw2_problem* p, const StepArgs& a, cudaStream_t st, bool chained = false)
{
    int nbx, nby;
    tiles(p, &nbx, &nby);
    const bool split = p->transverse < 0;
    switch (p->rp) {
    case CLAW2_RP_ACOUSTICS:
        return split ? launch_step_t<RpAcoustics, true>(a, nbx, nby, st, chained) : launch_step_t<RpAcoustics, false>(a, nbx, nby, st, chained);
    case CLAW2_RP_VC_ACOUSTICS:
        return split ? launch_step_t<RpVcAcoustics, true>(a, nbx, nby, st, chained) : launch_step_t<RpVcAcoustics, false>(a, nbx, nby, st, chained);
    case CLAW2_RP_EULER_4WAVE:
        return split ? launch_step_t<RpEuler<false>, true>(a, nbx, nby, st, chained) : launch_step_t<RpEuler<false>, false>(a, nbx, nby, st, chained);
    case CLAW2_RP_EULER_5WAVE:
        return split ? launch_step_t<RpEuler<true>, true>(a, nbx, nby, st, chained) : launch_step_t<RpEuler<true>, false>(a, nbx, nby, st, chained);
    case CLAW2_RP_SHALLOW_ROE:
        return split ? launch_step_t<RpShallow, true>(a, nbx, nby, st, chained) : launch_step_t<RpShallow, false>(a, nbx, nby, st, chained);
    case CLAW2_RP_PSYSTEM:
        return split ? launch_step_t<RpPsystem, true>(a, nbx, nby, st, chained) : launch_step_t<RpPsystem, false>(a, nbx, nby, st, chained);
    default:
        return CLAW2_ERR_INVALID;
    }
}

int launch_fill(const claw2_problem* p, double* q, int ncomp, const int* bl, const int* bu, bool is_aux,
                double* q0, double* q1, const claw2_control* ctrl, cudaStream_t st)
{
    claw2_layout L;
    claw2_get_layout(p, &L);
    for (int axis = 0; axis < 2; axis++) {
        FillArgs f;
        f.q = q; f.ld = L.ld; f.plane = L.plane; f.mx = p->mx; f.my = p->my; f.ncomp = ncomp;
        f.bl = bl[axis]; f.bu = bu[axis];
        f.negate = is_aux ? -1 : axis + 1;
        const int other = (axis == 0 ? p->my : p->mx) + 2 * CLAW2_NUM_GHOST;
        const long long total = (long long)ncomp * other * 2 * CLAW2_NUM_GHOST;
        const int threads = 256;
        const int blocks = (int)((total + threads - 1) / threads);
        if (ctrl) {
            if (axis == 0) fill_kernel_ctrl<0><<<blocks, threads, 0, st>>>(f, q0, q1, ctrl);
            else fill_kernel_ctrl<1><<<blocks, threads, 0, st>>>(f, q0, q1, ctrl);
        } else {
            if (axis == 0) fill_kernel<0><<<blocks, threads, 0, st>>>(f);
            else fill_kernel<1><<<blocks, threads, 0, st>>>(f);
        }
        if (cudaGetLastError() != cudaSuccess) return CLAW2_ERR_CUDA;
    }
    return CLAW2_OK;
}

int conv(const claw2_problem* p, int ncomp, const double* src, double* dst, bool to_dev, bool ghosts, cudaStream_t st)
{
    claw2_layout L;
    int rc = claw2_get_layout(p, &L);
    if (rc) return rc;
    const int g = ghosts ? 2 * CLAW2_NUM_GHOST : 0;
    const int nx = p->mx + g, ny = p->my + g;
    const long long total = (long long)ncomp * nx * ny;
    const int threads = 256;
    int blocks = (int)((total + threads - 1) / threads);
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    if (to_dev) ref_to_dev_kernel<<<blocks, threads, 0, st>>>(src, dst, ncomp, nx, ny, L.ld, L.plane, ghosts ? 1 : 0);
    else dev_to_ref_kernel<<<blocks, threads, 0, st>>>(src, dst, ncomp, nx, ny, L.ld, L.plane, ghosts ? 1 : 0);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

}  // namespace

// ===========================================================================
// extern "C" ABI
// ===========================================================================
extern "C" {

int claw2_abi_version(void) { return CLAW2_ABI_VERSION; }

int claw2_debug_halo_shortfall(int bytes)
{
    if (bytes < 0 || bytes > 65536 || (bytes & 7)) return CLAW2_ERR_INVALID;
    g_halo_shortfall.store(bytes, std::memory_order_relaxed);
    return CLAW2_OK;
}

const char* claw2_strerror(int status)
{
    switch (status) {
    case CLAW2_OK: return "ok";
    case CLAW2_ERR_INVALID: return "invalid problem description or argument";
    case CLAW2_ERR_UNSUPPORTED: return "feature not supported by this build";
    case CLAW2_ERR_CUDA: return "CUDA runtime error";
    case CLAW2_ERR_CFL: return "CFL too large, giving up!";
    case CLAW2_ERR_MAX_STEPS: return "Maximum number of timesteps have been taken";
    case CLAW2_ERR_NONFINITE: return "non-finite or non-physical state produced";
    case CLAW2_ERR_TIMEOUT: return "bounded device wait gave up";
    case CLAW2_ERR_NOMEM: return "out of memory";
    case CLAW2_ERR_SIZE: return "size beyond the documented maximum";
    default: return "unknown claw2 status";
    }
}

int claw2_validate(const claw2_problem* p)
{
    int meqn, mw, maux;
    if (!p) return CLAW2_ERR_INVALID;
    if (solver_shape(p->rp, &meqn, &mw, &maux)) return CLAW2_ERR_INVALID;
    if (p->num_eqn != meqn || p->num_waves != mw || p->num_aux < maux) return CLAW2_ERR_INVALID;
    if (p->num_ghost != CLAW2_NUM_GHOST) return CLAW2_ERR_UNSUPPORTED;
    if (p->mx < 2 || p->my < 2) return CLAW2_ERR_INVALID;
    if (p->num_aux < 0 || p->num_aux > CLAW2_MAX_EQN) return CLAW2_ERR_INVALID;
    if (p->order < 1 || p->order > 2) return CLAW2_ERR_INVALID;
    if (p->transverse < -1 || p->transverse > 2) return CLAW2_ERR_INVALID;
    if (p->index_capa < -1 || p->index_capa >= p->num_aux) return CLAW2_ERR_INVALID;
    if (!(p->dx > 0.0) || !(p->dy > 0.0)) return CLAW2_ERR_INVALID;
    for (int w = 0; w < p->num_waves; w++)
        if (p->mthlim[w] < 0) return CLAW2_ERR_INVALID;
    for (int d = 0; d < 2; d++) {
        if (p->bc_lower[d] < 0 || p->bc_lower[d] > 3 || p->bc_upper[d] < 0 || p->bc_upper[d] > 3) return CLAW2_ERR_INVALID;
        if (!periodic_ok(p->bc_lower[d], p->bc_upper[d])) return CLAW2_ERR_UNSUPPORTED;
        if (p->num_aux > 0 && (p->aux_bc_lower[d] < 0 || p->aux_bc_lower[d] > 3 ||
                               p->aux_bc_upper[d] < 0 || p->aux_bc_upper[d] > 3)) return CLAW2_ERR_INVALID;
    }
    return CLAW2_OK;
}

int claw2_get_layout(const claw2_problem* p, claw2_layout* out)
{
    if (!p || !out || p->mx < 1 || p->my < 1) return CLAW2_ERR_INVALID;
    const long long nx = (long long)p->mx + 2 * CLAW2_NUM_GHOST;
    out->ld = (nx + 15) / 16 * 16;              // 128-byte row pitch
    out->rows = (long long)p->my + 2 * CLAW2_NUM_GHOST;
    out->plane = out->ld * out->rows;
    out->q_elems = (long long)p->num_eqn * out->plane;
    out->aux_elems = (long long)p->num_aux * out->plane;
    return CLAW2_OK;
}

size_t claw2_scratch_bytes(const claw2_problem* p)
{
    if (!p || p->mx < 1 || p->my < 1) return 0;
    return scratch_bytes(p);
}

int claw2_fill_ghosts(const claw2_problem* p, double* q, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    return launch_fill(p, q, p->num_eqn, p->bc_lower, p->bc_upper, false, nullptr, nullptr, nullptr, S(stream));
}

int claw2_fill_aux_ghosts(const claw2_problem* p, double* aux, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (p->num_aux == 0) return CLAW2_OK;
    return launch_fill(p, aux, p->num_aux, p->aux_bc_lower, p->aux_bc_upper, true, nullptr, nullptr, nullptr, S(stream));
}

int claw2_step(const claw2_problem* p, const double* q_in, double* q_out, const double* aux, double dt,
               void* scratch, double* cfl_dev, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q_in || !q_out || !scratch || !cfl_dev || (p->num_aux > 0 && !aux) || q_in == q_out) return CLAW2_ERR_INVALID;
    StepArgs a;
    fill_args(p, q_out, a);
    a.qin = q_in; a.qout = q_out; a.aux = aux; a.dt = dt;
    set_scratch(scratch, a);
    a.cfl_out = cfl_dev;
    if ((rc = launch_step(p, a, S(stream)))) return rc;
    if (!a.ghost_fused)
        return launch_fill(p, q_out, p->num_eqn, p->bc_lower, p->bc_upper, false, nullptr, nullptr, nullptr, S(stream));
    return CLAW2_OK;
}

int claw2_advance(const claw2_problem* p, double* q0, double* q1, const double* aux, claw2_control* ctrl,
                  void* scratch, int nsteps, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q0 || !q1 || !ctrl || !scratch || (p->num_aux > 0 && !aux) || nsteps < 0) return CLAW2_ERR_INVALID;
    StepArgs a;
    fill_args(p, q0, a);
    a.q0 = q0; a.q1 = q1; a.aux = aux; a.ctrl = ctrl;
    set_scratch(scratch, a);
    for (int n = 0; n < nsteps; n++) {
        // from the second step on, a step follows a step kernel directly
        if ((rc = launch_step(p, a, S(stream), n > 0 && a.ghost_fused))) return rc;
        if (!a.ghost_fused &&
            (rc = launch_fill(p, nullptr, p->num_eqn, p->bc_lower, p->bc_upper, false, q0, q1, ctrl, S(stream))))
            return rc;
    }
    return CLAW2_OK;
}

}  // extern "C"

namespace {
// Checks claw2_hooks against the problem and sets the source term in a.
int apply_hooks(const claw2_problem* p, const claw2_hooks* hooks, StepArgs& a)
{
    if (hooks->source != CLAW2_SRC_NONE && hooks->source != CLAW2_SRC_EULER_RADIAL) return CLAW2_ERR_INVALID;
    if (hooks->source == CLAW2_SRC_EULER_RADIAL &&
        ((p->rp != CLAW2_RP_EULER_4WAVE && p->rp != CLAW2_RP_EULER_5WAVE) || hooks->source_aux < 0 ||
         hooks->source_aux >= p->num_aux))
        return CLAW2_ERR_UNSUPPORTED;
    if (hooks->aux_from_q != 0) {
        const int k = hooks->aux_from_q - 1, m = hooks->aux_q - 1;
        if (k < 0 || k >= p->num_aux || m < 0 || m >= p->num_eqn) return CLAW2_ERR_INVALID;
        for (int d = 0; d < 2; d++)
            if (p->aux_bc_lower[d] != p->bc_lower[d] || p->aux_bc_upper[d] != p->bc_upper[d] ||
                p->bc_lower[d] == CLAW2_BC_CUSTOM || p->bc_upper[d] == CLAW2_BC_CUSTOM)
                return CLAW2_ERR_UNSUPPORTED;
    }
    a.src = hooks->source;
    a.src_aux = hooks->source_aux;
    return CLAW2_OK;
}

int launch_aux_from_q(const claw2_hooks* hooks, const StepArgs& a, double* aux, double* q0, double* q1,
                      claw2_control* ctrl, cudaStream_t st)
{
    if (!hooks || hooks->aux_from_q == 0) return CLAW2_OK;
    const long long n = a.plane;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    aux_from_q_kernel<<<blocks, 256, 0, st>>>(aux, q0, q1, ctrl, a.plane, hooks->aux_q - 1, hooks->aux_from_q - 1);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}
}  // namespace

extern "C" {

int claw2_advance_hooked(const claw2_problem* p, double* q0, double* q1, const double* aux, claw2_control* ctrl,
                         void* scratch, int nsteps, const claw2_hooks* hooks, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q0 || !q1 || !ctrl || !scratch || !hooks || (p->num_aux > 0 && !aux) || nsteps < 0) return CLAW2_ERR_INVALID;
    StepArgs a;
    fill_args(p, q0, a);
    a.q0 = q0; a.q1 = q1; a.aux = aux; a.ctrl = ctrl;
    set_scratch(scratch, a);
    if ((rc = apply_hooks(p, hooks, a))) return rc;
    for (int n = 0; n < nsteps; n++) {
        if ((rc = launch_aux_from_q(hooks, a, const_cast<double*>(aux), q0, q1, ctrl, S(stream)))) return rc;
        if ((rc = launch_step(p, a, S(stream)))) return rc;
        if (!a.ghost_fused &&
            (rc = launch_fill(p, nullptr, p->num_eqn, p->bc_lower, p->bc_upper, false, q0, q1, ctrl, S(stream))))
            return rc;
    }
    return CLAW2_OK;
}

int claw2_advance_gauged(const claw2_problem* p, double* q0, double* q1, const double* aux, claw2_control* ctrl,
                         void* scratch, int nsteps, const claw2_hooks* hooks, const claw2_gauges* g, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q0 || !q1 || !ctrl || !scratch || !g || (p->num_aux > 0 && !aux) || nsteps < 0) return CLAW2_ERR_INVALID;
    if (g->ngauges < 1 || g->capacity < 1 || !g->cells || !g->record || !g->state) return CLAW2_ERR_INVALID;
    StepArgs a;
    fill_args(p, q0, a);
    a.q0 = q0; a.q1 = q1; a.aux = aux; a.ctrl = ctrl;
    set_scratch(scratch, a);
    if (hooks && (rc = apply_hooks(p, hooks, a))) return rc;
    const int threads = 128;
    for (int n = 0; n < nsteps; n++) {
        if ((rc = launch_aux_from_q(hooks, a, const_cast<double*>(aux), q0, q1, ctrl, S(stream)))) return rc;
        if ((rc = launch_step(p, a, S(stream)))) return rc;
        if (!a.ghost_fused &&
            (rc = launch_fill(p, nullptr, p->num_eqn, p->bc_lower, p->bc_upper, false, q0, q1, ctrl, S(stream))))
            return rc;
        gauge_record_kernel<<<1, threads, 0, S(stream)>>>(*g, q0, q1, ctrl, p->num_eqn, a.ld, a.plane, p->mx, p->my);
        if (cudaGetLastError() != cudaSuccess) return CLAW2_ERR_CUDA;
    }
    return CLAW2_OK;
}

int claw2_step_ctrl(const claw2_problem* p, double* q0, double* q1, const double* aux, claw2_control* ctrl,
                    void* scratch, double* cfl_dev, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q0 || !q1 || !ctrl || !scratch || !cfl_dev || (p->num_aux > 0 && !aux)) return CLAW2_ERR_INVALID;
    StepArgs a;
    fill_args(p, q0, a);
    a.q0 = q0; a.q1 = q1; a.aux = aux; a.ctrl = ctrl;
    a.ctrl_readonly = 1;
    a.cfl_out = cfl_dev;
    a.ghost_fused = 0;
    set_scratch(scratch, a);
    return launch_step(p, a, S(stream));
}

int claw2_control_apply(claw2_control* ctrl, const double* cfl_dev, void* stream)
{
    if (!ctrl || !cfl_dev) return CLAW2_ERR_INVALID;
    control_apply_kernel<<<1, 1, 0, S(stream)>>>(ctrl, cfl_dev);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

int claw2_fill_ghosts_ctrl(const claw2_problem* p, double* q0, double* q1, const claw2_control* ctrl, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q0 || !q1 || !ctrl) return CLAW2_ERR_INVALID;
    return launch_fill(p, nullptr, p->num_eqn, p->bc_lower, p->bc_upper, false, q0, q1, ctrl, S(stream));
}

static int halo(const claw2_problem* p, double* q0, double* q1, const claw2_control* ctrl, int upper, double* buf,
                int unpack, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q0 || !q1 || !ctrl || !buf || (upper != 0 && upper != 1) || p->my < 2) return CLAW2_ERR_INVALID;
    claw2_layout L;
    claw2_get_layout(p, &L);
    const int total = p->num_eqn * 2 * (p->mx + 2 * CLAW2_NUM_GHOST);
    halo_kernel<<<(total + 255) / 256, 256, 0, S(stream)>>>(q0, q1, ctrl, buf, L.ld, L.plane, p->mx, p->my,
                                                           p->num_eqn, upper, unpack);
    return cudaGetLastError() == cudaSuccess ? CLAW2_OK : CLAW2_ERR_CUDA;
}

int claw2_halo_pack(const claw2_problem* p, const double* q0, const double* q1, const claw2_control* ctrl, int upper,
                    double* buf, void* stream)
{
    return halo(p, const_cast<double*>(q0), const_cast<double*>(q1), ctrl, upper, buf, 0, stream);
}

int claw2_halo_unpack(const claw2_problem* p, double* q0, double* q1, const claw2_control* ctrl, int upper,
                      const double* buf, void* stream)
{
    return halo(p, q0, q1, ctrl, upper, const_cast<double*>(buf), 1, stream);
}

int claw2_control_init(claw2_control* c, double t, double dt, double tend, double cfl_max, double cfl_desired,
                       double dt_max, int dt_variable, int take_one_step, int64_t max_steps, double prev_cfl)
{
    if (!c) return CLAW2_ERR_INVALID;
    std::memset(c, 0, sizeof *c);
    c->t = t; c->dt = dt; c->tstart = t; c->tend = tend;
    c->cfl = prev_cfl;
    c->cfl_max = cfl_max; c->cfl_desired = cfl_desired; c->dt_max = dt_max;
    c->status_cflmax = prev_cfl; c->status_dtmin = dt; c->status_dtmax = dt;
    c->dt_variable = dt_variable; c->take_one_step = take_one_step;
    c->max_steps = max_steps;
    if (!dt_variable) {                                       // solver.py:618-624
        if (take_one_step) c->max_steps = 1;
        else {
            c->max_steps = (int64_t)((tend - t + 1e-10) / dt);
            if (std::fabs(c->max_steps * dt - (tend - t)) > 1e-5 * (tend - t)) return CLAW2_ERR_INVALID;
        }
    }
    if (dt_variable && cfl_desired > cfl_max) return CLAW2_ERR_INVALID;   // :625-626
    if (tend <= t && !take_one_step) c->max_steps = 0;                     // :627-629
    if (c->max_steps <= 0) { c->done = 1; return CLAW2_OK; }
    if (!take_one_step) {                                                  // :637-641
        if (c->t + c->dt > c->tend && c->tstart < c->tend) c->dt = c->tend - c->t;
        if (c->tend - c->t - c->dt < 1.e-14 * c->t) c->dt = c->tend - c->t;
    }
    return CLAW2_OK;
}

int claw2_ref_to_device(const claw2_problem* p, int ncomp, const double* ref, double* dev, void* stream)
{
    if (!p || !ref || !dev || ncomp < 1) return CLAW2_ERR_INVALID;
    return conv(p, ncomp, ref, dev, true, true, S(stream));
}

int claw2_device_to_ref(const claw2_problem* p, int ncomp, const double* dev, double* ref, void* stream)
{
    if (!p || !ref || !dev || ncomp < 1) return CLAW2_ERR_INVALID;
    return conv(p, ncomp, dev, ref, false, true, S(stream));
}

// ---------------------------------------------------------------------------
// batched form
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {
// threads per CTA, resident CTAs per SM, tile edge (cells per CTA per work
// item = tile^2).  Variants 4.. exist for the light acoustics body only
// (claw2_batch_advance returns CLAW2_ERR_UNSUPPORTED for them with the other
// solvers); a line of the light body has 32 lanes for tile + 3 interfaces, so
// smaller tiles leave lanes idle but waste fewer cells at instance edges.
// persistent: a grid of SMs x resident CTAs walking contiguous runs of tiles
// (batch_kernel); otherwise one CTA per tile (batch_tile_kernel)
struct BatchVariant { int threads, minb, tile, persistent; };
constexpr BatchVariant kBatchVariants[] = {{256, 2, 29, 1}, {128, 4, 29, 1}, {128, 3, 29, 1}, {512, 1, 29, 1},
                                           {256, 3, 29, 1}, {256, 4, 29, 1}, {256, 3, 21, 1}, {256, 4, 21, 1},
                                           {256, 3, 13, 1}, {256, 4, 13, 1}, {256, 3, 29, 0}, {256, 4, 29, 0},
                                           {128, 6, 29, 0}, {512, 2, 29, 0}};
constexpr int kNumBatchVariants = sizeof(kBatchVariants) / sizeof(kBatchVariants[0]);

bool batch_tile_ok(int tile) { return tile == 29 || tile == 21 || tile == 13; }

template <class RP, int NT, int MINB, bool LIGHT, int T>
int batch_launch_t(const StepArgs& common, const claw2_batch_instance* inst, int ninst, int ntiles, int nsteps,
                   cudaStream_t st)
{
    constexpr int SMB = LIGHT ? LightSmem<T, T, NT>::bytes : TileSmem<RP, 29, 29, NT, false>::bytes;
    constexpr int kSmemLimit = 227 * 1024;        // dynamic shared memory a CTA can opt in to
    constexpr int SMMAX = SMB + 4 * kBatchTableMax < kSmemLimit ? SMB + 4 * kBatchTableMax : SMB;
    auto kern = batch_kernel<RP, NT, MINB, LIGHT, T>;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, kern, SMMAX) != cudaSuccess) return CLAW2_ERR_CUDA;
    // the persistent grid: SMs x the CTAs that fit with this launch's table
    const int tbytes = (4 * ninst + 15) / 16 * 16;
    const int table = ninst <= kBatchTableMax && SMB + tbytes <= SMMAX;
    const int smem = SMB + (table ? tbytes : 0);
    int dev = 0, nsm = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT, smem) != cudaSuccess || occ < 1)
        return CLAW2_ERR_CUDA;
    const int grid = nsm * occ;
    const int g = ntiles < grid ? ntiles : grid;
    for (int n = 0; n < nsteps; n++) {
        kern<<<g, NT, smem, st>>>(inst, ninst, ntiles, common, SMB / 8, table);
        if (cudaGetLastError() != cudaSuccess) return CLAW2_ERR_CUDA;
    }
    return CLAW2_OK;
}

template <class RP, int NT, int MINB, bool LIGHT, int T>
int batch_launch_tiles(const StepArgs& common, const claw2_batch_instance* inst, int ninst, int ntiles, int nsteps,
                       const int32_t* tile_inst, cudaStream_t st)
{
    constexpr int SMB = LIGHT ? LightSmem<T, T, NT>::bytes : TileSmem<RP, 29, 29, NT, false>::bytes;
    auto kern = batch_tile_kernel<RP, NT, MINB, LIGHT, T>;
    static std::atomic<uint64_t> optin{0};
    if (smem_optin(optin, kern, SMB) != cudaSuccess) return CLAW2_ERR_CUDA;
    for (int n = 0; n < nsteps; n++) {
        kern<<<ntiles, NT, SMB, st>>>(inst, ninst, common, tile_inst);
        if (cudaGetLastError() != cudaSuccess) return CLAW2_ERR_CUDA;
    }
    return CLAW2_OK;
}

template <class RP>
int batch_launch_rp(int variant, const StepArgs& c, const claw2_batch_instance* inst, int ninst, int ntiles,
                    int nsteps, const int32_t* tile_inst, cudaStream_t st)
{
    if constexpr (HasLight<RP>::value) {
        if (c.capa < 0 && !c.fwave) {
            switch (variant) {
            case 0: return batch_launch_t<RP, 256, 2, true, 29>(c, inst, ninst, ntiles, nsteps, st);
            case 1: return batch_launch_t<RP, 128, 4, true, 29>(c, inst, ninst, ntiles, nsteps, st);
            case 2: return batch_launch_t<RP, 128, 3, true, 29>(c, inst, ninst, ntiles, nsteps, st);
            case 3: return batch_launch_t<RP, 512, 1, true, 29>(c, inst, ninst, ntiles, nsteps, st);
            case 4: return batch_launch_t<RP, 256, 3, true, 29>(c, inst, ninst, ntiles, nsteps, st);
            case 5: return batch_launch_t<RP, 256, 4, true, 29>(c, inst, ninst, ntiles, nsteps, st);
            case 6: return batch_launch_t<RP, 256, 3, true, 21>(c, inst, ninst, ntiles, nsteps, st);
            case 7: return batch_launch_t<RP, 256, 4, true, 21>(c, inst, ninst, ntiles, nsteps, st);
            case 8: return batch_launch_t<RP, 256, 3, true, 13>(c, inst, ninst, ntiles, nsteps, st);
            case 9: return batch_launch_t<RP, 256, 4, true, 13>(c, inst, ninst, ntiles, nsteps, st);
            case 10: return batch_launch_tiles<RP, 256, 3, true, 29>(c, inst, ninst, ntiles, nsteps, tile_inst, st);
            case 11: return batch_launch_tiles<RP, 256, 4, true, 29>(c, inst, ninst, ntiles, nsteps, tile_inst, st);
            case 12: return batch_launch_tiles<RP, 128, 6, true, 29>(c, inst, ninst, ntiles, nsteps, tile_inst, st);
            case 13: return batch_launch_tiles<RP, 512, 2, true, 29>(c, inst, ninst, ntiles, nsteps, tile_inst, st);
            default: return CLAW2_ERR_INVALID;
            }
        }
    }
    switch (variant) {
    case 0: return batch_launch_t<RP, 256, 2, false, 29>(c, inst, ninst, ntiles, nsteps, st);
    case 1: return batch_launch_t<RP, 128, 4, false, 29>(c, inst, ninst, ntiles, nsteps, st);
    case 2: return batch_launch_t<RP, 128, 3, false, 29>(c, inst, ninst, ntiles, nsteps, st);
    case 3: return batch_launch_t<RP, 512, 1, false, 29>(c, inst, ninst, ntiles, nsteps, st);
    default: return variant < kNumBatchVariants ? CLAW2_ERR_UNSUPPORTED : CLAW2_ERR_INVALID;
    }
}

int batch_launch(const claw2_problem* p, const claw2_batch_instance* inst, int ninst, int ntiles, int nsteps,
                 int variant, const int32_t* tile_inst, cudaStream_t st)
{
    StepArgs c;
    fill_args(p, nullptr, c);
    c.ghost_fused = 1;
    for (int d = 0; d < 2; d++)
        if (p->bc_lower[d] == CLAW2_BC_CUSTOM || p->bc_upper[d] == CLAW2_BC_CUSTOM) return CLAW2_ERR_UNSUPPORTED;
    switch (p->rp) {
    case CLAW2_RP_ACOUSTICS: return batch_launch_rp<RpAcoustics>(variant, c, inst, ninst, ntiles, nsteps, tile_inst, st);
    case CLAW2_RP_VC_ACOUSTICS: return batch_launch_rp<RpVcAcoustics>(variant, c, inst, ninst, ntiles, nsteps, tile_inst, st);
    case CLAW2_RP_EULER_4WAVE: return batch_launch_rp<RpEuler<false>>(variant, c, inst, ninst, ntiles, nsteps, tile_inst, st);
    case CLAW2_RP_EULER_5WAVE: return batch_launch_rp<RpEuler<true>>(variant, c, inst, ninst, ntiles, nsteps, tile_inst, st);
    case CLAW2_RP_SHALLOW_ROE: return batch_launch_rp<RpShallow>(variant, c, inst, ninst, ntiles, nsteps, tile_inst, st);
    case CLAW2_RP_PSYSTEM: return batch_launch_rp<RpPsystem>(variant, c, inst, ninst, ntiles, nsteps, tile_inst, st);
    default: return CLAW2_ERR_INVALID;
    }
}

int batch_check(const claw2_problem* p, const claw2_batch_instance* inst, int ninst, int ntiles, int nsteps,
                int variant)
{
    if (!p || !inst || ninst < 1 || ntiles < 1 || nsteps < 0) return CLAW2_ERR_INVALID;
    if (variant < 0 || variant >= kNumBatchVariants) return CLAW2_ERR_INVALID;
    if (p->transverse < 0) return CLAW2_ERR_UNSUPPORTED;
    int meqn, mw, maux;
    if (solver_shape(p->rp, &meqn, &mw, &maux) || p->num_eqn != meqn || p->num_waves != mw || p->num_aux < maux)
        return CLAW2_ERR_INVALID;
    if (p->num_ghost != CLAW2_NUM_GHOST || p->index_capa >= p->num_aux) return CLAW2_ERR_INVALID;
    for (int d = 0; d < 2; d++)
        if (!periodic_ok(p->bc_lower[d], p->bc_upper[d])) return CLAW2_ERR_UNSUPPORTED;
    return CLAW2_OK;
}
}  // namespace

extern "C" {

int claw2_batch_num_variants(void) { return kNumBatchVariants; }

int claw2_batch_variant_info(int v, int* threads, int* ctas_per_sm)
{
    if (v < 0 || v >= kNumBatchVariants || !threads || !ctas_per_sm) return CLAW2_ERR_INVALID;
    *threads = kBatchVariants[v].threads;
    *ctas_per_sm = kBatchVariants[v].minb;
    return CLAW2_OK;
}

int claw2_batch_tiles(int mx, int my, int* nbx, int* nby)
{
    return claw2_batch_tiles_for(UTX, mx, my, nbx, nby);
}

int claw2_batch_variant_tile(int v)
{
    if (v < 0 || v >= kNumBatchVariants) return -1;
    return kBatchVariants[v].tile;
}

int claw2_batch_tiles_for(int tile, int mx, int my, int* nbx, int* nby)
{
    if (!batch_tile_ok(tile) || mx < 4 || my < 4 || !nbx || !nby) return CLAW2_ERR_INVALID;
    *nbx = (mx + tile - 1) / tile;
    *nby = (my + tile - 1) / tile;
    return CLAW2_OK;
}

int claw2_batch_advance(const claw2_problem* p, const claw2_batch_instance* inst, int ninst, int ntiles, int nsteps,
                        int variant, void* stream)
{
    return claw2_batch_advance_map(p, inst, ninst, ntiles, nullptr, nsteps, variant, stream);
}

int claw2_batch_advance_map(const claw2_problem* p, const claw2_batch_instance* inst, int ninst, int ntiles,
                            const int32_t* tile_inst, int nsteps, int variant, void* stream)
{
    int rc = batch_check(p, inst, ninst, ntiles, nsteps, variant);
    if (rc) return rc;
    return batch_launch(p, inst, ninst, ntiles, nsteps, variant, tile_inst, S(stream));
}

int claw2_batch_graph_create(const claw2_problem* p, const claw2_batch_instance* inst, int ninst, int ntiles,
                             int nsteps, int variant, void** graph_exec)
{
    return claw2_batch_graph_create_map(p, inst, ninst, ntiles, nullptr, nsteps, variant, graph_exec);
}

int claw2_batch_graph_create_map(const claw2_problem* p, const claw2_batch_instance* inst, int ninst, int ntiles,
                                 const int32_t* tile_inst, int nsteps, int variant, void** graph_exec)
{
    int rc = batch_check(p, inst, ninst, ntiles, nsteps, variant);
    if (rc) return rc;
    if (!graph_exec) return CLAW2_ERR_INVALID;
    // one launch outside the capture configures the kernel (shared-memory
    // attribute, occupancy) so that the capture itself only records launches
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return CLAW2_ERR_CUDA;
    rc = batch_launch(p, inst, ninst, ntiles, 0, variant, tile_inst, st);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (!rc && cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = CLAW2_ERR_CUDA;
    if (!rc) {
        const int r2 = batch_launch(p, inst, ninst, ntiles, nsteps, variant, tile_inst, st);
        if (cudaStreamEndCapture(st, &graph) != cudaSuccess || r2) rc = r2 ? r2 : CLAW2_ERR_CUDA;
    }
    if (!rc && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) rc = CLAW2_ERR_CUDA;
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(st);
    if (rc) return rc;
    *graph_exec = exec;
    return CLAW2_OK;
}

int claw2_graph_launch(void* graph_exec, void* stream)
{
    if (!graph_exec) return CLAW2_ERR_INVALID;
    return cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(graph_exec), S(stream)) == cudaSuccess ? CLAW2_OK
                                                                                                     : CLAW2_ERR_CUDA;
}

int claw2_graph_destroy(void* graph_exec)
{
    if (!graph_exec) return CLAW2_OK;
    return cudaGraphExecDestroy(reinterpret_cast<cudaGraphExec_t>(graph_exec)) == cudaSuccess ? CLAW2_OK
                                                                                               : CLAW2_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// allocation-free step
//
// Some callers cannot allocate GPU memory: a host code that hands all device
// memory to its own pool at start-up, a time loop that must not enter the CUDA
// allocator (an allocation can synchronise the device), or a foreign-language
// binding that can pass pointers to existing buffers but cannot own device
// allocations.  claw2_step_noalloc serves them: its scratch (the block-arrival
// counter and one CFL partial per tile) is the static array below, which every
// GPU that loads this library holds until the process exits.
// ---------------------------------------------------------------------------
}  // extern "C"

static __device__ __align__(256) unsigned char g_noalloc_scratch[64 + 8 * CLAW2_NOALLOC_MAX_TILES];

namespace {
constexpr int kMaxDevices = 64;
std::atomic<void*> g_noalloc_addr[kMaxDevices];   // device address of g_noalloc_scratch, per device
}

extern "C" {

int claw2_step_noalloc(const claw2_problem* p, const double* q_in, double* q_out, const double* aux, double dt,
                       double* cfl_dev, void* stream)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!q_in || !q_out || !cfl_dev || (p->num_aux > 0 && !aux) || q_in == q_out) return CLAW2_ERR_INVALID;
    int nbx, nby;
    tiles(p, &nbx, &nby);
    if ((long long)nbx * (long long)nby > CLAW2_NOALLOC_MAX_TILES) return CLAW2_ERR_SIZE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return CLAW2_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return CLAW2_ERR_UNSUPPORTED;
    // Set-up, once per device, with that device current: the name of a
    // __device__ variable is only a host-side stand-in, so the kernel gets the
    // address the runtime reports for this device.
    void* scratch = g_noalloc_addr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess || !scratch) return CLAW2_ERR_CUDA;
        g_noalloc_addr[dev].store(scratch, std::memory_order_release);
    }
    // the array keeps the previous call's contents; the arrival counter must start at zero
    if (cudaMemsetAsync(scratch, 0, 64, S(stream)) != cudaSuccess) return CLAW2_ERR_CUDA;
    return claw2_step(p, q_in, q_out, aux, dt, scratch, cfl_dev, stream);
}

// ---------------------------------------------------------------------------
// host-buffer session
// ---------------------------------------------------------------------------
struct claw2_session {
    claw2_problem p;
    claw2_layout L;
    double *q0, *q1, *aux, *ref, *cfl;
    void* scratch;
    claw2_control* ctrl;       // device
    claw2_control* ctrl_host;  // pinned
    cudaStream_t stream;
};

int claw2_session_create(const claw2_problem* p, claw2_session** out)
{
    int rc = claw2_validate(p);
    if (rc) return rc;
    if (!out) return CLAW2_ERR_INVALID;
    claw2_session* s = new (std::nothrow) claw2_session;
    if (!s) return CLAW2_ERR_NOMEM;
    std::memset(s, 0, sizeof *s);
    s->p = *p;
    claw2_get_layout(p, &s->L);
    const size_t qb = sizeof(double) * s->L.q_elems;
    const size_t nref = (size_t)(p->num_eqn > p->num_aux ? p->num_eqn : p->num_aux) *
                        (p->mx + 2 * CLAW2_NUM_GHOST) * (p->my + 2 * CLAW2_NUM_GHOST);
    bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&s->q0, qb) == cudaSuccess && cudaMalloc(&s->q1, qb) == cudaSuccess;
    ok = ok && cudaMalloc(&s->ref, sizeof(double) * nref) == cudaSuccess;
    ok = ok && cudaMalloc(&s->cfl, sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->scratch, claw2_scratch_bytes(p)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->ctrl, sizeof(claw2_control)) == cudaSuccess;
    ok = ok && cudaMallocHost(&s->ctrl_host, sizeof(claw2_control)) == cudaSuccess;
    if (ok && p->num_aux > 0) ok = cudaMalloc(&s->aux, sizeof(double) * s->L.aux_elems) == cudaSuccess;
    ok = ok && cudaMemset(s->q0, 0, qb) == cudaSuccess && cudaMemset(s->q1, 0, qb) == cudaSuccess;
    ok = ok && cudaMemset(s->scratch, 0, claw2_scratch_bytes(p)) == cudaSuccess;
    if (!ok) { claw2_session_destroy(s); return CLAW2_ERR_NOMEM; }
    *out = s;
    return CLAW2_OK;
}

int claw2_session_destroy(claw2_session* s)
{
    if (!s) return CLAW2_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->q0); cudaFree(s->q1); cudaFree(s->ref); cudaFree(s->cfl); cudaFree(s->scratch);
    cudaFree(s->ctrl); cudaFree(s->aux);
    if (s->ctrl_host) cudaFreeHost(s->ctrl_host);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return CLAW2_OK;
}

static int upload_aux(claw2_session* s, const double* aux, bool ghosts)
{
    const claw2_problem* p = &s->p;
    if (p->num_aux == 0) return CLAW2_OK;
    if (!aux) return CLAW2_ERR_INVALID;
    const size_t n = (size_t)p->num_aux * (p->mx + (ghosts ? 2 * CLAW2_NUM_GHOST : 0)) *
                     (p->my + (ghosts ? 2 * CLAW2_NUM_GHOST : 0));
    if (cudaMemcpyAsync(s->ref, aux, n * sizeof(double), cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    int rc = conv(p, p->num_aux, s->ref, s->aux, true, ghosts, s->stream);
    if (rc) return rc;
    if (!ghosts) return claw2_fill_aux_ghosts(p, s->aux, s->stream);
    return CLAW2_OK;
}

int claw2_session_step2(claw2_session* s, const double* qold, double* qnew, const double* aux, double dt,
                        double* cfl)
{
    if (!s || !qold || !qnew || !cfl) return CLAW2_ERR_INVALID;
    const claw2_problem* p = &s->p;
    const size_t n = (size_t)p->num_eqn * (p->mx + 2 * CLAW2_NUM_GHOST) * (p->my + 2 * CLAW2_NUM_GHOST);
    int rc;
    if ((rc = upload_aux(s, aux, true))) return rc;
    if (cudaMemcpyAsync(s->ref, qold, n * sizeof(double), cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    if ((rc = conv(p, p->num_eqn, s->ref, s->q0, true, true, s->stream))) return rc;
    if ((rc = claw2_step(p, s->q0, s->q1, s->aux, dt, s->scratch, s->cfl, s->stream))) return rc;
    if ((rc = conv(p, p->num_eqn, s->q1, s->ref, false, true, s->stream))) return rc;
    if (cudaMemcpyAsync(qnew, s->ref, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    if (cudaMemcpyAsync(cfl, s->cfl, sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return CLAW2_ERR_CUDA;
    return std::isnan(*cfl) ? CLAW2_ERR_NONFINITE : CLAW2_OK;
}

int claw2_session_evolve(claw2_session* s, double* q, const double* aux, double* t, double* dt, double tend,
                         double cfl_max, double cfl_desired, double dt_max, int64_t max_steps, double* status)
{
    if (!s || !q || !t || !dt) return CLAW2_ERR_INVALID;
    const claw2_problem* p = &s->p;
    const size_t n = (size_t)p->num_eqn * p->mx * p->my;
    int rc;
    if ((rc = upload_aux(s, aux, false))) return rc;
    if (cudaMemcpyAsync(s->ref, q, n * sizeof(double), cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    if ((rc = conv(p, p->num_eqn, s->ref, s->q0, true, false, s->stream))) return rc;
    if ((rc = claw2_fill_ghosts(p, s->q0, s->stream))) return rc;
    if ((rc = claw2_control_init(s->ctrl_host, *t, *dt, tend, cfl_max, cfl_desired, dt_max, 1, 0, max_steps, cfl_desired)))
        return rc;
    if (cudaMemcpyAsync(s->ctrl, s->ctrl_host, sizeof(claw2_control), cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    for (;;) {
        // the controller's own estimate of the steps left (to tend and to
        // max_steps), at most 256 per batch: the host reads the controller
        // only between batches, and steps launched after it is done return
        // at once
        const claw2_control* h = s->ctrl_host;
        double left = (double)(h->max_steps - h->iter);
        if (h->dt > 0.0) left = std::min(left, (h->tend - h->t) / h->dt + 1.0);
        const int batch = (int)std::max(1.0, std::min(256.0, left));
        if ((rc = claw2_advance(p, s->q0, s->q1, s->aux, s->ctrl, s->scratch, batch, s->stream))) return rc;
        if (cudaMemcpyAsync(s->ctrl_host, s->ctrl, sizeof(claw2_control), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
            return CLAW2_ERR_CUDA;
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) return CLAW2_ERR_CUDA;
        if (s->ctrl_host->done) break;
    }
    const claw2_control* c = s->ctrl_host;
    double* cur = c->cur ? s->q1 : s->q0;
    if ((rc = conv(p, p->num_eqn, cur, s->ref, false, false, s->stream))) return rc;
    if (cudaMemcpyAsync(q, s->ref, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
        return CLAW2_ERR_CUDA;
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return CLAW2_ERR_CUDA;
    *t = c->t;
    *dt = c->dt;
    if (status) {
        status[0] = c->status_cflmax; status[1] = c->status_dtmin; status[2] = c->status_dtmax;
        status[3] = (double)c->numsteps; status[4] = (double)c->rejected;
    }
    return c->error;
}

}  // extern "C"
