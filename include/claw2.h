/*
 * claw2.h -- C ABI of the B200 (sm_100a) Clawpack 2D wave-propagation step.
 *
 * This header is the drop-in boundary for PyClaw's 2D classic solver.  In the
 * reference, ClawSolver2D.step_hyperbolic (src/pyclaw/classic/solver.py:498-547)
 * hands the ghosted state array qbc to the f2py module classic2:
 *
 *     self.qbc, cfl = self.fmod.step2(maxm, num_ghost, mx, my, qold, self.qbc,
 *                                     self.auxbc, dx, dy, self.dt, self._method,
 *                                     self._mthlim, aux1, aux2, aux3, work,
 *                                     self.fwave, rpn2, rpt2)
 *
 * (solver.py:537-539; split mode calls step2ds twice, :525-533).  Every entry
 * point below names the reference routine it replaces.  All functions are
 * plain C: integers, doubles, and untyped pointers.  Device pointers are CUDA
 * global-memory pointers on the current device; `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  Nothing here aborts the
 * process: every call returns a claw2 status code (0 = success).
 *
 * Two memory layouts are used:
 *
 *  - "reference layout": the Fortran-ordered ghosted array of the reference,
 *    qbc(num_eqn, 1-g:mx+g, 1-g:my+g), i.e. element (m,i,j) (0-based m, padded
 *    i in [0,mx+2g), padded j in [0,my+2g)) lives at m + num_eqn*(i + (mx+2g)*j).
 *    Used by the claw2_ref_* and claw2_session_* entry points.
 *
 *  - "device layout": one plane per component, rows along x, with a padded row
 *    pitch; element (m,i,j) lives at m*plane + j*ld + i (padded i, j as above).
 *    claw2_get_layout() returns ld/plane.  Used by every device-resident entry
 *    point (claw2_fill_ghosts, claw2_step, claw2_advance).
 */
#ifndef CLAW2_H
#define CLAW2_H

#include <stddef.h>
#include <stdint.h>

#ifndef CLAW2_EXPORT
#define CLAW2_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CLAW2_ABI_VERSION 1
#define CLAW2_MAX_EQN 8
#define CLAW2_MAX_WAVES 8
#define CLAW2_MAX_PARAMS 8
#define CLAW2_NUM_GHOST 2

/* ---- status codes ------------------------------------------------------ */
enum claw2_status {
    CLAW2_OK = 0,
    CLAW2_ERR_INVALID = 1,        /* bad problem description or argument        */
    CLAW2_ERR_UNSUPPORTED = 2,    /* valid in the reference, not built here      */
    CLAW2_ERR_CUDA = 3,           /* a CUDA runtime call failed                  */
    CLAW2_ERR_CFL = 4,            /* fixed dt and CFL > cfl_max ("giving up")    */
    CLAW2_ERR_MAX_STEPS = 5,      /* max_steps reached before tend               */
    CLAW2_ERR_NONFINITE = 6,      /* NaN/Inf or non-physical state produced      */
    CLAW2_ERR_TIMEOUT = 7,        /* a bounded device wait gave up               */
    CLAW2_ERR_NOMEM = 8,          /* allocation failed                           */
    CLAW2_ERR_SIZE = 9            /* size beyond a documented maximum            */
};

/* ---- Riemann solvers (solver.rp in the reference; clawpack.riemann modules) */
enum claw2_rp {
    CLAW2_RP_ACOUSTICS = 1,       /* rp2_acoustics: q=(p,u,v); params rho,bulk,cc,zz  */
    CLAW2_RP_VC_ACOUSTICS = 2,    /* rp2_vc_acoustics: q=(p,u,v), aux=(rho,c)         */
    CLAW2_RP_EULER_4WAVE = 3,     /* rp2_euler_4wave: q=(rho,rhou,rhov,E); gamma,gamma1 */
    CLAW2_RP_EULER_5WAVE = 4,     /* rp2_euler_5wave: + tracer; gamma,gamma1          */
    CLAW2_RP_SHALLOW_ROE = 5,     /* rp2_shallow_roe_with_efix: q=(h,hu,hv); grav     */
    CLAW2_RP_PSYSTEM = 6          /* rp2_psystem (f-waves): q=(eps,rho u,rho v),
                                     aux=(rho, K, linearity 1|2, eps for rpt2)      */
};

/* ---- boundary conditions (pyclaw.BC, src/pyclaw/solver.py:12-18) ------- */
enum claw2_bc {
    CLAW2_BC_CUSTOM = 0,          /* ghost cells are filled by the caller        */
    CLAW2_BC_EXTRAP = 1,
    CLAW2_BC_PERIODIC = 2,
    CLAW2_BC_WALL = 3
};

/*
 * Problem description.  Mirrors what the reference packs into method(7) and
 * mthlim(num_waves) (ClawSolver.set_method / set_mthlim,
 * src/pyclaw/classic/solver.py:167-198) plus the Riemann-solver scalars that
 * State.set_cparam copies into the /cparam/ common block (state.py:162-182).
 */
typedef struct claw2_problem {
    int32_t rp;                       /* enum claw2_rp                              */
    int32_t num_eqn;
    int32_t num_waves;
    int32_t num_aux;
    int32_t mx, my;                   /* interior cells                             */
    int32_t num_ghost;                /* must be CLAW2_NUM_GHOST                    */
    int32_t order;                    /* method(2): 1 or 2                          */
    int32_t transverse;               /* method(3): 0,1,2; -1 = dimensional split   */
    int32_t index_capa;               /* method(6)-1: 0-based aux index, -1 = none  */
    int32_t use_fwave;                /* solver.fwave                               */
    int32_t mthlim[CLAW2_MAX_WAVES];  /* solver.limiters per wave family            */
    int32_t bc_lower[2], bc_upper[2]; /* solver.bc_lower / bc_upper (x, y)          */
    int32_t aux_bc_lower[2], aux_bc_upper[2];
    double dx, dy;
    double params[CLAW2_MAX_PARAMS];  /* acoustics: rho,bulk,cc,zz; euler: gamma,gamma1;
                                         shallow: grav                              */
} claw2_problem;

/* Device layout of one ghosted array (see top of file). */
typedef struct claw2_layout {
    int64_t ld;        /* row pitch in doubles                                      */
    int64_t rows;      /* my + 2*num_ghost                                          */
    int64_t plane;     /* doubles per component plane                               */
    int64_t q_elems;   /* num_eqn * plane                                           */
    int64_t aux_elems; /* num_aux * plane                                           */
} claw2_layout;

/*
 * Time-step controller kept in device memory.  It restates the loop body of
 * Solver.evolve_to_time (src/pyclaw/solver.py:632-691): dt clamping to tend,
 * CFL accept/reject with restore, dt <- min(dt_max, dt*cfl_desired/cfl), and
 * the status dictionary {cflmax, dtmin, dtmax, numsteps}.  The step kernel's
 * last block runs that logic on the device, so many steps can be launched (or
 * replayed from a CUDA graph) without a host round trip per step.
 */
typedef struct claw2_control {
    double t, dt, tstart, tend;
    double cfl;                 /* CFL number of the last step taken            */
    double cfl_max, cfl_desired, dt_max;
    double status_cflmax, status_dtmin, status_dtmax;
    int64_t numsteps;           /* accepted steps (status['numsteps'])          */
    int64_t iter;               /* loop iterations including rejected ones      */
    int64_t max_steps;
    int64_t rejected;
    int32_t cur;                /* index (0/1) of the buffer holding the state  */
    int32_t done;               /* 1 once t >= tend (or one step taken)         */
    int32_t error;              /* claw2_status of the device loop              */
    int32_t dt_variable;
    int32_t take_one_step;
    uint32_t reserved_;         /* keep 0 (the block-arrival counter lives in scratch) */
    int32_t pad_[2];
} claw2_control;

/* ---- queries --------------------------------------------------------- */
CLAW2_EXPORT int claw2_abi_version(void);
CLAW2_EXPORT const char* claw2_strerror(int status);
/* Validates a problem; mirrors the checks the reference performs before it
 * steps (limiter list length, classic/solver.py:173-176; cparam keys,
 * state.py:176-180; workspace sizes, step2.f90:66-71). */
CLAW2_EXPORT int claw2_validate(const claw2_problem* p);
CLAW2_EXPORT int claw2_get_layout(const claw2_problem* p, claw2_layout* out);
/* Bytes of device scratch (per-block CFL partials) that claw2_step and
 * claw2_advance need. */
CLAW2_EXPORT size_t claw2_scratch_bytes(const claw2_problem* p);

/* ---- device-resident path (device layout, device pointers) ----------- */

/* Fill the ghost cells of q: Solver.apply_q_bcs / qbc_lower / qbc_upper
 * (src/pyclaw/solver.py:299-434) for extrap/periodic/wall; CUSTOM sides are
 * left untouched. x first, then y, so corners follow the reference. */
CLAW2_EXPORT int claw2_fill_ghosts(const claw2_problem* p, double* q, void* stream);
/* Same for aux: Solver.apply_aux_bcs / auxbc_lower / auxbc_upper (:438-576). */
CLAW2_EXPORT int claw2_fill_aux_ghosts(const claw2_problem* p, double* aux, void* stream);

/* One homogeneous step q_in -> q_out with a given dt: the work of
 * step2 (src/pyclaw/classic/step2.f90:2-251) when p->transverse >= 0, or of the
 * two step2ds sweeps (step2ds.f90:2-258, called from classic/solver.py:525-533)
 * when p->transverse == -1.  q_in's ghost cells must be filled.  Writes the
 * interior of q_out and, for non-CUSTOM sides, its ghost cells for the next
 * step.  The CFL number is written to *cfl_dev (device memory).  scratch must
 * hold claw2_scratch_bytes(p) bytes; its first 64 bytes must be zero on the
 * first call (the kernel leaves them zero). */
CLAW2_EXPORT int claw2_step(const claw2_problem* p, const double* q_in, double* q_out,
               const double* aux, double dt, void* scratch, double* cfl_dev,
               void* stream);

/* Largest number of tiles that claw2_step_noalloc accepts (claw2_scratch_bytes
 * counts them: 29x29 cells for the acoustics solvers, 13x13 on their grids of
 * fewer than 148 such tiles, 28x28 for Euler and shallow water and with
 * dimensional splitting): about 25 to 27 million cells. */
#define CLAW2_NOALLOC_MAX_TILES 32768

/* For testing the bounded wait of the TMA-staged tile bodies only (no
 * counterpart in the reference): from now on every such CTA of this process
 * waits for `bytes` (a multiple of 8, at most 65536; 0 restores normal
 * operation) more than its halo copies deliver, so its wait on the copies runs
 * out after about a second; the step then reports CLAW2_ERR_TIMEOUT through
 * the controller (a NaN CFL number without one) and writes no cells. */
CLAW2_EXPORT int claw2_debug_halo_shortfall(int bytes);

/* claw2_step without any device allocation, for callers that may not allocate
 * GPU memory (their memory belongs to a pool they manage, their time loop must
 * not call the allocator, or their language binding cannot own device memory).
 * No counterpart in the reference.  Same arguments and results as claw2_step
 * minus `scratch`: the scratch is a static array inside this library
 * (64 + 8*CLAW2_NOALLOC_MAX_TILES bytes, held by every GPU that loads the
 * library until the process exits).  The first call on a device looks up that
 * array's address for the current device; make that first call before any
 * stream capture begins.  Problems with more tiles than the maximum return
 * CLAW2_ERR_SIZE.  All calls share the one array, so calls that overlap on the
 * GPU (different streams, or different host threads, on the same device) race;
 * order them on one stream.  The address is remembered per device ordinal for
 * the device's primary context (the one the CUDA runtime uses): do not call
 * this entry point with another driver-API context current, nor after a
 * cudaDeviceReset of a device it has already run on. */
CLAW2_EXPORT int claw2_step_noalloc(const claw2_problem* p, const double* q_in, double* q_out,
                                    const double* aux, double dt, double* cfl_dev, void* stream);

/* Launch nsteps controlled steps.  q0/q1 are the two state buffers; ctrl->cur
 * says which holds the current state.  Each launch reads dt from ctrl, steps
 * q[cur] -> q[1-cur] and updates ctrl exactly as one iteration of
 * Solver.evolve_to_time (solver.py:632-691) does.  Launches after ctrl->done
 * become no-ops.  Nothing is synchronised; read ctrl back to see progress. */
CLAW2_EXPORT int claw2_advance(const claw2_problem* p, double* q0, double* q1,
                  const double* aux, claw2_control* ctrl, void* scratch,
                  int nsteps, void* stream);

/* Device-side forms of two application callbacks of the reference's Euler
 * shock-bubble app, so that a run using them needs no host round trip per step
 * (the reference passes Python functions: solver.step_source and a custom
 * boundary callback, apps/euler_2d/shockbubble.py:68-124).
 *  - source CLAW2_SRC_EULER_RADIAL: the geometric source of the Euler equations
 *    with radial symmetry, integrated with the app's two-stage second-order
 *    Runge-Kutta step (step_Euler_radial, shockbubble.py:89-124) on every
 *    interior cell after the hyperbolic step (Godunov splitting, source_split
 *    = 1), the radial coordinate read from aux component source_aux.  It is
 *    fused into the step's final write; a rejected step's output is discarded
 *    whole.  (One difference: the reference skips the source of a step whose
 *    CFL number equals cfl_max exactly and still accepts the step.)
 *  - a fixed inflow state on a side is expressed as a custom side (bc 0)
 *    whose ghost cells the caller fills once, in both state buffers: the step
 *    never writes the ghost cells of custom sides. */
enum claw2_source {
    CLAW2_SRC_NONE = 0,
    CLAW2_SRC_EULER_RADIAL = 1
};

typedef struct claw2_hooks {
    int32_t source;        /* claw2_source                                  */
    int32_t source_aux;    /* aux component holding the radial coordinate   */
    int32_t aux_from_q;    /* 0, or k: before every step aux component k     */
    int32_t aux_q;         /*   (1-based) is set to q component aux_q        */
                           /*   (1-based) of the current state, ghost cells  */
                           /*   included (aux is written: it must be device  */
                           /*   memory the library may change)               */
} claw2_hooks;

/* claw2_advance with the hooks applied to each step: the source term, and
 * the before-step copy of a state component into an aux component that the
 * Riemann solver reads (apps/psystem_2d/psystem.py:86-90 sets aux(4) = q(1)
 * before every step for its transverse solver).  The copy takes the ghost
 * cells of q too, so the aux boundary conditions of that component must be
 * those of q (checked: CLAW2_ERR_UNSUPPORTED otherwise).
 * CLAW2_ERR_UNSUPPORTED for a source the Riemann solver cannot take
 * (CLAW2_SRC_EULER_RADIAL needs the Euler solvers and aux). */
CLAW2_EXPORT int claw2_advance_hooked(const claw2_problem* p, double* q0, double* q1, const double* aux,
                                      claw2_control* ctrl, void* scratch, int nsteps, const claw2_hooks* hooks,
                                      void* stream);

/* ---- gauges recorded on the device ---------------------------------- */
/* Solver.write_gauge_values (src/pyclaw/solver.py:713-742) samples q at every
 * gauge cell after each accepted step (evolve_to_time, solver.py:654-656) and
 * hands it to compute_gauge_values on the host.  A recorder keeps those
 * samples on the device instead, so the time loop stays on the GPU: after a
 * step accepted by the controller, record row r = state[0] gets, for gauge k,
 * record[(r*ngauges + k)*(1+num_eqn) + 0] = t and [.. + 1 + m] = q(m, ix, iy)
 * of the new state, and state[0] grows by one.  The caller drains the rows
 * and sets state[0] back to 0 before `capacity` rows are full; a step
 * accepted with no free row sets state[2] = 1 and is not recorded.  A gauge
 * cell outside 0 <= ix < mx, 0 <= iy < my records NaN.  All pointers are
 * device memory. */
typedef struct claw2_gauges {
    int32_t ngauges;
    int32_t capacity;            /* rows of `record`                             */
    const int32_t* cells;        /* ngauges pairs (ix, iy) of interior cells     */
    double* record;              /* capacity x ngauges x (1 + num_eqn) doubles    */
    int64_t* state;              /* [0] rows written, [1] numsteps of the last
                                    row (set it to ctrl->numsteps at the start),
                                    [2] overflow flag                            */
} claw2_gauges;

/* claw2_advance (with the source term of `hooks` when hooks is not NULL) and
 * the gauge recorder `g` run after every step. */
CLAW2_EXPORT int claw2_advance_gauged(const claw2_problem* p, double* q0, double* q1, const double* aux,
                                      claw2_control* ctrl, void* scratch, int nsteps, const claw2_hooks* hooks,
                                      const claw2_gauges* g, void* stream);

/* ---- domain decomposition: one slab of a larger grid per process -------- */
/* The reference runs one grid per process under PETSc (PetClaw: a DA with a
 * halo exchange, src/petclaw/state.py:268, and a global CFL max,
 * src/petclaw/cfl.py:30-31).  Here a slab is a claw2_problem whose sides that
 * face another slab are custom (bc 0); per step every slab runs, in order:
 * claw2_halo_pack (its two boundary rows of q[cur] into a buffer),
 * the exchange of those buffers between neighbours (the caller's transport,
 * e.g. NCCL), claw2_halo_unpack (the neighbours' rows into the ghost rows),
 * claw2_step_ctrl, a max-reduction of the CFL numbers over all slabs (the
 * caller's transport), claw2_control_apply and claw2_fill_ghosts_ctrl.  All of
 * it is asynchronous on the stream; cur and dt are read on the device. */

/* One step q[cur] -> q[1-cur] with dt and cur read from ctrl (as
 * claw2_advance), writing the slab's CFL number to cfl_dev (+inf when the new
 * state is not finite) and leaving ctrl unchanged.  Ghost cells of the new
 * state are not written; fill them with claw2_fill_ghosts_ctrl after
 * claw2_control_apply. */
CLAW2_EXPORT int claw2_step_ctrl(const claw2_problem* p, double* q0, double* q1, const double* aux,
                                 claw2_control* ctrl, void* scratch, double* cfl_dev, void* stream);

/* One iteration of the controller (as claw2_advance's) with the CFL number
 * *cfl_dev (a max over all slabs; +inf or NaN: non-finite state). */
CLAW2_EXPORT int claw2_control_apply(claw2_control* ctrl, const double* cfl_dev, void* stream);

/* Ghost fill (claw2_fill_ghosts) of q[ctrl->cur]; custom sides untouched. */
CLAW2_EXPORT int claw2_fill_ghosts_ctrl(const claw2_problem* p, double* q0, double* q1, const claw2_control* ctrl,
                                        void* stream);

/* Halo rows of q[ctrl->cur], all components and all columns including the
 * ghost columns, as num_eqn x 2 x (mx+4) doubles (component, row, column).
 * pack: upper = 0 the rows 0,1, upper = 1 the rows my-2,my-1;
 * unpack: upper = 0 into the ghost rows -2,-1, upper = 1 into my,my+1. */
CLAW2_EXPORT int claw2_halo_pack(const claw2_problem* p, const double* q0, const double* q1,
                                 const claw2_control* ctrl, int upper, double* buf, void* stream);
CLAW2_EXPORT int claw2_halo_unpack(const claw2_problem* p, double* q0, double* q1, const claw2_control* ctrl,
                                   int upper, const double* buf, void* stream);

/* Host-side initialisation of a controller for evolve_to_time(solution, tend)
 * (solver.py:600-641): status reset, fixed-dt step count, first clamp. */
CLAW2_EXPORT int claw2_control_init(claw2_control* c, double t, double dt, double tend,
                       double cfl_max, double cfl_desired, double dt_max,
                       int dt_variable, int take_one_step, int64_t max_steps,
                       double prev_cfl);

/* Layout conversion between the reference layout and the device layout, on
 * the device (device pointers to both). */
CLAW2_EXPORT int claw2_ref_to_device(const claw2_problem* p, int ncomp, const double* ref,
                        double* dev, void* stream);
CLAW2_EXPORT int claw2_device_to_ref(const claw2_problem* p, int ncomp, const double* dev,
                        double* ref, void* stream);

/* ---- batched form: many independent instances per launch --------------- */
/* One instance of a batch: its own grid size, spacing, state buffers (device
 * layout of that grid), aux, controller and scratch.  All instances share the
 * solver settings of the claw2_problem passed with them (Riemann solver,
 * limiters, order, transverse mode, boundary conditions); its mx, my, dx, dy
 * are ignored.  No counterpart in the reference, which steps one patch per
 * call. */
typedef struct claw2_batch_instance {
    double* q0;                 /* state buffers (device layout for this grid) */
    double* q1;
    const double* aux;          /* may be NULL when num_aux == 0               */
    claw2_control* ctrl;        /* this instance's time-step controller        */
    double* partials;           /* one double per tile of this instance        */
    unsigned int* ticket;       /* arrival counter, zero between launches      */
    int64_t ld, plane;          /* layout of this grid (claw2_get_layout)      */
    int32_t mx, my;
    double dx, dy;
    int32_t nbx, nby;           /* tiles (claw2_batch_tiles_for the variant's edge) */
    int32_t tile_begin;         /* index of this instance's first tile         */
    int32_t pad_;
} claw2_batch_instance;

/* Launch configurations of the batched kernel the autotuner chooses from:
 * threads per CTA x resident CTAs per SM x tile edge, and the grid's form
 * (variants 0-9: a persistent grid of SMs x resident CTAs, each CTA walking a
 * contiguous run of tiles; 10-13: one CTA per tile). */
CLAW2_EXPORT int claw2_batch_num_variants(void);
/* Threads per CTA and resident CTAs per SM of variant v (for reporting). */
CLAW2_EXPORT int claw2_batch_variant_info(int v, int* threads, int* ctas_per_sm);
/* Tile edge (cells) of variant v: 29, 21 or 13; -1 for an invalid v.  The
 * descriptors passed with variant v must number the tiles of that edge. */
CLAW2_EXPORT int claw2_batch_variant_tile(int v);
/* Tiles of an mx x my instance for a tile edge of 29, 21 or 13 cells. */
CLAW2_EXPORT int claw2_batch_tiles_for(int tile, int mx, int my, int* nbx, int* nby);
/* Tiles of an mx x my instance with 29x29 tiles (variants 0-5). */
CLAW2_EXPORT int claw2_batch_tiles(int mx, int my, int* nbx, int* nby);
/* nsteps launches of the batched step: every launch takes one controlled step
 * (Solver.evolve_to_time's loop body, src/pyclaw/solver.py:632-691) of every
 * instance whose controller is not done, each with its own dt.  inst is a
 * device array of ninst descriptors whose tiles are numbered consecutively;
 * ntiles is their total.  Unsplit (transverse >= 0) only. */
CLAW2_EXPORT int claw2_batch_advance(const claw2_problem* p, const claw2_batch_instance* inst, int ninst,
                                     int ntiles, int nsteps, int variant, void* stream);
/* The same nsteps launches captured once into a CUDA graph; replay it with
 * claw2_graph_launch.  The descriptors and buffers must stay where they are. */
CLAW2_EXPORT int claw2_batch_graph_create(const claw2_problem* p, const claw2_batch_instance* inst, int ninst,
                                          int ntiles, int nsteps, int variant, void** graph_exec);
/* The same two with a tile -> instance map: tile_inst is a device array of
 * ntiles int32, entry t the instance whose tiles include tile t.  The
 * one-CTA-per-tile variants then find a tile's instance with one load
 * instead of a binary search over the descriptors (an entry that does not
 * hold its tile falls back to the search); the other variants ignore it.
 * NULL means no map. */
CLAW2_EXPORT int claw2_batch_advance_map(const claw2_problem* p, const claw2_batch_instance* inst, int ninst,
                                         int ntiles, const int32_t* tile_inst, int nsteps, int variant,
                                         void* stream);
CLAW2_EXPORT int claw2_batch_graph_create_map(const claw2_problem* p, const claw2_batch_instance* inst, int ninst,
                                              int ntiles, const int32_t* tile_inst, int nsteps, int variant,
                                              void** graph_exec);
CLAW2_EXPORT int claw2_graph_launch(void* graph_exec, void* stream);
CLAW2_EXPORT int claw2_graph_destroy(void* graph_exec);

/* ---- host-buffer session (reference layout, host pointers) ----------- */
/* A session owns device buffers for one problem so that callers holding host
 * arrays (the f2py calling convention of step2) can step without managing
 * device memory. */
typedef struct claw2_session claw2_session;
CLAW2_EXPORT int claw2_session_create(const claw2_problem* p, claw2_session** out);
CLAW2_EXPORT int claw2_session_destroy(claw2_session* s);
/* Exact f2py contract of step2/step2ds (classic/solver.py:525-539): qold and
 * qnew are host arrays in reference layout with ghost cells already filled by
 * the caller; on return qnew holds the updated array and *cfl the CFL number.
 * aux may be NULL when num_aux == 0. */
CLAW2_EXPORT int claw2_session_step2(claw2_session* s, const double* qold, double* qnew,
                        const double* aux, double dt, double* cfl);
/* Controller.run-style evolve from host data: q (reference layout interior,
 * shape (num_eqn, mx, my) Fortran order) is uploaded, the solution is advanced
 * from *t to tend with on-device dt control, and q is downloaded again.
 * *t and *dt are updated; status receives {cflmax, dtmin, dtmax, numsteps,
 * rejected} as doubles (5 entries, may be NULL). */
CLAW2_EXPORT int claw2_session_evolve(claw2_session* s, double* q, const double* aux,
                         double* t, double* dt, double tend, double cfl_max,
                         double cfl_desired, double dt_max, int64_t max_steps,
                         double* status);

#ifdef __cplusplus
}
#endif
#endif /* CLAW2_H */
