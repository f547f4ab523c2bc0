/* claw2_adjoint.h -- multi-shot variable-coefficient acoustics and the
 * hand-written adjoint of its unsplit wave-propagation step.
 *
 * There is no counterpart in the reference: PyClaw has no adjoint.  These
 * entry points serve gradient-based inversion.  S independent wavefields
 * ("shots") share one aux field (rho, c) and one fixed dt; each step is the
 * reference's unsplit step2 (src/pyclaw/classic/step2.f90) with the
 * variable-coefficient acoustics solvers (rpn2/rpt2 of clawpack's
 * vc_acoustics), followed by a point source per shot and receiver sampling.
 *
 * Layout: every shot's state is one device-layout array of claw2.h
 * (claw2_get_layout: num_eqn planes of `plane` doubles, ghost width 2), shot s
 * starting at q + s * shot_stride.  aux is one device-layout array with
 * planes (rho, c).  Cell indices passed as int32 are flat interior indices
 * i + mx * j (0-based).
 *
 * The adjoint is the exact transpose of the linearised step with the limiter
 * branches frozen at the forward state (the branch of philim taken, the
 * upwind side of each wave and the "zero wave norm" skip), i.e. the derivative
 * torch.autograd computes for a transcription of the same step.  The dt is
 * treated as a constant.  Supported: rp = CLAW2_RP_VC_ACOUSTICS, order 1 or
 * 2, transverse 0, 1 or 2, limiters 0..5, no capacity, no f-waves, extrap /
 * periodic / wall boundaries, mx, my >= 4.  Anything else returns
 * CLAW2_ERR_UNSUPPORTED.
 *
 * All functions are asynchronous on `stream` and allocate nothing.
 */
#ifndef CLAW2_ADJOINT_H
#define CLAW2_ADJOINT_H

#include "claw2.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bytes of device scratch claw2_shots_step needs for nshots shots (zero-filled
 * once before the first call; the step leaves it ready for the next call). */
CLAW2_EXPORT size_t claw2_shots_scratch_bytes(const claw2_problem* p, int nshots);

/* One unsplit step of every shot with the same dt.  q_in must have its ghost
 * cells filled; q_out receives the new interior and its ghost images.
 * cfl_dev[s] receives shot s's CFL number. */
CLAW2_EXPORT int claw2_shots_step(const claw2_problem* p, int nshots, long long shot_stride,
                                  const double* q_in, double* q_out, const double* aux, double dt,
                                  void* scratch, double* cfl_dev, void* stream);

/* Point sources and receivers after a step: for each shot s with
 * src_cell[s] >= 0, add src_amp[s] to the pressure of that cell (and of its
 * ghost images); then record the pressure at the nrec receiver cells into
 * traces[s * nrec + r].  src_cell/src_amp/rec_cell/traces are device arrays;
 * src_amp or traces may be null (nothing added / nothing recorded).  Cell
 * indices outside 0..mx*my-1 are skipped (a receiver there records 0). */
CLAW2_EXPORT int claw2_shots_inject_record(const claw2_problem* p, int nshots, long long shot_stride, double* q,
                                           const int32_t* src_cell, const double* src_amp, int nrec,
                                           const int32_t* rec_cell, double* traces, void* stream);

/* Adjoint of one step.  q: the state the step started from (ghosts filled);
 * lam_in: the adjoint of the step's output (interior values; ghost cells must
 * be zero).  lam_out receives the adjoint of the step's input over the
 * interior and the two-cell ghost ring (the ghost-ring values are the raw
 * adjoints of the ghost cells, to be folded by claw2_shots_adjoint_fold).
 * gaux + s * gaux_stride (device layout, planes rho and c, ghost ring
 * included) accumulates shot s's gradient with respect to aux. */
CLAW2_EXPORT int claw2_shots_adjoint_step(const claw2_problem* p, int nshots, long long shot_stride,
                                          const double* q, const double* aux, double dt, const double* lam_in,
                                          double* lam_out, double* gaux, long long gaux_stride, void* stream);

/* Transpose of the ghost fill (Solver.apply_q_bcs): adds the ghost-ring
 * adjoints of lam into the interior cells they were copied from (y sides
 * first, then x sides, walls negating the normal velocity) and zeroes the
 * ghost ring; then adds gtrace[s * nrec + r] (device, may be null) to the
 * pressure adjoint at receiver r.  */
CLAW2_EXPORT int claw2_shots_adjoint_fold(const claw2_problem* p, int nshots, long long shot_stride, double* lam,
                                          int nrec, const int32_t* rec_cell, const double* gtrace, void* stream);

/* Transpose of the aux ghost fill (Solver.apply_aux_bcs) on every shot's aux
 * gradient: folds the ghost ring into the interior and zeroes it. */
CLAW2_EXPORT int claw2_shots_fold_aux(const claw2_problem* p, int nshots, long long gaux_stride, double* gaux,
                                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CLAW2_ADJOINT_H */
