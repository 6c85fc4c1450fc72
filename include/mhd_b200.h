/*
 * mhd_b200.h -- C ABI of the B200 (sm_100a) SPMHD particle-update library.
 *
 * The library replaces the CUDA kernels that PySPH generates at run time for
 * the reference's equation groups (src/scheme.py:66-81) and its integrator
 * step (src/integrator.py), plus the PySPH neighbour search
 * (src/application.py:63-78, periodic_mode="minimum_image") that feeds them.
 *
 * Conventions
 *  - Every function returns MHD_OK (0) or a negative MHD_ERR_* code; no C++
 *    exception crosses the ABI.  mhd_last_error() gives a message.
 *  - Particle memory belongs to the caller (one device array per reference
 *    property name, structure of arrays).  A context owns only workspace.
 *  - All calls are ordered on the CUDA stream passed in (cudaStream_t as
 *    void*; NULL = legacy default stream).  One host thread per context.
 *  - Device-side failures (non-finite dt, neighbour capacity) are recorded in
 *    a device status word and reported at the next synchronising call.
 */
#ifndef MHD_B200_H
#define MHD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MHD_ABI_VERSION 1

#define MHD_OK 0
#define MHD_ERR_INVALID (-1)        /* bad argument, null required pointer, n > n_max */
#define MHD_ERR_CUDA (-2)           /* a CUDA runtime call failed */
#define MHD_ERR_NOT_CONVERGED (-3)  /* density iteration hit max_iter with unconverged particles */
#define MHD_ERR_NONFINITE (-4)      /* NaN/Inf met in the timestep reduction */
#define MHD_ERR_CAPACITY (-5)       /* cell grid larger than the supported maximum */
#define MHD_ERR_NO_DEVICE (-6)      /* no CUDA device, or not sm_100 */
#define MHD_ERR_RELIST (-7)         /* a captured run met a list rebuild: its state is invalid, replay it uncaptured */

/* Kernel ids: the reference's kernel map, src/scheme.py:48-56. */
#define MHD_KERNEL_CUBIC 0
#define MHD_KERNEL_QUINTIC 1
#define MHD_KERNEL_WENDLAND_C2 2
#define MHD_KERNEL_WENDLAND_C4 3
#define MHD_KERNEL_WENDLAND_C6 4
#define MHD_KERNEL_GAUSSIAN 5
#define MHD_KERNEL_SUPER_GAUSSIAN 6

/* Pair-sum precision of the force and density passes. */
#define MHD_PRECISION_FP64 0
#define MHD_PRECISION_FP32 1

/*
 * Scheme parameters.  Fields map to the reference's configuration
 * (src/config.py:8-57) and MHDScheme (src/scheme.py:32-44); dim, alpha_min,
 * alpha_max and precision are extensions whose defaults (3, 0, 1, FP64)
 * reproduce the reference.
 */
typedef struct MhdParams {
  int32_t dim;             /* 2 or 3 (reference: always 3, src/scheme.py:57) */
  int32_t kernel;          /* MHD_KERNEL_* */
  int32_t iterate;         /* numerics.density == "iterate" (src/scheme.py:69) */
  int32_t min_iter;        /* 2 (src/scheme.py:71) */
  int32_t max_iter;        /* 250, MAX_DENSITY_ITERATIONS (src/scheme.py:28) */
  int32_t precision;       /* MHD_PRECISION_* */
  int32_t periodic[3];     /* periodic_mode "minimum_image" per axis */
  int32_t reserved;
  double hfact;            /* numerics.hfact, the k of DensityIteration */
  double gamma;            /* physics.gamma */
  double mu0;              /* physics.mu0 */
  double av;               /* physics.artificial_viscosity */
  double ac;               /* physics.artificial_thermal_conductivity */
  double ar;               /* physics.artificial_magnetic_dissipation */
  double clean_speed;      /* numerics.cleaning_speed_factor */
  double clean_damp;       /* numerics.cleaning_damping_factor */
  double timestep_factor;  /* solver.timestep_factor */
  double alpha_min;        /* Cullen-Dehnen clip, reference literal 0 (src/equations.py:428) */
  double alpha_max;        /* reference literal 1 */
  double tf;               /* solver.tf: the last step is clipped to reach it */
  double lo[3];            /* periodic box (src/application.py:66-78) */
  double hi[3];
} MhdParams;

/*
 * Particle state: one device pointer per reference property name
 * (src/particles.py).  The X-macro lists the fields in layout order; all are
 * double except itype (int32).  "Required" fields must be non-null for the
 * step and RHS calls; "optional" ones are written only when non-null.
 */
#define MHD_STATE_REQUIRED(X)                                                                       \
  X(x) X(y) X(z) X(gid) X(u) X(v) X(w) X(rho) X(rho_sum) X(h) X(m) X(cs) X(p) X(e) X(au) X(av) X(aw) \
  X(ae) X(ah) X(upred) X(vpred) X(wpred) X(epred) X(h0) X(div) X(dt_cfl) X(dt_adapt) X(omega)       \
  X(converged) X(alpha1) X(Bx) X(By) X(Bz) X(Bevolx) X(Bevoly) X(Bevolz) X(psi) X(Bevolxpred)        \
  X(Bevolypred) X(Bevolzpred) X(psipred) X(Bxpred) X(Bypred) X(Bzpred) X(aBevolx) X(aBevoly)         \
  X(aBevolz) X(apsi) X(divBsymm) X(divBdiff) X(div_for_psi) X(alphaloc)
#define MHD_STATE_OPTIONAL(X)                                                                       \
  X(x0) X(y0) X(z0) X(u0) X(v0) X(w0) X(e0) X(alpha10) X(Bevolx0) X(Bevoly0) X(Bevolz0) X(psi0)      \
  X(xilimiter) X(divvdt) X(arho) X(grhox) X(grhoy) X(grhoz) X(dwdh)                                 \
  X(cd_rxx) X(cd_rxy) X(cd_rxz) X(cd_ryy) X(cd_ryz) X(cd_rzz) X(cd_vxx) X(cd_vxy) X(cd_vxz)           \
  X(cd_vyx) X(cd_vyy) X(cd_vyz) X(cd_vzx) X(cd_vzy) X(cd_vzz) X(cd_axx) X(cd_axy) X(cd_axz)           \
  X(cd_ayx) X(cd_ayy) X(cd_ayz) X(cd_azx) X(cd_azy) X(cd_azz) X(dvdx_xx) X(dvdx_xy) X(dvdx_xz)        \
  X(dvdx_yx) X(dvdx_yy) X(dvdx_yz) X(dvdx_zx) X(dvdx_zy) X(dvdx_zz)

typedef struct MhdState {
#define MHD_FIELD_(n) double* n;
  MHD_STATE_REQUIRED(MHD_FIELD_)
  MHD_STATE_OPTIONAL(MHD_FIELD_)
#undef MHD_FIELD_
  int32_t* itype; /* 1 = integrated fluid; other values are frozen (src/integrator.py:39,69) */
} MhdState;

/* Per-call statistics of a right-hand side (host memory). */
typedef struct MhdRhsStats {
  int32_t density_passes;   /* passes of the iterated DensityIteration group */
  int32_t grid_rebuilds;    /* neighbour grids built (1 + re-plans when h outgrew the cells) */
  int64_t n_unconverged;    /* particles unconverged when the group stopped */
  int64_t n_cells;          /* cells of the last grid */
} MhdRhsStats;

/* Kernel families timed with CUDA events when timing is enabled. */
#define MHD_TIMING_KINDS 7
#define MHD_TIMING_CELLS 0        /* cell keys, radix sort, cell table, gather */
#define MHD_TIMING_DENSITY 1      /* density passes */
#define MHD_TIMING_PROLOGUE 2     /* force prologue (G2, G3, G5) */
#define MHD_TIMING_FORCE 3        /* fused force pass (G4, G6-G10) */
#define MHD_TIMING_DT 4           /* timestep reduction */
#define MHD_TIMING_INTEGRATE 5    /* integrator stages / corrector-predictor */
#define MHD_TIMING_LISTS 6        /* neighbour-list build (gather, scatter, ordering) */

/* ---- library and context ---- */

int mhd_abi_version(void);
/* Names of the MhdState fields in layout order (for binding checks). */
int mhd_state_field_count(void);
const char* mhd_state_field_name(int32_t i);
/* Names of the fields mhd_cells_build permutes from src into dst (the
   caller needs distinct src/dst buffers for exactly these, itype last). */
int mhd_sorted_field_count(void);
const char* mhd_sorted_field_name(int32_t i);

/* Creates a context for up to n_max particles on the current CUDA device.
   Replaces PySPH's solver set-up of the generated kernels
   (MHDScheme.configure_solver, src/scheme.py:46-59). */
int mhd_ctx_create(const MhdParams* params, int64_t n_max, void** ctx);
int mhd_ctx_destroy(void* ctx);
int mhd_ctx_set_params(void* ctx, const MhdParams* params);
const char* mhd_last_error(void* ctx);
/* Number of this library's kernels launched through the context so far. */
int64_t mhd_launch_count(void* ctx);

/* Per-family device time with CUDA events recorded on the launching stream
   around each launch.  mhd_timing_read synchronises, returns the totals
   since the previous read (ms[MHD_TIMING_KINDS], launches[...]) and resets. */
int mhd_timing_enable(void* ctx, int32_t enable);
int mhd_timing_read(void* ctx, double* ms, int64_t* launches);

/* Measured FMA throughput (FLOP/s, FMA = 2 flops) of the FP64 or FP32 SIMT
   pipe on the current device: the compute roof of the pair passes. */
int mhd_probe_fma_peak(int32_t precision, double* flops_per_second, void* stream);

/* Neighbour pairs (self included) and distance tests of the force passes
   run with timing enabled (mhd_timing_enable) since the previous call
   (synchronises, then resets). */
int mhd_pair_counts(void* ctx, int64_t* pairs, int64_t* candidates, void* stream);

/* Particles whose neighbour lists were built or carried over across a sort
   (`listed`), and of those the lists built afresh (`rebuilt`), over all
   list builds since the previous call (synchronises, then resets).  No
   reference counterpart: PySPH rebuilds every neighbour structure on every
   update (its NNPS), which this library does when MHD_LIST_REUSE=0. */
int mhd_list_counts(void* ctx, int64_t* listed, int64_t* rebuilt, void* stream);

/* ---- neighbour search ----
   Sort the particles of `src` by cell of the neighbour grid (Morton-free
   linear cell order, stable LSD radix sort + prefix scan) and write the
   permuted persistent fields into `dst`: PySPH's NNPS update plus
   Solver.reorder_particles (src/solver.py:30-32).  `src` and `dst` may not
   alias.  The grid is kept in the context for the passes that follow. */
int mhd_cells_build(void* ctx, const MhdState* src, MhdState* dst, int64_t n, void* stream);

/* Neighbour count of every particle of `s` (device int32[n]) under the
   exact FP64 rule of the neighbour search -- r2 < (R h_i)^2 or
   r2 < (R h_j)^2, minimum image, self included -- with the current h; the
   check that the compacted lists hold PySPH's neighbour sets
   (src/application.py:63-78).  Needs a preceding mhd_cells_build. */
int mhd_neighbour_counts(void* ctx, MhdState* s, int64_t n, int32_t* counts, void* stream);

/* ---- equation groups (src/scheme.py:71-80) ----
   G1, DensityIteration with its iterated Group (src/equations.py:14-94,
   src/scheme.py:71); neighbours follow the current h in every pass. */
int mhd_density_iterate(void* ctx, MhdState* s, int64_t n, MhdRhsStats* stats, void* stream);
/* G2-G10 fused: SmoothingLengthRateFromDensityRelation, DensityFromSmoothingLength,
   IdealGasEOS, CullenDehnenAlphaDiagnostics, StrainDiagnostics,
   MagneticStateReconstruction, MHDAccelerations,
   SmoothingLengthRateFromForceDivergence, MagneticStressAccelerations,
   MagneticStateRates, EnergyLimiter, DivBCorrection, AdaptiveTimestep
   (src/equations.py:97-624) as one neighbour pass with prologue/epilogue. */
int mhd_force_pass(void* ctx, MhdState* s, int64_t n, void* stream);
/* One full right-hand side on `src` (grid build into `dst`, G1..G10 on
   `dst`): PySPH's Integrator.compute_accelerations. */
int mhd_rhs(void* ctx, const MhdState* src, MhdState* dst, int64_t n, MhdRhsStats* stats, void* stream);

/* ---- timestep (src/solver.py:40,61; src/equations.py:570-585) ----
   dt = min_i dt_adapt_i, clipped so that t + dt <= tf.  Writes dt to the
   device scalar the corrector reads and to *dt_host (synchronising) when
   dt_host is non-null. */
int mhd_timestep(void* ctx, const MhdState* s, int64_t n, double t, double* dt_host, void* stream);

/* Allocation-free timestep reduction.  No counterpart in the reference: it
   serves callers that cannot call cudaMalloc (code being captured into a
   CUDA graph, embedders whose allocator policy forbids library-owned device
   memory, real-time loops).  It needs no context: dt_adapt (device, n
   values) in, *dt_out (device) = min_i dt_adapt_i clipped so t + dt <= tf, or
   NaN if some dt_adapt is non-positive or non-finite.  Scratch is a
   file-scope __device__ array (32 KiB) kept on every GPU that loads the
   library; n above MHD_NOALLOC_MAX_N is rejected with MHD_ERR_INVALID.  The
   first call on a device looks up the array's device address (make it before
   any stream capture; the address is kept, so do not call again on a device
   after cudaDeviceReset); calls that overlap on the GPU race on the shared
   array. */
#define MHD_NOALLOC_MAX_N 67108864
int mhd_timestep_noalloc(const double* dt_adapt, int64_t n, double t, double tf, double* dt_out, void* stream);

/* Device clock of the fused loop: t = start of the current step, dt = its
   size.  mhd_corrector_predictor with device dt advances it. */
int mhd_clock_set(void* ctx, double t, double dt, void* stream);
int mhd_clock_get(void* ctx, double* t, double* dt, void* stream); /* synchronising */

/* ---- integrator (MHDStep, src/integrator.py:12-82) ----
   The literal stages: every property the reference writes is written. */
int mhd_step_initialize(void* ctx, MhdState* s, int64_t n, void* stream);
int mhd_step_stage1(void* ctx, MhdState* s, int64_t n, double dt, void* stream);
int mhd_step_stage2(void* ctx, MhdState* s, int64_t n, double dt, void* stream);
/* Fused corrector-predictor: stage2 of the current step with dt_cur, then
   initialize + stage1 of the next with dt_next, one pass over HBM.
   mode: 1 = stage2 only, 2 = initialize+stage1 only, 3 = both.
   A negative dt reads the value mhd_timestep left on the device.  The
   x0..psi0 copies are not materialised (they are consumed in registers). */
int mhd_corrector_predictor(void* ctx, MhdState* s, int64_t n, int32_t mode, double dt_cur, double dt_next,
                            void* stream);

/* One PEC step (PECIntegrator.one_timestep order: initialize, stage1, wrap,
   RHS, stage2, wrap) on `src`; the result is in `dst` (particle order
   changes with the neighbour sort).  dt < 0 uses the device dt. */
int mhd_step(void* ctx, MhdState* src, MhdState* dst, int64_t n, double dt, MhdRhsStats* stats, void* stream);

/* ---- batched form and captured runs ----
   No counterpart in the reference, which advances one case per Application
   (src/application.py) with its solver loop (src/solver.py:35-76). */

/* Declares the first start[n_inst] particles of the context as n_inst
   independent instances stored one after another: instance k holds
   [start[k], start[k+1]) (start[0] = 0, every instance non-empty).  The
   instances share the parameters and the domain; each keeps its own grid,
   clock and timestep, and its results equal a run of the instance alone
   while its grid stays within capacity.  Plans every grid from `s`
   (synchronising) and fixes its cell capacity at ceil(cells * cell_headroom)
   per axis (1 <= cell_headroom <= 16); from then on grids are planned on the
   device within those capacities (coarser cells when h shrinks further),
   without host synchronisation.  n_inst = 1 puts a single simulation on the
   device planner.  Resets every clock to t = dt = 0 and drops captured
   runs. */
int mhd_ctx_set_instances(void* ctx, const MhdState* s, int32_t n_inst, const int64_t* start, double cell_headroom,
                          void* stream);
int32_t mhd_instance_count(void* ctx);

/* Clocks of all instances, t[n_inst] and dt[n_inst] in host memory
   (synchronising).  mhd_clock_set / mhd_clock_get address instance 0. */
int mhd_clock_set_all(void* ctx, const double* t, const double* dt, void* stream);
int mhd_clock_get_all(void* ctx, double* t, double* dt, void* stream);

/* `steps` fused PEC steps on the device clocks: per step the right-hand side
   from the current state into the other buffer set, the per-instance
   timestep (tf clip per instance), then the fused corrector-predictor
   (mode 1 on the last step when `finish`, else 3).  The state starts in
   `a`; the sorted fields ping-pong between `a` and `b` (mhd_cells_build's
   src and dst), so after an odd number of steps it is in `b`.
   capture = 0 runs step by step with the host-checked density iteration
   and list rebuilds of mhd_rhs.  capture = 1 (after mhd_ctx_set_instances)
   captures the steps once into a CUDA graph -- cached per buffers, step
   count and context configuration -- and launches them as one graph: each
   density iteration runs its first min_iter passes, then a conditional
   while node repeats one pass until the group stops (the on-device stop
   test) or 256 passes ran, and nothing synchronises until the run ends.  A
   captured run whose lists stopped covering an h (or overflowed), or whose
   density iteration had not stopped after its captured passes, returns
   MHD_ERR_RELIST: its state is invalid; restore the input state and clocks
   and replay the run with capture = 0. */
int mhd_advance(void* ctx, MhdState* a, MhdState* b, int64_t n, int32_t steps, int32_t finish, int32_t capture,
                void* stream);

/* Autotuner hook: cells >= list cut-off / stencil wide (stencil 1..3) and the
   force pass's launch shape (0..3: 128x2, 128x3, 128x4, 256x2 threads x
   minimum resident blocks; -1 = per-precision default).  Drops captured
   runs; a batched context re-plans its capacities at the next
   mhd_ctx_set_instances. */
int mhd_ctx_tune(void* ctx, int32_t stencil, int32_t force_shape);

/* ---- derivative form (forward mode) ----
   No counterpart in the reference.  The literal PEC step (MHDStep with the
   ten groups of src/scheme.py:66-81, single density pass) on dual numbers:
   every double* of the MhdState points to n records of
   (1 + MHD_TANGENT_DIRS) doubles {value, d/dp_1, ..., d/dp_DIRS}, p being
   the caller's parameters (seeded through the initial state and through
   alpha_max).  The context's parameters must have iterate = 0.  The step
   size is a plain value: the adaptive rule is not differentiated (frozen
   dt).  Neighbours: a cell grid over each pass's positions and smoothing
   lengths with the exact rule (any n <= the context's n_max; the
   particles keep the caller's order).  alpha_max: host array of
   1 + MHD_TANGENT_DIRS doubles (value and derivatives), or null for the
   context's value. */
#define MHD_TANGENT_DIRS 2
int mhd_tangent_dirs(void);
/* src/application.py:99-108: Bevol = B / rho, psi = 0, predicted copies. */
int mhd_tangent_sync(void* ctx, MhdState* s, int64_t n, void* stream);
/* One right-hand side (Integrator.compute_accelerations). */
int mhd_tangent_rhs(void* ctx, MhdState* s, int64_t n, const double* alpha_max, void* stream);
/* One PEC step with step size dt (PECIntegrator.one_timestep). */
int mhd_tangent_step(void* ctx, MhdState* s, int64_t n, double dt, const double* alpha_max, void* stream);
/* sum_i m_i |B_i|^2 / (2 mu0 rho_i) and its derivatives into
   energy[1 + MHD_TANGENT_DIRS] (host; synchronising). */
int mhd_tangent_magnetic_energy(void* ctx, const MhdState* s, int64_t n, double* energy, void* stream);

/* ---- derivative form (reverse mode, checkpointed) ----
   No counterpart in the reference.  L = sum_i m_i |B_i|^2 / (2 mu0 rho_i)
   after `steps` literal PEC steps from the state in `s` (plain FP64 fields;
   single density pass, n <= the context's n_max), and its adjoint:
   lambda0 = dL/dS_0 over the MHD_ADJOINT_FIELDS step-state fields
   (mhd_adjoint_field_name order, field-major, device, fields x n) and
   dL/d alpha_max through the steps.  The step sizes are frozen: on input
   dts[k] >= 0 is used as given; a negative dts[k] (k >= 1) is replaced by
   the adaptive rule on the values of the state before step k (clipped to
   tf), so the forward call returns the sequence it used.  `checkpoints`:
   device array of (ceil(steps / every) + 1) x fields x n doubles; the
   forward call keeps the state every `every` steps there, the backward
   call re-runs each segment from its checkpoint with a tape and walks it
   backwards.  Local Jacobians come from dual-number evaluation of the same
   step functions; the energy limiter's time scale is frozen like dt. */
#define MHD_ADJOINT_FIELDS 24
int mhd_adjoint_field_count(void);
const char* mhd_adjoint_field_name(int32_t k);
int mhd_adjoint_forward(void* ctx, const MhdState* s, int64_t n, int32_t steps, double* dts, int32_t every,
                        double* checkpoints, double* loss, void* stream);
int mhd_adjoint_backward(void* ctx, const MhdState* s, int64_t n, int32_t steps, const double* dts, int32_t every,
                         const double* checkpoints, double* lambda0, double* dloss_dalpha_max, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MHD_B200_H */
