/*
 * erosion_b200 — C ABI of the B200 Stokes boundary-integral library.
 *
 * The first three entry points keep the names, argument order and by-reference
 * convention of the Fortran routines that quaife/erosion's Julia package binds
 * with `ccall` from `libstokes.so`, so the library drops in for that file.
 * Integer arguments are int64 (Julia's `Ref{Int}`); every array is caller
 * owned host memory and is final when the call returns.  Calls are serialised
 * by an internal mutex; the library keeps its device buffers between calls.
 *
 * Unknown layout (the reference's, stokesSolver.f:469-470, :636-660, :993-995):
 *   [ wall sigma_x (nouter) | wall sigma_y (nouter) |
 *     per body b: sigma_x (npts), sigma_y (npts) |
 *     per body b: stokeslet_x, stokeslet_y, rotlet ]
 *   length 2*nouter + 2*npts*nbods + 3*nbods.
 *
 * Errors: the reference has no error channel (its subroutines return nothing
 * and ignore DGMRES's IERR).  These entry points keep `void` and record an
 * outcome readable through erosion_last_status()/erosion_last_error().
 */
#ifndef EROSION_B200_H
#define EROSION_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum {
  EROSION_OK = 0,            /* converged / completed                          */
  EROSION_MAXITER = 1,       /* GMRES reached maxl without meeting tol         */
  EROSION_BREAKDOWN = 2,     /* GMRES stalled, or a NaN/Inf appeared           */
  EROSION_BAD_INPUT = 3,     /* sizes, geometry or arguments rejected          */
  EROSION_CUDA_ERROR = 4,    /* a CUDA call failed                             */
  EROSION_NO_DEVICE = 5      /* no usable CUDA device                          */
};

/* Replaces stokesSolver (ErosionPackage/fortran_code/stokesSolver.f:1-131),
 * bound at ErosionPackage/src/DensityStress.jl:48-51.  Builds the geometry and
 * right-hand side, then solves the double-layer boundary integral equation by
 * unrestarted GMRES to relative residual 1e-8.  density is the initial guess
 * on entry and the solution on exit; nits receives the GMRES iterations.
 * ifmm is accepted for ABI compatibility: the far field is an exact direct sum.
 * ibary = 1 applies the barycentric near-singular corrections with the
 * selection rules of matvec_DLP_fmmbary (ifmm = 1) or to every pair of
 * distinct curves as matvec_DLP_bary does (ifmm = 0); ibary = 0 is the
 * trapezoid rule everywhere.  ibc = 0 parabolic, 1 uniform wall velocity. */
void stokessolver_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter,
                   const int64_t* ifmm, const int64_t* ibary, const int64_t* ibc,
                   const int64_t* maxl, const double* xx, const double* yy,
                   double* density, int64_t* nits);

/* Replaces computeShearStress (stokesSolver.f:3002-3096), bound at
 * DensityStress.jl:195-198.  tau[npts*nbods] receives the wall shear stress on
 * every body node; ibary = 1 evaluates other curves' contributions with the
 * barycentric formulas (deformation_on_boundary), 0 with the trapezoid rule
 * (deformation_on_boundary_trap). */
void computeshearstress_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter,
                         const double* xx, const double* yy, const double* density,
                         const int64_t* ibary, double* tau);

/* Replaces computeQoiTargets (stokesSolver.f:3099-3323), bound at
 * DensityStress.jl:81-86: velocity, pressure and vorticity at ntargets points;
 * targets classified inside a body are zeroed. */
void computeqoitargets_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter,
                        const int64_t* ibary, const double* xx, const double* yy,
                        const double* density, const int64_t* ntargets,
                        const double* xtar, const double* ytar, double* utar,
                        double* vtar, double* ptar, double* vortar);

/* Outcome (EROSION_* code) and message of the last entry-point call made by
 * the calling thread; each thread has its own.  The string stays valid until
 * that thread's next call into the library. */
int erosion_last_status(void);
const char* erosion_last_error(void);

/* ------------------------------------------------------------------------
 * Extended interface (no counterpart in the reference's ABI): the knobs the
 * reference hard-codes, precision mode, device-resident operands, and the
 * pieces the parity tests compare one by one.
 * ------------------------------------------------------------------------ */
typedef struct {
  double wall_a;        /* wall semi-axis in x (reference 3, stokesSolver.f:189)   */
  double wall_b;        /* wall semi-axis in y (reference 1, :190); also the channel
                           half-height used by the near-wall tests (:717-719, 769)
                           and by the parabolic wall data (:398-404)               */
  double wall_order;    /* superellipse order (reference 8, :186)                  */
  double tol;           /* GMRES relative residual (reference 1e-8, :482)          */
  int64_t maxl;         /* iteration cap (reference ParamSet maxl = 8000)          */
  int32_t ibary;        /* 1 barycentric near field, 0 trapezoid                   */
  int32_t ifmm;         /* with ibary=1: 1 fmmbary selection rules, 0 all pairs    */
  int32_t ibc;          /* 0 parabolic, 1 uniform wall velocity                    */
  int32_t precision;    /* 0 FP64; 1 mixed: FP32 far field (FP64 accumulation) inside FP64
                           iterative refinement to the same tol                    */
  int32_t rhs_mode;     /* 0 production data; 1 the reference's manufactured
                           stokeslet (1,2) + rotlet 3 at the origin (:220-257);
                           2 homogeneous (all-zero) data                           */
  int32_t true_residual;/* 1: also evaluate ||b - A x||/||b|| with the FP64 operator */
  int32_t precond;      /* 0: none (the reference: JPRE = 0, stokesSolver.f:490);
                           1: block Gauss-Seidel right preconditioner - wall block
                           -2 I, wall-to-body coupling, exact inverse of every
                           body's (2 npts + 3) block in FP32; 2: as 1 after a
                           coarse correction on every body's rigid-motion
                           densities and stokeslet/rotlet unknowns (fewer
                           iterations at 10-30 bodies, many more at 100-400:
                           experimental).  The stopping test is unchanged:
                           ||b - A x||/||b|| <= tol                                 */
  int32_t learned_guess; /* 1: also try the learned initial guess (the network of
                           erosion_lw_train) and start GMRES from whichever of
                           {learned, supplied density, zero} has the smallest FP64
                           residual                                               */
  int32_t fast_fp64;    /* mixed mode: 1 (default) applies the fast FP64 far field
                           (reciprocal to ~1e-12 instead of FP64 rounding) while the
                           residual is above relax_tol and to the wall's sources
                           after, 0 the accurate one; true residuals always use
                           the accurate one                                       */
  int32_t precond_refresh; /* block preconditioner: 0 or 1 rebuilds the body blocks
                           at every set-up; k > 1 keeps the previous inverses for up
                           to k - 1 further set-ups of the same size (consecutive
                           stages and time steps of an erosion run, whose shapes
                           change little).  Flexible GMRES meets the same
                           tolerance with any fixed preconditioner; only the
                           iteration count can change                            */
  int32_t stress_all_bary; /* shear stress with ibary = 1: 0 (default) evaluates
                           another curve by the barycentric formulas only at body
                           nodes within 12 of its node spacings and by the
                           trapezoid rule beyond (where the two agree to
                           rounding); 1 evaluates every pair barycentrically, as
                           deformation_on_boundary does                          */
  int32_t sweep_decades;/* mixed mode: 0 runs the first refinement sweep to tol;
                           k > 0 (default 5) stops every sweep once its estimate has
                           fallen 10^-k below the residual it started from (a
                           sweep whose stopping point would lie within a decade
                           of tol runs to tol), and the next sweep restarts from
                           the true FP64 residual.  The error an FP32 operator leaves in a sweep
                           scales with the residual it starts from, so with
                           relax_tol >= 1 (FP32 far field from the first
                           iteration) the sweeps stay accurate while no FP64
                           far-field sum is needed outside the true residuals      */
  double relax_tol;     /* mixed mode: GMRES applies the FP32 far field once its
                           residual estimate is at or below relax_tol ||b||
                           (default 1: from the first iteration, the refinement
                           sweeps restoring FP64 accuracy); 0 selects 1e5 tol  */
} erosion_params;

/* Fills the reference's defaults: wall (3, 1, 8), tol 1e-8, maxl 8000, ibary 1,
 * ifmm 1, ibc 1, FP64, production right-hand side; for the mixed mode
 * (precision 1): fast_fp64 1, relax_tol 1, sweep_decades 5. */
void erosion_default_params(erosion_params* p);

/* Solve statistics of the last erosion_solve / stokessolver_ call. */
typedef struct {
  int64_t iterations;       /* GMRES iterations (sum over refinement sweeps)       */
  int64_t matvecs;          /* operator applications, all precisions               */
  int64_t matvecs_fp32;     /* of which with the FP32 far field                    */
  int64_t sweeps;           /* outer refinement sweeps (1 for FP64)                */
  double est_residual;      /* GMRES estimate rho/||b|| at exit                    */
  double true_residual;     /* ||b - A x||/||b|| (FP64 operator) when requested    */
  double ms_total;          /* device time of the solve                            */
  double ms_far;            /* device time inside the FP64 far-field kernel        */
  int64_t far_launches;     /* FP64 far-field kernel launches                      */
  int64_t near_pairs;       /* (target node, source curve) barycentric pairs       */
  double ms_far32;          /* device time inside the FP32 far-field kernel        */
  int64_t far32_launches;   /* FP32 far-field kernel launches                      */
  int64_t far32_pairs;      /* source-target pairs per FP32 far-field launch       */
  double true_residual_checks; /* FP64 true-residual evaluations (mixed mode)      */
  double sweep_residual[8]; /* true residual after each refinement sweep          */
  int64_t sweep_iterations[8]; /* GMRES iterations of each sweep                   */
  int64_t floor_accepted;   /* 1: refinement stopped at the true-residual rounding
                               floor (above tol) instead of below tol            */
  int64_t guess_used;       /* initial guess: 0 zero, 1 supplied/previous, 2 learned */
  double guess_residual[3]; /* ||b - A x0||/||b|| of each candidate (-1: not tried) */
  int64_t far64_pairs;      /* source-target pairs per full FP64 far-field launch   */
  double ms_farw;           /* mixed operator: device time of the FP64 wall-source
                               far-field launches                                  */
  int64_t farw_launches;    /* their count                                         */
  int64_t farw_pairs;       /* wall-source pairs per such launch                   */
  int64_t precond_active;   /* 1: the block preconditioner was applied             */
  int64_t precond_singular_blocks; /* bodies whose FP32 block had a zero pivot; each
                               such body is left unpreconditioned (identity block)
                               while the others keep theirs                        */
  double ms_setup;          /* host wall time of the last geometry set-up: node
                               geometry, near lists, far-field tiles, launch shapes
                               and the preconditioner                              */
  double ms_precond_setup;  /* device time of the preconditioner's block assembly
                               and inversion within that set-up                    */
  double ms_far64f;         /* mixed operator: device time of the fast FP64 far-field
                               launches (pairs per launch: far64_pairs)            */
  int64_t far64f_launches;  /* their count                                         */
} erosion_solve_stats;

/* Host-array solve.  density: initial guess in, solution out. */
int erosion_solve(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                  const double* xx, const double* yy, double* density, int64_t* nits);

/* Same with device pointers (inputs resident in HBM; density updated in place). */
int erosion_solve_device(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                         const double* d_xx, const double* d_yy, double* d_density, int64_t* nits);

void erosion_get_solve_stats(erosion_solve_stats* s);

/* Ensemble solve (extended API; the reference solves one geometry per call).
 * nbatch independent geometries, each with its own npts[g], nbods[g],
 * nouter[g]; xx, yy hold every geometry's body nodes one after another
 * (npts[g]*nbods[g] each), density every geometry's unknowns one after
 * another (2*npts*nbods + 3*nbods + 2*nouter each; initial guess in, solution
 * out), nits[g] receives each geometry's GMRES iterations.  Every geometry is
 * solved with the method erosion_solve applies for the same parameters (one
 * erosion_params for all); the geometries advance together, one Arnoldi
 * iteration per round: the far field of all of them is one persistent launch
 * per precision and the rest of a round replays one captured CUDA graph.
 * Returns EROSION_OK or the first non-OK status of a geometry. */
int erosion_solve_batch(const erosion_params* p, int32_t nbatch, const int64_t* npts, const int64_t* nbods,
                        const int64_t* nouter, const double* xx, const double* yy, double* density, int64_t* nits);

typedef struct {
  int64_t geometries;
  int64_t rounds;            /* lockstep Arnoldi rounds (graph replays)            */
  int64_t iterations;        /* GMRES iterations summed over the geometries        */
  int64_t graph_captures;    /* round graphs captured (pattern or buffer changes)   */
  double ms_total;           /* device time of the whole ensemble solve            */
  double pairs64_per_round;  /* FP64 far-field pairs of the last captured round     */
  double pairs32_per_round;  /* FP32 far-field pairs of the last captured round     */
  double pairs64_total;      /* FP64 far-field pairs over all rounds               */
  double pairs32_total;      /* FP32 far-field pairs over all rounds               */
  double max_true_residual;  /* largest final residual over the geometries         */
  int64_t shape64, shape32;  /* ensemble launch shapes (indices as erosion_get_far_shapes) */
  float tune_ms[8];          /* timed candidates: [0..3] FP64, [4..7] FP32 (0 = not timed) */
  double setup_host_ms;      /* host wall time of the members' set-ups (geometry,
                                near lists, tiles, preconditioners, initial residuals),
                                run on a pool of host threads                      */
} erosion_batch_stats;

void erosion_get_batch_stats(erosion_batch_stats* s);

/* One application of the boundary operator (host arrays) — the reference's
 * matvec_DLP_fmmbary / matvec_DLP_bary / matvec_DLP depending on ibary, ifmm;
 * precision = 1 applies the mixed-precision operator (FP32 far field from body
 * sources to the nodes of other curves, FP64 elsewhere, the wall's sources
 * included); precision = 2 the fast FP64 operator of the mixed solve's early
 * iterations (FP64 with a far-field reciprocal good to ~1e-12). */
int erosion_matvec(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                   const double* xx, const double* yy, const double* density, double* vel);

/* The trapezoid-rule boundary operator (erosion_matvec with ibary = 0 and
 * precision = 0) for callers that cannot allocate GPU memory — a caller whose
 * runtime owns all device memory or whose device memory is reserved up front,
 * running its own iterative solver around this operator.  No counterpart in
 * the reference (an addition of this library).  Inputs and output are DEVICE
 * pointers (d_xx, d_yy: [npts*nbods] body nodes; d_den, d_vel: [2*npts*nbods
 * + 3*nbods + 2*nouter]); the kernels run on 'stream' (a cudaStream_t, NULL
 * = the legacy default stream) and the call returns without waiting for them.
 * It allocates no device memory: every intermediate lives in one fixed 24 MiB
 * array that is part of the library on every GPU that loads it, which limits
 * the size to nouter <= 4096, npts <= 512, nbods <= 128 and nouter +
 * npts*nbods <= 32768 (larger sizes, ibary != 0 or precision != 0 return
 * EROSION_BAD_INPUT).  The first call on a device looks up that array's
 * device address; make it before capturing any stream.  Calls share the
 * array: calls whose kernels overlap on the GPU race and must be ordered by
 * the caller.  Inputs are not checked for finiteness or for bodies inside the
 * wall.  A CUDA error already pending on the calling thread when the call
 * starts is reported as EROSION_CUDA_ERROR (nothing is launched) and left
 * pending for the caller.  The call takes no library lock: it never waits on
 * the host for another thread's call into the library. */
int erosion_matvec_noalloc(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                           const double* d_xx, const double* d_yy, const double* d_den, double* d_vel,
                           void* stream);

/* Pressure on the body boundaries for a given density: replaces
 * computePressure (stokesSolver.f:4644-4885), which PostProcess.jl:103-113
 * (compute_pressure) binds as `computepressure_`.  Wall sources and other
 * bodies by the trapezoid rule, a body's own nodes by odd-even quadrature on
 * the density less its value at the target, plus the jump and the stokeslet
 * pressure.  pressure: [npts*nbods]. */
void computepressure_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter, const double* xx,
                      const double* yy, const double* density, double* pressure);

/* Same with the extended parameters (wall shape); returns a status. */
int erosion_pressure(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                     const double* yy, const double* density, double* pressure);

/* The right-hand side of bd_condition (stokesSolver.f:208-314). */
int erosion_rhs(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                const double* xx, const double* yy, double* rhs);

/* Geometry as compute_derivs/inner_geometry/outer_geometry build it; any
 * output may be NULL.  Body arrays npts*nbods, per-body nbods, wall nouter. */
int erosion_geometry(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                     const double* xx, const double* yy, double* px, double* py, double* cur,
                     double* speed, double* cx, double* cy, double* xo, double* yo,
                     double* px0, double* py0, double* cur0, double* speed0);

/* Shear stress (host arrays); E, if not NULL, receives E11, E12, E22 (3*npts*nbods). */
int erosion_shear_stress(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                         const double* xx, const double* yy, const double* density,
                         double* tau, double* E);

int erosion_shear_stress_device(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                                const double* d_xx, const double* d_yy, const double* d_density,
                                double* d_tau);

/* Velocity, pressure, vorticity at targets (host arrays). */
int erosion_qoi_targets(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                        const double* xx, const double* yy, const double* density,
                        int64_t ntargets, const double* xtar, const double* ytar,
                        double* utar, double* vtar, double* ptar, double* vortar);

/* Near-pair bookkeeping of the last geometry set up: the integer wall length
 * scale 'lw' of matvec_DLP_fmmbary (an INTEGER there, :705-709), the number
 * of near-wall bodies (written to wall_bodies, capacity nbods) and the total
 * number of barycentric (target node, source curve) pairs. */
int64_t erosion_near_info(int64_t* lw, int64_t* wall_bodies, int64_t* near_pairs);

/* ------------------------------------------------------------------------
 * Erosion time step (theta-L form).  Replaces the Julia time loop's step
 * rungekutta2 (ErosionPackage/src/TimeStepping.jl:189-202) with everything it
 * calls: getxy (ThetaLen.jl:92-101), getstress! (DensityStress.jl:23-36,
 * i.e. the solve, the optional fixed-pressure-drop rescale and the shear
 * stress), getderivs (TimeStepping.jl:63-95), delete_indices (:103-126) and
 * timestep! (:130-185), all on the device.
 * ------------------------------------------------------------------------ */
typedef struct {
  double dt;            /* time step (ParamSet dt, ThetaLen.jl:27)               */
  double epsilon;       /* curvature smoothing (epsfac/npts)                     */
  double sigma;         /* stress smoothing (sigfac/npts)                        */
  int32_t fixarea;      /* ParamSet fixarea                                      */
  int32_t fixpdrop;     /* ParamSet fixpdrop: rescale the density so that the
                           pressure drop between x = -2 and x = 2 is 8
                           (DensityStress.jl:129-167; meaningful for walls
                           that contain those slices)                            */
  int32_t warm_start;   /* 0: zero initial guess (the reference,
                           DensityStress.jl:45); 1: the most recent solve's
                           density (the other stage, half a step back) when
                           the body count is unchanged, each body's rigid part
                           carried to the new nodes; 2: as 1 plus the learned
                           increment, whichever candidate has the smallest
                           residual.  In the mixed or preconditioned solve a
                           guess no better than zero is replaced by zero      */
  int32_t reserved[5];
} erosion_step_params;

/* Fills the ParamSet defaults for npts: dt 1e-3, epsilon 15/npts,
 * sigma 10/npts, fixarea 0, fixpdrop 1, warm_start 0. */
void erosion_default_step_params(erosion_step_params* sp, int64_t npts);

/* Per-step statistics of the last erosion_rk2_step call. */
typedef struct {
  int64_t gmres_iterations[2];  /* per stage                                  */
  int64_t bodies_deleted;
  double ms_solve;              /* device time in the two solves              */
  double ms_stress;             /* device time in the two shear stresses      */
  double ms_thetalen;           /* device time in the theta-L arithmetic      */
  double ms_total;
  double max_residual;          /* largest GMRES estimate at exit             */
  double matau[2];              /* mean smoothed |tau| over bodies, per stage */
  int64_t guess_used[2];        /* initial guess per stage: 0 zero, 1 previous,
                                   2 learned                                  */
  double guess_residual[2];     /* its relative residual ||b - A x0||/||b||   */
  double ms_setup;              /* host wall time of the two geometry set-ups
                                   (included in ms_solve)                     */
  double ms_precond_setup;      /* device time of the two preconditioner
                                   set-ups (included in ms_setup)             */
  int64_t precond_active[2];    /* per stage: 1 when the block preconditioner
                                   was applied                                */
  int64_t precond_singular_blocks[2]; /* per stage: bodies left
                                   unpreconditioned (zero pivot)              */
  int64_t matvecs[2];           /* per stage: operator applications           */
  int64_t matvecs_fp32[2];      /* per stage: of which with the FP32 far field */
} erosion_step_stats;

/* One RK2 step of the theta-L state, host arrays, in place:
 * theta[nbods*npts], len/xsm/ysm[nbods]; *nbods is updated when bodies are
 * deleted and deleted[] (capacity nbods) receives their original indices.
 * *t is advanced by dt. */
int erosion_rk2_step(const erosion_params* p, const erosion_step_params* sp, int64_t npts,
                     int64_t* nbods, int64_t nouter, double* theta, double* len, double* xsm,
                     double* ysm, double* t, int64_t* deleted);

/* Same with the state resident on the device (in place). */
int erosion_rk2_step_device(const erosion_params* p, const erosion_step_params* sp, int64_t npts,
                            int64_t* nbods, int64_t nouter, double* d_theta, double* d_len,
                            double* d_xsm, double* d_ysm, double* t, int64_t* deleted);

void erosion_get_step_stats(erosion_step_stats* s);

/* The density solved in stage `stage` (0 or 1) of the last RK2 step (host
 * array of at least 2*npts*nbods + 3*nbods + 2*nouter entries, the body count
 * after that stage's deletions).  Stage 0 is solved on the state the step
 * started from.  EROSION_BAD_INPUT when there is none (no step yet, or the
 * body count changed after the solve). */
int erosion_get_step_density(int32_t stage, double* density, int64_t capacity);

/* The body node coordinates that density was solved on (npts*nbods each;
 * stage 1's nodes are those of the half-step state, which the caller does
 * not otherwise see). */
int erosion_get_step_nodes(int32_t stage, double* xx, double* yy, int64_t capacity);

/* Drag on the bodies of a theta-L state: replaces drag (PostProcess.jl:131-162)
 * with the shear stress and pressure it calls (compute_stress,
 * compute_pressure: computeshearstress_/computepressure_ semantics with
 * fixpdrop off, i.e. umax = 1).  Host arrays: theta[nbods*npts],
 * len/xsm/ysm[nbods]; density is the solved density of that state (with
 * rotation != 0: of the rotated problem, the bodies turned by xyrot,
 * DensityStress.jl:40).  Per body, ds = L/npts, tangent s = (cos th, sin th)
 * (rotated: (-sin th, cos th)) and inward normal n = (-s_y, s_x) (getns,
 * PostProcess.jl:23-33):
 *   pdrag = sum p n ds,   vdrag = sum tau s ds.
 * drag[4] receives the totals (pdragx, pdragy, vdragx, vdragy) summed in body
 * order; drag_bodies[4*nbods] (optional) the per-body parts; tau_all,
 * atau_all (gaussfilter(|tau|, sigma)) and press_all [npts*nbods] (optional)
 * the DragData arrays. */
int erosion_drag(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* theta,
                 const double* len, const double* xsm, const double* ysm, const double* density, int32_t rotation,
                 double sigma, double* drag, double* drag_bodies, double* tau_all, double* atau_all,
                 double* press_all);

/* Node coordinates of theta-L bodies (getxy, ThetaLen.jl:92-101), host arrays. */
int erosion_getxy(int64_t npts, int64_t nbods, const double* theta, const double* len,
                  const double* xsm, const double* ysm, double* xx, double* yy);

/* The CUDA stream every library kernel is launched on (a cudaStream_t), so a
 * caller can order its own work and events with the library's. */
void* erosion_stream(void);

/* Number of kernels the library has launched since the process started. */
int64_t erosion_launch_count(void);

/* Measured vector FMA throughput of this GPU in TFLOP/s (2 flops per FMA):
 * precision 0 = FP64, 1 = FP32 scalar FMA, 2 = FP32 packed two-lane FMA
 * (sm_100's f32x2 instructions), from a ~10 ms register-resident FMA loop
 * over every SM (the roofline denominator of the pair kernels). */
double erosion_peak_tflops(int32_t precision);

/* Far-field launch shapes (extended API; the reference's FMM has no
 * counterpart).  Each far-field kernel has a list of candidate CTA shapes
 * (threads per CTA x targets per thread x variant); by default an autotuner
 * times every candidate on the geometry at hand the first time a problem of
 * that size is set up (problems above 2e8 node pairs) and keeps the fastest.
 * erosion_set_far_shape(kind, shape) forces candidate 'shape' (kind 0 = the
 * accurate FP64 kernel, 1 = the FP32 kernel, 2 = the fast FP64 kernel of the
 * mixed solve's early iterations) from the next set-up on; shape = -1
 * returns to the autotuner.  Returns EROSION_BAD_INPUT for an unknown kind
 * or shape. */
int erosion_set_far_shape(int32_t kind, int32_t shape);

/* The shapes in use: shape[kind] = candidate index (3 kinds); desc[12*kind +
 * 3*i ..] = (threads, targets per thread, variant) of candidate i
 * (num_shapes[kind] of them, at most 4; capacity 36 entries).  The variant
 * is, for the FP64 kernels, the reciprocal: 1 FP32 estimate + 2
 * Newton-Raphson steps, 3 FP64 estimate + 2 steps (accurate kind), 2 FP32
 * estimate + 1 step, 4 FP64 estimate + 1 step (fast kind); for the FP32
 * kernel the unroll factor of the source loop plus 10 x the resident CTAs
 * per SM it is compiled for (its register budget).  ms[8*kind + i] = the
 * autotuner's time of candidate i in milliseconds (0 when not timed;
 * capacity 24).  Any pointer may be NULL. */
int erosion_get_far_shapes(int32_t* shape, int32_t* desc, float* ms, int32_t* num_shapes);

/* ------------------------------------------------------------------------
 * Learned initial guess (no counterpart in the reference).  A network of
 * 105 -> 256 -> 256 -> 256 -> 37 (GELU, BF16 weights, FP32 accumulation)
 * maps per-body geometry features (68: 32 Fourier shape coefficients, 4
 * position/size terms, 4 per nearest neighbour for 8 neighbours) and the
 * encoding of the body's density increment over the previous time step (37)
 * to the encoding of its increment over the current step.  The encoding of
 * a density is its Fourier modes -8..8 scaled by the body radius and its
 * stokeslet/rotlet strengths (linear in the density).  In an erosion step
 * with warm_start = 2 the guess is the previous step's density plus the
 * decoded prediction, used when its FP64 residual beats the previous
 * density's.
 * ------------------------------------------------------------------------ */
/* Widths: geometry features (68), network input (105), encoding (37). */
int erosion_lw_dims(int32_t* geo, int32_t* in, int32_t* out);
/* Per-body geometry features of a geometry: feat[nbods*68]. */
int erosion_lw_features(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                        const double* xx, const double* yy, float* feat);
/* Per-body encoding of a density (or of a density increment): targ[nbods*37]. */
int erosion_lw_encode(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                      const double* xx, const double* yy, const double* density, float* targ);
/* Density (body entries, wall zero) of per-body targets. */
int erosion_lw_decode(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                      const double* xx, const double* yy, const float* targ, double* density);
/* Initialises the weights (He normal, seeded); erosion_lw_train does this too. */
int erosion_lw_init(uint64_t seed);
int64_t erosion_lw_num_params(void);
int erosion_lw_get_params(float* out);
int erosion_lw_set_params(const float* in);
/* Mean squared error and its gradient with respect to every parameter for
 * rows (x, y) used as given (no standardisation); for checking the backward
 * kernels. */
int erosion_lw_loss_grad(const float* x, const float* y, int64_t nsamples, double* loss, float* grads);
/* Trains from scratch on rows feat[nsamples*105] (geometry features, then the
 * previous increment's encoding) and targ[nsamples*37] (the encoding of the
 * increment that followed): standardisation from the data, then mini-batch
 * Adam. */
int erosion_lw_train(const float* feat, const float* targ, int64_t nsamples, int64_t epochs, int64_t batch,
                     double lr, uint64_t seed, double* final_loss);
/* Targets predicted by the trained network for raw features. */
int erosion_lw_predict(const float* feat, int64_t nsamples, float* out);

/* Releases every device buffer the library holds. */
void erosion_release(void);

#ifdef __cplusplus
}
#endif

#endif /* EROSION_B200_H */
