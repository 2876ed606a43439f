/*
 * mycel_b200 — C ABI of the B200 (sm_100a) implementation of Mycel.Core's FEM + SIMP inner loop.
 *
 * The reference (zmalrobot/mycel, C#/.NET 10) has no FFI today; its seams are the public static entry points
 * TopologyOptimizer.Run and StaticAnalysis.Run plus the kernels they call. Each entry point below names the
 * reference member it replaces (file:line, paths inside the reference project). A C# host binds these with
 * [DllImport("mycel_b200")]; buffers are caller-owned, read or written only during the call (pin them with
 * `fixed`), and all device memory is owned by the library and stays resident between calls.
 *
 * Conventions: every function returns int32_t status (MYCEL_OK = 0). Vectors are box-sized like the
 * reference's: DOF vectors have 3*(nx+1)*(ny+1)*(nz+1) doubles (dof = 3*node + c), element arrays have
 * nx*ny*nz entries (e = ix + nx*(iy + ny*iz)); "active" arrays list active elements in ascending e.
 * Calls on one problem are not re-entrant (the reference serialises solves through FemWorkTeam's lock).
 */
#ifndef MYCEL_B200_H
#define MYCEL_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (reference exception each one maps to) ---- */
#define MYCEL_OK 0
#define MYCEL_E_ARG 1               /* ArgumentException / ArgumentOutOfRangeException */
#define MYCEL_E_UNDERCONSTRAINED 2  /* InvalidOperationException: < 6 fixed DOFs on active nodes (PcgSolver.cs:95-100) */
#define MYCEL_E_NOT_CONVERGED 3     /* InvalidOperationException: "FEM solver did not converge ..." (StaticAnalysis.cs:88-92) */
#define MYCEL_E_BREAKDOWN 4         /* PCG breakdown reported as a non-converged PcgResult (PcgSolver.cs:245-346) */
#define MYCEL_E_CANCELLED 5         /* OperationCanceledException / loop break on cancellation (TopologyOptimizer.cs:169-172) */
#define MYCEL_E_TIMEOUT 6           /* new: a bounded device wait gave up */
#define MYCEL_E_DEVICE 7            /* new: CUDA error */
#define MYCEL_E_OOM 8               /* new: device memory or admission budget exhausted */
#define MYCEL_E_INVALID_OPERATION 9 /* InvalidOperationException (FeModel.AssembleForces: empty patch with force) */

#define MYCEL_PRECISION_FP64 0  /* plain method: FP64 throughout, reproduces the reference's arithmetic */
/* FP32 inner PCG (K·u, Jacobi) inside FP64 iterative refinement. Per problem, a mixed solve may instead run
   the fast FP64 form below: after an FP32 stall, or when the problem's solves have shown the FP32 form needing
   more than 1.5x the fast FP64 form's iterations per decade of residual (second solve probes it, every 16th
   solve re-probes; decided on iteration counts, so deterministic). */
#define MYCEL_PRECISION_MIXED 1
/* FP64 throughout with the factorised cube-element operator (same tolerance test on the exact FP64 residual,
   not bit-exact with the reference's colour-ordered product); also what a stalled mixed solve goes on in */
#define MYCEL_PRECISION_FP64_FACTORED 2
/* FP64 flexible CG on the factorised operator, preconditioned by a geometric multigrid V-cycle in FP32
   (Galerkin coarse operators rebuilt from E at each solve, damped Jacobi smoothing, dense coarsest solve);
   same tolerance test on the exact FP64 residual. Falls back to MYCEL_PRECISION_FP64_FACTORED on a grid
   that does not coarsen (a 1x1x1 grid) or when it does not converge. */
#define MYCEL_PRECISION_FP64_MG 3
/* The multigrid form with the inner iteration in FP32: FP32 flexible CG (FP32 K·u and V-cycle, FP64 dot
   products) wrapped in FP64 iterative refinement (true residual f - K u in FP64 after each 1e-3 drop of the
   recursive one). Goes on in MYCEL_PRECISION_FP64_MG if it stalls or does not converge (and starts there for
   the rest of the problem's solves after a stall), then as MYCEL_PRECISION_FP64_FACTORED. */
#define MYCEL_PRECISION_MIXED_MG 4

typedef struct mycel_ctx mycel_ctx;
typedef struct mycel_problem mycel_problem;
typedef struct mycel_filter mycel_filter;
typedef struct mycel_simp_session mycel_simp_session;

/* GridSpec (Voxelization/GridSpec.cs:11-44); origin does not enter the path. h is float like GridSpec.H. */
typedef struct {
  int32_t nx, ny, nz;
  float h;
} mycel_grid;

/* FeMaterial(E0, Nu, EminRatio) (Fem/FeMaterial.cs:11-16); Emin = E0 * EminRatio. */
typedef struct {
  double e0, nu, emin_ratio;
} mycel_material;

/* LoadCase(SurfacePatch, Vector3 TotalForce) (Fem/LoadCase.cs:10-19; SurfacePatch.cs:25-49). */
typedef struct {
  int32_t n_nodes;
  const int32_t* nodes;
  const double* node_area;
  float force[3];
} mycel_load_case;

typedef struct {
  int64_t total_elements, total_nodes, total_dofs;
  int64_t active_elements, active_nodes, active_fixed_dofs;
  int64_t device_bytes; /* device memory held by the problem */
} mycel_problem_info;

/* PcgResult (Fem/PcgResult.cs:7-14) plus refinement bookkeeping of the mixed form. */
typedef struct {
  int32_t iterations;
  double final_residual;
  int32_t converged;
  double elapsed_ms;
  int32_t refinement_steps; /* mixed form: outer FP64 refinement steps; 0 for FP64 */
  int32_t inner_iterations; /* mixed form: FP32 PCG iterations summed over refinement steps */
  char message[256];
  /* mixed form: iterations of the FP64 PCG that finished a solve whose FP32 inner iteration stalled (a
     refinement cycle longer than 3x all earlier cycles together and than 2000 iterations), broke down or ran
     out of iterations: the solve goes
     on in the fast FP64 form (MYCEL_PRECISION_FP64_FACTORED) from the refined u, then, should that fail too,
     in the plain FP64 PCG. After a stall, later mixed solves of the same problem start in the fast FP64 form
     (inner_iterations 0). For MYCEL_PRECISION_FP64_FACTORED: the plain FP64 PCG's iterations.
     iterations = inner_iterations + fallback_iterations. */
  int32_t fallback_iterations;
} mycel_pcg_result;

/* StaticAnalysisOptions (Fem/StaticAnalysis.cs:8-17). The reference's IPreconditioner option
   (Fem/IPreconditioner.cs:9-20, default JacobiPreconditioner at Fem/StaticAnalysis.cs:74) is carried by
   precision: the FP64 forms and the mixed forms precondition with Jacobi, the MG forms with the geometric
   multigrid; a managed preconditioner has no device counterpart. */
typedef struct {
  double tolerance;        /* default 1e-6 */
  int32_t max_iterations;  /* default 5000 */
  int32_t throw_on_non_convergence; /* default 1 */
  int32_t precision;       /* MYCEL_PRECISION_* */
} mycel_static_options;

/* OptimizerOptions (Optimization/OptimizerOptions.cs:5-26). */
typedef struct {
  double volume_fraction;   /* 0.4 */
  double filter_radius_mm;  /* 2.0 */
  double penal;             /* 3.0 */
  double move_limit;        /* 0.2 */
  int32_t max_iterations;   /* 200 */
  double solver_tolerance_initial; /* 1e-4 */
  double solver_tolerance_final;   /* 1e-6 */
  int32_t solver_max_iterations;   /* 5000 */
  int32_t continuation;     /* 0 */
  int32_t enable_heaviside; /* 0 */
  double rho_min;           /* 1e-3 */
  const uint8_t* passive_mask; /* box-sized or NULL */
  int64_t passive_mask_len;
  int32_t protect_boundary_hinges; /* 1 */
  const float* initial_density;    /* box-sized or active-sized, or NULL */
  int64_t initial_density_len;
  int32_t start_iteration;         /* 1 */
  const double* warm_start_displacements; /* total_dofs or NULL (other lengths are ignored, as in the reference) */
  int64_t warm_start_len;
  int32_t enforce_minimum_filter_radius; /* 1 */
  int32_t precision;                     /* MYCEL_PRECISION_* */
  /* 0: the load cases are summed into one right-hand side (FeModel.AssembleForces, FeModel.cs:263-321; the
     reference's behaviour). 1: load cases kept apart (no counterpart in the reference): each case is solved on
     the shared stiffness from its own warm start, the objective is the sum of the cases' compliances (the
     record's compliance), the sensitivities are summed over the cases in case order, max_displacement is the
     largest over the cases, u is the sum of the cases' displacements, solver_iterations the sum and
     solver_residual the largest over the cases; warm_start_displacements is not used (every case starts from
     zero). With one load case both modes give the same results. */
  int32_t separate_load_cases;
} mycel_simp_options;

/* IterationSnapshot scalars + IterationTimings (Optimization/IterationSnapshot.cs:5-31). */
typedef struct {
  int32_t iteration;
  double compliance, volume_fraction, max_change, grey_level;
  int32_t solver_iterations;
  double solver_residual;
  double max_displacement;
  double solve_ms, sensitivity_ms, filter_ms, update_ms, total_ms;
  int32_t refinement_steps;
} mycel_iter_record;

/* IProgress<IterationSnapshot>.Report: called on the calling thread after every SIMP iteration with the
   record and box-sized float physical/design densities (valid during the call only). */
typedef void (*mycel_progress_fn)(void* user, const mycel_iter_record* rec, const float* physical_density,
                                  const float* design_density);

/* ---- context ---- */
int32_t mycel_version(void);
int32_t mycel_ctx_create(int32_t device, mycel_ctx** out);
int32_t mycel_ctx_destroy(mycel_ctx* ctx);
/* The CUDA stream (cudaStream_t) all work of this context is issued on. */
void* mycel_ctx_stream(mycel_ctx* ctx);
/* Message of the last failed call on this context (thread-local copy valid until the next call). */
const char* mycel_last_error(mycel_ctx* ctx);
/* Kernel launches issued by this context since creation (all of them are this library's own kernels). */
int64_t mycel_ctx_launch_count(mycel_ctx* ctx);
/* Right-hand sides solved through packed launches (mycel_simp_step_many) on this context since creation; no
   counterpart in the reference (a statistic of the packed form). */
int64_t mycel_ctx_packed_count(mycel_ctx* ctx);
/* Live timing of the dominant kernels: when enabled, PCG chunks record CUDA events around one stiffness matvec
   launch per chunk (on the context stream). which = 0: FP32 matvec of the mixed form, 1: FP64 matvec,
   2: FP64 matvec of the fast FP64 and multigrid forms, 3: the multigrid forms' level-1 residual product
   (event-record nodes inside the chunk graph; nodes = that level's nodes). Returns the summed device time, the
   number of timed launches and the nodes / active elements they covered. */
int32_t mycel_ctx_set_profiling(mycel_ctx* ctx, int32_t enable);
/* Device time of one launch of a solver kernel on this problem (no counterpart in the reference): `reps`
   launches back to back in one CUDA graph, as the solver's chunk graphs issue them, timed by CUDA events on the
   context stream after a warm-up launch; which = 0: the FP32 outer matvec of the mixed forms, 3: the multigrid
   level-1 residual product. Uses only work vectors that hold nothing between solves. */
int32_t mycel_problem_kernel_bench(mycel_problem* p, int32_t which, int32_t reps, double* avg_us);
int32_t mycel_ctx_kernel_timing(mycel_ctx* ctx, int32_t which, double* total_ms, int64_t* launches, int64_t* nodes,
                                int64_t* active_elements);
/* Bounded waits of the OC kernel (no counterpart in the reference, whose OC runs on the host). The OC update is
   one persistent kernel whose blocks meet at grid barriers; each wait polls at most max_polls times (about
   64 ns each) and then gives up, the kernel returns and the call reports MYCEL_E_TIMEOUT with the device still
   usable. max_polls = 0 restores the default (about 1 s plus 4 polls per element). unreachable = 1 is for
   testing that failure path: every barrier then waits for one block more than the grid holds, so each wait
   runs out. */
int32_t mycel_ctx_set_oc_wait(mycel_ctx* ctx, int64_t max_polls, int32_t unreachable);

/* ---- problem: FeModel + FemOperator (Fem/FeModel.cs:43-184, Fem/FemOperator.cs:33-108) ----
   element_density: box-sized (default 1.0 when NULL); penal: FeModel.Penal. */
int32_t mycel_problem_create(mycel_ctx* ctx, const mycel_grid* grid, const uint8_t* domain,
                             const mycel_material* material, const int32_t* fixed_dofs, int32_t n_fixed,
                             const mycel_load_case* loads, int32_t n_loads, const double* element_density,
                             double penal, mycel_problem** out);
/* Ends the problem's live SIMP sessions (as mycel_simp_end), then frees the problem; do not use those
   sessions afterwards. */
int32_t mycel_problem_destroy(mycel_problem* p);
int32_t mycel_problem_info_get(mycel_problem* p, mycel_problem_info* out);
/* Tuning of the kernels of one problem (no counterpart in the reference, which has one CPU kernel per step).
   MYCEL_TUNE_MATVEC32: FP32 stiffness matvec of the mixed form; 0 = chosen by timing all variants on first
   use (default), 1 = dense KE rows on the FMA pipe, 2 = dense KE on the tensor cores (tcgen05, 3xTF32),
   3 = factorised cube-element operator (Walsh-Hadamard basis, about 190 flops per element instead of 1152).
   get returns the variant in use (0 while not chosen yet). */
#define MYCEL_TUNE_MATVEC32 1
#define MYCEL_MV32_DENSE 1
#define MYCEL_MV32_TENSOR 2
#define MYCEL_MV32_FACTORED 3
int32_t mycel_problem_set_tuning(mycel_problem* p, int32_t key, int32_t value);
int32_t mycel_problem_get_tuning(mycel_problem* p, int32_t key, int32_t* value);
/* FeModel.AssembleForces (Fem/FeModel.cs:263-321): box-sized nodal forces. */
int32_t mycel_problem_forces(mycel_problem* p, double* f_out);
/* Load cases kept apart (multi-RHS over the shared stiffness; the reference sums its cases, FeModel.cs:267-318).
   mycel_problem_load_cases: the number of load cases given to mycel_problem_create. mycel_problem_case_forces:
   the nodal forces of case k alone (the same arithmetic as AssembleForces on a zero vector). */
int32_t mycel_problem_load_cases(mycel_problem* p, int32_t* n_cases);
int32_t mycel_problem_case_forces(mycel_problem* p, int32_t k, double* f_out);
/* StaticAnalysis.Run (Fem/StaticAnalysis.cs:35-142) for every load case apart, on one stiffness: E, DiagA and
   the solver set-up (the multigrid hierarchy of the MG precisions) are formed once and shared by the cases;
   case k equals mycel_static_solve on the problem holding case k alone. Each case starts from zero.
   u_out: n_cases * total_dofs (case-major); compliance_out, max_displacement_out, res: n_cases each, may be
   NULL. opt->throw_on_non_convergence reports the first case that does not converge. */
int32_t mycel_static_solve_cases(mycel_problem* p, const mycel_static_options* opt, double* u_out,
                                 double* compliance_out, double* max_displacement_out, mycel_pcg_result* res);

/* ---- kernel-level entry points ---- */
/* FemOperator.UpdateDensities (Fem/FemOperator.cs:114-138): E_e = Emin + rho^p (E0-Emin) and DiagA. */
int32_t mycel_update_densities(mycel_problem* p, const double* density_box, double penal);
/* FemOperator.DiagA after AssembleDiagonal (Fem/FemOperator.cs:143-172). */
int32_t mycel_diagonal(mycel_problem* p, double* diag_out);
/* FemOperator.ApplyK (projected=0, Fem/FemOperator.cs:196-243) / ApplyA with xIsAlreadyProjected (projected=1,
   :250-273): y = K(rho) x by node-centric gather in the reference's colour order. precision selects the
   FP64 kernel or the FP32 kernel (x, y converted at the boundary). */
int32_t mycel_apply_k(mycel_problem* p, const double* x, double* y, int32_t projected, int32_t precision);
/* PcgSolver.Solve with JacobiPreconditioner (Fem/PcgSolver.cs:80-370): x is the warm start in, solution out. */
int32_t mycel_pcg_solve(mycel_problem* p, const double* b, double* x, double tol, int32_t max_iterations,
                        int32_t precision, mycel_pcg_result* res);
/* StaticAnalysis.Run (Fem/StaticAnalysis.cs:35-142). warm_start may be NULL; a non-NULL warm_start whose
   length differs from total_dofs is MYCEL_E_ARG (:62-67). reactions_out / von_mises_out may be NULL. */
int32_t mycel_static_solve(mycel_problem* p, const mycel_static_options* opt, const double* warm_start,
                           int64_t warm_start_len, double* u_out, double* reactions_out, double* von_mises_out,
                           double* compliance_out, double* max_displacement_out, mycel_pcg_result* res);
/* StaticAnalysis.AverageElementToNode (Fem/StaticAnalysis.cs:222-268): nodal_out[node] = mean of
   element_scalar over the problem's active elements meeting at the node (0 where none does), summed in the
   reference's element order. len must equal the element count (else MYCEL_E_ARG with the reference's text). */
int32_t mycel_average_element_to_node(mycel_problem* p, const double* element_scalar, int64_t len,
                                      double* nodal_out);

/* Math.Pow as the kernels evaluate it (FemOperator.cs:100,133 E_e = Emin + Math.Pow(rho, p)(E0 - Emin);
   SensitivityAnalysis.cs:93-95 p Math.Pow(rho, p - 1) dE): the host C library's pow (GNU libc 2.28+ algorithm)
   with its rounding sequence, so the device returns the library's bits. out[i] = x[i]^y[i] (y_len == n) or
   x[i]^y[0] (y_len == 1); host buffers. */
int32_t mycel_pow(mycel_ctx* ctx, int64_t n, const double* x, const double* y, int64_t y_len, double* out);

/* DensityFilter (Optimization/DensityFilter.cs:34-199) over the problem's active elements, radius in elements. */
int32_t mycel_filter_create(mycel_problem* p, double rmin, mycel_filter** out);
int32_t mycel_filter_destroy(mycel_filter* f);
/* ApplyFilter (DensityFilter.cs:205-251), ApplySensitivityFilter (:257-303); active-indexed in/out. */
int32_t mycel_filter_apply(mycel_filter* f, const double* in_active, double* out_active);
int32_t mycel_filter_adjoint(mycel_filter* f, const double* in_active, double* out_active);
/* DensityFilter.S (:187-198). */
int32_t mycel_filter_s(mycel_filter* f, double* s_active);

/* SensitivityAnalysis.ComputeComplianceSensitivities (Optimization/SensitivityAnalysis.cs:13-146). */
int32_t mycel_sensitivities(mycel_problem* p, const double* u, const double* rho_phys_active, double penal,
                            double* dc_active);
/* OcOptimizer.Update (Optimization/OcOptimizer.cs:12-132); passive may be NULL; rho_new may alias rho. */
int32_t mycel_oc_update(mycel_ctx* ctx, int32_t n, const double* rho, const double* dc, const double* s,
                        const uint8_t* passive, double* rho_new, double target_volume_fraction, double move_limit,
                        double rho_min, double lambda_guess, int32_t max_bisection_steps, double volume_tolerance,
                        double* lambda_out);

/* OC update that allocates no device memory. No counterpart in the reference: it is for callers that cannot
   allocate device memory when they run this step (a host whose device memory is all reserved by another
   allocator in the process, or a loop that must not take the synchronisation of a cudaMalloc/cudaFree).
   rho, dc, s, passive (may be NULL) and rho_new are device pointers owned by the caller; lambda_out is a host
   pointer. The kernel's scratch is a fixed 65.6 KB array inside the library, held by every GPU that loads it
   until the process exits, sized for 1024 persistent blocks (devices that need more return MYCEL_E_ARG).
   The first call on a device looks up that array's device address, so make it before any stream capture.
   The work runs on the context's stream, which is not ordered after the caller's streams: the caller's writes
   to rho, dc, s and passive must be complete (e.g. their stream synchronised) before the call. Each call
   synchronises the context's stream to read lambda, so rho_new is ready when it returns.
   All calls share the array: calls that overlap on the GPU (other streams, other threads) race. */
int32_t mycel_oc_update_noalloc(mycel_ctx* ctx, int32_t n, const double* rho, const double* dc, const double* s,
                                const uint8_t* passive, double* rho_new, double target_volume_fraction,
                                double move_limit, double rho_min, double lambda_guess, int32_t max_bisection_steps,
                                double volume_tolerance, double* lambda_out);

/* HeavisideProjection.Project / Derivative (Optimization/HeavisideProjection.cs:12-37), host arrays of n values;
   the reference's default eta is 0.5. */
int32_t mycel_heaviside_project(mycel_ctx* ctx, int64_t n, const double* rho_tilde, double* rho_bar, double beta,
                                double eta);
int32_t mycel_heaviside_derivative(mycel_ctx* ctx, int64_t n, const double* rho_tilde, double* deriv, double beta,
                                   double eta);

/* ---- SIMP loop: TopologyOptimizer.Run (Optimization/TopologyOptimizer.cs:16-407) ----
   cancel / pause: polled between iterations (CancellationToken, IterationController.CheckAndBlock);
   history: room for history_cap records; u_out (total_dofs), physical/design_density_out (box, float) may
   be NULL. Non-convergence of a solve returns MYCEL_E_NOT_CONVERGED with the reference's message. */
int32_t mycel_simp_run(mycel_problem* p, const mycel_simp_options* opt, mycel_progress_fn progress, void* user,
                       const volatile int32_t* cancel, const volatile int32_t* pause, mycel_iter_record* history,
                       int32_t history_cap, int32_t* n_iterations, int32_t* converged, double* u_out,
                       float* physical_density_out, float* design_density_out);

/* Session form of the same loop for callers that keep the state (rho, u, PCG vectors, lambda) resident and
   step it themselves (the serving loop, the benchmark). step runs one SIMP iteration; *done is set when the
   stop rule fires or max_iterations is reached. */
int32_t mycel_simp_begin(mycel_problem* p, const mycel_simp_options* opt, mycel_simp_session** out);
int32_t mycel_simp_step(mycel_simp_session* s, mycel_iter_record* rec, int32_t* done);
int32_t mycel_simp_read(mycel_simp_session* s, double* u_out, float* physical_density_out, float* design_density_out,
                        double* rho_phys_active_out, double* rho_design_active_out, double* lambda_out);
int32_t mycel_simp_end(mycel_simp_session* s);
/* 1 once the session's stop rule has fired (TopologyOptimizationResult.Converged,
   Optimization/TopologyOptimizationResult.cs:6-17; set by the rule at TopologyOptimizer.cs:374-390), else 0. */
int32_t mycel_simp_converged(const mycel_simp_session* s);

/* One SIMP iteration of each of n sessions, with their solves packed. No counterpart in the reference, which
   runs one optimisation at a time (Optimization/OptimizationCoordinator.cs:229 through FemWorkTeam's lock,
   Fem/FemWorkTeam.cs:109); it replaces n calls of mycel_simp_step. The sessions share one context and each
   has its own problem. Those in MYCEL_PRECISION_MIXED_MG advance their FP32 outer iterations (and those of
   their load cases kept apart) together: every kernel of an outer iteration is one launch for all of them,
   whose CTAs are split between the problems by a per-problem table (grid, vectors, CTA range); the other
   sessions are solved one after another. Every session takes the iteration mycel_simp_step would take, to the
   bit. recs, done and status (each n entries, may be NULL) get each session's record, done flag and status;
   the call returns the first failure. cancel is polled between chunks of outer iterations. */
int32_t mycel_simp_step_many(mycel_simp_session* const* sessions, int32_t n, mycel_iter_record* recs, int32_t* done,
                             int32_t* status, const volatile int32_t* cancel);
/* Whole optimisations of n sessions (one context, one session per problem), each to its stop rule or
   max_iterations, as mycel_simp_step in a loop would take them, to the bit; no counterpart in the reference
   (same seams as mycel_simp_step_many). When every session is in MYCEL_PRECISION_MIXED_MG, the solves share
   one packed plan for the whole run and each problem goes on to its next SIMP iteration as soon as its own
   solve has ended, while the others still solve (no SIMP iteration waits for the slowest problem); otherwise
   the sessions are stepped together by mycel_simp_step_many. Records go to history[i * cap ...], n_iters[i] of
   them (only the first cap are kept); status[i] is each session's status (all three may be NULL); the call
   returns the first failure. cancel is polled between chunks of outer iterations. */
int32_t mycel_simp_run_many(mycel_simp_session* const* sessions, int32_t n, mycel_iter_record* history, int32_t cap,
                            int32_t* n_iters, int32_t* status, const volatile int32_t* cancel);

/* RunWriter snapshot frames (Persistence/RunWriter.cs:132-160 WriteSnapshotAsync, :199-245 the it_NNNNNN
   frame, :344-356 ComputeQuantizedChecksum) of the last completed iteration, without stalling the loop:
   frame_begin quantises the physical density to one byte per box element on the device
   (round(clamp(rho, 0, 1) * 255f), half away from zero) and starts its copy to pinned host memory; it returns a
   slot (two alternate, so one frame can be in flight while the next iteration runs). frame_end waits for that
   copy and returns the bytes (box-sized), the 72-byte little-endian header and the FNV-1a checksum of the
   bytes (computed on the host: FNV-1a is sequential). The stream checksum of RunWriter is then
   rolling = (rolling ^ checksum) * 16777619, starting from 2166136261. Brotli compression and file writing
   stay with the host. Any output may be NULL. */
int32_t mycel_simp_frame_begin(mycel_simp_session* s, int32_t* slot_out);
int32_t mycel_simp_frame_end(mycel_simp_session* s, int32_t slot, uint8_t* frame_out, uint8_t* header_out,
                             uint32_t* checksum_out);

/* ---- iso-surface: SurfaceNetsExtractor.Extract (PostProcessing/SurfaceNetsExtractor.cs:31-312) ----
   Closed 2-manifold triangle mesh of the level set density >= threshold of a box-sized float density field
   (element order x fastest) on a grid with spacing h and the given origin, by constrained Surface Nets with a
   1-voxel zero border: the reference's well-composedness passes, one vertex per dual cell with mixed corners,
   two triangles per sign-changing grid edge. Vertices, triangles and their orders are the reference's
   (sequential semantics, float arithmetic rounded per operation). density_len shorter than nx*ny*nz is
   MYCEL_E_ARG with the reference's message. The mesh (IndexedMesh: positions, 3 floats per vertex; indices, 3
   per triangle) is returned in host memory; mycel_mesh_info also gives the well-composedness passes run and
   the voxels' saddle/corner-kiss resolutions made. */
typedef struct mycel_mesh mycel_mesh;
int32_t mycel_surface_nets(mycel_ctx* ctx, int32_t nx, int32_t ny, int32_t nz, float h, const float* origin,
                           const float* density, int64_t density_len, float threshold, mycel_mesh** out);
/* The same extraction from a SIMP session's physical density of its last iteration, which stays on the device
   (the float field the snapshots read), for a per-iteration preview without copying the density to the host.
   origin may be NULL (0, 0, 0). */
int32_t mycel_simp_surface_nets(mycel_simp_session* s, const float* origin, float threshold, mycel_mesh** out);
int32_t mycel_mesh_info(const mycel_mesh* m, int64_t* n_vertices, int64_t* n_indices, int32_t* passes,
                        int64_t* changes);
int32_t mycel_mesh_copy(const mycel_mesh* m, float* positions, int32_t* indices);
void mycel_mesh_destroy(mycel_mesh* m);
/* TaubinSmoother.Smooth (PostProcessing/TaubinSmoother.cs:15-134): positions (3 floats per vertex, host) are
   replaced by the smoothed ones; per vertex the sorted de-duplicated triangle neighbours, then `iterations`
   times a lambda and a mu Laplacian step (reference defaults 3, 0.5, -0.53), bit-identical to the sequential
   code. iterations <= 0 or an empty mesh leaves positions unchanged; an index outside the vertex array is
   MYCEL_E_ARG. */
int32_t mycel_taubin_smooth(mycel_ctx* ctx, float* positions, int64_t n_vertices, const int32_t* indices,
                            int64_t n_indices, int32_t iterations, float lambda, float mu);

/* ---- serving: continuous batching of SIMP jobs on one GPU ----
   No counterpart in the reference, whose App runs one optimisation at a time (OptimizationCoordinator.cs:229
   through the FemWorkTeam lock, FemWorkTeam.cs:109). A server runs `slots` jobs at once, each on its own CUDA
   stream and host thread, so their PCG iterations interleave on the device; a queued job is admitted, in
   arrival order with backfill of later jobs that fit, when a slot is free and the device memory of the
   running jobs plus its own (mycel_job_device_bytes) stays within hbm_budget_bytes. A job's state (rho, u,
   PCG vectors, lambda) stays resident on the device from its first to its last iteration. Each job's results
   do not depend on what else runs: every reduction has a fixed order. */
typedef struct mycel_server mycel_server;

typedef struct {
  int32_t device;
  int32_t slots;             /* jobs running at once (>= 1) */
  int64_t hbm_budget_bytes;  /* admission limit on the summed device memory of running jobs */
} mycel_server_options;

/* One optimisation job: the arguments of mycel_problem_create and mycel_simp_run. Every array (including
   those inside loads and options) is copied by mycel_server_submit. */
typedef struct {
  mycel_grid grid;
  const uint8_t* domain;
  mycel_material material;
  const int32_t* fixed_dofs;
  int32_t n_fixed;
  const mycel_load_case* loads;
  int32_t n_loads;
  const double* element_density; /* box-sized or NULL */
  double penal;
  mycel_simp_options options;
  int32_t keep_u;                /* keep the final u for mycel_server_job_result */
} mycel_job_spec;

#define MYCEL_JOB_QUEUED 0
#define MYCEL_JOB_RUNNING 1
#define MYCEL_JOB_DONE 2
#define MYCEL_JOB_FAILED 3

typedef struct {
  int32_t state;            /* MYCEL_JOB_* */
  int32_t status;           /* MYCEL_* of a failed job, else MYCEL_OK */
  int32_t iterations, converged;
  int64_t device_bytes;     /* admission estimate */
  double submit_s, start_s, finish_s; /* seconds since the server was created */
  double final_compliance;
  int64_t solver_iterations; /* PCG iterations summed over the job's SIMP iterations */
  char message[256];
} mycel_job_info;

typedef struct {
  int64_t submitted, completed, failed, running, queued;
  int64_t simp_iterations;   /* summed over completed jobs */
  double first_submit_s, last_finish_s;
  double p50_latency_s, p99_latency_s, mean_latency_s, max_latency_s; /* submit -> finish, completed jobs */
  double p50_queue_s, p99_queue_s;                                    /* submit -> start */
  int64_t admitted_bytes, peak_admitted_bytes;
} mycel_server_stats;

int32_t mycel_server_create(const mycel_server_options* opt, mycel_server** out);
int32_t mycel_server_submit(mycel_server* s, const mycel_job_spec* job, int64_t* job_id);
int32_t mycel_server_job_info(mycel_server* s, int64_t job_id, mycel_job_info* out);
/* Waits for one job (job_id >= 0) or for every submitted job (job_id < 0); MYCEL_E_TIMEOUT after timeout_s
   (timeout_s < 0: no limit). */
int32_t mycel_server_wait(mycel_server* s, int64_t job_id, double timeout_s);
/* Results of a finished job; any output may be NULL. history: up to cap records; densities box-sized float;
   u total_dofs (when the job kept it). */
int32_t mycel_server_job_result(mycel_server* s, int64_t job_id, mycel_iter_record* history, int32_t cap,
                                float* physical_density_out, float* design_density_out, double* u_out);
int32_t mycel_server_stats_get(mycel_server* s, mycel_server_stats* out);
/* Lets running jobs finish, fails queued ones, joins the workers and frees everything. */
int32_t mycel_server_destroy(mycel_server* s);
const char* mycel_server_last_error(mycel_server* s);
/* Device memory a job holds while it runs (problem, PCG and mixed workspaces, SIMP session, filter): the
   admission estimate, an upper bound of mycel_problem_info.device_bytes for the same job. */
int64_t mycel_job_device_bytes(const mycel_job_spec* job);

#ifdef __cplusplus
}
#endif
#endif
