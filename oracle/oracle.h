/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement of Mycel.Core's FEM + SIMP inner loop (zmalrobot/mycel, C#/.NET 10), used as the
 * correctness checker for the CUDA library. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it. The product path never links or calls it.
 *
 * Pinning: the reference is C# and cannot be built here (no .NET runtime), so the restatement is pinned
 * against the reference's own known-answer tests and published numbers (Hex8 patch tests, V1 axial bar,
 * V3 cantilever deflections, E_min ablation compliances) — see tests/test_oracle_*.py.
 *
 * One detail of the reference cannot be observed here and is a runtime switch:
 *   lane mode  — how Vector256<double>.Sum combines its four lanes
 *                (0: (l0+l1)+(l2+l3) [.NET 8+ Sum(lower)+Sum(upper)], 1: (l0+l2)+(l1+l3), 2: ((l0+l1)+l2)+l3)
 * Math.Pow is the C library's pow, as .NET calls it on Linux.
 */
#ifndef MYCEL_ORACLE_H
#define MYCEL_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (match include/mycel.h) */
#define ORC_OK 0
#define ORC_E_ARG 1
#define ORC_E_UNDERCONSTRAINED 2
#define ORC_E_NOT_CONVERGED 3
#define ORC_E_INVALID_OPERATION 9

void orc_set_lane_mode(int mode);
/* Math.Pow as the restatement evaluates it (the C library's pow): out[i] = x[i]^y[y_len == 1 ? 0 : i]. */
void orc_math_pow(int64_t n, const double* x, const double* y, int64_t y_len, double* out);
void orc_set_threads(int n);
int orc_get_threads(void);
/* RunWriter.ComputeQuantizedChecksum and the 8-bit frame quantisation (Persistence/RunWriter.cs:211-217,
   344-356); out (n bytes) may be NULL. */
uint32_t orc_quantized_checksum(const float* v, int64_t n, uint8_t* out);

/* Hex8Element.CreateKe(h, nu) -> ke[576] row-major. */
int orc_create_ke(double h, double nu, double* ke);

/* FeModel */
typedef struct orc_model orc_model;
orc_model* orc_model_create(int nx, int ny, int nz, float h, const uint8_t* domain, double e0, double nu,
                            double emin_ratio, const int32_t* fixed, int32_t n_fixed,
                            const double* element_density, double penal, int* status, char* msg, int msglen);
int orc_model_add_load(orc_model* m, int32_t n_nodes, const int32_t* nodes, const double* areas, float fx, float fy,
                       float fz);
void orc_model_free(orc_model* m);
/* counts: [active elements, active nodes, active fixed dofs, total dofs, total elements, total nodes] */
void orc_model_counts(const orc_model* m, int64_t* out6);
void orc_model_active_elements(const orc_model* m, int32_t* out);
void orc_model_constrained(const orc_model* m, uint8_t* out);
int orc_model_assemble_forces(const orc_model* m, double* f, char* msg, int msglen);
/* load case k alone, and the number of load cases */
int orc_model_assemble_case_forces(const orc_model* m, int32_t k, double* f, char* msg, int msglen);
int32_t orc_model_load_case_count(const orc_model* m);
void orc_model_set_density(orc_model* m, const double* density_box, double penal);

/* FemOperator */
typedef struct orc_op orc_op;
orc_op* orc_op_create(orc_model* m);
void orc_op_free(orc_op* op);
void orc_op_update_densities(orc_op* op, const double* density_box, double penal);
void orc_op_diag(const orc_op* op, double* out);
void orc_op_apply_k(orc_op* op, const double* x, double* y);
void orc_op_apply_k_scalar_reference(orc_op* op, const double* x, double* y);
void orc_op_apply_a(orc_op* op, const double* x, double* y, int projected);
void orc_op_element_e(const orc_op* op, double* e_box);

/* PcgSolver.Solve with the Jacobi preconditioner */
typedef struct {
  int32_t iterations;
  double final_residual;
  int32_t converged;
  char message[256];
} orc_pcg_result;
int orc_pcg_solve(orc_op* op, const double* b, double* x, double tol, int32_t max_iter, orc_pcg_result* res,
                  char* msg, int msglen);

/* StaticAnalysis.Run (without von Mises) */
int orc_static_run(orc_model* m, double tol, int32_t max_iter, const double* warm, int64_t warm_len,
                   int throw_on_nonconv, double* u, double* reactions, double* compliance, double* max_disp,
                   orc_pcg_result* res, char* msg, int msglen);
/* StaticAnalysis.ComputeElementVonMises (centroid B, D·B·u_e, box-sized, 0 for inactive) */
void orc_von_mises(orc_op* op, const double* u, double* vm_box);

/* DensityFilter */
typedef struct orc_filter orc_filter;
orc_filter* orc_filter_create(int nx, int ny, int nz, const uint8_t* domain, const int32_t* active, int32_t n_active,
                              double rmin);
void orc_filter_free(orc_filter* f);
void orc_filter_apply(const orc_filter* f, const double* in, double* out);
void orc_filter_adjoint(const orc_filter* f, const double* in, double* out);
void orc_filter_s(const orc_filter* f, double* out);
int64_t orc_filter_nnz(const orc_filter* f);

/* SensitivityAnalysis.ComputeComplianceSensitivities */
void orc_sensitivities(orc_op* op, const double* u, const double* rho_phys, double* dc, double penal);

/* OcOptimizer.Update (rho_new may alias rho) */
double orc_oc_update(const double* rho, const double* dc, const double* s, const uint8_t* passive, double* rho_new,
                     int32_t n, double f, double move, double rho_min, double lambda_guess, int32_t max_bisect,
                     double vol_tol);
/* The same update, recording each volume evaluation in order: lam_out[k], vol_out[k] (up to cap of them);
   returns the number of evaluations; total_s_out: the sum of s in element order. */
int32_t orc_oc_trace(const double* rho, const double* dc, const double* s, const uint8_t* pas, int32_t n, double f,
                     double move, double rmin, double lg, int32_t maxb, double voltol, double* lam_out,
                     double* vol_out, int32_t cap, double* total_s_out);

/* HeavisideProjection */
void orc_heaviside_project(const double* rt, double* rb, int32_t n, double beta, double eta);
void orc_heaviside_derivative(const double* rt, double* d, int32_t n, double beta, double eta);

/* PassiveRegion.Build */
void orc_passive_region(int nx, int ny, int nz, const int32_t* nodes, int32_t n_nodes, int radius, uint8_t* out);

/* TopologyOptimizer.Run */
typedef struct {
  double volume_fraction, filter_radius_mm, penal, move_limit;
  int32_t max_iterations;
  double solver_tol_initial, solver_tol_final;
  int32_t solver_max_iterations;
  int32_t continuation, enable_heaviside;
  double rho_min;
  const uint8_t* passive_mask;
  int64_t passive_len;
  int32_t protect_boundary_hinges;
  const float* initial_density;
  int64_t initial_density_len;
  int32_t start_iteration;
  const double* warm_start;
  int64_t warm_start_len;
  int32_t enforce_min_filter_radius;
  /* 0: load cases summed into one right-hand side (the reference); 1: one solve per load case, objective the
     sum of the cases' compliances, sensitivities summed in case order, u reported as the sum of the cases' u */
  int32_t separate_load_cases;
} orc_simp_options;

typedef struct {
  int32_t iteration;
  double compliance, volume_fraction, max_change, grey_level;
  int32_t solver_iterations;
  double solver_residual;
  double max_displacement;
  double total_ms;
} orc_iter_record;

/* history has room for history_cap records; phys/design receive the final snapshot (float, box-sized);
   rho_phys_active (optional) receives the final filtered density in double (active-indexed). */
int orc_topopt_run(orc_model* m, const orc_simp_options* o, orc_iter_record* history, int32_t history_cap,
                   int32_t* n_iters, int32_t* converged, double* u_out, float* phys_out, float* design_out,
                   double* rho_phys_active, double* rho_design_active, double* lambda_out, char* msg, int msglen);

/* SurfaceNetsExtractor.Extract: padded threshold field, well-composedness passes, one vertex per mixed dual
   cell, two triangles per sign-changing grid edge. orc_mesh_info: {vertices, indices, passes, changes}. */
/* StaticAnalysis.AverageElementToNode: nodal means of an element scalar over the active elements. */
void orc_average_element_to_node(const orc_model* m, const double* element_scalar, double* nodal_out);
typedef struct orc_mesh orc_mesh;
/* TaubinSmoother.Smooth on positions (3 floats per vertex) in place. */
void orc_taubin_smooth(float* pos, int64_t nv, const int32_t* idx, int64_t ni, int iterations, float lambda, float mu);
orc_mesh* orc_surface_nets(int nx, int ny, int nz, float h, const float* origin, const float* density, float thr);
void orc_mesh_info(const orc_mesh* m, int64_t* out);
void orc_mesh_copy(const orc_mesh* m, float* pos, int32_t* idx);
void orc_mesh_free(orc_mesh* m);

#ifdef __cplusplus
}
#endif
#endif
