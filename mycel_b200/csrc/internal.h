// Internal declarations of libmycel_b200: device state of a problem, kernel launchers, helpers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/mycel.h"

namespace mycel {

// ---- small POD passed by value to kernels (kernel parameter space is broadcast like constant memory) ----
struct GridDims {
  int nx, ny, nz;    // elements per axis
  int nx1, ny1, nz1; // nodes per axis
  int64_t ne, nn, nd;
  // FP32 vectors of the mixed form use a padded layout: each node row (fixed j, k) holds its 3 nx1 DOFs
  // contiguously from a 16-byte aligned start, row pitch rp floats (multiple of 4); pads stay zero.
  int rp;
  int64_t n32;       // rp * ny1 * nz1
  // FP64 work vectors of the fast FP64 form: the same layout with row pitch rp64 doubles (multiple of 2)
  int rp64;
  int64_t n64;       // rp64 * ny1 * nz1
};

inline GridDims make_dims(int nx, int ny, int nz) {
  GridDims g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.nx1 = nx + 1; g.ny1 = ny + 1; g.nz1 = nz + 1;
  g.ne = (int64_t)nx * ny * nz;
  g.nn = (int64_t)g.nx1 * g.ny1 * g.nz1;
  g.nd = 3 * g.nn;
  g.rp = (3 * g.nx1 + 3) & ~3;
  g.n32 = (int64_t)g.rp * g.ny1 * g.nz1;
  g.rp64 = (3 * g.nx1 + 1) & ~1;
  g.n64 = (int64_t)g.rp64 * g.ny1 * g.nz1;
  return g;
}

// index of DOF c of node (i, j, k) in the padded FP32 layout
#ifdef __CUDACC__
__host__ __device__
#endif
inline int64_t pidx(const GridDims& g, int i, int64_t jk, int c) { return (int64_t)g.rp * jk + 3 * i + c; }

struct KeD { double v[576]; };  // element stiffness (row-major), FP64
struct KeF { float v[576]; };   // FP32 copy for the mixed form
// KE split for 3xTF32 tensor-core products: rows padded to 32 (rows 24..31 zero), row-major [32][24]
struct KeTf { float hi[32 * 24]; float lo[32 * 24]; };
// Hex8 operator of a cube element in the per-axis (sum, difference) basis, FP32, scaled by h / 8 (see
// build_hexop). dcl[pc][n]: eigenvalue of component c at a basis function whose c-axis factor is even (0) or
// odd (1) and with n odd factors on the other two axes; lam[pk], mu[pk]: coupling constants lambda m(pk),
// mu m(pk) of two different components, pk the parity on the third axis.
struct HexOpF { float dcl[2][3]; float lam[2]; float mu[2]; };
struct HexOpD { double dcl[2][3]; double lam[2]; double mu[2]; };  // the same constants in FP64

// Node flag bits (one byte per node): bits 0-2 = DOF c constrained, bit 3 = node active.
enum : uint8_t { NF_CX = 1, NF_CY = 2, NF_CZ = 4, NF_ACTIVE = 8 };

// PCG status word (device). 0 = running.
enum PcgStatus : int {
  PCG_RUNNING = 0,
  PCG_CONVERGED = 1,
  PCG_BREAK_CURVATURE = 2,
  PCG_BREAK_ALPHA = 3,
  PCG_STAGNATED = 4,
  PCG_BREAK_BETA = 5,
  PCG_MAXITER = 6,
  PCG_INIT_CONVERGED = 7,
  PCG_RHS_ZERO = 8,
};

// Device-resident scalar state of one PCG solve (PcgSolver.cs:231-357 locals).
struct PcgState {
  int status;
  int iter;
  int max_iter;
  int stag;
  int nonzero_x;
  int pad_;
  double tol, bnorm, bn2, rho0, rel, prev, alpha, beta, pap, rn2, last_bad;
  unsigned int counter;  // completion counter for the last-block pattern
  unsigned int counter2;
  double dot_acc;        // scratch (mixed form)
};

// ---- device memory helpers ----
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct MgHier;  // multigrid hierarchy of a problem (fp32_kernels.cu)
}  // namespace mycel

// ---- opaque handles of the C ABI ----
struct mycel_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // second stream for set-up work that can overlap the main stream's (joined back)
  int num_sms = 148;
  int oc_grid = 0;                  // blocks of the persistent OC kernel: num_sms x oc_blocks_per_sm(), set at creation
  int64_t oc_wait_polls = 0;        // polls of each OC grid-barrier wait before it gives up (0: the default)
  int oc_wait_unreachable = 0;      // test switch: the OC barrier waits for one block more than the grid holds
  int64_t launches = 0;
  std::string last_error;
  void* pinned = nullptr;  // small pinned scratch for scalar readbacks
  size_t pinned_bytes = 0;
  // optional live timing of the dominant kernel (CUDA events captured around one matvec per PCG chunk)
  int profile = 0;
  double prof_ms[4] = {0, 0, 0, 0};  // [0] FP32 matvec, [1] FP64 matvec
  int64_t prof_n[4] = {0, 0, 0, 0};
  int64_t prof_nodes[4] = {0, 0, 0, 0};     // nodes processed by the timed launches
  int64_t prof_elems[4] = {0, 0, 0, 0};     // active elements processed by the timed launches
  void* pack = nullptr;    // packed-solve workspace (fp32_kernels.cu), built on first use
  void* fan = nullptr;     // side streams for independent per-problem work of a batch step (mycel::fan_*)
  cudaStream_t main_stream = nullptr, main_side = nullptr;  // the context's own streams while a fan slot is in use
  int64_t packed_rhs = 0;  // right-hand sides whose solves ran through packed launches (a statistic)
};

struct mycel_problem {
  mycel_ctx* ctx = nullptr;
  uint64_t serial = 0;  // distinct for every problem the process creates (cached plans compare it)
  mycel::GridDims g{};
  float h = 1.0f;
  double e0 = 1, nu = 0.3, emin_ratio = 1e-6, emin = 1e-6, penal = 3.0;
  mycel::KeD ke{};
  mycel::KeF kef{};
  mycel::KeTf ketf{};
  mycel::HexOpF hexop{};
  mycel::HexOpD hexop64{};
  int mv32 = -1;                  // FP32 matvec variant in use: -1 not chosen yet, else MYCEL_MV32_* (1..3)
  int tune_mv32 = 0;              // requested variant: 0 autotune, else MYCEL_MV32_*
  bool mixed_prefers_f64f = false; // a mixed solve of this problem stalled: later ones start in fast FP64
  // mixed form's choice between its FP32 and fast FP64 inner forms: solves so far and the latest iterations
  // per decade of residual reduction of each (deterministic: counts, not timings)
  int mix_solves = 0;
  double it32_per_dec = -1.0, it64_per_dec = -1.0;
  int* d_err = nullptr;           // device error word (bounded waits that gave up)
  double diag_ke[24];
  int64_t n_active = 0, n_active_nodes = 0, n_active_fixed = 0;
  std::vector<mycel_simp_session*> sessions;  // live SIMP sessions on this problem (ended by problem_destroy)
  std::vector<int32_t> fixed_host;        // FixedDofs as given (may repeat)
  std::vector<int32_t> load_nodes_host;   // union of load patch nodes (hinge shell)
  std::vector<int32_t> f_idx;             // AssembleForces result: DOFs with a non-zero force, ascending
  std::vector<double> f_val;              //   and their forces
  // load cases kept apart (multi-RHS solves over the shared stiffness): each case's nodal forces alone, as
  // (DOF, value) contributions in assembly order; device right-hand sides built on first use
  std::vector<std::vector<std::pair<int64_t, double>>> case_terms;
  int32_t n_cases = 0;
  double* d_case_F = nullptr;             // [n_cases * nd] F_k
  double* d_case_b = nullptr;             // [n_cases * nd] P F_k
  int32_t* d_case_nz = nullptr;           // non-zero lists of F_k (ascending), concatenated
  std::vector<int32_t> case_nz_off, case_nz_cnt;
  uint64_t e_version = 0;                 // bumped whenever E changes (shared set-ups compare it)
  int assemble_status = 0;
  std::string assemble_msg;
  // device arrays
  uint8_t* d_domain = nullptr;    // [ne]
  uint8_t* d_nflags = nullptr;    // [nn]
  int32_t* d_fixed = nullptr;     // FixedDofs as given
  int32_t* d_active = nullptr;    // [n_active] ascending box element index
  int32_t* d_e2a = nullptr;       // [ne] active index or -1
  double* d_F = nullptr;          // [nd] nodal forces
  double* d_b = nullptr;          // [nd] P F
  int32_t* d_fnz = nullptr;       // indices i with F[i] != 0, ascending
  int32_t n_fnz = 0;
  int32_t* d_bnz = nullptr;       // indices with b[i] != 0, ascending
  int32_t n_bnz = 0;
  double* d_rho_box = nullptr;    // [ne] FeModel.ElementDensity
  double* d_E = nullptr;          // [ne] E_e (active elements)
  float* d_Ef = nullptr;          // [ne] FP32 copy
  double* d_diag = nullptr;       // [nd] DiagA
  double* d_invd = nullptr;       // [nd] Jacobi inverse diagonal
  float* d_invdf = nullptr;       // [n32] FP32 copy, padded layout
  // PCG workspace (FP64)
  double *d_r = nullptr, *d_z = nullptr, *d_p = nullptr, *d_ap = nullptr, *d_x = nullptr;
  double* d_part = nullptr;       // [2*nblocks] partial sums
  mycel::PcgState* d_state = nullptr;
  // mixed-form workspace
  float *f_x = nullptr, *f_r = nullptr, *f_z = nullptr, *f_p0 = nullptr, *f_p1 = nullptr, *f_ap = nullptr;
  CUtensorMap f_tmap[4];          // TMA descriptors of f_r, f_z, f_p0, f_p1 (node-plane boxes of the FP32 matvec)
  // fast FP64 form (factorised operator, FP64 recurrences): padded FP64 work vectors, TMA maps, graphs
  double *g_x = nullptr, *g_r = nullptr, *g_z = nullptr, *g_p0 = nullptr, *g_p1 = nullptr, *g_ap = nullptr,
         *g_invd = nullptr;
  CUtensorMap g_tmap[4];          // g_r, g_z, g_p0, g_p1
  cudaGraphExec_t pcg64f_graph[2] = {nullptr, nullptr};
  int pcg64f_graph_profiled = 0;
  cudaEvent_t prof64f_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  mycel::MgHier* mg = nullptr;     // multigrid hierarchy (MYCEL_PRECISION_FP64_MG), built on first use
  // TMA descriptors of the per-case FP32 work vectors of batched multigrid solves (owned by the hierarchy)
  int n_case_tmaps = 0;
  const float* case_tmap_ptr[32] = {};
  const CUtensorMap* case_tmap[32] = {};
  double* d_r64 = nullptr;        // refinement residual
  double* d_part2 = nullptr;      // [many] FP64 partials for mixed dots
  int64_t n_part2 = 0;
  int64_t device_bytes = 0;
  // scratch for API calls
  double* d_tmp0 = nullptr;       // [nd]
  double* d_tmp1 = nullptr;       // [nd]
  int lane_mode = 0;
  cudaGraphExec_t pcg_graph[2] = {nullptr, nullptr};
  int pcg_graph_chunk = 0;
  cudaEvent_t prof64_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  cudaGraphExec_t pcg32_graph[2] = {nullptr, nullptr};
  int pcg32_graph_chunk = 0;
  int pcg32_graph_profiled = 0;
  cudaEvent_t prof_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int pcg_graph_profiled = 0;
};

struct mycel_filter {
  mycel_problem* p = nullptr;
  double rmin = 1.5;
  int n_off = 0;
  int rc = 0;                   // offset radius ceil(rmin), in elements
  int4* d_off = nullptr;        // (dx, dy, dz, unused) in the reference's loop order
  double* d_w = nullptr;        // rmin - dist per offset
  double* d_invhs = nullptr;    // [ne]
  double* d_s = nullptr;        // [ne]
};

namespace mycel {

// ---- error plumbing ----
int32_t set_error(mycel_ctx* ctx, int32_t code, const std::string& msg);
#define MYCEL_CUDA(ctx, call)                                                                      \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return ::mycel::set_error((ctx), MYCEL_E_DEVICE, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

// ---- host setup ----
void build_ke(double h, double nu, double* ke);  // Hex8Element.CreateKe semantics
void split_ke_tf32(const double* ke, KeTf* out);   // hi = tf32(KE), lo = tf32(KE - hi), rows padded to 32
void build_hexop(double h, double nu, HexOpF* out);  // factorised form of KE(h, nu), FP32
void build_hexop64(double h, double nu, HexOpD* out);  // the same in FP64
int64_t num_blocks8192(int64_t n);

// ---- FP64 plain-path launchers (fp64_kernels.cu, compiled with -fmad=false) ----
void launch_setup_nodes(mycel_problem* p, const int32_t* d_fixed, int32_t n_fixed, int32_t* d_count);
void launch_update_E(mycel_problem* p, const double* d_rho_box, double penal);
void launch_diag(mycel_problem* p);
void launch_matvec64(mycel_problem* p, const double* x, double* y, int projected, const int* d_status);
void launch_project_x(mycel_problem* p, double* x, int* d_flag);
void launch_pcg_bnorm(mycel_problem* p);
void launch_pcg_init_r(mycel_problem* p, int nonzero);
void launch_pcg_dot_rr(mycel_problem* p);
void launch_pcg_init_z(mycel_problem* p);
void launch_pcg_iteration(mycel_problem* p, bool skip_matvec = false);
void launch_compliance(mycel_problem* p, const double* u, double* d_out);
void launch_compliance(mycel_problem* p, const double* F, const int32_t* fnz, int32_t n_fnz, const double* u,
                       double* d_out);
void launch_max_disp(mycel_problem* p, const double* u, double* d_out);
void launch_max_disp(mycel_problem* p, const double* const* us, int m, int64_t stride, double* d_out);
void launch_reactions(mycel_problem* p, const double* ku, double* out, const int32_t* d_fixed, int32_t n_fixed);
void launch_von_mises(mycel_problem* p, const double* u, double* vm);
void launch_average_e2n(mycel_problem* p, const double* es, double* out);
int32_t surface_nets_core(mycel_ctx* ctx, int32_t nx, int32_t ny, int32_t nz, float h, const float* origin,
                          const float* h_density, const float* d_density, float threshold, mycel_mesh** out);
void launch_scatter_active(mycel_problem* p, const double* src_active, double* dst_box, double fill);
void launch_gather_active(mycel_problem* p, const double* src_box, double* dst_active);

// filter
int filter_setup(mycel_filter* f);
void launch_filter_fwd(mycel_filter* f, const double* in_box, double* out_box);
void launch_filter_adj(mycel_filter* f, const double* in_box, double* out_box);
void launch_sens(mycel_problem* p, const double* u, const double* rho_box, double penal, double* dc_box,
                 bool accumulate = false);

// OC (persistent cooperative kernel); returns 0 or MYCEL_E_TIMEOUT / MYCEL_E_DEVICE
struct OcParams {
  double f, move, rho_min, lambda_guess, vol_tol;
  int max_bisect;
  int heaviside;
  // 1: every decision of the bisection is the one the reference's sequential sums give (the tree sums are used
  // where they are farther from the threshold than their error bound, the sequential sum otherwise), and the
  // total S and the volume and grey metrics are summed in element order. 0: tree sums throughout.
  int exact = 1;
  double total_s = -1.0;  // >= 0: sum of S in element order, known from an earlier call; < 0: computed here
};
struct OcOut {
  double lambda;
  double max_change;
  double vol_sum;
  double grey_sum;
  int err;
  int trials;  // volume evaluations; 0 when a grid barrier timed out
  double total_s;
};
// HeavisideProjection (HeavisideProjection.cs:12-37) over the elements idx[0..n) (all n when idx is null):
// mode 0 out = Project(rt); mode 1 out = dcb * Derivative(rt) (TopologyOptimizer.cs:283-287); mode 2
// out = Derivative(rt).
void launch_heaviside(mycel_ctx* ctx, int64_t n, const int32_t* idx, const double* rt, const double* dcb,
                      double* out, double beta, double eta, int mode);
// Blocks of the persistent OC kernel per SM on the current device (occupancy, clamped to [1, 2]).
int oc_blocks_per_sm(int* out);
// Scratch the OC kernel needs for a grid of `grid` blocks: partial sums, broadcast cells, barrier words.
inline size_t oc_scratch_doubles(int grid) { return (size_t)7 * grid + 4 + 4; }
int launch_oc(mycel_ctx* ctx, int64_t n, const int32_t* d_index /*box index of element i or null*/,
              const double* rho, const double* dc, const double* s, const uint8_t* passive, double* rho_new,
              const double* rho_phys_for_metrics, const double* rho_tilde_for_grey, const OcParams& prm,
              double* d_scratch, size_t scratch_doubles, OcOut* d_out);

// ---- mixed form (fp32_kernels.cu) ----
void launch_E_to_f32(mycel_problem* p);
void launch_matvec32(mycel_problem* p, const float* x, float* y, int projected);
int32_t mixed_apply_k_f64io(mycel_problem* p, const double* x, double* y, int projected);
bool simp_session_converged(const mycel_simp_session* s);  // the SIMP stop rule fired
int32_t mixed_solve_entry(mycel_problem* p, const double* d_b, const int32_t* d_nz, int32_t n_nz, double* d_u,
                          double tol, int max_iter, const volatile int32_t* cancel, mycel_pcg_result* res);
// Load cases 0 .. ncase-1 of the problem solved together in the mixed multigrid form (one V-cycle's coarse
// levels for all cases); d_u: ncase x total_dofs, case-major, warm starts in, solutions out; res: ncase.
int32_t mg_solve_cases(mycel_problem* p, int ncase, double* d_u, double tol, int max_iter,
                       const volatile int32_t* cancel, mycel_pcg_result* res);
constexpr int kMaxBatchedCases = 8;
// One problem's part of a packed solve (mixed multigrid form): its single right-hand side (ncase 1: p->d_b, the
// solution in d_u) or its load cases 0 .. ncase-1 solved together (p->d_case_b; d_u: ncase x total_dofs,
// case-major); warm starts in, solutions out, res: ncase results.
struct PackJob {
  mycel_problem* p;
  int ncase;
  double* d_u;
  double tol;
  int max_iter;
  mycel_pcg_result* res;
};
// Solves the jobs (all problems of context c, one job per problem) with their FP32 outer iterations advanced
// together by packed launches; jobs the packed form cannot take are solved alone. Each result equals the
// problem's solve alone in the mixed multigrid form.
int32_t mg_solve_packed(mycel_ctx* c, int njobs, PackJob* jobs, const volatile int32_t* cancel);
void pack_release(mycel_ctx* c);
// Asynchronous packed run (mycel_simp_run_many): the right-hand sides of the jobs share one packed plan for a
// whole optimisation and each job's solves start and end on their own. pkr_open leaves out the jobs the
// packed form cannot take (packed[j] 0: the caller steps them alone). pkr_begin issues the start of job j's next solve; after the caller synchronises the
// context stream, pkr_after_begin lets the started right-hand sides run; pkr_advance runs one chunk of outer
// iterations (synchronised), refines and restarts what stopped, and appends the jobs whose solves ended;
// pkr_results gives an ended job's results (ncase of them).
struct PackRunJob {
  mycel_problem* p;
  int ncase;
  double* d_u;
};
struct PackRun;
int32_t pkr_open(mycel_ctx* c, const std::vector<PackRunJob>& jobs, PackRun** out, std::vector<char>* packed);
void pkr_close(PackRun* r);
int32_t pkr_begin(PackRun* r, int j, double tol, int max_iter);
int32_t pkr_after_begin(PackRun* r);
int32_t pkr_after_begin_job(PackRun* r, int j);  // the same for job j only (its start read back already)
bool pkr_running(const PackRun* r);
int32_t pkr_advance(PackRun* r, const volatile int32_t* cancel, std::vector<int>* ended);
const mycel_pcg_result* pkr_results(const PackRun* r, int j);
// Fan-out of independent per-problem work of a batch step over side streams: fan_begin makes them wait for
// the context stream's work so far; fan_use(c, k) issues the following work of the context on side stream k
// (the context's stream and side stream are swapped, so every launch helper follows); fan_end returns to the
// context's streams, which then wait for everything issued on the side streams.
int32_t fan_begin(mycel_ctx* c);
void fan_use(mycel_ctx* c, int slot);
void fan_end(mycel_ctx* c);
void fan_release(mycel_ctx* c);
// The same side stream k for work that depends on nothing queued on the context stream (the caller orders it
// by events): fan_use_free issues the following work of the context there, fan_restore returns.
int32_t fan_use_free(mycel_ctx* c, int slot, cudaStream_t* fan_stream);
void fan_restore(mycel_ctx* c);
bool cases_together_enabled();
int32_t kernel_bench(mycel_problem* p, int which, int reps, double* avg_us);  // MYCEL_CASES_TOGETHER=0 turns the batched case solve off
int32_t refined_solve_entry(mycel_problem* p, const double* d_b, const int32_t* d_nz, int32_t n_nz, double* d_u,
                            double tol, int max_iter, const volatile int32_t* cancel, int precision,
                            mycel_pcg_result* res);
int32_t fast64_apply_k(mycel_problem* p, const double* x, double* y, int projected);
void mg_release(mycel_problem* p);
int64_t mg_device_bytes(int nx, int ny, int nz, int n_cases, bool cases_together);  // hierarchy of a grid; 0 when it does not coarsen

// ---- drivers (api.cu) ----
int32_t pcg_solve_fp64(mycel_problem* p, const double* d_b, const int32_t* d_nz, int32_t n_nz, double* d_x,
                       double tol, int max_iter, const volatile int32_t* cancel, mycel_pcg_result* res);
// load cases apart: device right-hand sides of every case (built on first use) and a solve of one of them
int32_t ensure_cases(mycel_problem* p);
int32_t solve_case(mycel_problem* p, int k, double* d_u, double tol, int max_iter, int precision,
                   const volatile int32_t* cancel, mycel_pcg_result* res);
int32_t solve_dispatch(mycel_problem* p, double* d_u, double tol, int max_iter, int precision,
                       const volatile int32_t* cancel, mycel_pcg_result* res);
int32_t ensure_pcg_workspace(mycel_problem* p);

}  // namespace mycel
