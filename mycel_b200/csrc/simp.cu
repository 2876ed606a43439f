// SIMP loop: TopologyOptimizer.Run (src/Mycel.Core/Optimization/TopologyOptimizer.cs:16-407) with the design
// state resident on the device. Per iteration: filter -> (Heaviside) -> E/DiagA -> tolerance schedule -> warm
// PCG -> compliance, max |u| -> sensitivities -> adjoint filter -> OC bisection -> metrics. Only scalars (and
// requested snapshots) cross PCIe.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "internal.h"

using namespace mycel;

struct mycel_simp_session {
  mycel_problem* p = nullptr;
  mycel_simp_options o{};
  mycel_filter* filt = nullptr;
  double rmin = 1.5;
  std::vector<std::string> warnings;
  double *d_rho = nullptr, *d_rho_new = nullptr, *d_rt = nullptr, *d_rb = nullptr, *d_dcb = nullptr,
         *d_dct = nullptr, *d_dc = nullptr, *d_u = nullptr, *d_scal = nullptr, *d_oc_scr = nullptr;
  OcOut* d_oc = nullptr;
  uint8_t* d_pas = nullptr;
  float *d_phys_f = nullptr, *d_des_f = nullptr;
  int ncase = 1;               // load cases solved apart (separate_load_cases with more than one case), else 1
  double* d_uc = nullptr;      // [ncase * nd] each case's displacements (its warm start)
  int iter = 1, start = 1, maxit = 200;
  double lambda = 1.0, max_change = 1.0, beta = 1.0;
  double total_s = -1.0;       // sum of the filter's S over the active elements (fixed per filter), once known
  std::deque<double> chist;
  bool converged = false, done = false;
  int count = 0;
  cudaEvent_t ev[5] = {};
  std::vector<float> h_phys, h_des;
  mycel_iter_record last{};        // record of the last completed iteration (frame headers)
  // RunWriter frames: two device byte frames and pinned host copies, filled without waiting
  uint8_t* d_frame[2] = {nullptr, nullptr};
  uint8_t* h_frame[2] = {nullptr, nullptr};
  cudaEvent_t frame_ev[2] = {nullptr, nullptr};
  mycel_iter_record frame_rec[2] = {};
  bool frame_busy[2] = {false, false};
  int frame_next = 0;
  void* h_pin = nullptr;           // pinned host slot of the per-iteration scalar read-backs
};

namespace {

// RunWriter's 8-bit quantisation (Persistence/RunWriter.cs:211-217): round(clamp(v, 0, 1) * 255f), half away
// from zero, in FP32
__global__ void k_quantize(int64_t ne, const float* __restrict__ v, uint8_t* __restrict__ q) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const float c = fminf(fmaxf(v[e], 0.0f), 1.0f);
  q[e] = (uint8_t)roundf(__fmul_rn(c, 255.0f));
}

// u += v (the superposition of the load cases' displacements, added in case order)
__global__ void k_add_into(int64_t n, double* __restrict__ u, const double* __restrict__ v) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) u[i] = u[i] + v[i];
}

// out = 0 + c[0] + c[1] + ... in case order (the objective: the sum of the cases' compliances)
__global__ void k_sum_in_order(const double* __restrict__ c, int m, double* out) {
  double t = 0.0;
  for (int k = 0; k < m; ++k) t = t + c[k];
  *out = t;
}

__global__ void k_snapshot(int64_t ne, const uint8_t* __restrict__ dom, const double* __restrict__ rb,
                           const double* __restrict__ rho, float* __restrict__ pf, float* __restrict__ df) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  bool a = dom[e] != 0;
  pf[e] = a ? (float)rb[e] : 0.0f;
  df[e] = a ? (float)rho[e] : 0.0f;
}

template <class T>
cudaError_t salloc(mycel_simp_session* s, T** ptr, size_t count) {
  size_t bytes = std::max<size_t>(sizeof(T) * count, 16);
  cudaError_t e = cudaMallocAsync((void**)ptr, bytes, s->p->ctx->stream);  // stream-ordered, no device sync
  if (e == cudaSuccess) s->p->device_bytes += (int64_t)bytes;
  return e;
}

double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace

extern "C" int32_t mycel_simp_end(mycel_simp_session* s);

extern "C" int32_t mycel_simp_begin(mycel_problem* p, const mycel_simp_options* opt, mycel_simp_session** out) {
  if (!p || !opt || !out) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  *out = nullptr;
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  (void)cudaGetLastError();  // do not report a stale error of an earlier, unrelated call
  cudaStream_t st = c->stream;
  const GridDims& g = p->g;
  mycel_simp_session* s = new mycel_simp_session();
  s->p = p;
  s->o = *opt;
  const mycel_simp_options& o = s->o;
  // filter radius in voxels (TopologyOptimizer.cs:28-39)
  double h = (double)p->h;
  s->rmin = o.filter_radius_mm / h;
  if (s->rmin < 1.5) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "Filter radius %.2f mm (%.2f voxels) is below 1.5h (%.2f mm).", o.filter_radius_mm,
                  s->rmin, 1.5 * h);
    s->warnings.push_back(buf);
    if (o.enforce_minimum_filter_radius) s->rmin = 1.5;
  }
  if (p->assemble_status) {
    int32_t code = p->assemble_status;
    std::string m = p->assemble_msg;
    delete s;
    return set_error(c, code, m);
  }
  // passive mask (TopologyOptimizer.cs:45-84): option mask and hinge shell PassiveRegion.Build(r = 1)
  std::vector<uint8_t> pas((size_t)g.ne, 0);
  std::vector<uint8_t> dom((size_t)g.ne);
  cudaMemcpyAsync(dom.data(), p->d_domain, g.ne, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (o.passive_mask)
    for (int64_t e = 0; e < g.ne; ++e)
      if (dom[e] && e < o.passive_mask_len && o.passive_mask[e] != 0) pas[e] = 1;
  if (o.protect_boundary_hinges) {
    std::vector<int32_t> nodes(p->load_nodes_host);
    std::unordered_set<int32_t> seen(nodes.begin(), nodes.end());
    for (int32_t d : p->fixed_host)
      if (seen.insert(d / 3).second) nodes.push_back(d / 3);
    for (int32_t n : nodes) {
      int64_t nx1 = g.nx1, ny1 = g.ny1;
      int nk = (int)(n / (nx1 * ny1));
      int64_t rem = n % (nx1 * ny1);
      int nj = (int)(rem / nx1), ni = (int)(rem % nx1);
      auto cl = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
      int x0 = cl(ni - 1, 0, g.nx - 1), x1 = cl(ni, 0, g.nx - 1);
      int y0 = cl(nj - 1, 0, g.ny - 1), y1 = cl(nj, 0, g.ny - 1);
      int z0 = cl(nk - 1, 0, g.nz - 1), z1 = cl(nk, 0, g.nz - 1);
      for (int iz = z0; iz <= z1; ++iz)
        for (int iy = y0; iy <= y1; ++iy)
          for (int ix = x0; ix <= x1; ++ix) {
            int64_t e = ix + (int64_t)g.nx * (iy + (int64_t)g.ny * iz);
            if (dom[e]) pas[e] = 1;
          }
    }
  }
  // initial design (TopologyOptimizer.cs:90-122)
  std::vector<double> rho((size_t)g.ne, 0.0);
  if (o.initial_density) {
    if (o.initial_density_len == g.ne) {
      for (int64_t e = 0; e < g.ne; ++e)
        if (dom[e]) rho[e] = (double)o.initial_density[e];
    } else if (o.initial_density_len == p->n_active) {
      int64_t i = 0;
      for (int64_t e = 0; e < g.ne; ++e)
        if (dom[e]) rho[e] = (double)o.initial_density[i++];
    } else {
      delete s;
      return set_error(c, MYCEL_E_ARG, "InitialDensity length (" + std::to_string(o.initial_density_len) +
                                           ") must match either TotalElements (" + std::to_string(g.ne) +
                                           ") or ActiveElementCount (" + std::to_string(p->n_active) + ").");
    }
  } else {
    for (int64_t e = 0; e < g.ne; ++e)
      if (dom[e]) rho[e] = pas[e] ? 1.0 : o.volume_fraction;
  }
  for (int64_t e = 0; e < g.ne; ++e)
    if (pas[e]) rho[e] = 1.0;
  int32_t rc = ensure_pcg_workspace(p);
  if (rc) {
    delete s;
    return rc;
  }
  s->ncase = o.separate_load_cases && p->n_cases > 1 ? p->n_cases : 1;
  if (s->ncase > 1 && (rc = ensure_cases(p))) {
    delete s;
    return rc;
  }
  bool ok = !salloc(s, &s->d_rho, g.ne) && !salloc(s, &s->d_rho_new, g.ne) && !salloc(s, &s->d_rt, g.ne) &&
            !salloc(s, &s->d_dcb, g.ne) && !salloc(s, &s->d_dc, g.ne) && !salloc(s, &s->d_u, g.nd) &&
            !salloc(s, &s->d_scal, 16 + (s->ncase > 1 ? s->ncase : 0)) &&
            !salloc(s, &s->d_oc_scr, oc_scratch_doubles(c->oc_grid)) &&
            !salloc(s, &s->d_oc, 1) && !salloc(s, &s->d_pas, g.ne) && !salloc(s, &s->d_phys_f, g.ne) &&
            !salloc(s, &s->d_des_f, g.ne);
  if (ok && o.enable_heaviside) ok = !salloc(s, &s->d_rb, g.ne) && !salloc(s, &s->d_dct, g.ne);
  if (ok && s->ncase > 1) ok = !salloc(s, &s->d_uc, (size_t)(s->ncase * g.nd));
  if (!ok) {
    mycel_simp_end(s);
    return set_error(c, MYCEL_E_OOM, "out of device memory for the SIMP state");
  }
  if (!o.enable_heaviside) s->d_rb = s->d_rt;
  cudaMemcpyAsync(s->d_rho, rho.data(), sizeof(double) * g.ne, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->d_rho_new, rho.data(), sizeof(double) * g.ne, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->d_pas, pas.data(), g.ne, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(s->d_rt, 0, sizeof(double) * g.ne, st);
  cudaMemsetAsync(s->d_dcb, 0, sizeof(double) * g.ne, st);
  cudaMemsetAsync(s->d_dc, 0, sizeof(double) * g.ne, st);
  if (o.warm_start_displacements && o.warm_start_len == g.nd && s->ncase == 1)
    cudaMemcpyAsync(s->d_u, o.warm_start_displacements, sizeof(double) * g.nd, cudaMemcpyHostToDevice, st);
  else
    cudaMemsetAsync(s->d_u, 0, sizeof(double) * g.nd, st);
  if (s->d_uc) cudaMemsetAsync(s->d_uc, 0, sizeof(double) * s->ncase * g.nd, st);
  for (auto& e : s->ev) cudaEventCreate(&e);
  if (cudaMallocHost(&s->h_pin, 256) != cudaSuccess) s->h_pin = nullptr;
  cudaError_t pe = cudaGetLastError();
  if (pe == cudaSuccess && !s->h_pin) pe = cudaErrorMemoryAllocation;
  if (pe != cudaSuccess) {
    mycel_simp_end(s);
    return set_error(c, MYCEL_E_DEVICE, std::string("SIMP set-up: ") + cudaGetErrorString(pe));
  }
  rc = mycel_filter_create(p, s->rmin, &s->filt);
  if (rc) {
    mycel_simp_end(s);
    return rc;
  }
  s->start = s->iter = o.start_iteration;
  s->maxit = o.max_iterations;
  s->done = s->iter > s->maxit;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    mycel_simp_end(s);
    return set_error(c, MYCEL_E_DEVICE, std::string("SIMP set-up: ") + cudaGetErrorString(e));
  }
  // initial options' pointers are not kept beyond begin
  s->o.passive_mask = nullptr;
  s->o.initial_density = nullptr;
  s->o.warm_start_displacements = nullptr;
  p->sessions.push_back(s);
  *out = s;
  return MYCEL_OK;
}

// One SIMP iteration in four phases, so that a batch of sessions can run each phase for all of them (their
// solves packed): simp_pre (continuation, filter, E/DiagA, tolerance), the solve, simp_post_issue
// (compliance, sensitivities, adjoint filter, OC, read-backs queued) and, after the stream is synchronised,
// simp_post_finish (host state, record, stop rule).
struct SimpPre {
  double penal = 3.0, tol = 1e-8;
  std::chrono::steady_clock::time_point t0;
};

static void simp_pre(mycel_simp_session* s, SimpPre* pre) {
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  cudaStream_t st = c->stream;
  const mycel_simp_options& o = s->o;
  const int iter = s->iter;
  pre->t0 = std::chrono::steady_clock::now();
  // 1. penalisation continuation (:176-183)
  double penal = o.penal;
  if (o.continuation) penal = iter < 20 ? 1.0 : (iter < 40 ? 2.0 : o.penal);
  cudaEventRecord(s->ev[0], st);
  // 2. filter (:191-202); passive elements are kept at 1 by the OC kernel and the initial design
  launch_filter_fwd(s->filt, s->d_rho, s->d_rt);
  if (o.enable_heaviside) {
    launch_heaviside(c, p->n_active, p->d_active, s->d_rt, nullptr, s->d_rb, s->beta, 0.5, 0);
  }
  cudaEventRecord(s->ev[1], st);
  // E_e and DiagA from the physical densities (:204-209)
  launch_update_E(p, s->d_rb, penal);
  launch_diag(p);
  // 3. solver tolerance schedule (:211-224): host scalar control, glibc log10/pow as Math.Log10/Math.Pow
  double tol;
  if (iter == s->start) {
    tol = o.solver_tolerance_initial;
  } else {
    double ta = clampd((s->max_change - 0.01) / 0.09, 0.0, 1.0);
    double li = std::log10(std::max(o.solver_tolerance_initial, 1e-15));
    double lf = std::log10(std::max(o.solver_tolerance_final, 1e-15));
    double lt = lf + ta * (li - lf);
    tol = std::pow(10.0, lt);
  }
  pre->penal = penal;
  pre->tol = tol;
}

// the load cases' results folded into one (iterations and times summed, the largest residual, the first failure)
static void fold_cases(const mycel_pcg_result* rs, int n, mycel_pcg_result* pr) {
  std::memset(pr, 0, sizeof *pr);
  pr->converged = 1;
  for (int k = 0; k < n && pr->converged; ++k) {
    const mycel_pcg_result& rk = rs[k];
    pr->iterations += rk.iterations;
    pr->inner_iterations += rk.inner_iterations;
    pr->fallback_iterations += rk.fallback_iterations;
    pr->refinement_steps += rk.refinement_steps;
    pr->elapsed_ms += rk.elapsed_ms;
    pr->final_residual = std::max(pr->final_residual, rk.final_residual);
    pr->converged = rk.converged;
    std::memcpy(pr->message, rk.message, sizeof pr->message);
  }
}

// the load cases of a session are solved together (packed or alone) in the mixed multigrid form
static bool cases_solved_together(const mycel_simp_session* s) {
  return s->o.precision == MYCEL_PRECISION_MIXED_MG && s->ncase <= kMaxBatchedCases && cases_together_enabled();
}

// 4. warm-started PCG (:226-253); with the load cases apart one solve per case from its own warm start, all
// on this iteration's stiffness (the solver set-up is shared)
static int32_t simp_solve(mycel_simp_session* s, const SimpPre& pre, const volatile int32_t* cancel,
                          mycel_pcg_result* pr) {
  mycel_problem* p = s->p;
  const mycel_simp_options& o = s->o;
  int32_t rc;
  const int64_t nd = p->g.nd;
  if (s->ncase == 1) return solve_dispatch(p, s->d_u, pre.tol, o.solver_max_iterations, o.precision, cancel, pr);
  if (cases_solved_together(s)) {  // one V-cycle's coarse levels for all cases
    mycel_pcg_result rs[kMaxBatchedCases];
    if ((rc = mg_solve_cases(p, s->ncase, s->d_uc, pre.tol, o.solver_max_iterations, cancel, rs))) return rc;
    fold_cases(rs, s->ncase, pr);
    return MYCEL_OK;
  }
  std::memset(pr, 0, sizeof *pr);
  pr->converged = 1;
  for (int k = 0; k < s->ncase && pr->converged; ++k) {
    mycel_pcg_result rk;
    if ((rc = solve_case(p, k, s->d_uc + k * nd, pre.tol, o.solver_max_iterations, o.precision, cancel, &rk)))
      return rc;
    pr->iterations += rk.iterations;
    pr->inner_iterations += rk.inner_iterations;
    pr->fallback_iterations += rk.fallback_iterations;
    pr->refinement_steps += rk.refinement_steps;
    pr->elapsed_ms += rk.elapsed_ms;
    pr->final_residual = std::max(pr->final_residual, rk.final_residual);
    pr->converged = rk.converged;
    std::memcpy(pr->message, rk.message, sizeof pr->message);
  }
  return MYCEL_OK;
}

static int32_t simp_post_issue(mycel_simp_session* s, const SimpPre& pre, const mycel_pcg_result& pr) {
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  cudaStream_t st = c->stream;
  const mycel_simp_options& o = s->o;
  const double penal = pre.penal;
  const int64_t nd = p->g.nd;
  cudaEventRecord(s->ev[2], st);
  if (!pr.converged)
    return set_error(c, MYCEL_E_NOT_CONVERGED,
                     "FEM solver did not converge in " + std::to_string(pr.iterations) + " iterations (" + pr.message +
                         "). Is the model not sufficiently constrained?");
  if (s->ncase == 1) {
    // compliance and max |u| (:255-276)
    launch_compliance(p, s->d_u, s->d_scal);
    launch_max_disp(p, s->d_u, s->d_scal + 1);
    // 5. sensitivities and adjoint filter (:278-294)
    launch_sens(p, s->d_u, s->d_rb, penal, s->d_dcb);
  } else {
    // objective sum_k F_k . u_k, the largest |u| over the cases, sensitivities summed in case order, and the
    // reported u = sum_k u_k
    for (int k = 0; k < s->ncase; ++k) {
      launch_compliance(p, p->d_case_F + k * nd, p->d_case_nz + p->case_nz_off[2 * k], p->case_nz_cnt[2 * k],
                        s->d_uc + k * nd, s->d_scal + 16 + k);
      launch_sens(p, s->d_uc + k * nd, s->d_rb, penal, s->d_dcb, k > 0);
    }
    k_sum_in_order<<<1, 1, 0, st>>>(s->d_scal + 16, s->ncase, s->d_scal);
    const double* uc = s->d_uc;
    launch_max_disp(p, &uc, s->ncase, nd, s->d_scal + 1);
    MYCEL_CUDA(c, cudaMemcpyAsync(s->d_u, s->d_uc, sizeof(double) * nd, cudaMemcpyDeviceToDevice, st));
    for (int k = 1; k < s->ncase; ++k)
      k_add_into<<<(unsigned)((nd + 255) / 256), 256, 0, st>>>(nd, s->d_u, s->d_uc + k * nd);
    c->launches += s->ncase;
  }
  if (o.enable_heaviside) {
    launch_heaviside(c, p->n_active, p->d_active, s->d_rt, s->d_dcb, s->d_dct, s->beta, 0.5, 1);
    launch_filter_adj(s->filt, s->d_dct, s->d_dc);
  } else {
    launch_filter_adj(s->filt, s->d_dcb, s->d_dc);
  }
  cudaEventRecord(s->ev[3], st);
  // 6. OC update with lambda carried over (:296-311) + metrics (:322-338)
  // the plain method takes every bisection decision as the reference's sequential sums do; the other forms
  // (not bit-exact anyway) decide on the grid's tree sums
  OcParams prm{o.volume_fraction, o.move_limit, o.rho_min, s->lambda, 1e-8, 60, o.enable_heaviside};
  prm.exact = o.precision == MYCEL_PRECISION_FP64 ? 1 : 0;
  prm.total_s = s->total_s;
  int32_t rc = launch_oc(c, p->n_active, p->d_active, s->d_rho, s->d_dc, s->filt->d_s, s->d_pas, s->d_rho_new,
                         s->d_rb, o.enable_heaviside ? s->d_rt : s->d_rb, prm, s->d_oc_scr,
                         oc_scratch_doubles(c->oc_grid), s->d_oc);
  if (rc) return set_error(c, rc, "OC kernel launch failed");
  cudaEventRecord(s->ev[4], st);
  double* hsc = (double*)s->h_pin;
  OcOut* ho = (OcOut*)((char*)s->h_pin + 64);
  MYCEL_CUDA(c, cudaMemcpyAsync(hsc, s->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  MYCEL_CUDA(c, cudaMemcpyAsync(ho, s->d_oc, sizeof(OcOut), cudaMemcpyDeviceToHost, st));
  return MYCEL_OK;
}

static int32_t simp_post_finish(mycel_simp_session* s, const SimpPre& pre, const mycel_pcg_result& pr,
                                mycel_iter_record* rec, int32_t* done) {
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  const mycel_simp_options& o = s->o;
  const int iter = s->iter;
  const double* hsc = (const double*)s->h_pin;
  const OcOut* ho = (const OcOut*)((const char*)s->h_pin + 64);
  if (ho->trials == 0) return set_error(c, MYCEL_E_TIMEOUT, "OC grid barrier timed out");
  std::swap(s->d_rho, s->d_rho_new);
  s->lambda = ho->lambda;
  s->total_s = ho->total_s;
  if (o.enable_heaviside && iter % 25 == 0 && s->beta < 8.0) s->beta = std::min(8.0, s->beta * 2.0);
  s->max_change = ho->max_change;
  double na = (double)p->n_active;
  mycel_iter_record r{};
  r.iteration = iter;
  r.compliance = hsc[0];
  r.volume_fraction = ho->vol_sum / na;
  r.max_change = ho->max_change;
  r.grey_level = (4.0 * ho->grey_sum / na) * 100.0;
  r.solver_iterations = pr.iterations;
  r.solver_residual = pr.final_residual;
  r.max_displacement = hsc[1];
  r.refinement_steps = pr.refinement_steps;
  float ms = 0;
  cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]);
  r.filter_ms = ms;
  r.solve_ms = pr.elapsed_ms;
  cudaEventElapsedTime(&ms, s->ev[2], s->ev[3]);
  r.sensitivity_ms = ms;
  cudaEventElapsedTime(&ms, s->ev[3], s->ev[4]);
  r.update_ms = ms;
  r.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - pre.t0).count();
  if (rec) *rec = r;
  s->last = r;
  s->count++;
  // stop rule (:374-390)
  s->chist.push_back(r.compliance);
  if (s->chist.size() > 6) s->chist.pop_front();
  if (s->chist.size() == 6) {
    double rel = std::fabs(r.compliance - s->chist.front()) / r.compliance;
    if (s->max_change < 0.01 && rel < 1e-3) {
      s->converged = true;
      s->done = true;
    }
  }
  s->iter++;
  if (s->iter > s->maxit) s->done = true;
  if (done) *done = s->done ? 1 : 0;
  return MYCEL_OK;
}

static int32_t simp_step_impl(mycel_simp_session* s, mycel_iter_record* rec, int32_t* done,
                              const volatile int32_t* cancel) {
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  if (done) *done = s->done ? 1 : 0;
  if (s->done) return MYCEL_OK;
  SimpPre pre;
  simp_pre(s, &pre);
  mycel_pcg_result pr;
  int32_t rc = simp_solve(s, pre, cancel, &pr);
  if (rc) return rc;
  if ((rc = simp_post_issue(s, pre, pr))) return rc;
  MYCEL_CUDA(c, cudaStreamSynchronize(c->stream));
  return simp_post_finish(s, pre, pr, rec, done);
}

extern "C" int32_t mycel_simp_step(mycel_simp_session* s, mycel_iter_record* rec, int32_t* done) {
  if (!s) return set_error(nullptr, MYCEL_E_ARG, "NULL session");
  return simp_step_impl(s, rec, done, nullptr);
}

// One SIMP iteration of each of n sessions (one context, one session per problem). The sessions in the mixed
// multigrid form have their solves packed (mg_solve_packed: every kernel of an FP32 outer iteration one launch
// for all of them); the others are solved one after another. Each session's iteration is the one
// mycel_simp_step would take. status[i] (optional) gets each session's own status; the call returns the
// first failure (MYCEL_OK when none). A session that is done is left as it is.
extern "C" int32_t mycel_simp_step_many(mycel_simp_session* const* ss, int32_t n, mycel_iter_record* recs,
                                        int32_t* done, int32_t* status, const volatile int32_t* cancel) {
  if (!ss || n < 1) return set_error(nullptr, MYCEL_E_ARG, "NULL sessions or count below 1");
  for (int i = 0; i < n; ++i)
    if (!ss[i]) return set_error(nullptr, MYCEL_E_ARG, "NULL session");
  mycel_ctx* c = ss[0]->p->ctx;
  for (int i = 0; i < n; ++i) {
    if (ss[i]->p->ctx != c) return set_error(c, MYCEL_E_ARG, "the sessions of a batch step share one context");
    for (int j = 0; j < i; ++j)
      if (ss[j]->p == ss[i]->p) return set_error(c, MYCEL_E_ARG, "each session of a batch step has its own problem");
  }
  cudaSetDevice(c->device);
  // MYCEL_VERBOSE: host time of each phase, each ended by a synchronisation (for breakdowns only)
  const bool verbose = std::getenv("MYCEL_VERBOSE") != nullptr;
  auto tp = std::chrono::steady_clock::now();
  auto lap = [&](const char* what) {
    if (!verbose) return;
    cudaStreamSynchronize(c->stream);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "mycel: step_many %s %.3f ms\n", what, std::chrono::duration<double, std::milli>(now - tp).count());
    tp = now;
  };
  std::vector<SimpPre> pre(n);
  std::vector<mycel_pcg_result> pr(n);
  std::vector<int32_t> st(n, MYCEL_OK);
  std::vector<char> live(n, 0);
  std::vector<std::vector<mycel_pcg_result>> cres(n);
  std::vector<PackJob> jobs;
  std::vector<int> job_of;
  bool fan_on = false;
  for (int i = 0; i < n; ++i) {
    mycel_simp_session* s = ss[i];
    if (done) done[i] = s->done ? 1 : 0;
    if (s->done) continue;
    live[i] = 1;
    if (!fan_on) fan_on = fan_begin(c) == MYCEL_OK;  // the sessions' filters and E side by side
    if (fan_on) fan_use(c, i);
    simp_pre(s, &pre[i]);
    const bool packable = s->o.precision == MYCEL_PRECISION_MIXED_MG && (s->ncase == 1 || cases_solved_together(s));
    if (!packable) continue;
    cres[i].resize(s->ncase);
    jobs.push_back(PackJob{s->p, s->ncase, s->ncase == 1 ? s->d_u : s->d_uc, pre[i].tol, s->o.solver_max_iterations,
                           cres[i].data()});
    job_of.push_back(i);
  }
  if (fan_on) fan_end(c);
  lap("filter, E, diagonal");
  if (!jobs.empty()) {
    int32_t rc = mg_solve_packed(c, (int)jobs.size(), jobs.data(), cancel);
    for (size_t q = 0; q < jobs.size(); ++q) {
      const int i = job_of[q];
      if (rc) st[i] = rc;
      else fold_cases(cres[i].data(), ss[i]->ncase, &pr[i]);
    }
  }
  for (int i = 0; i < n; ++i) {
    mycel_simp_session* s = ss[i];
    if (!live[i] || !cres[i].empty() || st[i]) continue;
    st[i] = simp_solve(s, pre[i], cancel, &pr[i]);
  }
  lap("solves");
  fan_on = fan_begin(c) == MYCEL_OK;  // sensitivities, adjoint filters and OC updates side by side
  for (int i = 0; i < n; ++i)
    if (live[i] && !st[i]) {
      if (fan_on) fan_use(c, i);
      st[i] = simp_post_issue(ss[i], pre[i], pr[i]);
    }
  if (fan_on) fan_end(c);
  lap("sensitivities, adjoint, OC");
  cudaError_t e = cudaStreamSynchronize(c->stream);
  int32_t first = MYCEL_OK;
  for (int i = 0; i < n; ++i) {
    if (live[i] && !st[i]) {
      if (e != cudaSuccess) st[i] = set_error(c, MYCEL_E_DEVICE, std::string("SIMP step: ") + cudaGetErrorString(e));
      else st[i] = simp_post_finish(ss[i], pre[i], pr[i], recs ? recs + i : nullptr, done ? done + i : nullptr);
    }
    if (status) status[i] = st[i];
    if (!first && st[i]) first = st[i];
  }
  return first;
}

static int32_t snapshot(mycel_simp_session* s) {
  mycel_problem* p = s->p;
  cudaStream_t st = p->ctx->stream;
  k_snapshot<<<(unsigned)((p->g.ne + 255) / 256), 256, 0, st>>>(p->g.ne, p->d_domain, s->d_rb, s->d_rho, s->d_phys_f,
                                                                 s->d_des_f);
  p->ctx->launches++;
  return MYCEL_OK;
}

extern "C" int32_t mycel_simp_read(mycel_simp_session* s, double* u, float* phys, float* des, double* rpa,
                                   double* rda, double* lambda) {
  if (!s) return set_error(nullptr, MYCEL_E_ARG, "NULL session");
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  cudaStream_t st = c->stream;
  if (phys || des) {
    snapshot(s);
    if (phys) MYCEL_CUDA(c, cudaMemcpyAsync(phys, s->d_phys_f, sizeof(float) * p->g.ne, cudaMemcpyDeviceToHost, st));
    if (des) MYCEL_CUDA(c, cudaMemcpyAsync(des, s->d_des_f, sizeof(float) * p->g.ne, cudaMemcpyDeviceToHost, st));
  }
  if (u) MYCEL_CUDA(c, cudaMemcpyAsync(u, s->d_u, sizeof(double) * p->g.nd, cudaMemcpyDeviceToHost, st));
  if (rpa) {
    launch_gather_active(p, s->d_rb, p->d_tmp0);
    MYCEL_CUDA(c, cudaMemcpyAsync(rpa, p->d_tmp0, sizeof(double) * p->n_active, cudaMemcpyDeviceToHost, st));
    MYCEL_CUDA(c, cudaStreamSynchronize(st));
  }
  if (rda) {
    launch_gather_active(p, s->d_rho, p->d_tmp1);
    MYCEL_CUDA(c, cudaMemcpyAsync(rda, p->d_tmp1, sizeof(double) * p->n_active, cudaMemcpyDeviceToHost, st));
  }
  MYCEL_CUDA(c, cudaStreamSynchronize(st));
  if (lambda) *lambda = s->lambda;
  return MYCEL_OK;
}

// ---- RunWriter frames (Persistence/RunWriter.cs:132-160, 199-245, 344-356) ----
extern "C" int32_t mycel_simp_frame_begin(mycel_simp_session* s, int32_t* slot_out) {
  if (!s || !slot_out) return set_error(s ? s->p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  if (s->count == 0) return set_error(c, MYCEL_E_INVALID_OPERATION, "no iteration has been run yet");
  const int slot = s->frame_next;
  if (s->frame_busy[slot])
    return set_error(c, MYCEL_E_INVALID_OPERATION, "both frame slots are pending: end one first");
  const int64_t ne = p->g.ne;
  if (!s->d_frame[slot]) {
    MYCEL_CUDA(c, cudaMallocAsync((void**)&s->d_frame[slot], (size_t)ne, c->stream));
    MYCEL_CUDA(c, cudaMallocHost((void**)&s->h_frame[slot], (size_t)ne));
    MYCEL_CUDA(c, cudaEventCreateWithFlags(&s->frame_ev[slot], cudaEventDisableTiming));
  }
  snapshot(s);
  k_quantize<<<(unsigned)((ne + 255) / 256), 256, 0, c->stream>>>(ne, s->d_phys_f, s->d_frame[slot]);
  c->launches++;
  MYCEL_CUDA(c, cudaMemcpyAsync(s->h_frame[slot], s->d_frame[slot], (size_t)ne, cudaMemcpyDeviceToHost, c->stream));
  MYCEL_CUDA(c, cudaEventRecord(s->frame_ev[slot], c->stream));
  s->frame_rec[slot] = s->last;
  s->frame_busy[slot] = true;
  s->frame_next = slot ^ 1;
  *slot_out = slot;
  return MYCEL_OK;
}

extern "C" int32_t mycel_simp_frame_end(mycel_simp_session* s, int32_t slot, uint8_t* frame_out, uint8_t* header_out,
                                        uint32_t* checksum_out) {
  if (!s) return set_error(nullptr, MYCEL_E_ARG, "NULL session");
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  if (slot < 0 || slot > 1 || !s->frame_busy[slot])
    return set_error(c, MYCEL_E_ARG, "frame slot is not pending");
  cudaSetDevice(c->device);
  MYCEL_CUDA(c, cudaEventSynchronize(s->frame_ev[slot]));
  s->frame_busy[slot] = false;
  const int64_t ne = p->g.ne;
  const uint8_t* q = s->h_frame[slot];
  // ComputeQuantizedChecksum (:344-356): FNV-1a over the bytes in order (sequential by definition)
  uint32_t h = 2166136261u;
  for (int64_t i = 0; i < ne; ++i) h = (h ^ q[i]) * 16777619u;
  if (frame_out) std::memcpy(frame_out, q, (size_t)ne);
  if (checksum_out) *checksum_out = h;
  if (header_out) {
    // WriteIterationFileAtomic header (:223-235): little-endian fields at fixed offsets
    const mycel_iter_record& r = s->frame_rec[slot];
    uint8_t hd[72] = {};
    auto put32 = [&](int o, uint32_t v) { for (int b = 0; b < 4; ++b) hd[o + b] = (uint8_t)(v >> (8 * b)); };
    auto putd = [&](int o, double v) {
      uint64_t u;
      std::memcpy(&u, &v, 8);
      for (int b = 0; b < 8; ++b) hd[o + b] = (uint8_t)(u >> (8 * b));
    };
    hd[0] = 'T'; hd[1] = 'O'; hd[2] = 'P'; hd[3] = 'O';
    put32(4, 1u);
    put32(8, (uint32_t)p->g.nx);
    put32(12, (uint32_t)p->g.ny);
    put32(16, (uint32_t)p->g.nz);
    put32(20, (uint32_t)r.iteration);
    putd(24, r.compliance);
    putd(32, r.volume_fraction);
    putd(40, r.max_change);
    putd(48, r.grey_level);
    put32(56, (uint32_t)r.solver_iterations);
    putd(60, r.total_ms);
    put32(68, h);
    std::memcpy(header_out, hd, 72);
  }
  return MYCEL_OK;
}

extern "C" int32_t mycel_simp_end(mycel_simp_session* s) {
  if (!s) return MYCEL_OK;
  auto& live = s->p->sessions;
  live.erase(std::remove(live.begin(), live.end(), s), live.end());
  cudaSetDevice(s->p->ctx->device);
  cudaStreamSynchronize(s->p->ctx->stream);
  if (s->filt) mycel_filter_destroy(s->filt);
  cudaStream_t st = s->p->ctx->stream;
  double* dptr[] = {s->d_rho, s->d_rho_new, s->d_rt, s->d_dcb, s->d_dc, s->d_u, s->d_scal, s->d_oc_scr, s->d_uc};
  for (double* q : dptr)
    if (q) cudaFreeAsync(q, st);
  if (s->o.enable_heaviside) {
    if (s->d_rb) cudaFreeAsync(s->d_rb, st);
    if (s->d_dct) cudaFreeAsync(s->d_dct, st);
  }
  if (s->d_oc) cudaFreeAsync(s->d_oc, st);
  if (s->d_pas) cudaFreeAsync(s->d_pas, st);
  if (s->d_phys_f) cudaFreeAsync(s->d_phys_f, st);
  if (s->d_des_f) cudaFreeAsync(s->d_des_f, st);
  for (auto& e : s->ev)
    if (e) cudaEventDestroy(e);
  if (s->h_pin) cudaFreeHost(s->h_pin);
  for (int k = 0; k < 2; ++k) {
    if (s->d_frame[k]) cudaFreeAsync(s->d_frame[k], st);
    if (s->h_frame[k]) cudaFreeHost(s->h_frame[k]);
    if (s->frame_ev[k]) cudaEventDestroy(s->frame_ev[k]);
  }
  delete s;
  return MYCEL_OK;
}

extern "C" int32_t mycel_simp_run(mycel_problem* p, const mycel_simp_options* opt, mycel_progress_fn progress,
                                  void* user, const volatile int32_t* cancel, const volatile int32_t* pause,
                                  mycel_iter_record* history, int32_t cap, int32_t* n_iters, int32_t* converged,
                                  double* u_out, float* phys_out, float* des_out) {
  if (n_iters) *n_iters = 0;
  if (converged) *converged = 0;
  mycel_simp_session* s = nullptr;
  int32_t rc = mycel_simp_begin(p, opt, &s);
  if (rc) return rc;
  mycel_ctx* c = p->ctx;
  if (progress) {
    s->h_phys.resize((size_t)p->g.ne);
    s->h_des.resize((size_t)p->g.ne);
  }
  int32_t err = MYCEL_OK;
  while (!s->done) {
    // IterationController.CheckAndBlock / CancellationToken (:168-172)
    if (cancel && *cancel) break;
    while (pause && *pause && !(cancel && *cancel)) std::this_thread::sleep_for(std::chrono::milliseconds(1));
    if (cancel && *cancel) break;
    mycel_iter_record r;
    int32_t d = 0;
    err = simp_step_impl(s, &r, &d, cancel);
    if (err == MYCEL_E_CANCELLED) {
      err = MYCEL_OK;
      break;
    }
    if (err) break;
    if (history && s->count - 1 < cap) history[s->count - 1] = r;
    if (progress) {
      snapshot(s);
      cudaMemcpyAsync(s->h_phys.data(), s->d_phys_f, sizeof(float) * p->g.ne, cudaMemcpyDeviceToHost, c->stream);
      cudaMemcpyAsync(s->h_des.data(), s->d_des_f, sizeof(float) * p->g.ne, cudaMemcpyDeviceToHost, c->stream);
      cudaStreamSynchronize(c->stream);
      progress(user, &r, s->h_phys.data(), s->h_des.data());
    }
  }
  if (n_iters) *n_iters = s->count;
  if (converged) *converged = s->converged ? 1 : 0;
  std::string msg = c->last_error;
  if (s->count > 0 || !err) {
    int32_t rr = mycel_simp_read(s, u_out, phys_out, des_out, nullptr, nullptr, nullptr);
    if (!err) err = rr;
  }
  mycel_simp_end(s);
  if (err) c->last_error = msg;
  return err;
}

// Whole optimisations of n sessions (one context, one session per problem) to their ends: every session runs
// until its stop rule fires or max_iterations is reached, as with mycel_simp_step in a loop, and its records
// go to history[i * cap ...] (n_iters[i] of them, at most cap). When every session is in the mixed multigrid
// form (load cases summed, or kept apart and solved together) their solves share one packed plan for the
// whole run and each problem goes on to its next SIMP iteration as soon as its own solve ends (the others may
// still be solving); otherwise the sessions are stepped together by mycel_simp_step_many. Each session's
// iterates are those of its run alone.
extern "C" int32_t mycel_simp_run_many(mycel_simp_session* const* ss, int32_t n, mycel_iter_record* history,
                                       int32_t cap, int32_t* n_iters, int32_t* status,
                                       const volatile int32_t* cancel) {
  if (!ss || n < 1) return set_error(nullptr, MYCEL_E_ARG, "NULL sessions or count below 1");
  for (int i = 0; i < n; ++i)
    if (!ss[i]) return set_error(nullptr, MYCEL_E_ARG, "NULL session");
  mycel_ctx* c = ss[0]->p->ctx;
  for (int i = 0; i < n; ++i) {
    if (ss[i]->p->ctx != c) return set_error(c, MYCEL_E_ARG, "the sessions of a batch run share one context");
    for (int j = 0; j < i; ++j)
      if (ss[j]->p == ss[i]->p) return set_error(c, MYCEL_E_ARG, "each session of a batch run has its own problem");
  }
  cudaSetDevice(c->device);
  std::vector<int32_t> st(n, MYCEL_OK);
  auto record = [&](int i, const mycel_iter_record& r) {
    if (n_iters) {
      if (history && n_iters[i] < cap) history[(int64_t)i * cap + n_iters[i]] = r;
      n_iters[i]++;
    }
  };
  if (n_iters)
    for (int i = 0; i < n; ++i) n_iters[i] = 0;
  std::vector<PackRunJob> jobs;
  for (int i = 0; i < n; ++i) {
    mycel_simp_session* s = ss[i];
    const bool form = s->o.precision == MYCEL_PRECISION_MIXED_MG && (s->ncase == 1 || cases_solved_together(s));
    jobs.push_back(PackRunJob{s->p, form ? s->ncase : 0, s->ncase == 1 ? s->d_u : s->d_uc});
  }
  PackRun* run = nullptr;
  std::vector<char> pmask(n, 0);
  if (pkr_open(c, jobs, &run, &pmask) != MYCEL_OK) run = nullptr;
  if (!run) {  // sessions stepped together, each SIMP iteration a barrier
    std::vector<mycel_iter_record> recs(n);
    std::vector<int32_t> dn(n), sst(n);
    for (;;) {
      std::vector<mycel_simp_session*> live;
      std::vector<int> idx;
      for (int i = 0; i < n; ++i)
        if (!ss[i]->done && !st[i]) live.push_back(ss[i]), idx.push_back(i);
      if (live.empty()) break;
      if (cancel && *cancel) break;
      mycel_simp_step_many(live.data(), (int)live.size(), recs.data(), dn.data(), sst.data(), cancel);
      for (size_t q = 0; q < live.size(); ++q) {
        if (sst[q]) st[idx[q]] = sst[q];
        else record(idx[q], recs[q]);
      }
    }
  } else {
    // Each packed session cycles through: solving (its right-hand sides in the packed chunks), SIMP update
    // (sensitivities, adjoint filter, OC) and start of the next solve (filter, E, set-up, start of the solve)
    // on a side stream of the context while the chunks of the others go on; the host polls the side stream's
    // event and takes the next step when it has passed.
    enum : int { J_SOLVE = 0, J_POST = 1, J_BEGIN = 2, J_OFF = 3 };
    std::vector<SimpPre> pre(n);
    std::vector<char> live(n, 0);
    std::vector<int> phase(n, J_OFF);
    std::vector<cudaEvent_t> ev(n, nullptr);
    std::vector<mycel_pcg_result> pr(n);
    int32_t rc = MYCEL_OK;
    for (int i = 0; i < n && !rc; ++i)
      if (pmask[i] && cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess)
        rc = set_error(c, MYCEL_E_DEVICE, "packed run: events");
    for (int i = 0; i < n && !rc; ++i) {  // first starts on the context stream, then one wait
      if (ss[i]->done) continue;
      live[i] = 1;
      if (!pmask[i]) continue;
      simp_pre(ss[i], &pre[i]);
      if ((st[i] = pkr_begin(run, i, pre[i].tol, ss[i]->o.solver_max_iterations))) live[i] = 0;
      else phase[i] = J_SOLVE;
    }
    if (!rc) rc = cudaStreamSynchronize(c->stream) == cudaSuccess ? pkr_after_begin(run)
                                                                  : set_error(c, MYCEL_E_DEVICE, "packed run start");
    // MYCEL_VERBOSE: host time in the chunks (with the refinement of what stopped) and waiting for side work
    const bool verbose = std::getenv("MYCEL_VERBOSE") != nullptr;
    double t_adv = 0.0, t_wait = 0.0;
    int64_t n_adv = 0, n_end = 0;
    std::vector<int> ended;
    while (!rc) {
      bool any = false;
      for (int i = 0; i < n; ++i) any = any || live[i];
      if (!any) break;
      for (int i = 0; i < n; ++i) {  // the sessions the packed form cannot take: one SIMP iteration each
        if (!live[i] || pmask[i]) continue;
        mycel_iter_record r{};
        int32_t d = 0;
        if ((st[i] = simp_step_impl(ss[i], &r, &d, cancel))) {
          live[i] = 0;
          continue;
        }
        record(i, r);
        if (d || (cancel && *cancel)) live[i] = 0;
      }
      ended.clear();
      const auto ta = std::chrono::steady_clock::now();
      if ((rc = pkr_advance(run, cancel, &ended))) break;
      t_adv += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count();
      ++n_adv;
      n_end += (int64_t)ended.size();
      for (int i : ended) {  // the solve has ended: the SIMP update on the session's side stream
        fold_cases(pkr_results(run, i), ss[i]->ncase, &pr[i]);
        cudaStream_t fs = nullptr;
        if ((rc = fan_use_free(c, i, &fs))) break;
        st[i] = simp_post_issue(ss[i], pre[i], pr[i]);
        if (!st[i] && cudaEventRecord(ev[i], fs) != cudaSuccess) st[i] = set_error(c, MYCEL_E_DEVICE, "packed run: event");
        fan_restore(c);
        if (st[i]) live[i] = 0, phase[i] = J_OFF;
        else phase[i] = J_POST;
      }
      if (rc) break;
      bool waiting = false;
      for (int i = 0; i < n && !rc; ++i) {
        if (!live[i] || (phase[i] != J_POST && phase[i] != J_BEGIN)) continue;
        const cudaError_t q = cudaEventQuery(ev[i]);
        if (q == cudaErrorNotReady) {
          waiting = true;
          continue;
        }
        if (q != cudaSuccess) {
          rc = set_error(c, MYCEL_E_DEVICE, std::string("packed run: ") + cudaGetErrorString(q));
          break;
        }
        if (phase[i] == J_BEGIN) {  // its start has been read back: it joins the chunks
          if ((st[i] = pkr_after_begin_job(run, i))) live[i] = 0, phase[i] = J_OFF;
          else phase[i] = J_SOLVE;
          continue;
        }
        mycel_iter_record r{};
        int32_t d = 0;
        if ((st[i] = simp_post_finish(ss[i], pre[i], pr[i], &r, &d))) {
          live[i] = 0;
          phase[i] = J_OFF;
          continue;
        }
        record(i, r);
        if (d || (cancel && *cancel)) {
          live[i] = 0;
          phase[i] = J_OFF;
          continue;
        }
        cudaStream_t fs = nullptr;  // the next iteration's filter, E, set-up and solve start, on the side stream
        if ((rc = fan_use_free(c, i, &fs))) break;
        simp_pre(ss[i], &pre[i]);
        st[i] = pkr_begin(run, i, pre[i].tol, ss[i]->o.solver_max_iterations);
        if (!st[i] && cudaEventRecord(ev[i], fs) != cudaSuccess) st[i] = set_error(c, MYCEL_E_DEVICE, "packed run: event");
        fan_restore(c);
        if (st[i]) live[i] = 0, phase[i] = J_OFF;
        else phase[i] = J_BEGIN, waiting = true;
      }
      if (rc) break;
      bool stepped_alone = false;
      for (int i = 0; i < n; ++i) stepped_alone = stepped_alone || (live[i] && !pmask[i]);
      if (!waiting && ended.empty() && !stepped_alone && !pkr_running(run)) {
        bool solving = false;  // a session that solves but has nothing running would never go on
        for (int i = 0; i < n; ++i) solving = solving || (live[i] && phase[i] == J_SOLVE);
        if (solving) rc = set_error(c, MYCEL_E_TIMEOUT, "packed run: a solve has nothing left to run");
        break;
      }
      if (waiting && !pkr_running(run)) {  // nothing to iterate: wait for the first pending side work
        const auto tw = std::chrono::steady_clock::now();
        for (int i = 0; i < n; ++i)
          if (live[i] && (phase[i] == J_POST || phase[i] == J_BEGIN)) {
            cudaEventSynchronize(ev[i]);
            break;
          }
        t_wait += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tw).count();
      }
    }
    cudaStreamSynchronize(c->stream);
    for (int i = 0; i < n; ++i)  // side work still in flight after an error or a cancellation
      if (ev[i]) cudaEventSynchronize(ev[i]);
    if (verbose)
      std::fprintf(stderr, "mycel: run_many chunks %lld (%.1f ms), solves ended %lld, waiting for side work %.1f ms\n",
                   (long long)n_adv, t_adv, (long long)n_end, t_wait);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    pkr_close(run);
    if (rc && rc != MYCEL_E_CANCELLED)
      for (int i = 0; i < n; ++i)
        if (live[i] && !st[i]) st[i] = rc;
  }
  int32_t first = MYCEL_OK;
  for (int i = 0; i < n; ++i) {
    if (status) status[i] = st[i];
    if (!first && st[i]) first = st[i];
  }
  return first;
}

namespace mycel {
bool simp_session_converged(const mycel_simp_session* s) { return s && s->converged; }
}  // namespace mycel

extern "C" int32_t mycel_simp_converged(const mycel_simp_session* s) { return s && s->converged ? 1 : 0; }

extern "C" int32_t mycel_simp_surface_nets(mycel_simp_session* s, const float* origin, float threshold,
                                           mycel_mesh** out) {
  if (!s || !out) return set_error(s ? s->p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  mycel_problem* p = s->p;
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  if (s->count == 0) return set_error(c, MYCEL_E_INVALID_OPERATION, "no iteration has been run yet");
  const float zero[3] = {0.0f, 0.0f, 0.0f};
  snapshot(s);  // the float physical density of the last iteration, on the device
  return surface_nets_core(c, p->g.nx, p->g.ny, p->g.nz, p->h, origin ? origin : zero, nullptr, s->d_phys_f,
                           threshold, out);
}
