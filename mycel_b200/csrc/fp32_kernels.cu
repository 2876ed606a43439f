// Mixed-precision form: FP32 inner Jacobi-PCG (K·u and the preconditioner in FP32 with FP32 accumulation)
// inside FP64 iterative refinement. FP64 is kept only for the refinement residual f - K u, the CG alpha/beta
// dot products (FP32 operands, products and sums in FP64), and the outer update u += s d.
//
// Per inner iteration two kernels:
//   k_mv32   p_t = z + beta p_{t-1} (on the fly for every gathered node), Ap_t = K p_t, and the FP64 partials of
//            p_t . Ap_t; the last CTA forms alpha.
//   k_xr32   x += alpha p, r -= alpha Ap, z = r invD, FP64 partials of r.r and r.z; the last CTA forms the inner
//            residual, the stop test and beta.
// Reductions use a fixed CTA decomposition and a block-ordered final sum, so results do not depend on timing.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <chrono>
#include <cstring>
#include <string>

#include "internal.h"

namespace mycel {

enum MixStatus : int { MIX_RUNNING = 0, MIX_DONE = 1, MIX_BREAKDOWN = 2, MIX_MAXITER = 3 };

struct MixState {
  int status;
  int iter;      // inner iterations of this refinement step
  int max_iter;
  int pad;
  double eta;    // inner relative tolerance
  double r0n2;   // ||r32_0||^2
  double rho0, alpha, beta, rel_in, rn2, pap;
  unsigned int counter;
  unsigned int pad2;
};

constexpr int kT = 256;

__device__ __forceinline__ int local_index32(int ox, int oy, int oz) {
  int base = oy ? (ox ? 2 : 3) : (ox ? 1 : 0);
  return base + 4 * oz;
}

__device__ __forceinline__ double ld_vol(const double* p) { return *(const volatile double*)p; }

__device__ __forceinline__ bool elect_last32(unsigned int* counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x * gridDim.y - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// deterministic block sum of a double (result valid in thread 0)
__device__ __forceinline__ double bsum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
  return t;
}

// ---------------------------------------------------------------------------------------------------------
// FP32 K p with on-the-fly p update (parity-class node mapping as in the FP64 kernel)
// ---------------------------------------------------------------------------------------------------------
template <int MODE>  // 0: y = K x (plain), 1: inner-PCG step (p update + pAp partials)
__global__ void __launch_bounds__(kT) k_mv32(GridDims g, const __grid_constant__ KeF ke, const float* __restrict__ xin,
                                             const float* __restrict__ z, const float* __restrict__ pold,
                                             float* __restrict__ pnew, float* __restrict__ y,
                                             const float* __restrict__ E, const uint8_t* __restrict__ dom,
                                             const uint8_t* __restrict__ nf, int projected, MixState* st,
                                             double* part) {
  __shared__ double sh[32];
  if (MODE == 1 && st->status != MIX_RUNNING) return;
  const float beta = MODE == 1 ? (float)st->beta : 0.0f;
  const bool first = MODE == 1 ? (st->iter == 0) : true;
  const int cls = blockIdx.y;
  const int px = cls & 1, py = (cls >> 1) & 1, pz = (cls >> 2) & 1;
  const int cx = (g.nx1 - px + 1) >> 1, cy = (g.ny1 - py + 1) >> 1, cz = (g.nz1 - pz + 1) >> 1;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = t < (int64_t)cx * cy * cz;
  double pap = 0.0;
  if (valid) {
    int a_ = (int)(t % cx);
    int64_t rest = t / cx;
    int i = px + 2 * a_, j = py + 2 * (int)(rest % cy), k = pz + 2 * (int)(rest / cy);
    const int64_t sy = g.nx1, sz = (int64_t)g.nx1 * g.ny1;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
#pragma unroll 1
    for (int col = 0; col < 8; ++col) {
      int ox = (col & 1) ^ px, oy = ((col >> 1) & 1) ^ py, oz = ((col >> 2) & 1) ^ pz;
      int ie = i - ox, je = j - oy, kk = k - oz;
      if (ie < 0 || ie >= g.nx || je < 0 || je >= g.ny || kk < 0 || kk >= g.nz) continue;
      int64_t e = ie + (int64_t)g.nx * (je + (int64_t)g.ny * kk);
      if (!__ldg(dom + e)) continue;
      float ee = __ldg(E + e);
      int64_t n0 = ie + sy * je + sz * kk;
      const int64_t off[8] = {0, 1, 1 + sy, sy, sz, sz + 1, sz + 1 + sy, sz + sy};
      float ue[24];
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        int64_t q = 3 * (n0 + off[b]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float v;
          if (MODE == 1) v = first ? __ldg(z + q + c) : fmaf(beta, __ldg(pold + q + c), __ldg(z + q + c));
          else v = __ldg(xin + q + c);
          ue[3 * b + c] = v * ee;
        }
      }
      const int a = local_index32(ox, oy, oz);
      const float* r0 = ke.v + (3 * a) * 24;
      float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
      for (int c = 0; c < 24; ++c) {
        s0 = fmaf(r0[c], ue[c], s0);
        s1 = fmaf(r0[24 + c], ue[c], s1);
        s2 = fmaf(r0[48 + c], ue[c], s2);
      }
      acc0 += s0;
      acc1 += s1;
      acc2 += s2;
    }
    int64_t n = i + sy * j + sz * k;
    uint8_t f = projected ? nf[n] : 0;
    float out[3] = {acc0, acc1, acc2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      int64_t q = 3 * n + c;
      float pv;
      if (MODE == 1) {
        pv = first ? z[q] : fmaf(beta, pold[q], z[q]);
        pnew[q] = pv;
      } else {
        pv = xin[q];
      }
      float yv = (f & (1 << c)) ? pv : out[c];
      y[q] = yv;
      if (MODE == 1) pap += (double)pv * (double)yv;
    }
  }
  if (MODE != 1) return;
  double b = bsum(pap, sh);
  const unsigned nblk = gridDim.x * gridDim.y;
  const unsigned bid = blockIdx.y * gridDim.x + blockIdx.x;
  if (threadIdx.x == 0) part[bid] = b;
  if (!elect_last32(&st->counter)) return;
  if (threadIdx.x != 0) return;
  st->counter = 0;
  double s = 0.0;
  for (unsigned q = 0; q < nblk; ++q) s += ld_vol(part + q);
  st->pap = s;
  if (!(s > 0.0) || !isfinite(s)) {
    st->status = MIX_BREAKDOWN;
    return;
  }
  st->alpha = st->rho0 / s;
}

// x += alpha p, r -= alpha Ap, z = r invD; partials of r.r and r.z (FP64)
__global__ void __launch_bounds__(kT) k_xr32(int64_t n, float* __restrict__ x, float* __restrict__ r,
                                             float* __restrict__ z, const float* __restrict__ p,
                                             const float* __restrict__ ap, const float* __restrict__ invd,
                                             MixState* st, double* part, int init) {
  __shared__ double sh[32];
  if (st->status != MIX_RUNNING) return;
  const float alpha = init ? 0.f : (float)st->alpha;
  double rr = 0.0, rz = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float rv = r[i];
    if (!init) {
      x[i] = fmaf(alpha, p[i], x[i]);
      rv = fmaf(-alpha, ap[i], rv);
      r[i] = rv;
    }
    float zv = rv * invd[i];
    z[i] = zv;
    rr += (double)rv * (double)rv;
    rz += (double)rv * (double)zv;
  }
  double brr = bsum(rr, sh);
  double brz = bsum(rz, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = brr;
    part[gridDim.x + blockIdx.x] = brz;
  }
  if (!elect_last32(&st->counter)) return;
  if (threadIdx.x != 0) return;
  st->counter = 0;
  double srr = 0.0, srz = 0.0;
  for (unsigned q = 0; q < gridDim.x; ++q) {
    srr += ld_vol(part + q);
    srz += ld_vol(part + gridDim.x + q);
  }
  if (init) {
    st->r0n2 = srr;
    st->rho0 = srz;
    st->iter = 0;
    st->rel_in = 1.0;
    if (!(srr > 0.0)) st->status = MIX_DONE;
    return;
  }
  st->iter += 1;
  st->rn2 = srr;
  double rel = sqrt(srr / st->r0n2);
  st->rel_in = rel;
  if (rel <= st->eta) {
    st->status = MIX_DONE;
    return;
  }
  double beta = srz / st->rho0;
  if (!isfinite(beta) || beta < 0.0) {
    st->status = MIX_BREAKDOWN;
    return;
  }
  st->beta = beta;
  st->rho0 = srz;
  if (st->iter >= st->max_iter) st->status = MIX_MAXITER;
}

// FP64 refinement residual r64 = P(b - A u) with partials of r64.r64; scaled FP32 copy r32 = r64 / ||r64||
__global__ void k_resid64(int64_t n, const uint8_t* __restrict__ nf, const double* __restrict__ b,
                          const double* __restrict__ au, double* __restrict__ r64, double* part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    bool con = nf[i / 3] & (1 << (i % 3));
    double v = con ? 0.0 : (b[i] - au[i]);
    r64[i] = v;
    s += v * v;
  }
  double bs = bsum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
}

__global__ void k_sum_part(const double* part, int nb, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int q = 0; q < nb; ++q) s += part[q];
  *out = s;
}

__global__ void k_scale_to_f32(int64_t n, const double* __restrict__ r64, const double* __restrict__ n2,
                               float* __restrict__ r32, float* __restrict__ x32) {
  double inv = 1.0 / sqrt(*n2);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    r32[i] = (float)(r64[i] * inv);
    x32[i] = 0.f;
  }
}

__global__ void k_axpy_u(int64_t n, double* __restrict__ u, const float* __restrict__ d, const double* __restrict__ n2) {
  double s = sqrt(*n2);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    u[i] += s * (double)d[i];
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_to_f64(int64_t n, const float* __restrict__ a, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

static dim3 cls_grid(const GridDims& g) {
  int cx = (g.nx1 + 1) >> 1, cy = (g.ny1 + 1) >> 1, cz = (g.nz1 + 1) >> 1;
  int64_t tot = (int64_t)cx * cy * cz;
  return dim3((unsigned)((tot + kT - 1) / kT), 8, 1);
}

static int stream_blocks(mycel_problem* p) { return p->ctx->num_sms * 8; }

void launch_E_to_f32(mycel_problem* p) {
  (void)p;  // k_update_E writes the FP32 copy of E alongside the FP64 one
}

void mixed_apply_k_f64io(mycel_problem* p, const double* x, double* y, int projected) {
  cudaStream_t s = p->ctx->stream;
  int64_t n = p->g.nd;
  float* fx = (float*)p->d_r;  // borrow FP64 workspace as FP32 staging
  float* fy = fx + n;
  k_to_f32<<<stream_blocks(p), kT, 0, s>>>(n, x, fx);
  k_mv32<0><<<cls_grid(p->g), kT, 0, s>>>(p->g, p->kef, fx, nullptr, nullptr, nullptr, fy, p->d_Ef, p->d_domain,
                                         p->d_nflags, projected, nullptr, nullptr);
  k_to_f64<<<stream_blocks(p), kT, 0, s>>>(n, fy, y);
  p->ctx->launches += 3;
}

static int32_t ensure_mixed(mycel_problem* p) {
  if (p->f_x) return MYCEL_OK;
  int64_t n = p->g.nd;
  size_t fb = sizeof(float) * (size_t)n + 64;
  cudaError_t e = cudaSuccess;
  float** bufs[] = {&p->f_x, &p->f_r, &p->f_z, &p->f_p0, &p->f_p1, &p->f_ap};
  for (float** b : bufs) {
    if ((e = cudaMalloc((void**)b, fb)) != cudaSuccess) break;
    p->device_bytes += (int64_t)fb;
  }
  if (e == cudaSuccess) {
    e = cudaMalloc((void**)&p->d_r64, sizeof(double) * (size_t)n + 64);
    p->device_bytes += (int64_t)(sizeof(double) * n);
  }
  if (e != cudaSuccess) return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the mixed-precision workspace");
  return MYCEL_OK;
}

static MixState* mix_state(mycel_problem* p) {
  // lives after the FP64 PcgState in the same allocation? use the tail of d_part2
  return (MixState*)(p->d_part2 + p->n_part2 - 64);
}

__global__ void k_mix_init(MixState* st, double eta, int max_iter) {
  MixState s = {};
  s.status = MIX_RUNNING;
  s.eta = eta;
  s.max_iter = max_iter;
  *st = s;
}

static int32_t capture_mixed_graph(mycel_problem* p, int chunk) {
  if (p->pcg32_graph) return MYCEL_OK;
  cudaStream_t s = p->ctx->stream;
  int64_t n = p->g.nd;
  MixState* st = mix_state(p);
  double* part = p->d_part2;
  int sb = stream_blocks(p);
  int64_t before = p->ctx->launches;
  cudaGraph_t graph;
  MYCEL_CUDA(p->ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int t = 0; t < chunk; ++t) {
    float* pcur = (t & 1) ? p->f_p1 : p->f_p0;
    float* pprev = (t & 1) ? p->f_p0 : p->f_p1;
    k_mv32<1><<<cls_grid(p->g), kT, 0, s>>>(p->g, p->kef, nullptr, p->f_z, pprev, pcur, p->f_ap, p->d_Ef,
                                           p->d_domain, p->d_nflags, 1, st, part);
    k_xr32<<<sb, kT, 0, s>>>(n, p->f_x, p->f_r, p->f_z, pcur, p->f_ap, p->d_invdf, st, part, 0);
  }
  MYCEL_CUDA(p->ctx, cudaStreamEndCapture(s, &graph));
  p->ctx->launches = before;
  MYCEL_CUDA(p->ctx, cudaGraphInstantiate(&p->pcg32_graph, graph, 0));
  cudaGraphDestroy(graph);
  p->pcg32_graph_chunk = chunk;
  return MYCEL_OK;
}

// Mixed solve of A u = b (A = P K P + I - P) to ||P(b - A u)|| / ||P b|| <= tol, measured in FP64.
int32_t mixed_solve_entry(mycel_problem* p, const double* d_b, const int32_t* d_nz, int32_t n_nz, double* d_u,
                          double tol, int max_iter, const volatile int32_t* cancel, mycel_pcg_result* res) {
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  auto t0 = std::chrono::steady_clock::now();
  std::memset(res, 0, sizeof *res);
  if (p->n_active_fixed < 6)
    return set_error(c, MYCEL_E_UNDERCONSTRAINED,
                     "Model has fewer than 6 unique fixed DOFs on active nodes (found " +
                         std::to_string(p->n_active_fixed) +
                         "). At least 6 fixed DOFs are required to prevent rigid body modes in 3D.");
  int32_t st = ensure_pcg_workspace(p);
  if (st) return st;
  if ((st = ensure_mixed(p))) return st;
  const int64_t n = p->g.nd;
  const int sb = stream_blocks(p);
  double* part = p->d_part2;
  double* scal = p->d_part2 + p->n_part2 - 128;  // [0] ||r64||^2
  MixState* ms = mix_state(p);
  // project u and ||P b|| (same kernels as the FP64 path)
  double* saved_b = p->d_b;
  int32_t* saved_nz = p->d_bnz;
  int32_t saved_n = p->n_bnz;
  p->d_b = const_cast<double*>(d_b);
  p->d_bnz = const_cast<int32_t*>(d_nz);
  p->n_bnz = n_nz;
  struct Restore {
    mycel_problem* p; double* b; int32_t* nz; int32_t n;
    ~Restore() { p->d_b = b; p->d_bnz = nz; p->n_bnz = n; }
  } restore{p, saved_b, saved_nz, saved_n};
  cudaMemsetAsync(p->d_state, 0, sizeof(PcgState), s);
  launch_project_x(p, d_u, &p->d_state->nonzero_x);
  launch_pcg_bnorm(p);
  PcgState* hs = (PcgState*)c->pinned;
  MYCEL_CUDA(c, cudaMemcpyAsync(hs, p->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  const double bnorm = hs->bnorm;
  if (bnorm <= 1e-30) {
    MYCEL_CUDA(c, cudaMemsetAsync(d_u, 0, sizeof(double) * n, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    res->converged = 1;
    std::snprintf(res->message, sizeof res->message, "RHS is zero. Solution is zero.");
    return MYCEL_OK;
  }
  if ((st = capture_mixed_graph(p, 16))) return st;
  int total_inner = 0, steps = 0;
  double rel = 0.0;
  bool ok = false, broke = false;
  const int max_steps = 30;
  double* hsc = (double*)((char*)c->pinned + 1024);
  MixState* hms = (MixState*)((char*)c->pinned + 2048);
  for (;;) {
    // r64 = P(b - A u), ||r64||
    launch_matvec64(p, d_u, p->d_ap, 1, nullptr);
    k_resid64<<<sb, kT, 0, s>>>(n, p->d_nflags, d_b, p->d_ap, p->d_r64, part);
    k_sum_part<<<1, 32, 0, s>>>(part, sb, scal);
    c->launches += 2;
    MYCEL_CUDA(c, cudaMemcpyAsync(hsc, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    rel = std::sqrt(hsc[0]) / bnorm;
    if (rel <= tol) {
      ok = true;
      break;
    }
    if (steps >= max_steps || total_inner >= max_iter || broke) break;
    if (cancel && *cancel) return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
    // inner FP32 solve of A d = r64 / ||r64|| to relative accuracy eta
    double eta = std::max(0.5 * tol / rel, 1e-5);
    eta = std::min(eta, 0.1);
    k_scale_to_f32<<<sb, kT, 0, s>>>(n, p->d_r64, scal, p->f_r, p->f_x);
    k_mix_init<<<1, 1, 0, s>>>(ms, eta, max_iter - total_inner);
    k_xr32<<<sb, kT, 0, s>>>(n, p->f_x, p->f_r, p->f_z, p->f_p0, p->f_ap, p->d_invdf, ms, part, 1);
    c->launches += 3;
    int64_t launched = 0;
    for (;;) {
      MYCEL_CUDA(c, cudaMemcpyAsync(hms, ms, sizeof(MixState), cudaMemcpyDeviceToHost, s));
      MYCEL_CUDA(c, cudaStreamSynchronize(s));
      if (hms->status != MIX_RUNNING) break;
      if (launched > (int64_t)(max_iter - total_inner) + 4 * p->pcg32_graph_chunk)
        return set_error(c, MYCEL_E_TIMEOUT, "inner PCG device state did not reach a final status");
      launched += p->pcg32_graph_chunk;
      if (cancel && *cancel) return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
      MYCEL_CUDA(c, cudaGraphLaunch(p->pcg32_graph, s));
      c->launches += 2 * p->pcg32_graph_chunk;
    }
    total_inner += hms->iter;
    if (hms->status == MIX_BREAKDOWN && hms->iter == 0) broke = true;
    k_axpy_u<<<sb, kT, 0, s>>>(n, d_u, p->f_x, scal);
    c->launches++;
    ++steps;
  }
  res->iterations = total_inner;
  res->inner_iterations = total_inner;
  res->refinement_steps = steps;
  res->final_residual = rel;
  res->converged = ok ? 1 : 0;
  if (!ok)
    std::snprintf(res->message, sizeof res->message,
                  "PCG reached maximum iterations without converging. Is the model not sufficiently constrained?");
  res->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return MYCEL_OK;
}

}  // namespace mycel
