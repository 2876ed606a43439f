// C ABI of libmycel_b200: context, problem residency, the PCG driver, StaticAnalysis.Run and the SIMP loop
// (TopologyOptimizer.Run). Host code here only marshals descriptors, sequences kernels and reads back scalars;
// every vector operation of the path runs in this library's kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "internal.h"

using namespace mycel;

namespace mycel {

static thread_local std::string tls_error;

int32_t set_error(mycel_ctx* ctx, int32_t code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  tls_error = msg;
  return code;
}

}  // namespace mycel

namespace {

template <class T>
cudaError_t dalloc(mycel_problem* p, T** ptr, size_t count) {
  size_t bytes = std::max<size_t>(sizeof(T) * count, 16);
  bytes = (bytes + 15) & ~size_t(15);
  // stream-ordered: no device-wide synchronisation, so set-up and tear-down of one problem do not stall the
  // work of others running on other streams (the serving loop)
  cudaError_t e = cudaMallocAsync((void**)ptr, bytes, p->ctx->stream);
  if (e == cudaSuccess) p->device_bytes += (int64_t)bytes;
  return e;
}

void dfree(cudaStream_t s, void* ptr) {
  if (ptr) cudaFreeAsync(ptr, s);
}

std::string fmt_e3(double v) {
  // .NET "E3": one digit, '.', three digits, 'E', sign, at least three exponent digits
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v > 0 ? "\xe2\x88\x9e" : "-\xe2\x88\x9e";
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.3E", v);
  char* e = std::strchr(buf, 'E');
  if (e) {
    char sign = e[1];
    int ex = std::atoi(e + 2);
    std::snprintf(e, sizeof buf - (size_t)(e - buf), "E%c%03d", sign, ex);
  }
  return buf;
}

std::string underconstrained_msg(int64_t n) {
  return "Model has fewer than 6 unique fixed DOFs on active nodes (found " + std::to_string(n) +
         "). At least 6 fixed DOFs are required to prevent rigid body modes in 3D.";
}

// PcgResult.Message for a finished device state (PcgSolver.cs:149-367)
void fill_result(const PcgState& st, mycel_pcg_result* res) {
  res->iterations = st.iter;
  res->final_residual = st.rel;
  res->converged = 0;
  std::string m;
  switch (st.status) {
    case PCG_CONVERGED: res->converged = 1; break;
    case PCG_INIT_CONVERGED:
      res->converged = 1;
      m = "Initial guess already converged.";
      break;
    case PCG_RHS_ZERO:
      res->converged = 1;
      res->final_residual = 0.0;
      m = "RHS is zero. Solution is zero.";
      break;
    case PCG_BREAK_CURVATURE:
      m = "PCG curvature breakdown (p\xe1\xb5\x80" "Ap = " + fmt_e3(st.last_bad) +
          " <= 0). Is the model not sufficiently constrained?";
      break;
    case PCG_BREAK_ALPHA:
      m = "PCG step breakdown (alpha = " + fmt_e3(st.last_bad) + "). Is the model not sufficiently constrained?";
      break;
    case PCG_STAGNATED: m = "PCG stagnated: residual stopped decreasing. Is the model not sufficiently constrained?"; break;
    case PCG_BREAK_BETA:
      m = "PCG search direction breakdown (beta = " + fmt_e3(st.last_bad) +
          "). Is the model not sufficiently constrained?";
      break;
    default: m = "PCG reached maximum iterations without converging. Is the model not sufficiently constrained?"; break;
  }
  std::snprintf(res->message, sizeof res->message, "%s", m.c_str());
}

}  // namespace
namespace mycel {
int32_t ensure_pcg_workspace(mycel_problem* p) {
  if (p->d_x) return MYCEL_OK;
  int64_t nd = p->g.nd;
  int64_t nb = num_blocks8192(nd);
  if (dalloc(p, &p->d_x, nd) || dalloc(p, &p->d_r, nd) || dalloc(p, &p->d_z, nd) || dalloc(p, &p->d_p, nd) ||
      dalloc(p, &p->d_ap, nd) || dalloc(p, &p->d_part, 2 * nb + 64) || dalloc(p, &p->d_state, 1))
    return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the PCG workspace");
  cudaMemsetAsync(p->d_state, 0, sizeof(PcgState), p->ctx->stream);
  return MYCEL_OK;
}
}  // namespace mycel
namespace {

PcgState* pinned_state(mycel_ctx* c) { return (PcgState*)c->pinned; }

int32_t read_state(mycel_problem* p, PcgState* out) {
  PcgState* hs = pinned_state(p->ctx);
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(hs, p->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, p->ctx->stream));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(p->ctx->stream));
  *out = *hs;
  return MYCEL_OK;
}

__global__ void k_state_init(PcgState* st, double tol, int max_iter) {
  PcgState s = {};
  s.status = PCG_RUNNING;
  s.max_iter = max_iter;
  s.tol = tol;
  *st = s;
}

__global__ void k_state_rel_from_b(PcgState* st) {
  // zero warm start: rNormSq = bNormSq (PcgSolver.cs:185-192)
  st->rn2 = st->bn2;
  double rel = sqrt(st->bn2) / st->bnorm;
  st->rel = rel;
  st->prev = rel;
  if (rel <= st->tol) st->status = PCG_INIT_CONVERGED;
}

// ordered list of indices i with b[i] != 0 and DOF i unconstrained (P b non-zeros, ascending)
// F[idx[q]] = val[q]: the assembled forces' non-zero entries
__global__ void k_scatter_forces(int32_t n, const int32_t* __restrict__ idx, const double* __restrict__ val,
                                 double* __restrict__ F) {
  const int32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) F[idx[q]] = val[q];
}

// b = P F: F with the constrained DOFs zeroed
__global__ void k_project_rhs(int64_t n, const double* __restrict__ F, const uint8_t* __restrict__ nf,
                              double* __restrict__ b) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (nf[i / 3] & (1 << (i % 3))) ? 0.0 : F[i];
}

__global__ void k_nz_count(int64_t n, const double* __restrict__ b, const uint8_t* __restrict__ nf, int32_t* cnt) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int v = 0;
  if (i < n) v = (b[i] != 0.0) && !(nf[i / 3] & (1 << (i % 3)));
  v = __syncthreads_count(v);
  if (threadIdx.x == 0) cnt[blockIdx.x] = v;
}
__global__ void k_nz_write(int64_t n, const double* __restrict__ b, const uint8_t* __restrict__ nf,
                           const int32_t* __restrict__ cnt, int32_t* out, int32_t* total) {
  __shared__ int32_t base;
  __shared__ int32_t wsum[32];
  if (threadIdx.x == 0) {
    int32_t s = 0;
    for (unsigned k = 0; k < blockIdx.x; ++k) s += cnt[k];
    base = s;
    if (blockIdx.x == gridDim.x - 1) *total = s + cnt[blockIdx.x];
  }
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int v = 0;
  if (i < n) v = (b[i] != 0.0) && !(nf[i / 3] & (1 << (i % 3)));
  unsigned m = __ballot_sync(0xffffffffu, v);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wsum[w] = __popc(m);
  __syncthreads();
  if (v) {
    int32_t off = base;
    for (int k = 0; k < w; ++k) off += wsum[k];
    off += __popc(m & ((1u << lane) - 1u));
    out[off] = (int32_t)i;
  }
}

// Build the ordered P b non-zero list for an arbitrary device vector b into dst (capacity nd); returns count.
int32_t build_nz_list(mycel_problem* p, const double* d_bvec, int32_t* dst, int32_t* count) {
  int64_t n = p->g.nd;
  unsigned nb = (unsigned)((n + 255) / 256);
  int32_t* cnt = (int32_t*)p->d_part2;  // borrow: needs nb + 1 ints
  cudaStream_t s = p->ctx->stream;
  k_nz_count<<<nb, 256, 0, s>>>(n, d_bvec, p->d_nflags, cnt);
  k_nz_write<<<nb, 256, 0, s>>>(n, d_bvec, p->d_nflags, cnt, dst, cnt + nb);
  p->ctx->launches += 2;
  int32_t* h = (int32_t*)p->ctx->pinned;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(h, cnt + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  *count = *h;
  return MYCEL_OK;
}

const int kChunkIters = 16;

int32_t capture_pcg_graph(mycel_problem* p) {
  mycel_ctx* c = p->ctx;
  if (p->pcg_graph[0] && p->pcg_graph_profiled == c->profile) return MYCEL_OK;
  cudaStream_t s = c->stream;
  int64_t before = c->launches;
  for (int k = 0; k < 2; ++k) {
    if (p->pcg_graph[k]) cudaGraphExecDestroy(p->pcg_graph[k]);
    p->pcg_graph[k] = nullptr;
    for (int j = 0; j < 2; ++j)
      if (!p->prof64_ev[k][j]) cudaEventCreate(&p->prof64_ev[k][j]);
    cudaGraph_t graph;
    MYCEL_CUDA(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < kChunkIters; ++i) launch_pcg_iteration(p, c->profile && i == 0);
    MYCEL_CUDA(c, cudaStreamEndCapture(s, &graph));
    MYCEL_CUDA(c, cudaGraphInstantiate(&p->pcg_graph[k], graph, 0));
    cudaGraphDestroy(graph);
  }
  c->launches = before;  // captured launches are counted when the graph is replayed
  p->pcg_graph_chunk = kChunkIters;
  p->pcg_graph_profiled = c->profile;
  return MYCEL_OK;
}

// Chunk launch; when profiling, the first matvec runs directly between two stream events (outside the graph).
void launch_pcg_chunk(mycel_problem* p, int gi) {
  cudaStream_t s = p->ctx->stream;
  if (p->pcg_graph_profiled) {
    cudaEventRecord(p->prof64_ev[gi][0], s);
    launch_matvec64(p, p->d_p, p->d_ap, 1, &p->d_state->status);
    cudaEventRecord(p->prof64_ev[gi][1], s);
  }
  cudaGraphLaunch(p->pcg_graph[gi], s);
}

}  // namespace

namespace mycel {

// FP64 PCG (PcgSolver.Solve with Jacobi) on device vectors. d_b: right-hand side; nz list: ascending indices of
// the non-zero entries of P b; d_xv: warm start in, solution out. cancel may be NULL.
int32_t pcg_solve_fp64(mycel_problem* p, const double* d_bv, const int32_t* d_nz, int32_t n_nz, double* d_xv,
                       double tol, int max_iter, const volatile int32_t* cancel, mycel_pcg_result* res) {
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  auto t0 = std::chrono::steady_clock::now();
  std::memset(res, 0, sizeof *res);
  if (p->n_active_fixed < 6) return set_error(c, MYCEL_E_UNDERCONSTRAINED, underconstrained_msg(p->n_active_fixed));
  int32_t st = ensure_pcg_workspace(p);
  if (st) return st;
  // The kernels work on p->d_x / p->d_b; bind the caller's vectors.
  if (d_xv != p->d_x) MYCEL_CUDA(c, cudaMemcpyAsync(p->d_x, d_xv, sizeof(double) * p->g.nd, cudaMemcpyDeviceToDevice, s));
  double* saved_b = p->d_b;
  int32_t* saved_nz = p->d_bnz;
  int32_t saved_n = p->n_bnz;
  p->d_b = const_cast<double*>(d_bv);
  p->d_bnz = const_cast<int32_t*>(d_nz);
  p->n_bnz = n_nz;
  struct Restore {
    mycel_problem* p; double* b; int32_t* nz; int32_t n;
    ~Restore() { p->d_b = b; p->d_bnz = nz; p->n_bnz = n; }
  } restore{p, saved_b, saved_nz, saved_n};

  k_state_init<<<1, 1, 0, s>>>(p->d_state, tol, max_iter);
  c->launches++;
  launch_project_x(p, p->d_x, &p->d_state->nonzero_x);
  launch_pcg_bnorm(p);
  PcgState hs;
  if ((st = read_state(p, &hs))) return st;
  if (hs.bnorm <= 1e-30) {
    MYCEL_CUDA(c, cudaMemsetAsync(p->d_x, 0, sizeof(double) * p->g.nd, s));
    if (d_xv != p->d_x) MYCEL_CUDA(c, cudaMemcpyAsync(d_xv, p->d_x, sizeof(double) * p->g.nd, cudaMemcpyDeviceToDevice, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    hs.status = PCG_RHS_ZERO;
    hs.iter = 0;
    fill_result(hs, res);
    res->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return MYCEL_OK;
  }
  if (hs.nonzero_x) {
    launch_matvec64(p, p->d_x, p->d_ap, 1, nullptr);
    launch_pcg_init_r(p, 1);
    launch_pcg_dot_rr(p);
  } else {
    launch_pcg_init_r(p, 0);
    k_state_rel_from_b<<<1, 1, 0, s>>>(p->d_state);
    c->launches++;
  }
  launch_pcg_init_z(p);
  if ((st = capture_pcg_graph(p))) return st;
  if ((st = read_state(p, &hs))) return st;
  if (hs.status == PCG_RUNNING) {
    // pipeline: chunk k is queued while the status after chunk k-1 is read
    PcgState* slot[2] = {(PcgState*)((char*)c->pinned + 4096), (PcgState*)((char*)c->pinned + 4096 + 512)};
    cudaEvent_t evs[2];
    cudaEventCreateWithFlags(&evs[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&evs[1], cudaEventDisableTiming);
    struct EvGuard { cudaEvent_t* e; ~EvGuard() { cudaEventDestroy(e[0]); cudaEventDestroy(e[1]); } } evg{evs};
    int64_t launched = 0;
    for (int64_t k = 0;; ++k) {
      if (cancel && *cancel) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
      }
      // the device state machine stops by itself at max_iter; this bound only guards against a broken state
      if (launched > (int64_t)max_iter + 4 * p->pcg_graph_chunk) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_TIMEOUT, "PCG device state did not reach a final status");
      }
      int gi = (int)(k & 1);
      launch_pcg_chunk(p, gi);
      MYCEL_CUDA(c, cudaGetLastError());
      launched += p->pcg_graph_chunk;
      c->launches += 4 * p->pcg_graph_chunk - (p->pcg_graph_profiled ? 1 : 0);  // direct matvec counted itself
      MYCEL_CUDA(c, cudaMemcpyAsync(slot[gi], p->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
      MYCEL_CUDA(c, cudaEventRecord(evs[gi], s));
      if (k == 0) continue;
      int pi = (int)((k - 1) & 1);
      MYCEL_CUDA(c, cudaEventSynchronize(evs[pi]));
      if (slot[pi]->status != PCG_RUNNING) break;
      if (c->profile) {
        float ms_ = 0.f;
        if (cudaEventElapsedTime(&ms_, p->prof64_ev[pi][0], p->prof64_ev[pi][1]) == cudaSuccess) {
          c->prof_ms[1] += ms_;
          c->prof_n[1] += 1;
          c->prof_nodes[1] += p->g.nn;
          c->prof_elems[1] += p->n_active;
        }
      }
    }
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    if ((st = read_state(p, &hs))) return st;
  }
  if (d_xv != p->d_x) MYCEL_CUDA(c, cudaMemcpyAsync(d_xv, p->d_x, sizeof(double) * p->g.nd, cudaMemcpyDeviceToDevice, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  fill_result(hs, res);
  res->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return MYCEL_OK;
}

}  // namespace mycel

// ======================================================================================================
// context
// ======================================================================================================
extern "C" int32_t mycel_version(void) { return 100; }

extern "C" int32_t mycel_ctx_create(int32_t device, mycel_ctx** out) {
  if (!out) return set_error(nullptr, MYCEL_E_ARG, "out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return set_error(nullptr, MYCEL_E_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= n) return set_error(nullptr, MYCEL_E_ARG, "device index out of range");
  mycel_ctx* c = new mycel_ctx();
  c->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
      (e = cudaMallocHost(&c->pinned, 1 << 16)) != cudaSuccess) {
    std::string m = cudaGetErrorString(e);
    delete c;
    return set_error(nullptr, MYCEL_E_DEVICE, m);
  }
  c->pinned_bytes = 1 << 16;
  int oc_bpsm = 0;
  if (oc_blocks_per_sm(&oc_bpsm) != MYCEL_OK) {
    cudaFreeHost(c->pinned);
    cudaStreamDestroy(c->stream);
    if (c->side) cudaStreamDestroy(c->side);
    delete c;
    return set_error(nullptr, MYCEL_E_DEVICE, "occupancy query of the OC kernel failed");
  }
  c->oc_grid = c->num_sms * oc_bpsm;
  // Device memory freed by a problem stays in the device's stream-ordered pool for the next problem instead of
  // going back to the driver at the next synchronisation (re-mapping gigabytes for every job cost up to a few
  // hundred ms per job). A host that needs it released calls cudaMemPoolTrimTo on the default pool.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  *out = c;
  return MYCEL_OK;
}

extern "C" int32_t mycel_ctx_destroy(mycel_ctx* c) {
  if (!c) return MYCEL_OK;
  cudaSetDevice(c->device);
  pack_release(c);  // frees on the stream: before it goes
  fan_release(c);
  if (c->stream) {
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
  }
  if (c->side) {
    cudaStreamSynchronize(c->side);
    cudaStreamDestroy(c->side);
  }
  if (c->pinned) cudaFreeHost(c->pinned);
  delete c;
  return MYCEL_OK;
}

extern "C" void* mycel_ctx_stream(mycel_ctx* c) { return c ? (void*)c->stream : nullptr; }
extern "C" const char* mycel_last_error(mycel_ctx* c) { return c ? c->last_error.c_str() : tls_error.c_str(); }
extern "C" int64_t mycel_ctx_launch_count(mycel_ctx* c) { return c ? c->launches : 0; }
extern "C" int64_t mycel_ctx_packed_count(mycel_ctx* c) { return c ? c->packed_rhs : 0; }

extern "C" int32_t mycel_ctx_set_profiling(mycel_ctx* c, int32_t enable) {
  if (!c) return set_error(nullptr, MYCEL_E_ARG, "NULL context");
  c->profile = enable ? 1 : 0;
  for (int k = 0; k < 4; ++k) c->prof_ms[k] = 0, c->prof_n[k] = 0, c->prof_nodes[k] = 0, c->prof_elems[k] = 0;
  return MYCEL_OK;
}

extern "C" int32_t mycel_ctx_set_oc_wait(mycel_ctx* c, int64_t max_polls, int32_t unreachable) {
  if (!c || max_polls < 0) return set_error(c, MYCEL_E_ARG, "invalid argument");
  c->oc_wait_polls = max_polls;
  c->oc_wait_unreachable = unreachable ? 1 : 0;
  return MYCEL_OK;
}

extern "C" int32_t mycel_problem_kernel_bench(mycel_problem* p, int32_t which, int32_t reps, double* avg_us) {
  if (!p || !avg_us) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  return kernel_bench(p, which, reps, avg_us);
}

extern "C" int32_t mycel_ctx_kernel_timing(mycel_ctx* c, int32_t which, double* total_ms, int64_t* launches,
                                           int64_t* nodes, int64_t* elems) {
  if (!c || which < 0 || which > 3) return set_error(c, MYCEL_E_ARG, "invalid argument");
  if (total_ms) *total_ms = c->prof_ms[which];
  if (launches) *launches = c->prof_n[which];
  if (nodes) *nodes = c->prof_nodes[which];
  if (elems) *elems = c->prof_elems[which];
  return MYCEL_OK;
}

// ======================================================================================================
// problem
// ======================================================================================================
extern "C" int32_t mycel_problem_create(mycel_ctx* c, const mycel_grid* grid, const uint8_t* domain,
                                        const mycel_material* mat, const int32_t* fixed, int32_t n_fixed,
                                        const mycel_load_case* loads, int32_t n_loads, const double* density,
                                        double penal, mycel_problem** out) {
  if (!c || !grid || !domain || !mat || !out) return set_error(c, MYCEL_E_ARG, "NULL argument");
  *out = nullptr;
  if (grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0)
    return set_error(c, MYCEL_E_ARG, "Grid dimensions must be strictly positive.");
  if (!(grid->h > 0.0f)) return set_error(c, MYCEL_E_ARG, "Voxel pitch must be positive.");
  if (n_fixed < 0 || n_loads < 0 || (n_fixed > 0 && !fixed) || (n_loads > 0 && !loads))
    return set_error(c, MYCEL_E_ARG, "invalid fixed DOF or load arrays");
  GridDims g = make_dims(grid->nx, grid->ny, grid->nz);
  if (g.nd >= (int64_t)INT32_MAX) return set_error(c, MYCEL_E_ARG, "grid too large for 32-bit DOF indices");
  for (int32_t i = 0; i < n_fixed; ++i)
    if (fixed[i] < 0 || (int64_t)fixed[i] >= g.nd)
      return set_error(c, MYCEL_E_ARG, "Fixed DOF " + std::to_string(fixed[i]) + " is out of bounds [0, " +
                                           std::to_string(g.nd - 1) + "].");
  cudaSetDevice(c->device);
  (void)cudaGetLastError();  // do not report a stale error of an earlier, unrelated call
  mycel_problem* p = new mycel_problem();
  static std::atomic<uint64_t> next_serial{1};
  p->serial = next_serial.fetch_add(1);
  p->ctx = c;
  p->g = g;
  p->h = grid->h;
  p->e0 = mat->e0;
  p->nu = mat->nu;
  p->emin_ratio = mat->emin_ratio;
  p->emin = mat->e0 * mat->emin_ratio;  // FeMaterial.Emin
  p->penal = penal;
  build_ke((double)grid->h, mat->nu, p->ke.v);
  for (int i = 0; i < 576; ++i) p->kef.v[i] = (float)p->ke.v[i];
  split_ke_tf32(p->ke.v, &p->ketf);
  build_hexop((double)grid->h, mat->nu, &p->hexop);
  build_hexop64((double)grid->h, mat->nu, &p->hexop64);
  for (int i = 0; i < 24; ++i) p->diag_ke[i] = p->ke.v[i * 24 + i];
  p->fixed_host.assign(fixed, fixed + n_fixed);

  // FeModel.AssembleForces (FeModel.cs:263-321): descriptor marshalling of the load patches, O(patch nodes).
  // per DOF the terms are added in assembly order from 0.0, as into the reference's zeroed vector
  std::unordered_map<int64_t, double> facc;
  std::unordered_set<int32_t> seen;
  p->n_cases = std::max<int32_t>(n_loads, 0);
  p->case_terms.assign((size_t)p->n_cases, {});
  for (int32_t li = 0; li < n_loads && !p->assemble_status; ++li) {
    const mycel_load_case& L = loads[li];
    auto& terms = p->case_terms[(size_t)li];
    for (int32_t q = 0; q < L.n_nodes; ++q)
      if (seen.insert(L.nodes[q]).second) p->load_nodes_host.push_back(L.nodes[q]);
    if (L.n_nodes == 0) {
      if (L.force[0] != 0.0f || L.force[1] != 0.0f || L.force[2] != 0.0f) {
        p->assemble_status = MYCEL_E_INVALID_OPERATION;
        p->assemble_msg = "Cannot assemble load case: surface patch contains 0 nodes.";
      }
      continue;
    }
    double total = 0.0;
    for (int32_t q = 0; q < L.n_nodes; ++q) total += L.node_area[q];
    for (int32_t q = 0; q < L.n_nodes; ++q)
      if (L.nodes[q] < 0 || (int64_t)L.nodes[q] >= g.nn) {
        p->assemble_status = MYCEL_E_INVALID_OPERATION;
        p->assemble_msg = "Patch node index " + std::to_string(L.nodes[q]) + " is out of bounds [0, " +
                          std::to_string(g.nn - 1) + "].";
      }
    if (p->assemble_status) break;
    if (total <= 0.0) {
      double inv = 1.0 / L.n_nodes;
      double fx = (double)L.force[0] * inv, fy = (double)L.force[1] * inv, fz = (double)L.force[2] * inv;
      for (int32_t q = 0; q < L.n_nodes; ++q) {
        int64_t n = L.nodes[q];
        facc[3 * n] += fx;
        facc[3 * n + 1] += fy;
        facc[3 * n + 2] += fz;
        terms.push_back({3 * n, fx});
        terms.push_back({3 * n + 1, fy});
        terms.push_back({3 * n + 2, fz});
      }
    } else {
      double inv = 1.0 / total;
      for (int32_t q = 0; q < L.n_nodes; ++q) {
        int64_t n = L.nodes[q];
        double w = L.node_area[q] * inv;
        facc[3 * n] += (double)L.force[0] * w;
        facc[3 * n + 1] += (double)L.force[1] * w;
        facc[3 * n + 2] += (double)L.force[2] * w;
        terms.push_back({3 * n, (double)L.force[0] * w});
        terms.push_back({3 * n + 1, (double)L.force[1] * w});
        terms.push_back({3 * n + 2, (double)L.force[2] * w});
      }
    }
  }
  std::vector<int32_t> active;
  active.reserve((size_t)g.ne);
  for (int64_t e = 0; e < g.ne; ++e)
    if (domain[e]) active.push_back((int32_t)e);
  p->n_active = (int64_t)active.size();
  for (const auto& kv : facc)
    if (kv.second != 0.0) p->f_idx.push_back((int32_t)kv.first);
  std::sort(p->f_idx.begin(), p->f_idx.end());
  p->f_val.resize(p->f_idx.size());
  for (size_t q = 0; q < p->f_idx.size(); ++q) p->f_val[q] = facc[p->f_idx[q]];
  const std::vector<int32_t>& fnz = p->f_idx;
  p->n_fnz = (int32_t)fnz.size();

  cudaStream_t s = c->stream;
  int32_t* d_cnt = nullptr;
  bool ok = !dalloc(p, &p->d_domain, g.ne) && !dalloc(p, &p->d_nflags, (g.nn + 3) & ~int64_t(3)) &&
            !dalloc(p, &p->d_active, std::max<int64_t>(p->n_active, 1)) && !dalloc(p, &p->d_F, g.nd) &&
            !dalloc(p, &p->d_b, g.nd) && !dalloc(p, &p->d_fnz, std::max<int32_t>(p->n_fnz, 1)) &&
            !dalloc(p, &p->d_bnz, std::max<int32_t>(p->n_fnz, 1)) && !dalloc(p, &p->d_rho_box, g.ne) &&
            !dalloc(p, &p->d_E, g.ne) && !dalloc(p, &p->d_Ef, g.ne) && !dalloc(p, &p->d_diag, g.nd) &&
            !dalloc(p, &p->d_invd, g.nd) && !dalloc(p, &p->d_invdf, g.n32) && !dalloc(p, &p->d_tmp0, g.nd) &&
            !dalloc(p, &p->d_tmp1, g.nd) && !dalloc(p, &p->d_fixed, std::max<int32_t>(n_fixed, 1)) &&
            !dalloc(p, &p->d_err, 4) &&
            !dalloc(p, &d_cnt, 4);
  if (ok) ok = !dalloc(p, &p->d_part2, std::max<int64_t>(g.nd / 256 + 1024, 65536));
  p->n_part2 = std::max<int64_t>(g.nd / 256 + 1024, 65536);
  if (!ok) {
    dfree(c->stream, d_cnt);
    mycel_problem_destroy(p);
    return set_error(c, MYCEL_E_OOM, "out of device memory for the problem");
  }
  cudaMemsetAsync(p->d_invdf, 0, sizeof(float) * g.n32, s);  // pads of the padded FP32 layout stay zero
  cudaMemcpyAsync(p->d_domain, domain, g.ne, cudaMemcpyHostToDevice, s);
  if (p->n_active) cudaMemcpyAsync(p->d_active, active.data(), sizeof(int32_t) * p->n_active, cudaMemcpyHostToDevice, s);
  // F: zero, then its non-zero entries scattered (their values staged in tmp0)
  cudaMemsetAsync(p->d_F, 0, sizeof(double) * g.nd, s);
  if (p->n_fnz) {
    cudaMemcpyAsync(p->d_fnz, fnz.data(), sizeof(int32_t) * p->n_fnz, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(p->d_tmp0, p->f_val.data(), sizeof(double) * p->n_fnz, cudaMemcpyHostToDevice, s);
    k_scatter_forces<<<(unsigned)((p->n_fnz + 255) / 256), 256, 0, s>>>(p->n_fnz, p->d_fnz, p->d_tmp0, p->d_F);
    c->launches++;
  }
  if (n_fixed) cudaMemcpyAsync(p->d_fixed, fixed, sizeof(int32_t) * n_fixed, cudaMemcpyHostToDevice, s);
  if (density) {
    cudaMemcpyAsync(p->d_rho_box, density, sizeof(double) * g.ne, cudaMemcpyHostToDevice, s);
  } else {
    std::vector<double> ones((size_t)g.ne, 1.0);
    cudaMemcpyAsync(p->d_rho_box, ones.data(), sizeof(double) * g.ne, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
  }
  cudaMemsetAsync(d_cnt, 0, 16, s);
  cudaMemsetAsync(p->d_err, 0, 16, s);
  cudaMemsetAsync(p->d_E, 0, sizeof(double) * g.ne, s);
  cudaMemsetAsync(p->d_Ef, 0, sizeof(float) * g.ne, s);
  launch_setup_nodes(p, p->d_fixed, n_fixed, d_cnt);
  // b = P F and its ordered non-zero list
  int32_t nb_cnt = 0;
  k_project_rhs<<<(unsigned)((g.nd + 255) / 256), 256, 0, s>>>(g.nd, p->d_F, p->d_nflags, p->d_b);
  c->launches++;
  int32_t st = build_nz_list(p, p->d_F, p->d_bnz, &nb_cnt);
  if (st) {
    dfree(c->stream, d_cnt);
    mycel_problem_destroy(p);
    return st;
  }
  p->n_bnz = nb_cnt;
  // zero b on constrained DOFs: download flags once (set-up) to count active nodes and fixed DOFs
  std::vector<uint8_t> nf((size_t)g.nn);
  int32_t hcnt = 0;
  cudaMemcpyAsync(nf.data(), p->d_nflags, g.nn, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&hcnt, d_cnt, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dfree(c->stream, d_cnt);
  if (e != cudaSuccess) {
    mycel_problem_destroy(p);
    return set_error(c, MYCEL_E_DEVICE, std::string("problem set-up: ") + cudaGetErrorString(e));
  }
  int64_t an = 0;
  for (int64_t n = 0; n < g.nn; ++n) an += (nf[n] & NF_ACTIVE) ? 1 : 0;
  p->n_active_nodes = an;
  p->n_active_fixed = hcnt;
  launch_update_E(p, p->d_rho_box, penal);
  launch_diag(p);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    mycel_problem_destroy(p);
    return set_error(c, MYCEL_E_DEVICE, std::string("problem set-up: ") + cudaGetErrorString(e));
  }
  *out = p;
  return MYCEL_OK;
}

extern "C" int32_t mycel_problem_destroy(mycel_problem* p) {
  if (!p) return MYCEL_OK;
  while (!p->sessions.empty()) mycel_simp_end(p->sessions.back());  // sessions cannot outlive their problem
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  for (int k = 0; k < 2; ++k) {
    if (p->pcg_graph[k]) cudaGraphExecDestroy(p->pcg_graph[k]);
    for (int j = 0; j < 2; ++j)
      if (p->prof64_ev[k][j]) cudaEventDestroy(p->prof64_ev[k][j]);
  }
  for (int k = 0; k < 2; ++k) {
    if (p->pcg32_graph[k]) cudaGraphExecDestroy(p->pcg32_graph[k]);
    if (p->pcg64f_graph[k]) cudaGraphExecDestroy(p->pcg64f_graph[k]);
    for (int j = 0; j < 2; ++j) {
      if (p->prof_ev[k][j]) cudaEventDestroy(p->prof_ev[k][j]);
      if (p->prof64f_ev[k][j]) cudaEventDestroy(p->prof64f_ev[k][j]);
    }
  }
  mg_release(p);
  void* ptrs[] = {p->d_domain, p->d_nflags, p->d_fixed, p->d_err, p->d_active, p->d_e2a, p->d_F, p->d_b, p->d_fnz, p->d_bnz, p->d_rho_box,
                  p->d_case_F, p->d_case_b, p->d_case_nz,
                  p->d_E, p->d_Ef, p->d_diag, p->d_invd, p->d_invdf, p->d_r, p->d_z, p->d_p, p->d_ap, p->d_x,
                  p->d_part, p->d_state, p->f_x, p->f_r, p->f_z, p->f_p0, p->f_p1, p->f_ap, p->d_r64, p->d_part2,
                  p->d_tmp0, p->d_tmp1, p->g_x, p->g_r, p->g_z, p->g_p0, p->g_p1, p->g_ap, p->g_invd};
  for (void* q : ptrs) dfree(p->ctx->stream, q);
  delete p;
  return MYCEL_OK;
}

extern "C" int32_t mycel_problem_info_get(mycel_problem* p, mycel_problem_info* o) {
  if (!p || !o) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  o->total_elements = p->g.ne;
  o->total_nodes = p->g.nn;
  o->total_dofs = p->g.nd;
  o->active_elements = p->n_active;
  o->active_nodes = p->n_active_nodes;
  o->active_fixed_dofs = p->n_active_fixed;
  o->device_bytes = p->device_bytes;
  return MYCEL_OK;
}

extern "C" int32_t mycel_problem_set_tuning(mycel_problem* p, int32_t key, int32_t value) {
  if (!p) return set_error(nullptr, MYCEL_E_ARG, "NULL problem");
  if (key == MYCEL_TUNE_MATVEC32) {
    if (value < 0 || value > MYCEL_MV32_FACTORED)
      return set_error(p->ctx, MYCEL_E_ARG, "matvec variant must be 0 (auto), 1, 2 or 3");
    p->tune_mv32 = value;
    p->mv32 = value == 0 ? -1 : value;
    for (int k = 0; k < 2; ++k)
      if (p->pcg32_graph[k]) {
        cudaGraphExecDestroy(p->pcg32_graph[k]);
        p->pcg32_graph[k] = nullptr;
      }
    return MYCEL_OK;
  }
  return set_error(p->ctx, MYCEL_E_ARG, "unknown tuning key");
}

extern "C" int32_t mycel_problem_get_tuning(mycel_problem* p, int32_t key, int32_t* value) {
  if (!p || !value) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  if (key == MYCEL_TUNE_MATVEC32) {
    *value = p->mv32 < 0 ? 0 : p->mv32;
    return MYCEL_OK;
  }
  return set_error(p->ctx, MYCEL_E_ARG, "unknown tuning key");
}

extern "C" int32_t mycel_problem_forces(mycel_problem* p, double* f) {
  if (!p || !f) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  if (p->assemble_status) return set_error(p->ctx, p->assemble_status, p->assemble_msg);
  std::fill(f, f + p->g.nd, 0.0);
  for (size_t q = 0; q < p->f_idx.size(); ++q) f[p->f_idx[q]] = p->f_val[q];
  return MYCEL_OK;
}

// ---- load cases apart (multi-RHS over one stiffness; the reference sums its cases, FeModel.cs:267-318) ----
static void case_forces_host(const mycel_problem* p, int k, double* f) {
  std::fill(f, f + p->g.nd, 0.0);
  for (const auto& t : p->case_terms[(size_t)k]) f[t.first] += t.second;  // assembly order, as the summed F
}

extern "C" int32_t mycel_problem_load_cases(mycel_problem* p, int32_t* n) {
  if (!p || !n) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  *n = p->n_cases;
  return MYCEL_OK;
}

extern "C" int32_t mycel_problem_case_forces(mycel_problem* p, int32_t k, double* f) {
  if (!p || !f) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  if (p->assemble_status) return set_error(p->ctx, p->assemble_status, p->assemble_msg);
  if (k < 0 || k >= p->n_cases)
    return set_error(p->ctx, MYCEL_E_ARG, "Load case index " + std::to_string(k) + " is out of range [0, " +
                                              std::to_string(p->n_cases) + ").");
  case_forces_host(p, k, f);
  return MYCEL_OK;
}

namespace mycel {
// Device right-hand sides of every load case (first use): F_k, P F_k, and the ascending non-zero lists of F_k
// (compliance F_k . u_k, as k_compliance sums F . u) and of P F_k (the PCG's ||P b||), at case_nz_off[2k] and
// case_nz_off[2k + 1].
int32_t ensure_cases(mycel_problem* p) {
  if (p->d_case_nz || p->n_cases <= 0) return MYCEL_OK;  // the non-zero lists are written last
  if (p->assemble_status) return set_error(p->ctx, p->assemble_status, p->assemble_msg);
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  const int64_t nd = p->g.nd;
  const int m = p->n_cases;
  std::vector<uint8_t> nf((size_t)p->g.nn);
  MYCEL_CUDA(c, cudaMemcpyAsync(nf.data(), p->d_nflags, p->g.nn, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  std::vector<double> f((size_t)nd), b((size_t)nd);
  std::vector<int32_t> lists;
  p->case_nz_off.assign(2 * (size_t)m, 0);
  p->case_nz_cnt.assign(2 * (size_t)m, 0);
  auto release = [&] {  // after a failure nothing is kept, so a later call starts over
    const int64_t fb = ((int64_t)(8 * m * nd) + 15) & ~int64_t(15);
    if (p->d_case_F) p->device_bytes -= fb;
    if (p->d_case_b) p->device_bytes -= fb;
    dfree(s, p->d_case_F);
    dfree(s, p->d_case_b);
    p->d_case_F = p->d_case_b = nullptr;
  };
  if ((!p->d_case_F && dalloc(p, &p->d_case_F, (size_t)(m * nd))) ||
      (!p->d_case_b && dalloc(p, &p->d_case_b, (size_t)(m * nd)))) {
    release();
    return set_error(c, MYCEL_E_OOM, "out of device memory for the load cases");
  }
  for (int k = 0; k < m; ++k) {
    case_forces_host(p, k, f.data());
    p->case_nz_off[2 * k] = (int32_t)lists.size();
    for (int64_t i = 0; i < nd; ++i)
      if (f[i] != 0.0) lists.push_back((int32_t)i);
    p->case_nz_cnt[2 * k] = (int32_t)lists.size() - p->case_nz_off[2 * k];
    p->case_nz_off[2 * k + 1] = (int32_t)lists.size();
    for (int64_t i = 0; i < nd; ++i) {
      b[i] = (nf[i / 3] & (1 << (i % 3))) ? 0.0 : f[i];
      if (b[i] != 0.0) lists.push_back((int32_t)i);
    }
    p->case_nz_cnt[2 * k + 1] = (int32_t)lists.size() - p->case_nz_off[2 * k + 1];
    MYCEL_CUDA(c, cudaMemcpyAsync(p->d_case_F + k * nd, f.data(), sizeof(double) * nd, cudaMemcpyHostToDevice, s));
    MYCEL_CUDA(c, cudaMemcpyAsync(p->d_case_b + k * nd, b.data(), sizeof(double) * nd, cudaMemcpyHostToDevice, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));  // f and b are refilled for the next case
  }
  if (dalloc(p, &p->d_case_nz, std::max<size_t>(lists.size(), 1))) {
    p->d_case_nz = nullptr;
    release();
    return set_error(c, MYCEL_E_OOM, "out of device memory for the load cases");
  }
  if (!lists.empty())
    MYCEL_CUDA(c, cudaMemcpyAsync(p->d_case_nz, lists.data(), sizeof(int32_t) * lists.size(), cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

// PCG solve of load case k (right-hand side P F_k) into d_u, in the given precision
int32_t solve_case(mycel_problem* p, int k, double* d_u, double tol, int max_iter, int precision,
                   const volatile int32_t* cancel, mycel_pcg_result* res) {
  const double* b = p->d_case_b + (int64_t)k * p->g.nd;
  const int32_t* nz = p->d_case_nz + p->case_nz_off[2 * k + 1];
  const int32_t cnt = p->case_nz_cnt[2 * k + 1];
  if (precision == MYCEL_PRECISION_MIXED || precision == MYCEL_PRECISION_FP64_FACTORED ||
      precision == MYCEL_PRECISION_FP64_MG || precision == MYCEL_PRECISION_MIXED_MG)
    return refined_solve_entry(p, b, nz, cnt, d_u, tol, max_iter, cancel, precision, res);
  return pcg_solve_fp64(p, b, nz, cnt, d_u, tol, max_iter, cancel, res);
}
}  // namespace mycel

// ======================================================================================================
// kernel-level entry points
// ======================================================================================================
extern "C" int32_t mycel_update_densities(mycel_problem* p, const double* dens, double penal) {
  if (!p || !dens) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  cudaStream_t s = p->ctx->stream;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_rho_box, dens, sizeof(double) * p->g.ne, cudaMemcpyHostToDevice, s));
  p->penal = penal;
  launch_update_E(p, p->d_rho_box, penal);
  launch_diag(p);
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

extern "C" int32_t mycel_diagonal(mycel_problem* p, double* out) {
  if (!p || !out) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(out, p->d_diag, sizeof(double) * p->g.nd, cudaMemcpyDeviceToHost, p->ctx->stream));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(p->ctx->stream));
  return MYCEL_OK;
}

extern "C" int32_t mycel_apply_k(mycel_problem* p, const double* x, double* y, int32_t projected, int32_t precision) {
  if (!p || !x || !y) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  cudaStream_t s = p->ctx->stream;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_tmp0, x, sizeof(double) * p->g.nd, cudaMemcpyHostToDevice, s));
  if (precision == MYCEL_PRECISION_MIXED || precision == MYCEL_PRECISION_MIXED_MG) {
    int32_t st = ensure_pcg_workspace(p);
    if (st) return st;
    launch_E_to_f32(p);
    // FP32 operator on the FP32-rounded input
    if ((st = mixed_apply_k_f64io(p, p->d_tmp0, p->d_tmp1, projected))) return st;
  } else if (precision == MYCEL_PRECISION_FP64_FACTORED || precision == MYCEL_PRECISION_FP64_MG) {
    int32_t st = fast64_apply_k(p, p->d_tmp0, p->d_tmp1, projected);
    if (st) return st;
  } else {
    launch_matvec64(p, p->d_tmp0, p->d_tmp1, projected, nullptr);
  }
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(y, p->d_tmp1, sizeof(double) * p->g.nd, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

extern "C" int32_t mycel_pcg_solve(mycel_problem* p, const double* b, double* x, double tol, int32_t max_iter,
                                   int32_t precision, mycel_pcg_result* res) {
  if (!p || !b || !x || !res) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  cudaStream_t s = p->ctx->stream;
  int32_t st = ensure_pcg_workspace(p);
  if (st) return st;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_tmp1, b, sizeof(double) * p->g.nd, cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_x, x, sizeof(double) * p->g.nd, cudaMemcpyHostToDevice, s));
  int32_t* nz = (int32_t*)p->d_tmp0;
  int32_t cnt = 0;
  if ((st = build_nz_list(p, p->d_tmp1, nz, &cnt))) return st;
  if (precision == MYCEL_PRECISION_MIXED || precision == MYCEL_PRECISION_FP64_FACTORED ||
      precision == MYCEL_PRECISION_FP64_MG || precision == MYCEL_PRECISION_MIXED_MG) {
    st = refined_solve_entry(p, p->d_tmp1, nz, cnt, p->d_x, tol, max_iter, nullptr, precision, res);
  } else {
    st = pcg_solve_fp64(p, p->d_tmp1, nz, cnt, p->d_x, tol, max_iter, nullptr, res);
  }
  if (st) return st;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(x, p->d_x, sizeof(double) * p->g.nd, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

namespace mycel {
struct Fan {
  static constexpr int kN = 8;
  cudaStream_t s[kN] = {}, side[kN] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kN] = {};
  bool used[kN] = {};
  bool active = false;
};

int32_t fan_begin(mycel_ctx* c) {
  Fan* f = (Fan*)c->fan;
  if (!f) {
    f = new Fan();
    c->fan = f;
    for (int k = 0; k < Fan::kN; ++k) {
      MYCEL_CUDA(c, cudaStreamCreateWithFlags(&f->s[k], cudaStreamNonBlocking));
      MYCEL_CUDA(c, cudaStreamCreateWithFlags(&f->side[k], cudaStreamNonBlocking));
      MYCEL_CUDA(c, cudaEventCreateWithFlags(&f->join_ev[k], cudaEventDisableTiming));
    }
    MYCEL_CUDA(c, cudaEventCreateWithFlags(&f->fork_ev, cudaEventDisableTiming));
  }
  c->main_stream = c->stream;
  c->main_side = c->side;
  MYCEL_CUDA(c, cudaEventRecord(f->fork_ev, c->stream));
  for (int k = 0; k < Fan::kN; ++k) f->used[k] = false;
  f->active = true;
  return MYCEL_OK;
}

void fan_use(mycel_ctx* c, int slot) {
  Fan* f = (Fan*)c->fan;
  if (!f || !f->active) return;
  const int k = slot % Fan::kN;
  if (!f->used[k]) {  // the side stream starts after the context stream's work so far
    cudaStreamWaitEvent(f->s[k], f->fork_ev, 0);
    cudaStreamWaitEvent(f->side[k], f->fork_ev, 0);
    f->used[k] = true;
  }
  c->stream = f->s[k];
  c->side = f->side[k];
}

void fan_end(mycel_ctx* c) {
  Fan* f = (Fan*)c->fan;
  if (!f || !f->active) return;
  c->stream = c->main_stream;
  c->side = c->main_side;
  for (int k = 0; k < Fan::kN; ++k)
    if (f->used[k]) {  // a side stream's side work is joined into it by the work itself (mg_setup)
      cudaEventRecord(f->join_ev[k], f->s[k]);
      cudaStreamWaitEvent(c->stream, f->join_ev[k], 0);
    }
  f->active = false;
}

int32_t fan_use_free(mycel_ctx* c, int slot, cudaStream_t* fan_stream) {
  Fan* f = (Fan*)c->fan;
  if (!f) {  // the streams, made as fan_begin makes them
    if (int32_t st = fan_begin(c)) return st;
    fan_end(c);
    f = (Fan*)c->fan;
  }
  const int k = slot % Fan::kN;
  c->main_stream = c->stream;
  c->main_side = c->side;
  c->stream = f->s[k];
  c->side = f->side[k];
  if (fan_stream) *fan_stream = f->s[k];
  return MYCEL_OK;
}

void fan_restore(mycel_ctx* c) {
  c->stream = c->main_stream;
  c->side = c->main_side;
}

void fan_release(mycel_ctx* c) {
  Fan* f = (Fan*)c->fan;
  if (!f) return;
  for (int k = 0; k < Fan::kN; ++k) {
    if (f->s[k]) cudaStreamSynchronize(f->s[k]), cudaStreamDestroy(f->s[k]);
    if (f->side[k]) cudaStreamSynchronize(f->side[k]), cudaStreamDestroy(f->side[k]);
    if (f->join_ev[k]) cudaEventDestroy(f->join_ev[k]);
  }
  if (f->fork_ev) cudaEventDestroy(f->fork_ev);
  delete f;
  c->fan = nullptr;
}

int32_t solve_dispatch(mycel_problem* p, double* d_u, double tol, int max_iter, int precision,
                       const volatile int32_t* cancel, mycel_pcg_result* res) {
  if (precision == MYCEL_PRECISION_MIXED || precision == MYCEL_PRECISION_FP64_FACTORED ||
      precision == MYCEL_PRECISION_FP64_MG || precision == MYCEL_PRECISION_MIXED_MG) {
    return refined_solve_entry(p, p->d_b, p->d_bnz, p->n_bnz, d_u, tol, max_iter, cancel, precision, res);
  }
  return pcg_solve_fp64(p, p->d_b, p->d_bnz, p->n_bnz, d_u, tol, max_iter, cancel, res);
}
}  // namespace mycel

extern "C" int32_t mycel_average_element_to_node(mycel_problem* p, const double* element_scalar, int64_t len,
                                                 double* nodal_out) {
  if (!p || !element_scalar || !nodal_out) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  if (len != p->g.ne) return set_error(p->ctx, MYCEL_E_ARG, "elementScalar length must equal TotalElements.");
  cudaSetDevice(p->ctx->device);
  cudaStream_t s = p->ctx->stream;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_tmp0, element_scalar, sizeof(double) * p->g.ne, cudaMemcpyHostToDevice, s));
  launch_average_e2n(p, p->d_tmp0, p->d_tmp1);
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(nodal_out, p->d_tmp1, sizeof(double) * p->g.nn, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

extern "C" int32_t mycel_static_solve(mycel_problem* p, const mycel_static_options* opt, const double* warm,
                                      int64_t warm_len, double* u_out, double* reactions_out, double* vm_out,
                                      double* compliance_out, double* maxdisp_out, mycel_pcg_result* res) {
  if (!p || !u_out) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  mycel_static_options o = opt ? *opt : mycel_static_options{1e-6, 5000, 1, MYCEL_PRECISION_FP64};
  if (p->n_active_fixed < 6) return set_error(c, MYCEL_E_UNDERCONSTRAINED, underconstrained_msg(p->n_active_fixed));
  if (p->assemble_status) return set_error(c, p->assemble_status, p->assemble_msg);
  if (warm && warm_len != p->g.nd)
    return set_error(c, MYCEL_E_ARG, "WarmStartDisplacements length (" + std::to_string(warm_len) +
                                         ") must match TotalDofs (" + std::to_string(p->g.nd) + "). (Parameter 'options')");
  int32_t st = ensure_pcg_workspace(p);
  if (st) return st;
  // new FemOperator(model): E from ElementDensity and Penal
  launch_update_E(p, p->d_rho_box, p->penal);
  launch_diag(p);
  if (warm) MYCEL_CUDA(c, cudaMemcpyAsync(p->d_x, warm, sizeof(double) * p->g.nd, cudaMemcpyHostToDevice, s));
  else MYCEL_CUDA(c, cudaMemsetAsync(p->d_x, 0, sizeof(double) * p->g.nd, s));
  mycel_pcg_result local;
  mycel_pcg_result* r = res ? res : &local;
  st = solve_dispatch(p, p->d_x, o.tolerance, o.max_iterations, o.precision, nullptr, r);
  if (st) return st;
  if (o.throw_on_non_convergence && !r->converged)
    return set_error(c, MYCEL_E_NOT_CONVERGED,
                     "FEM solver did not converge in " + std::to_string(r->iterations) + " iterations (" + r->message +
                         "). Is the model not sufficiently constrained?");
  double* d_sc = p->d_part2;  // [0] compliance, [1] max disp
  launch_compliance(p, p->d_x, d_sc);
  launch_max_disp(p, p->d_x, d_sc + 1);
  if (reactions_out) {
    launch_matvec64(p, p->d_x, p->d_ap, 0, nullptr);  // ApplyK(u) (StaticAnalysis.cs:103-110)
    launch_reactions(p, p->d_ap, p->d_tmp1, p->d_fixed, (int32_t)p->fixed_host.size());
    MYCEL_CUDA(c, cudaMemcpyAsync(reactions_out, p->d_tmp1, sizeof(double) * p->g.nd, cudaMemcpyDeviceToHost, s));
  }
  if (vm_out) {
    launch_von_mises(p, p->d_x, p->d_tmp0);
    MYCEL_CUDA(c, cudaMemcpyAsync(vm_out, p->d_tmp0, sizeof(double) * p->g.ne, cudaMemcpyDeviceToHost, s));
  }
  double* hsc = (double*)c->pinned;
  MYCEL_CUDA(c, cudaMemcpyAsync(hsc, d_sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(c, cudaMemcpyAsync(u_out, p->d_x, sizeof(double) * p->g.nd, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  if (compliance_out) *compliance_out = hsc[0];
  if (maxdisp_out) *maxdisp_out = hsc[1];
  return MYCEL_OK;
}

extern "C" int32_t mycel_static_solve_cases(mycel_problem* p, const mycel_static_options* opt, double* u_out,
                                            double* compliance_out, double* maxdisp_out, mycel_pcg_result* res) {
  if (!p || !u_out) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  mycel_ctx* c = p->ctx;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  mycel_static_options o = opt ? *opt : mycel_static_options{1e-6, 5000, 1, MYCEL_PRECISION_FP64};
  if (p->n_active_fixed < 6) return set_error(c, MYCEL_E_UNDERCONSTRAINED, underconstrained_msg(p->n_active_fixed));
  if (p->assemble_status) return set_error(c, p->assemble_status, p->assemble_msg);
  int32_t st = ensure_pcg_workspace(p);
  if (st || (st = ensure_cases(p))) return st;
  // one stiffness for all cases: E and DiagA here, the solver's own set-up (multigrid hierarchy) on the first
  // case's solve, reused by the others while E is unchanged
  launch_update_E(p, p->d_rho_box, p->penal);
  launch_diag(p);
  const int64_t nd = p->g.nd;
  double* d_sc = p->d_part2;  // [0] compliance, [1] max disp
  double* hsc = (double*)c->pinned;
  // the mixed multigrid form solves the cases together (one V-cycle's coarse levels for all of them)
  const bool together = o.precision == MYCEL_PRECISION_MIXED_MG && p->n_cases > 1 &&
                        p->n_cases <= kMaxBatchedCases && cases_together_enabled();
  double* d_ucs = nullptr;
  std::vector<mycel_pcg_result> rs((size_t)std::max(p->n_cases, 1));
  struct Free {
    double*& q; cudaStream_t s;
    ~Free() { if (q) cudaFreeAsync(q, s); }
  } free_ucs{d_ucs, s};
  if (together) {
    MYCEL_CUDA(c, cudaMallocAsync((void**)&d_ucs, sizeof(double) * nd * p->n_cases, s));
    MYCEL_CUDA(c, cudaMemsetAsync(d_ucs, 0, sizeof(double) * nd * p->n_cases, s));
    if ((st = mg_solve_cases(p, p->n_cases, d_ucs, o.tolerance, o.max_iterations, nullptr, rs.data()))) return st;
  }
  for (int k = 0; k < p->n_cases; ++k) {
    mycel_pcg_result local;
    mycel_pcg_result* r = res ? res + k : &local;
    if (together) {
      *r = rs[(size_t)k];
      MYCEL_CUDA(c, cudaMemcpyAsync(p->d_x, d_ucs + k * nd, sizeof(double) * nd, cudaMemcpyDeviceToDevice, s));
    } else {
      MYCEL_CUDA(c, cudaMemsetAsync(p->d_x, 0, sizeof(double) * nd, s));
      if ((st = solve_case(p, k, p->d_x, o.tolerance, o.max_iterations, o.precision, nullptr, r))) return st;
    }
    if (o.throw_on_non_convergence && !r->converged)
      return set_error(c, MYCEL_E_NOT_CONVERGED,
                       "FEM solver did not converge in " + std::to_string(r->iterations) + " iterations (" +
                           r->message + ") for load case " + std::to_string(k) +
                           ". Is the model not sufficiently constrained?");
    launch_compliance(p, p->d_case_F + k * nd, p->d_case_nz + p->case_nz_off[2 * k], p->case_nz_cnt[2 * k], p->d_x,
                      d_sc);
    launch_max_disp(p, p->d_x, d_sc + 1);
    MYCEL_CUDA(c, cudaMemcpyAsync(hsc, d_sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaMemcpyAsync(u_out + k * nd, p->d_x, sizeof(double) * nd, cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    if (compliance_out) compliance_out[k] = hsc[0];
    if (maxdisp_out) maxdisp_out[k] = hsc[1];
  }
  return MYCEL_OK;
}

// ---- filter ----
extern "C" int32_t mycel_filter_create(mycel_problem* p, double rmin, mycel_filter** out) {
  if (!p || !out) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  (void)cudaGetLastError();
  mycel_filter* f = new mycel_filter();
  f->p = p;
  f->rmin = rmin;
  int st = filter_setup(f);
  if (st) {
    std::string m = p->ctx->last_error;
    mycel_filter_destroy(f);
    return set_error(p->ctx, st, m.empty() ? std::string("filter set-up failed") : m);
  }
  *out = f;
  return MYCEL_OK;
}

extern "C" int32_t mycel_filter_destroy(mycel_filter* f) {
  if (!f) return MYCEL_OK;
  cudaStreamSynchronize(f->p->ctx->stream);
  dfree(f->p->ctx->stream, f->d_off);
  dfree(f->p->ctx->stream, f->d_w);
  dfree(f->p->ctx->stream, f->d_invhs);
  dfree(f->p->ctx->stream, f->d_s);
  delete f;
  return MYCEL_OK;
}

static int32_t filter_io(mycel_filter* f, const double* in, double* out, int adj) {
  if (!f || !in || !out) return set_error(f ? f->p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  mycel_problem* p = f->p;
  cudaSetDevice(p->ctx->device);
  cudaStream_t s = p->ctx->stream;
  double* d_in = p->d_tmp0;   // active-sized staging
  double* d_box = p->d_tmp1;  // box
  int32_t st = ensure_pcg_workspace(p);
  if (st) return st;
  double* d_outbox = p->d_z;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(d_in, in, sizeof(double) * p->n_active, cudaMemcpyHostToDevice, s));
  launch_scatter_active(p, d_in, d_box, 0.0);
  if (adj) launch_filter_adj(f, d_box, d_outbox);
  else launch_filter_fwd(f, d_box, d_outbox);
  launch_gather_active(p, d_outbox, d_in);
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(out, d_in, sizeof(double) * p->n_active, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

extern "C" int32_t mycel_filter_apply(mycel_filter* f, const double* in, double* out) { return filter_io(f, in, out, 0); }
extern "C" int32_t mycel_filter_adjoint(mycel_filter* f, const double* in, double* out) { return filter_io(f, in, out, 1); }

extern "C" int32_t mycel_filter_s(mycel_filter* f, double* out) {
  if (!f || !out) return set_error(f ? f->p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  mycel_problem* p = f->p;
  cudaSetDevice(p->ctx->device);
  launch_gather_active(p, f->d_s, p->d_tmp0);
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(out, p->d_tmp0, sizeof(double) * p->n_active, cudaMemcpyDeviceToHost, p->ctx->stream));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(p->ctx->stream));
  return MYCEL_OK;
}

extern "C" int32_t mycel_sensitivities(mycel_problem* p, const double* u, const double* rho_active, double penal,
                                       double* dc_active) {
  if (!p || !u || !rho_active || !dc_active) return set_error(p ? p->ctx : nullptr, MYCEL_E_ARG, "NULL argument");
  cudaSetDevice(p->ctx->device);
  cudaStream_t s = p->ctx->stream;
  int32_t st = ensure_pcg_workspace(p);
  if (st) return st;
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_r, u, sizeof(double) * p->g.nd, cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(p->d_tmp0, rho_active, sizeof(double) * p->n_active, cudaMemcpyHostToDevice, s));
  launch_scatter_active(p, p->d_tmp0, p->d_tmp1, 0.0);
  launch_sens(p, p->d_r, p->d_tmp1, penal, p->d_z);
  launch_gather_active(p, p->d_z, p->d_tmp0);
  MYCEL_CUDA(p->ctx, cudaMemcpyAsync(dc_active, p->d_tmp0, sizeof(double) * p->n_active, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(p->ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}

extern "C" int32_t mycel_oc_update(mycel_ctx* c, int32_t n, const double* rho, const double* dc, const double* sv,
                                   const uint8_t* passive, double* rho_new, double f, double move, double rho_min,
                                   double lambda_guess, int32_t max_bisect, double vol_tol, double* lambda_out) {
  if (!c || n < 0 || (n > 0 && (!rho || !dc || !sv || !rho_new)))
    return set_error(c, MYCEL_E_ARG, "All spans must have length >= rho.Length.");
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  size_t nn = (size_t)std::max(n, 1);
  double *d_rho, *d_dc, *d_s, *d_new, *d_scr;
  uint8_t* d_pas = nullptr;
  OcOut* d_out;
  size_t scr = oc_scratch_doubles(c->oc_grid);
  MYCEL_CUDA(c, cudaMallocAsync((void**)&d_rho, nn * 8, s));
  MYCEL_CUDA(c, cudaMallocAsync((void**)&d_dc, nn * 8, s));
  MYCEL_CUDA(c, cudaMallocAsync((void**)&d_s, nn * 8, s));
  MYCEL_CUDA(c, cudaMallocAsync((void**)&d_new, nn * 8, s));
  MYCEL_CUDA(c, cudaMallocAsync((void**)&d_scr, scr * 8, s));
  MYCEL_CUDA(c, cudaMallocAsync((void**)&d_out, sizeof(OcOut), s));
  if (passive) MYCEL_CUDA(c, cudaMallocAsync((void**)&d_pas, nn, s));
  MYCEL_CUDA(c, cudaMemsetAsync(d_out, 0, sizeof(OcOut), s));
  if (n) {
    cudaMemcpyAsync(d_rho, rho, n * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_dc, dc, n * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_s, sv, n * 8, cudaMemcpyHostToDevice, s);
    if (passive) cudaMemcpyAsync(d_pas, passive, n, cudaMemcpyHostToDevice, s);
  }
  OcParams prm{f, move, rho_min, lambda_guess, vol_tol, max_bisect, 0};
  int st = launch_oc(c, n, nullptr, d_rho, d_dc, d_s, d_pas, d_new, nullptr, nullptr, prm, d_scr, scr, d_out);
  OcOut* ho = (OcOut*)c->pinned;
  std::memset(ho, 0, sizeof(OcOut));
  if (!st) {
    cudaMemcpyAsync(ho, d_out, sizeof(OcOut), cudaMemcpyDeviceToHost, s);
    if (n) cudaMemcpyAsync(rho_new, d_new, n * 8, cudaMemcpyDeviceToHost, s);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  OcOut h = *ho;
  cudaFreeAsync(d_rho, s); cudaFreeAsync(d_dc, s); cudaFreeAsync(d_s, s); cudaFreeAsync(d_new, s);
  cudaFreeAsync(d_scr, s); cudaFreeAsync(d_out, s);
  if (d_pas) cudaFreeAsync(d_pas, s);
  cudaStreamSynchronize(s);
  if (st || e != cudaSuccess) return set_error(c, MYCEL_E_DEVICE, std::string("OC kernel: ") + cudaGetErrorString(e));
  if (h.trials == 0) return set_error(c, MYCEL_E_TIMEOUT, "OC grid barrier timed out");
  if (lambda_out) *lambda_out = h.lambda;
  return MYCEL_OK;
}
