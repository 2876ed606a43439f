// Plain FP64 path: reproduces Mycel.Core's arithmetic on sm_100a.
// This translation unit is compiled with -fmad=false: no a*b+c is contracted, as in the reference (RyuJIT).
//
// Kernels and the reference code whose rounding sequence they reproduce:
//   k_matvec64      FemOperator.ApplyK/ApplyA (Fem/FemOperator.cs:196-294, MultiplyElementUnsafe :379-422).
//                   Node-centric gather: one thread per node sums its <= 8 element contributions in the
//                   8-colour order the reference scatters them, each contribution computed with the
//                   reference's scale-then-dot order (ue = x*E; four lane chains; Vector256.Sum).
//                   Threads are grouped by node parity class so every warp follows the same colour order and
//                   reads the same KE rows (broadcast from the kernel parameter bank).
//   k_diag          FemOperator.AssembleDiagonal (:143-172), same colour order; Jacobi inverse (JacobiPreconditioner.cs:25).
//   k_dot_exact     PcgSolver DotParallel/ProcessDotChunk (Fem/PcgSolver.cs:385-450): one CTA per 8192-block,
//                   producer warps stage products in shared memory, lanes 0-3 of warp 0 run the four
//                   sequential lane chains, the last CTA adds the block partials in block order.
//   k_xr_exact      ProcessUpdateXrNormChunk + ProcessApplyPrecDotChunk (:452-527) fused: two chain sets.
//   k_update_p      ProcessUpdatePChunk (:529-553).
//   k_filter_*      DensityFilter (Optimization/DensityFilter.cs:34-303) as a stencil in the reference's
//                   neighbour order (jz, jy, jx ascending), weights (rmin - dist) * invHs_row.
//   k_sens          SensitivityAnalysis (Optimization/SensitivityAnalysis.cs:98-144).
//   k_oc            OcOptimizer.Update (Optimization/OcOptimizer.cs:12-175): one persistent cooperative kernel.
#include <algorithm>
#include <mutex>
#include <string>
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "internal.h"
#include "libm_pow.h"

namespace mycel {

constexpr int kBlock = 8192;  // PcgSolver.BlockSize
constexpr int kChunk = 1024;  // products staged per shared-memory buffer
constexpr int kDotThreads = 256;

// ---------------------------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double lane_sum(int mode, double a0, double a1, double a2, double a3) {
  // Vector256<double>.Sum: Sum(lower) + Sum(upper) on .NET 8+ (mode 0); alternatives for the noise-floor study.
  if (mode == 1) return (a0 + a2) + (a1 + a3);
  if (mode == 2) return ((a0 + a1) + a2) + a3;
  return (a0 + a1) + (a2 + a3);
}

// Math.Pow on the path (FemOperator.cs:100,133; SensitivityAnalysis.cs:93-95): the host C library's pow,
// restated with its rounding sequence (libm_pow.h), so E_e and dE/drho carry the reference's bits for every
// exponent.
__device__ __forceinline__ double path_pow(double x, double y) { return libm_pow::pow(x, y); }

__device__ __forceinline__ int local_index(int ox, int oy, int oz) {
  // Hex8 local node order (Hex8Element.cs:8-16): (0,0,0),(1,0,0),(1,1,0),(0,1,0), then the same at z=1
  int base = oy ? (ox ? 2 : 3) : (ox ? 1 : 0);
  return base + 4 * oz;
}

__device__ __forceinline__ double ld_volatile(const double* p) { return *(const volatile double*)p; }

// Parity-class node mapping: blockIdx.y = class (px | py<<1 | pz<<2); nodes of one class have the same
// parity in i, j, k, so the colour order of their incident elements is the same for the whole warp.
struct ClassNode {
  int i, j, k, px, py, pz;
  bool valid;
};
__device__ __forceinline__ ClassNode class_node(const GridDims& g, int cls, int64_t t) {
  ClassNode c;
  c.px = cls & 1; c.py = (cls >> 1) & 1; c.pz = (cls >> 2) & 1;
  int cx = (g.nx1 - c.px + 1) >> 1, cy = (g.ny1 - c.py + 1) >> 1, cz = (g.nz1 - c.pz + 1) >> 1;
  int64_t tot = (int64_t)cx * cy * cz;
  c.valid = t < tot;
  if (!c.valid) { c.i = c.j = c.k = 0; return c; }
  int a = (int)(t % cx);
  int64_t rest = t / cx;
  int b = (int)(rest % cy);
  int cc = (int)(rest / cy);
  c.i = c.px + 2 * a; c.j = c.py + 2 * b; c.k = c.pz + 2 * cc;
  return c;
}

inline dim3 class_grid(const GridDims& g, int threads) {
  int cx = (g.nx1 + 1) >> 1, cy = (g.ny1 + 1) >> 1, cz = (g.nz1 + 1) >> 1;
  int64_t tot = (int64_t)cx * cy * cz;
  return dim3((unsigned)((tot + threads - 1) / threads), 8, 1);
}

// ---------------------------------------------------------------------------------------------------------
// problem set-up: active nodes, constrained mask (FeModel.cs:80-183)
// ---------------------------------------------------------------------------------------------------------
__global__ void k_node_flags(GridDims g, const uint8_t* __restrict__ dom, uint8_t* __restrict__ nf) {
  int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= g.nn) return;
  int i = (int)(n % g.nx1);
  int64_t r = n / g.nx1;
  int j = (int)(r % g.ny1), k = (int)(r / g.ny1);
  bool act = false;
  for (int dz = -1; dz <= 0; ++dz)
    for (int dy = -1; dy <= 0; ++dy)
      for (int dx = -1; dx <= 0; ++dx) {
        int ie = i + dx, je = j + dy, ke = k + dz;
        if (ie >= 0 && ie < g.nx && je >= 0 && je < g.ny && ke >= 0 && ke < g.nz)
          act |= dom[ie + (int64_t)g.nx * (je + (int64_t)g.ny * ke)] != 0;
      }
  nf[n] = act ? NF_ACTIVE : (uint8_t)(NF_CX | NF_CY | NF_CZ);
}

__global__ void k_fixed_flags(GridDims g, const int32_t* __restrict__ fixed, int32_t nfix, uint8_t* nf) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nfix) return;
  int32_t d = fixed[t];
  int64_t node = d / 3;
  int c = d % 3;
  // several threads may touch one node byte: use a 32-bit atomicOr on the containing word
  unsigned int* w = (unsigned int*)((uintptr_t)(nf + node) & ~(uintptr_t)3);
  int sh = (int)(((uintptr_t)(nf + node) & 3) * 8);
  atomicOr(w, (unsigned int)(1u << c) << sh);
}

// count unique fixed DOFs on active nodes (FeModel.ActiveFixedDofCount, :165-183)
__global__ void k_count_active_fixed(GridDims g, const uint8_t* __restrict__ nf, const uint8_t* __restrict__ fixmask,
                                     int32_t* count) {
  int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int v = 0;
  if (d < g.nd) v = (fixmask[d] != 0) && (nf[d / 3] & NF_ACTIVE);
  v = __syncthreads_count(v);
  if (threadIdx.x == 0 && v) atomicAdd(count, v);
}

__global__ void k_mark_fixed(const int32_t* __restrict__ fixed, int32_t nfix, uint8_t* fixmask) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nfix) fixmask[fixed[t]] = 1;
}

void launch_setup_nodes(mycel_problem* p, const int32_t* d_fixed, int32_t n_fixed, int32_t* d_count) {
  const GridDims& g = p->g;
  cudaStream_t s = p->ctx->stream;
  k_node_flags<<<(unsigned)((g.nn + 255) / 256), 256, 0, s>>>(g, p->d_domain, p->d_nflags);
  p->ctx->launches++;
  if (n_fixed > 0) {
    k_fixed_flags<<<(n_fixed + 255) / 256, 256, 0, s>>>(g, d_fixed, n_fixed, p->d_nflags);
    p->ctx->launches++;
    // reuse tmp0 as a byte mask of fixed DOFs
    uint8_t* fixmask = (uint8_t*)p->d_tmp0;
    cudaMemsetAsync(fixmask, 0, (size_t)g.nd, s);
    k_mark_fixed<<<(n_fixed + 255) / 256, 256, 0, s>>>(d_fixed, n_fixed, fixmask);
    k_count_active_fixed<<<(unsigned)((g.nd + 255) / 256), 256, 0, s>>>(g, p->d_nflags, fixmask, d_count);
    p->ctx->launches += 2;
  }
}

// ---------------------------------------------------------------------------------------------------------
// E_e = Emin + rho^p (E0 - Emin)   (FemOperator.cs:100, :133)
// ---------------------------------------------------------------------------------------------------------
__global__ void k_update_E(int64_t na, const int32_t* __restrict__ active, const double* __restrict__ rho,
                           double emin, double e0, double penal, double* __restrict__ E, float* __restrict__ Ef) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= na) return;
  int32_t e = active[t];
  double v = emin + path_pow(rho[e], penal) * (e0 - emin);
  E[e] = v;
  if (Ef) Ef[e] = (float)v;
}

void launch_update_E(mycel_problem* p, const double* d_rho_box, double penal) {
  p->e_version++;
  if (p->n_active == 0) return;
  k_update_E<<<(unsigned)((p->n_active + 255) / 256), 256, 0, p->ctx->stream>>>(
      p->n_active, p->d_active, d_rho_box, p->emin, p->e0, penal, p->d_E, p->d_Ef);
  p->ctx->launches++;
}

// DiagA[dof] = sum over colours of E_e * DiagKe[k]; constrained -> 1; invD = |d| > 1e-30 ? 1/d : 1
struct Diag24 { double v[24]; };
__global__ void __launch_bounds__(256) k_diag(GridDims g, const __grid_constant__ Diag24 dk, const double* __restrict__ E,
                                              const uint8_t* __restrict__ dom, const uint8_t* __restrict__ nf,
                                              double* __restrict__ diag, double* __restrict__ invd,
                                              float* __restrict__ invdf) {
  ClassNode cn = class_node(g, blockIdx.y, blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
  if (!cn.valid) return;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
#pragma unroll 1
  for (int col = 0; col < 8; ++col) {
    int ox = (col & 1) ^ cn.px, oy = ((col >> 1) & 1) ^ cn.py, oz = ((col >> 2) & 1) ^ cn.pz;
    int ie = cn.i - ox, je = cn.j - oy, ke = cn.k - oz;
    if (ie < 0 || ie >= g.nx || je < 0 || je >= g.ny || ke < 0 || ke >= g.nz) continue;
    int64_t e = ie + (int64_t)g.nx * (je + (int64_t)g.ny * ke);
    if (!dom[e]) continue;
    double ee = E[e];
    int a = local_index(ox, oy, oz);
    d0 = d0 + ee * dk.v[3 * a];
    d1 = d1 + ee * dk.v[3 * a + 1];
    d2 = d2 + ee * dk.v[3 * a + 2];
  }
  int64_t n = cn.i + (int64_t)g.nx1 * (cn.j + (int64_t)g.ny1 * cn.k);
  uint8_t f = nf[n];
  double dd[3] = {d0, d1, d2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double d = (f & (1 << c)) ? 1.0 : dd[c];
    double iv = fabs(d) > 1e-30 ? 1.0 / d : 1.0;
    diag[3 * n + c] = d;
    invd[3 * n + c] = iv;
    if (invdf) invdf[pidx(g, cn.i, cn.j + (int64_t)g.ny1 * cn.k, c)] = (float)iv;
  }
}

void launch_diag(mycel_problem* p) {
  Diag24 dk;
  for (int i = 0; i < 24; ++i) dk.v[i] = p->diag_ke[i];
  k_diag<<<class_grid(p->g, 256), 256, 0, p->ctx->stream>>>(p->g, dk, p->d_E, p->d_domain, p->d_nflags, p->d_diag,
                                                            p->d_invd, p->d_invdf);
  p->ctx->launches++;
}

// ---------------------------------------------------------------------------------------------------------
// y = K x (projected: y = x on constrained DOFs, ApplyA with xIsAlreadyProjected)
// z-marching shared-memory tiles: a CTA owns 64 x 4 nodes and marches over ZSEG node planes; three planes of x
// (one-node halo) and two element planes of E and the domain live in shared memory. Warp w handles the nodes
// of one parity in x (i = i0 + 2 lane + (w & 1)) of row j0 + (w >> 1), so the colour order of the incident
// elements, and the KE rows they read, are the same for the whole warp. The shared planes are stored
// parity-split in x, so a warp's 8-byte loads hit consecutive words.
// ---------------------------------------------------------------------------------------------------------
constexpr int MX = 64, MY = 4;
constexpr int MPX = MX + 2, MPY = MY + 2;   // node plane with halo
constexpr int MEX = MX + 1, MEY = MY + 1;   // element plane
constexpr int MPXH = (MPX + 1) / 2, MEXH = (MEX + 1) / 2;

__device__ __forceinline__ int psplit(int lx, int half) { return (lx & 1) * half + (lx >> 1); }

__global__ void __launch_bounds__(256) k_matvec64(GridDims g, const __grid_constant__ KeD ke,
                                                  const double* __restrict__ x, double* __restrict__ y,
                                                  const double* __restrict__ E, const uint8_t* __restrict__ dom,
                                                  const uint8_t* __restrict__ nf, int projected, int mode,
                                                  const int* __restrict__ status, int zseg) {
  __shared__ double xs[3][3][MPY][2 * MPXH];  // [slot][c][ly][parity-split lx]
  __shared__ double es[2][MEY][2 * MEXH];
  __shared__ uint8_t ds[2][MEY][2 * MEXH];
  if (status && *status != PCG_RUNNING) return;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int px = w & 1, ty = w >> 1;
  const int i0 = blockIdx.x * MX, j0 = blockIdx.y * MY, k0 = blockIdx.z * zseg;
  const int k1 = min(k0 + zseg, g.nz1);
  const int64_t sy = g.nx1, sz = (int64_t)g.nx1 * g.ny1;

  auto load_plane = [&](int kk, int slot) {
    for (int q = tid; q < MPY * MPX * 3; q += 256) {
      int c = q % 3, rest = q / 3, lx = rest % MPX, ly = rest / MPX;
      int i = i0 - 1 + lx, j = j0 - 1 + ly;
      double v = 0.0;
      if (kk >= 0 && kk < g.nz1 && i >= 0 && i < g.nx1 && j >= 0 && j < g.ny1) v = __ldg(x + 3 * (i + sy * j + sz * kk) + c);
      xs[slot][c][ly][psplit(lx, MPXH)] = v;
    }
  };
  auto load_eplane = [&](int ke_, int slot) {
    for (int q = tid; q < MEY * MEX; q += 256) {
      int lx = q % MEX, ly = q / MEX;
      int ie = i0 - 1 + lx, je = j0 - 1 + ly;
      double v = 0.0;
      uint8_t d = 0;
      if (ke_ >= 0 && ke_ < g.nz && ie >= 0 && ie < g.nx && je >= 0 && je < g.ny) {
        int64_t e = ie + (int64_t)g.nx * (je + (int64_t)g.ny * ke_);
        d = __ldg(dom + e);
        if (d) v = __ldg(E + e);
      }
      es[slot][ly][psplit(lx, MEXH)] = v;
      ds[slot][ly][psplit(lx, MEXH)] = d;
    }
  };

  load_plane(k0 - 1, (k0 + 2) % 3);
  load_plane(k0, k0 % 3);
  load_eplane(k0 - 1, (k0 + 1) & 1);
  const int lxn = 1 + 2 * lane + px;  // plane-local x of this thread's node
  const int i = i0 + lxn - 1, j = j0 + ty;
  const bool mine = i < g.nx1 && j < g.ny1;
  for (int k = k0; k < k1; ++k) {
    load_plane(k + 1, (k + 1) % 3);
    load_eplane(k, k & 1);
    __syncthreads();
    if (mine) {
      double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
      for (int col = 0; col < 8; ++col) {
        // node offset inside the element of colour col, and the element's local position
        const int ox = (col & 1) ^ (i & 1), oy = ((col >> 1) & 1) ^ (j & 1), oz = ((col >> 2) & 1) ^ (k & 1);
        const int sx = 1 - ox, sy_ = 1 - oy, sz_ = 1 - oz;  // element offset from (i-1, j-1, k-1)
        const int lxe = lxn - 1 + sx, lye = ty + sy_;      // element plane coordinates
        const int eslot = (k - 1 + sz_) & 1;
        const uint8_t act = ds[eslot][lye][psplit(lxe, MEXH)];
        if (!act) continue;  // outside the grid or inactive: no contribution
        const double ee = es[eslot][lye][psplit(lxe, MEXH)];
        double ue[24];
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const int bx = (b == 1 || b == 2 || b == 5 || b == 6) ? 1 : 0;
          const int by = (b == 2 || b == 3 || b == 6 || b == 7) ? 1 : 0;
          const int bz = b >= 4 ? 1 : 0;
          const int slot = (k - 1 + sz_ + bz + 3) % 3;
          const int lx = lxn - 1 + sx + bx, ly = ty + sy_ + by;
#pragma unroll
          for (int c = 0; c < 3; ++c) ue[3 * b + c] = xs[slot][c][ly][psplit(lx, MPXH)] * ee;
        }
        const int a = (oy ? (ox ? 2 : 3) : (ox ? 1 : 0)) + 4 * oz;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double* row = ke.v + (3 * a + c) * 24;
          double l[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            double s = row[q] * ue[q] + row[4 + q] * ue[4 + q];
            s = s + row[8 + q] * ue[8 + q];
            s = s + row[12 + q] * ue[12 + q];
            s = s + row[16 + q] * ue[16 + q];
            s = s + row[20 + q] * ue[20 + q];
            l[q] = s;
          }
          acc[c] = acc[c] + lane_sum(mode, l[0], l[1], l[2], l[3]);
        }
      }
      const int64_t n = i + sy * j + sz * k;
      const uint8_t f = projected ? nf[n] : 0;
      const int cslot = k % 3;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        y[3 * n + c] = (f & (1 << c)) ? xs[cslot][c][ty + 1][psplit(lxn, MPXH)] : acc[c];
    }
    __syncthreads();
  }
}

// z-segment length giving about 8 CTAs per SM (at least 2 planes per segment)
inline int matvec64_zseg(const GridDims& g, int num_sms) {
  int64_t txy = (int64_t)((g.nx1 + MX - 1) / MX) * ((g.ny1 + MY - 1) / MY);
  int64_t segs = std::max<int64_t>(1, (8 * (int64_t)num_sms + txy - 1) / txy);
  return (int)std::max<int64_t>(2, (g.nz1 + segs - 1) / segs);
}

void launch_matvec64(mycel_problem* p, const double* x, double* y, int projected, const int* d_status) {
  const GridDims& g = p->g;
  int zs = matvec64_zseg(g, p->ctx->num_sms);
  dim3 grid((unsigned)((g.nx1 + MX - 1) / MX), (unsigned)((g.ny1 + MY - 1) / MY), (unsigned)((g.nz1 + zs - 1) / zs));
  k_matvec64<<<grid, 256, 0, p->ctx->stream>>>(g, p->ke, x, y, p->d_E, p->d_domain, p->d_nflags, projected,
                                               p->lane_mode, d_status, zs);
  p->ctx->launches++;
}

// ---------------------------------------------------------------------------------------------------------
// exact block/lane reductions
// ---------------------------------------------------------------------------------------------------------
// Sequential 4-lane chain consumer: lanes 0..3 of the calling warp add buf[lane], buf[lane+4], ... in order.
__device__ __forceinline__ double chain4(double acc, const double* buf, int m, int lane4) {
  int q = lane4;
  for (; q + 28 < m; q += 32) {
    double v0 = buf[q], v1 = buf[q + 4], v2 = buf[q + 8], v3 = buf[q + 12];
    double v4 = buf[q + 16], v5 = buf[q + 20], v6 = buf[q + 24], v7 = buf[q + 28];
    acc = acc + v0; acc = acc + v1; acc = acc + v2; acc = acc + v3;
    acc = acc + v4; acc = acc + v5; acc = acc + v6; acc = acc + v7;
  }
  for (; q < m; q += 4) acc = acc + buf[q];
  return acc;
}

// Last-CTA election for the final, block-ordered sum (returns true in exactly one CTA, for all its threads).
__device__ __forceinline__ bool elect_last(unsigned int* counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Phases of the single-chain dot kernel.
enum DotPhase : int { PH_PAP = 0, PH_INIT_RR = 1 };

__global__ void __launch_bounds__(kDotThreads) k_dot_exact(const double* __restrict__ a, const double* __restrict__ b,
                                                           int64_t n, double* part, PcgState* st, int mode,
                                                           int phase) {
  if (st->status != PCG_RUNNING) return;
  __shared__ double buf[2][kChunk];
  const int64_t start = (int64_t)blockIdx.x * kBlock;
  const int cnt = (int)min((int64_t)kBlock, n - start);
  const int vc4 = cnt & ~3;
  const int nch = (vc4 + kChunk - 1) / kChunk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double acc = 0.0;
  for (int t = 0; t <= nch; ++t) {
    if (warp > 0 && t < nch) {
      const int base = t * kChunk;
      double* dst = buf[t & 1];
      for (int q = tid - 32; q < kChunk; q += kDotThreads - 32) {
        int idx = base + q;
        if (idx < vc4) dst[q] = a[start + idx] * b[start + idx];
      }
    }
    if (warp == 0 && t > 0 && lane < 4) {
      const int base = (t - 1) * kChunk;
      acc = chain4(acc, buf[(t - 1) & 1], min(kChunk, vc4 - base), lane);
    }
    __syncthreads();
  }
  if (warp == 0) {
    double l0 = __shfl_sync(0xffffffffu, acc, 0), l1 = __shfl_sync(0xffffffffu, acc, 1);
    double l2 = __shfl_sync(0xffffffffu, acc, 2), l3 = __shfl_sync(0xffffffffu, acc, 3);
    if (lane == 0) {
      double s = lane_sum(mode, l0, l1, l2, l3);
      for (int idx = vc4; idx < cnt; ++idx) s = s + a[start + idx] * b[start + idx];
      part[blockIdx.x] = s;
    }
  }
  if (!elect_last(&st->counter)) return;
  if (tid != 0) return;
  double sum = 0.0;
  for (unsigned k = 0; k < gridDim.x; ++k) sum = sum + ld_volatile(part + k);
  st->counter = 0;
  if (phase == PH_PAP) {
    st->iter += 1;
    double pap = sum;
    st->pap = pap;
    if (!(pap > 1e-30) || !isfinite(pap)) {
      st->last_bad = pap;
      st->status = PCG_BREAK_CURVATURE;
      return;
    }
    double alpha = st->rho0 / pap;
    if (!isfinite(alpha) || alpha <= 0.0) {
      st->last_bad = alpha;
      st->status = PCG_BREAK_ALPHA;
      return;
    }
    st->alpha = alpha;
  } else {  // PH_INIT_RR: rNormSq for a non-zero warm start (PcgSolver.cs:176-197)
    st->rn2 = sum;
    double rel = sqrt(sum) / st->bnorm;
    st->rel = rel;
    st->prev = rel;
    if (rel <= st->tol) st->status = PCG_INIT_CONVERGED;
  }
}

// Fused x/r update with ||r||^2 and z = r*invD with r.z. init=1: only the z part (rho0, p = z).
__global__ void __launch_bounds__(kDotThreads) k_xr_exact(double* __restrict__ x, double* __restrict__ r,
                                                          double* __restrict__ z, double* __restrict__ p,
                                                          const double* __restrict__ ap,
                                                          const double* __restrict__ invd, int64_t n, double* part,
                                                          PcgState* st, int mode, int init) {
  if (st->status != PCG_RUNNING) return;
  __shared__ double bufA[2][kChunk];
  __shared__ double bufB[2][kChunk];
  const double alpha = st->alpha;
  const int64_t start = (int64_t)blockIdx.x * kBlock;
  const int cnt = (int)min((int64_t)kBlock, n - start);
  const int vc4 = cnt & ~3;
  const int nch = (vc4 + kChunk - 1) / kChunk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double acc = 0.0;
  for (int t = 0; t <= nch; ++t) {
    if (warp > 0 && t < nch) {
      const int base = t * kChunk;
      double* da = bufA[t & 1];
      double* db = bufB[t & 1];
      for (int q = tid - 32; q < kChunk; q += kDotThreads - 32) {
        int idx = base + q;
        if (idx < vc4) {
          int64_t j = start + idx;
          double rv;
          if (!init) {
            double xv = x[j] + alpha * p[j];
            rv = r[j] - alpha * ap[j];
            x[j] = xv;
            r[j] = rv;
            da[q] = rv * rv;
          } else {
            rv = r[j];
          }
          double zv = rv * invd[j];
          z[j] = zv;
          if (init) p[j] = zv;
          db[q] = rv * zv;
        }
      }
    }
    if (warp == 0 && t > 0 && lane < 8) {
      const int base = (t - 1) * kChunk;
      const int m = min(kChunk, vc4 - base);
      if (lane < 4) {
        if (!init) acc = chain4(acc, bufA[(t - 1) & 1], m, lane);
      } else {
        acc = chain4(acc, bufB[(t - 1) & 1], m, lane - 4);
      }
    }
    __syncthreads();
  }
  if (warp == 0) {
    double a0 = __shfl_sync(0xffffffffu, acc, 0), a1 = __shfl_sync(0xffffffffu, acc, 1);
    double a2 = __shfl_sync(0xffffffffu, acc, 2), a3 = __shfl_sync(0xffffffffu, acc, 3);
    double b0 = __shfl_sync(0xffffffffu, acc, 4), b1 = __shfl_sync(0xffffffffu, acc, 5);
    double b2 = __shfl_sync(0xffffffffu, acc, 6), b3 = __shfl_sync(0xffffffffu, acc, 7);
    if (lane == 0) {
      double sa = lane_sum(mode, a0, a1, a2, a3);
      double sb = lane_sum(mode, b0, b1, b2, b3);
      if (!init) {
        for (int idx = vc4; idx < cnt; ++idx) {
          int64_t j = start + idx;
          double xi = x[j] + alpha * p[j];
          double ri = r[j] - alpha * ap[j];
          x[j] = xi;
          r[j] = ri;
          sa = sa + ri * ri;
        }
      }
      for (int idx = vc4; idx < cnt; ++idx) {
        int64_t j = start + idx;
        double zi = r[j] * invd[j];
        z[j] = zi;
        if (init) p[j] = zi;
        sb = sb + r[j] * zi;
      }
      part[blockIdx.x] = sa;
      part[gridDim.x + blockIdx.x] = sb;
    }
  }
  if (!elect_last(&st->counter)) return;
  if (tid != 0) return;
  st->counter = 0;
  const unsigned nb = gridDim.x;
  if (init) {
    double rho = 0.0;
    for (unsigned k = 0; k < nb; ++k) rho = rho + ld_volatile(part + nb + k);
    st->rho0 = rho;
    if (st->max_iter <= 0) st->status = PCG_MAXITER;
    return;
  }
  double rn2 = 0.0;
  for (unsigned k = 0; k < nb; ++k) rn2 = rn2 + ld_volatile(part + k);
  st->rn2 = rn2;
  double rel = sqrt(rn2) / st->bnorm;
  st->rel = rel;
  if (rel <= st->tol) {
    st->status = PCG_CONVERGED;
    return;
  }
  if (fabs(rel - st->prev) < 1e-15 * rel) {
    st->stag += 1;
    if (st->stag > 50) {
      st->status = PCG_STAGNATED;
      return;
    }
  } else {
    st->stag = 0;
  }
  st->prev = rel;
  double rho1 = 0.0;
  for (unsigned k = 0; k < nb; ++k) rho1 = rho1 + ld_volatile(part + nb + k);
  double beta = rho1 / st->rho0;
  if (!isfinite(beta) || beta < 0.0) {
    st->last_bad = beta;
    st->status = PCG_BREAK_BETA;
    return;
  }
  st->beta = beta;
  st->rho0 = rho1;
  if (st->iter >= st->max_iter) st->status = PCG_MAXITER;
}

__global__ void k_update_p(double* __restrict__ p, const double* __restrict__ z, int64_t n, const PcgState* st) {
  if (st->status != PCG_RUNNING) return;
  const double beta = st->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

// x projection (PcgSolver.cs:113-125) and "has non-zero x" flag
__global__ void k_project_x(int64_t nd, const uint8_t* __restrict__ nf, double* x, int* flag) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int nz = 0;
  if (i < nd) {
    if (nf[i / 3] & (1 << (i % 3))) x[i] = 0.0;
    else nz = x[i] != 0.0;
  }
  if (__syncthreads_or(nz) && threadIdx.x == 0) atomicOr(flag, 1);
}

// ||P b||^2: the reference adds b_i^2 over unconstrained i in index order; zero terms leave the running sum
// unchanged, so the sum over the ascending list of non-zero P b entries is the same number.
__global__ void k_bnorm_list(const double* __restrict__ b, const int32_t* __restrict__ idx, int32_t cnt,
                             PcgState* st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  constexpr int kB = 16;  // loads of 16 entries issued before they are added, in list order
  for (int32_t q0 = 0; q0 < cnt; q0 += kB) {
    double v[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) v[k] = q0 + k < cnt ? b[idx[q0 + k]] : 0.0;
#pragma unroll
    for (int k = 0; k < kB; ++k)
      if (q0 + k < cnt) s = s + v[k] * v[k];
  }
  st->bn2 = s;
  st->bnorm = sqrt(s);
}

void launch_project_x(mycel_problem* p, double* x, int* d_flag) {
  k_project_x<<<(unsigned)((p->g.nd + 255) / 256), 256, 0, p->ctx->stream>>>(p->g.nd, p->d_nflags, x, d_flag);
  p->ctx->launches++;
}

void launch_pcg_bnorm(mycel_problem* p) {
  k_bnorm_list<<<1, 32, 0, p->ctx->stream>>>(p->d_b, p->d_bnz, p->n_bnz, p->d_state);
  p->ctx->launches++;
}

// r = P(b - A x) or P b (PcgSolver.cs:176-192)
__global__ void k_init_r(int64_t nd, const uint8_t* __restrict__ nf, const double* __restrict__ b,
                         const double* __restrict__ ap, double* __restrict__ r, int nonzero) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nd) return;
  bool con = nf[i / 3] & (1 << (i % 3));
  r[i] = con ? 0.0 : (nonzero ? (b[i] - ap[i]) : b[i]);
}

void launch_pcg_init_r(mycel_problem* p, int nonzero) {
  k_init_r<<<(unsigned)((p->g.nd + 255) / 256), 256, 0, p->ctx->stream>>>(p->g.nd, p->d_nflags, p->d_b, p->d_ap,
                                                                         p->d_r, nonzero);
  p->ctx->launches++;
}

void launch_pcg_dot_rr(mycel_problem* p) {
  int64_t nb = num_blocks8192(p->g.nd);
  k_dot_exact<<<(unsigned)nb, kDotThreads, 0, p->ctx->stream>>>(p->d_r, p->d_r, p->g.nd, p->d_part, p->d_state,
                                                                p->lane_mode, PH_INIT_RR);
  p->ctx->launches++;
}

void launch_pcg_init_z(mycel_problem* p) {
  int64_t nb = num_blocks8192(p->g.nd);
  k_xr_exact<<<(unsigned)nb, kDotThreads, 0, p->ctx->stream>>>(p->d_x, p->d_r, p->d_z, p->d_p, p->d_ap, p->d_invd,
                                                               p->g.nd, p->d_part, p->d_state, p->lane_mode, 1);
  p->ctx->launches++;
}

// One PCG iteration (PcgSolver.cs:235-357): Ap = A p; pAp, alpha; x, r, ||r||; z, rho1, beta; p = z + beta p.
void launch_pcg_iteration(mycel_problem* p, bool skip_matvec) {
  cudaStream_t s = p->ctx->stream;
  int64_t nb = num_blocks8192(p->g.nd);
  if (!skip_matvec) launch_matvec64(p, p->d_p, p->d_ap, 1, &p->d_state->status);
  k_dot_exact<<<(unsigned)nb, kDotThreads, 0, s>>>(p->d_p, p->d_ap, p->g.nd, p->d_part, p->d_state, p->lane_mode,
                                                   PH_PAP);
  k_xr_exact<<<(unsigned)nb, kDotThreads, 0, s>>>(p->d_x, p->d_r, p->d_z, p->d_p, p->d_ap, p->d_invd, p->g.nd,
                                                  p->d_part, p->d_state, p->lane_mode, 0);
  k_update_p<<<(unsigned)std::min<int64_t>((p->g.nd + 255) / 256, 4096), 256, 0, s>>>(p->d_p, p->d_z, p->g.nd,
                                                                                        p->d_state);
  p->ctx->launches += 3;
}

// ---------------------------------------------------------------------------------------------------------
// compliance C = F.u (sequential over non-zero F in index order), max |u| over active nodes, reactions
// ---------------------------------------------------------------------------------------------------------
__global__ void k_compliance(const double* __restrict__ F, const double* __restrict__ u,
                             const int32_t* __restrict__ idx, int32_t cnt, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double c = 0.0;
  constexpr int kB = 16;  // loads of 16 terms issued before they are added, in list order
  for (int32_t q0 = 0; q0 < cnt; q0 += kB) {
    double fv[kB], uv[kB];
#pragma unroll
    for (int k = 0; k < kB; ++k) {
      const int32_t j = q0 + k < cnt ? idx[q0 + k] : 0;
      fv[k] = q0 + k < cnt ? F[j] : 0.0;
      uv[k] = q0 + k < cnt ? u[j] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kB; ++k)
      if (q0 + k < cnt) c = c + fv[k] * uv[k];
  }
  *out = c;
}

void launch_compliance(mycel_problem* p, const double* u, double* d_out) {
  launch_compliance(p, p->d_F, p->d_fnz, p->n_fnz, u, d_out);
}

void launch_compliance(mycel_problem* p, const double* F, const int32_t* fnz, int32_t n_fnz, const double* u,
                       double* d_out) {
  k_compliance<<<1, 32, 0, p->ctx->stream>>>(F, u, fnz, n_fnz, d_out);
  p->ctx->launches++;
}

__device__ __forceinline__ unsigned long long dbl_key(double v) {
  // non-negative doubles order like their bit patterns
  return (unsigned long long)__double_as_longlong(v);
}

__global__ void k_max_disp(GridDims g, const uint8_t* __restrict__ nf, const double* __restrict__ u,
                           unsigned long long* out) {
  double m = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < g.nn; n += (int64_t)gridDim.x * blockDim.x) {
    if (!(nf[n] & NF_ACTIVE)) continue;
    double ux = u[3 * n], uy = u[3 * n + 1], uz = u[3 * n + 2];
    double s = ux * ux + uy * uy + uz * uz;
    if (s > m) m = s;
  }
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_down_sync(0xffffffffu, m, o);
    if (v > m) m = v;
  }
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, dbl_key(m));
}

__global__ void k_sqrt_inplace(unsigned long long* v) {
  double d = __longlong_as_double((long long)*v);
  *(double*)v = sqrt(d);
}

void launch_max_disp(mycel_problem* p, const double* u, double* d_out) { launch_max_disp(p, &u, 1, 0, d_out); }

// largest |u| over the active nodes of m displacement vectors, u[k] at us[k] + k * stride
void launch_max_disp(mycel_problem* p, const double* const* us, int m, int64_t stride, double* d_out) {
  cudaMemsetAsync(d_out, 0, sizeof(double), p->ctx->stream);
  int blocks = std::max(1, std::min<int>((int)((p->g.nn + 255) / 256), p->ctx->num_sms * 8));
  for (int k = 0; k < m; ++k)
    k_max_disp<<<blocks, 256, 0, p->ctx->stream>>>(p->g, p->d_nflags, stride ? us[0] + k * stride : us[k],
                                                   (unsigned long long*)d_out);
  k_sqrt_inplace<<<1, 1, 0, p->ctx->stream>>>((unsigned long long*)d_out);
  p->ctx->launches += 1 + m;
}

__global__ void k_reactions(const double* __restrict__ ku, double* out, const int32_t* __restrict__ fixed, int32_t nf) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nf) out[fixed[t]] = ku[fixed[t]];
}

void launch_reactions(mycel_problem* p, const double* ku, double* out, const int32_t* d_fixed, int32_t n_fixed) {
  cudaMemsetAsync(out, 0, sizeof(double) * p->g.nd, p->ctx->stream);
  if (n_fixed > 0) {
    k_reactions<<<(n_fixed + 255) / 256, 256, 0, p->ctx->stream>>>(ku, out, d_fixed, n_fixed);
    p->ctx->launches++;
  }
}

// Element von Mises at the centroid (StaticAnalysis.cs:144-216)
struct VmConst {
  double bc[144];
  double d[36];
  double invh;
};
__global__ void k_von_mises(GridDims g, const __grid_constant__ VmConst vc, const double* __restrict__ u, const double* __restrict__ E,
                            const uint8_t* __restrict__ dom, double* __restrict__ vm) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= g.ne) return;
  if (!dom[e]) {
    vm[e] = 0.0;
    return;
  }
  int ix = (int)(e % g.nx);
  int64_t r = e / g.nx;
  int iy = (int)(r % g.ny), iz = (int)(r / g.ny);
  const int64_t sy = g.nx1, sz = (int64_t)g.nx1 * g.ny1;
  int64_t n0 = ix + sy * iy + sz * iz;
  const int64_t off[8] = {0, 1, 1 + sy, sy, sz, sz + 1, sz + 1 + sy, sz + sy};
  double ue[24];
  for (int b = 0; b < 8; ++b)
    for (int c = 0; c < 3; ++c) ue[3 * b + c] = u[3 * (n0 + off[b]) + c];
  double eps[6], sig[6];
  for (int q = 0; q < 6; ++q) {
    double s = 0.0;
    for (int k = 0; k < 24; ++k) s = s + vc.bc[q * 24 + k] * ue[k];
    eps[q] = s * vc.invh;
  }
  double ee = E[e];
  for (int q = 0; q < 6; ++q) {
    double s = 0.0;
    for (int k = 0; k < 6; ++k) s = s + vc.d[q * 6 + k] * eps[k];
    sig[q] = s * ee;
  }
  double d1 = sig[0] - sig[1], d2 = sig[1] - sig[2], d3 = sig[2] - sig[0];
  vm[e] = sqrt(0.5 * (d1 * d1 + d2 * d2 + d3 * d3) + 3.0 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5]));
}

void launch_von_mises(mycel_problem* p, const double* u, double* vm) {
  VmConst vc;
  // Hex8Element.BaseBc = EvaluateB(0,0,0,h=1) (Hex8Element.cs:71, :183-215)
  static const double xi[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, eta[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
                      zeta[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int i = 0; i < 144; ++i) vc.bc[i] = 0.0;
  for (int a = 0; a < 8; ++a) {
    double dx = (0.25 * 1.0) * xi[a] * (1.0 + eta[a] * 0.0) * (1.0 + zeta[a] * 0.0);
    double dy = (0.25 * 1.0) * eta[a] * (1.0 + xi[a] * 0.0) * (1.0 + zeta[a] * 0.0);
    double dz = (0.25 * 1.0) * zeta[a] * (1.0 + xi[a] * 0.0) * (1.0 + eta[a] * 0.0);
    vc.bc[0 * 24 + 3 * a] = dx; vc.bc[1 * 24 + 3 * a + 1] = dy; vc.bc[2 * 24 + 3 * a + 2] = dz;
    vc.bc[3 * 24 + 3 * a + 1] = dz; vc.bc[3 * 24 + 3 * a + 2] = dy;
    vc.bc[4 * 24 + 3 * a] = dz; vc.bc[4 * 24 + 3 * a + 2] = dx;
    vc.bc[5 * 24 + 3 * a] = dy; vc.bc[5 * 24 + 3 * a + 1] = dx;
  }
  double nu = p->nu;
  double factor = 1.0 / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double c1 = factor * (1.0 - nu), c2 = factor * nu, c3 = 1.0 / (2.0 * (1.0 + nu));
  for (int i = 0; i < 36; ++i) vc.d[i] = 0.0;
  vc.d[0] = c1; vc.d[1] = c2; vc.d[2] = c2; vc.d[6] = c2; vc.d[7] = c1; vc.d[8] = c2;
  vc.d[12] = c2; vc.d[13] = c2; vc.d[14] = c1; vc.d[21] = c3; vc.d[28] = c3; vc.d[35] = c3;
  vc.invh = 1.0 / (double)p->h;
  k_von_mises<<<(unsigned)((p->g.ne + 255) / 256), 256, 0, p->ctx->stream>>>(p->g, vc, u, p->d_E, p->d_domain, vm);
  p->ctx->launches++;
}

// StaticAnalysis.AverageElementToNode (Fem/StaticAnalysis.cs:222-268): per node, the mean of the scalars of the
// active elements meeting there, 0 where none does. A node gathers its (up to 8) elements in increasing element
// index, the order in which the reference's element loop adds to the node's sum, so the sums are bit-identical.
__global__ void k_avg_e2n(GridDims g, const double* __restrict__ es, const uint8_t* __restrict__ dom,
                          double* __restrict__ out) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= g.nn) return;
  const int i = (int)(n % g.nx1), j = (int)((n / g.nx1) % g.ny1), k = (int)(n / ((int64_t)g.nx1 * g.ny1));
  double sum = 0.0;
  int cnt = 0;
  for (int ez = k - 1; ez <= k; ++ez)
    for (int ey = j - 1; ey <= j; ++ey)
      for (int ex = i - 1; ex <= i; ++ex) {
        if (ex < 0 || ey < 0 || ez < 0 || ex >= g.nx || ey >= g.ny || ez >= g.nz) continue;
        const int64_t e = ex + (int64_t)g.nx * (ey + (int64_t)g.ny * ez);
        if (!dom[e]) continue;
        sum = sum + es[e];
        cnt++;
      }
  out[n] = cnt > 0 ? sum / (double)cnt : 0.0;
}

void launch_average_e2n(mycel_problem* p, const double* es, double* out) {
  k_avg_e2n<<<(unsigned)((p->g.nn + 255) / 256), 256, 0, p->ctx->stream>>>(p->g, es, p->d_domain, out);
  p->ctx->launches++;
}

// active <-> box index maps
__global__ void k_scatter_active(int64_t na, const int32_t* __restrict__ act, const double* __restrict__ src,
                                 double* __restrict__ dst) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < na) dst[act[t]] = src[t];
}
__global__ void k_gather_active(int64_t na, const int32_t* __restrict__ act, const double* __restrict__ src,
                                double* __restrict__ dst) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < na) dst[t] = src[act[t]];
}
__global__ void k_fill(int64_t n, double* p, double v) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) p[t] = v;
}

void launch_scatter_active(mycel_problem* p, const double* src_active, double* dst_box, double fill) {
  k_fill<<<(unsigned)((p->g.ne + 255) / 256), 256, 0, p->ctx->stream>>>(p->g.ne, dst_box, fill);
  p->ctx->launches++;
  if (p->n_active == 0) return;
  k_scatter_active<<<(unsigned)((p->n_active + 255) / 256), 256, 0, p->ctx->stream>>>(p->n_active, p->d_active,
                                                                                      src_active, dst_box);
  p->ctx->launches++;
}

void launch_gather_active(mycel_problem* p, const double* src_box, double* dst_active) {
  if (p->n_active == 0) return;
  k_gather_active<<<(unsigned)((p->n_active + 255) / 256), 256, 0, p->ctx->stream>>>(p->n_active, p->d_active,
                                                                                     src_box, dst_active);
  p->ctx->launches++;
}

// ---------------------------------------------------------------------------------------------------------
// Density filter as a stencil (DensityFilter.cs:61-198)
// ---------------------------------------------------------------------------------------------------------
// invHs per active element: hs accumulated over included neighbours in loop order.
__global__ void k_filter_invhs(GridDims g, const uint8_t* __restrict__ dom, const int4* __restrict__ off,
                               const double* __restrict__ w, int noff, double* __restrict__ invhs) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= g.ne || !dom[e]) return;
  int ex = (int)(e % g.nx);
  int64_t r = e / g.nx;
  int ey = (int)(r % g.ny), ez = (int)(r / g.ny);
  double hs = 0.0;
  for (int q = 0; q < noff; ++q) {
    int4 o = off[q];
    int jx = ex + o.x, jy = ey + o.y, jz = ez + o.z;
    if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) continue;
    if (!dom[jx + (int64_t)g.nx * (jy + (int64_t)g.ny * jz)]) continue;
    hs = hs + w[q];
  }
  invhs[e] = hs > 0.0 ? 1.0 / hs : 1.0;
}

// forward: out_r = sum_j (w_rj * invHs_r) * in_j, j in loop order.
// adjoint: out_i = sum_r (w_ri * invHs_r) * in_r, r ascending (the adjoint CSR rows are filled in forward-row
//          order, DensityFilter.cs:172-185); with in = 1 this is S_i (:188-198).
template <int ADJ>
__global__ void k_filter_apply(GridDims g, const uint8_t* __restrict__ dom, const int4* __restrict__ off,
                               const double* __restrict__ w, int noff, const double* __restrict__ invhs,
                               const double* __restrict__ in, double* __restrict__ out, int ones) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= g.ne || !dom[e]) return;
  int ex = (int)(e % g.nx);
  int64_t r = e / g.nx;
  int ey = (int)(r % g.ny), ez = (int)(r / g.ny);
  double s = 0.0;
  const double ih = invhs[e];
  for (int q = 0; q < noff; ++q) {
    int4 o = off[q];
    int jx = ex + o.x, jy = ey + o.y, jz = ez + o.z;
    if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) continue;
    int64_t j = jx + (int64_t)g.nx * (jy + (int64_t)g.ny * jz);
    if (!dom[j]) continue;
    if (ADJ) {
      double wt = w[q] * invhs[j];
      s = s + (ones ? wt : wt * in[j]);
    } else {
      s = s + (w[q] * ih) * in[j];
    }
  }
  out[e] = s;
}

// The forward filter as a shared-memory stencil: a CTA stages a 32 x 8 x 2 element tile with an rc-element halo
// (the input and the element flags; outside the grid or inactive: flag 0) and the offset list as index steps,
// then each thread forms its elements' sums from shared memory in the reference's neighbour order with the same
// operations, so the results are those of k_filter_apply<0> bit for bit (206 -> 147 us on the 192x96x96
// bridge). The adjoint stays per element: staged with 1/Hs its tile needs 74 KB, and at the occupancy that
// leaves it ran slower (237 against 201 us).
constexpr int kFtX = 32, kFtY = 8, kFtZ = 2;

__host__ __device__ inline size_t filter_tile_smem(int rc, int noff) {
  const size_t nt = (size_t)(kFtX + 2 * rc) * (kFtY + 2 * rc) * (kFtZ + 2 * rc);
  size_t b = nt * 8;
  b = (b + 15) & ~(size_t)15;
  b += (size_t)noff * 8 + (size_t)noff * 4 + nt;
  return b;
}

__global__ void __launch_bounds__(256) k_filter_tile(GridDims g, int rc, const uint8_t* __restrict__ dom,
                                                     const int4* __restrict__ off, const double* __restrict__ w,
                                                     int noff, const double* __restrict__ invhs,
                                                     const double* __restrict__ in, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char ftile[];
  const int PX = kFtX + 2 * rc, PY = kFtY + 2 * rc, PZ = kFtZ + 2 * rc, nt = PX * PY * PZ;
  double* sv = reinterpret_cast<double*>(ftile);
  size_t ob = (size_t)nt * 8;
  ob = (ob + 15) & ~(size_t)15;
  double* sw = reinterpret_cast<double*>(ftile + ob);
  int* so = reinterpret_cast<int*>(sw + noff);  // offsets as shared-memory index steps
  uint8_t* sd = reinterpret_cast<uint8_t*>(so + noff);
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kFtX - rc, y0 = blockIdx.y * kFtY - rc, z0 = blockIdx.z * kFtZ - rc;
  for (int i = tid; i < nt; i += blockDim.x) {
    const int gx = x0 + i % PX, gy = y0 + (i / PX) % PY, gz = z0 + i / (PX * PY);
    uint8_t d = 0;
    double v = 0.0;
    if (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz) {
      const int64_t j = gx + (int64_t)g.nx * (gy + (int64_t)g.ny * gz);
      d = dom[j];
      if (d) v = in[j];
    }
    sd[i] = d;
    sv[i] = v;
  }
  for (int q = tid; q < noff; q += blockDim.x) {
    const int4 o = off[q];
    so[q] = o.x + PX * (o.y + PY * o.z);
    sw[q] = w[q];
  }
  __syncthreads();
  const int tx = tid % kFtX, ty = tid / kFtX;
  for (int tz = 0; tz < kFtZ; ++tz) {
    const int ex = blockIdx.x * kFtX + tx, ey = blockIdx.y * kFtY + ty, ez = blockIdx.z * kFtZ + tz;
    if (ex >= g.nx || ey >= g.ny || ez >= g.nz) continue;
    const int li = (tx + rc) + PX * ((ty + rc) + PY * (tz + rc));
    if (!sd[li]) continue;
    const int64_t e = ex + (int64_t)g.nx * (ey + (int64_t)g.ny * ez);
    double s = 0.0;
    const double ih = invhs[e];
#pragma unroll 4
    for (int q = 0; q < noff; ++q) {
      const int lj = li + so[q];
      if (!sd[lj]) continue;
      s = s + (sw[q] * ih) * sv[lj];
    }
    out[e] = s;
  }
}

// largest shared-memory tile a CTA may use; beyond it (large filter radii) the per-element kernel runs
constexpr size_t kFilterTileMax = 200 * 1024;

static bool filter_tiled(mycel_filter* f) {
  static std::once_flag once;
  static bool ok = false;
  std::call_once(once, [] {
    ok = cudaFuncSetAttribute(k_filter_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFilterTileMax) ==
         cudaSuccess;
    cudaGetLastError();
  });
  return ok && filter_tile_smem(f->rc, f->n_off) <= kFilterTileMax;
}

static dim3 filter_tile_grid(const GridDims& g) {
  return dim3((unsigned)((g.nx + kFtX - 1) / kFtX), (unsigned)((g.ny + kFtY - 1) / kFtY),
              (unsigned)((g.nz + kFtZ - 1) / kFtZ));
}

int filter_setup(mycel_filter* f) {
  mycel_problem* p = f->p;
  double rmin = f->rmin;
  int rc = (int)ceil(rmin);
  double rsq = rmin * rmin;
  std::vector<int4> offs;
  std::vector<double> ws;
  for (int dz = -rc; dz <= rc; ++dz)
    for (int dy = -rc; dy <= rc; ++dy)
      for (int dx = -rc; dx <= rc; ++dx) {
        int ds = dz * dz + dy * dy + dx * dx;
        if (!((double)ds < rsq)) continue;
        double dist = sqrt((double)ds);
        if (!(dist < rmin)) continue;
        offs.push_back(make_int4(dx, dy, dz, 0));
        ws.push_back(rmin - dist);
      }
  f->n_off = (int)offs.size();
  f->rc = rc;
  cudaStream_t s = p->ctx->stream;
  if (cudaMallocAsync(&f->d_off, sizeof(int4) * offs.size(), s) != cudaSuccess) return MYCEL_E_OOM;
  if (cudaMallocAsync(&f->d_w, sizeof(double) * ws.size(), s) != cudaSuccess) return MYCEL_E_OOM;
  if (cudaMallocAsync(&f->d_invhs, sizeof(double) * p->g.ne, s) != cudaSuccess) return MYCEL_E_OOM;
  if (cudaMallocAsync(&f->d_s, sizeof(double) * p->g.ne, s) != cudaSuccess) return MYCEL_E_OOM;
  p->device_bytes += (int64_t)(sizeof(int4) * offs.size() + sizeof(double) * ws.size() + 16 * p->g.ne);
  cudaMemcpyAsync(f->d_off, offs.data(), sizeof(int4) * offs.size(), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(f->d_w, ws.data(), sizeof(double) * ws.size(), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(f->d_invhs, 0, sizeof(double) * p->g.ne, s);
  cudaMemsetAsync(f->d_s, 0, sizeof(double) * p->g.ne, s);
  unsigned nb = (unsigned)((p->g.ne + 127) / 128);
  k_filter_invhs<<<nb, 128, 0, s>>>(p->g, p->d_domain, f->d_off, f->d_w, f->n_off, f->d_invhs);
  k_filter_apply<1><<<nb, 128, 0, s>>>(p->g, p->d_domain, f->d_off, f->d_w, f->n_off, f->d_invhs, nullptr, f->d_s, 1);
  p->ctx->launches += 2;
  cudaError_t le = cudaGetLastError();
  cudaError_t se = cudaStreamSynchronize(s);  // host vectors above must outlive the copies
  if (le != cudaSuccess || se != cudaSuccess) {
    set_error(p->ctx, MYCEL_E_DEVICE, std::string("filter set-up: ") +
                                          cudaGetErrorString(le != cudaSuccess ? le : se));
    return MYCEL_E_DEVICE;
  }
  return MYCEL_OK;
}

void launch_filter_fwd(mycel_filter* f, const double* in_box, double* out_box) {
  mycel_problem* p = f->p;
  if (filter_tiled(f))
    k_filter_tile<<<filter_tile_grid(p->g), 256, filter_tile_smem(f->rc, f->n_off), p->ctx->stream>>>(
        p->g, f->rc, p->d_domain, f->d_off, f->d_w, f->n_off, f->d_invhs, in_box, out_box);
  else
    k_filter_apply<0><<<(unsigned)((p->g.ne + 127) / 128), 128, 0, p->ctx->stream>>>(
        p->g, p->d_domain, f->d_off, f->d_w, f->n_off, f->d_invhs, in_box, out_box, 0);
  p->ctx->launches++;
}

void launch_filter_adj(mycel_filter* f, const double* in_box, double* out_box) {
  mycel_problem* p = f->p;
  k_filter_apply<1><<<(unsigned)((p->g.ne + 127) / 128), 128, 0, p->ctx->stream>>>(
      p->g, p->d_domain, f->d_off, f->d_w, f->n_off, f->d_invhs, in_box, out_box, 0);
  p->ctx->launches++;
}

// ---------------------------------------------------------------------------------------------------------
// compliance sensitivities dc/drhoBar_e = -(p rho^(p-1) dE) * ue^T KE ue   (SensitivityAnalysis.cs:98-144)
// ---------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_sens(GridDims g, const __grid_constant__ KeD ke, const double* __restrict__ u,
                                              const double* __restrict__ rho, const uint8_t* __restrict__ dom,
                                              double penal, double dE, double* __restrict__ dc, int accumulate) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= g.ne || !dom[e]) return;
  int ix = (int)(e % g.nx);
  int64_t r = e / g.nx;
  int iy = (int)(r % g.ny), iz = (int)(r / g.ny);
  const int64_t sy = g.nx1, sz = (int64_t)g.nx1 * g.ny1;
  int64_t n0 = ix + sy * iy + sz * iz;
  const int64_t off[8] = {0, 1, 1 + sy, sy, sz, sz + 1, sz + 1 + sy, sz + sy};
  double ue[24];
#pragma unroll
  for (int b = 0; b < 8; ++b)
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[3 * b + c] = __ldg(u + 3 * (n0 + off[b]) + c);
  double se = 0.0;
#pragma unroll
  for (int rr = 0; rr < 24; ++rr) {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 24; ++c) s = s + ke.v[rr * 24 + c] * ue[c];
    se = se + ue[rr] * s;
  }
  double dEdr = penal * path_pow(rho[e], penal - 1.0) * dE;
  const double v = -dEdr * se;
  dc[e] = accumulate ? dc[e] + v : v;  // load cases apart: summed over the cases in case order
}

void launch_sens(mycel_problem* p, const double* u, const double* rho_box, double penal, double* dc_box,
                 bool accumulate) {
  k_sens<<<(unsigned)((p->g.ne + 127) / 128), 128, 0, p->ctx->stream>>>(p->g, p->ke, u, rho_box, p->d_domain, penal,
                                                                        p->e0 - p->emin, dc_box, accumulate ? 1 : 0);
  p->ctx->launches++;
}

// ---------------------------------------------------------------------------------------------------------
// HeavisideProjection (Optimization/HeavisideProjection.cs:12-37), an option of TopologyOptimizer.Run
// (:192-199, :279-290): the reference's expression order, every operation rounded once (this unit is built
// without contraction); Math.Clamp lets NaN through and Math.Max propagates it, as here. tanh is CUDA's, which
// can differ from the C library's in the last bit.
// ---------------------------------------------------------------------------------------------------------
__global__ void k_heaviside(int64_t n, const int32_t* __restrict__ idx, const double* __restrict__ rt,
                            const double* __restrict__ dcb, double* __restrict__ out, double beta, double eta,
                            int mode) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t e = idx ? (int64_t)idx[t] : t;
  const double den = tanh(beta * eta) + tanh(beta * (1.0 - eta));
  const double inv = 1.0 / den;
  if (mode == 0) {
    const double tbe = tanh(beta * eta);
    const double v = (tbe + tanh(beta * (rt[e] - eta))) * inv;
    out[e] = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);  // Math.Clamp(v, 0, 1)
    return;
  }
  const double th = tanh(beta * (rt[e] - eta));
  double d = beta * (1.0 - th * th) * inv;
  d = isnan(d) ? d : (d > 1e-12 ? d : 1e-12);  // Math.Max(d, 1e-12)
  out[e] = mode == 1 ? dcb[e] * d : d;
}

void launch_heaviside(mycel_ctx* ctx, int64_t n, const int32_t* idx, const double* rt, const double* dcb,
                      double* out, double beta, double eta, int mode) {
  if (n <= 0) return;
  k_heaviside<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, idx, rt, dcb, out, beta, eta, mode);
  ctx->launches++;
}

// Math.Pow over arrays, evaluated by the kernels' own path_pow (out[i] = x[i]^y[i], or x[i]^y[0] when y_len
// is 1): lets a host check the device's bits against its C library's pow.
__global__ void k_pow(int64_t n, const double* __restrict__ x, const double* __restrict__ y, int y_scalar,
                      double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = path_pow(x[i], y[y_scalar ? 0 : i]);
}

// ---------------------------------------------------------------------------------------------------------
// OC update: persistent cooperative kernel with a bounded grid barrier
// ---------------------------------------------------------------------------------------------------------
// Every wait gives up after OcArgs::max_polls polls of __nanosleep(64) (about 1 s by default, longer for large
// n, see launch_oc) and sets the error flag, so a grid that cannot meet ends with MYCEL_E_TIMEOUT on the host.
__device__ bool grid_sync_bounded(unsigned int* bar, int* err, long long max_polls, unsigned int extra) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = bar + 1;
    unsigned int gen = *vgen;
    __threadfence();
    unsigned int arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1 + extra) {
      bar[0] = 0;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*vgen == gen) {
        if (++spins > max_polls || *(volatile int*)err) {
          atomicExch(err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)err == 0;
}

__device__ __forceinline__ double clampd(double v, double lo, double hi) {
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}
__device__ __forceinline__ double maxd(double a, double b) {
  if (isnan(a) || isnan(b)) return __longlong_as_double(0x7ff8000000000000ll);
  return a > b ? a : b;
}
__device__ __forceinline__ double mind(double a, double b) {
  if (isnan(a) || isnan(b)) return __longlong_as_double(0x7ff8000000000000ll);
  return a < b ? a : b;
}

// volume term of element i for multiplier lam (OcOptimizer.EvaluateVolume :134-175) and the new density
__device__ __forceinline__ double oc_new_rho(double r, double dc, double si, bool pas, double lam, double move,
                                             double rmin) {
  if (pas) return 1.0;
  double lo = maxd(rmin, r - move), hi = mind(1.0, r + move);
  double nd = -dc;
  if (nd <= 0.0 || si <= 0.0) return lo;
  double b = nd / (lam * si);
  return clampd(r * sqrt(b), lo, hi);
}

__device__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t = t + sh[k];
  }
  return t;  // valid in thread 0
}

struct OcArgs {
  int64_t n;
  const int32_t* idx;
  const double* rho;
  const double* dc;
  const double* s;
  const uint8_t* pas;
  double* rho_new;
  const double* rho_phys;
  const double* rho_grey;
  double* scratch;  // oc_scratch_doubles(gridDim.x) doubles, layout below
  unsigned int* bar;
  int* err;
  OcOut* out;
  long long max_polls;    // polls of each wait before it gives up
  unsigned int extra;     // arrivals a barrier waits for beyond the grid (0; 1 only to test the time-out path)
};
// scratch layout (grid = gridDim.x): [0, 4 grid) two alternating pairs of per-block partial sums (value, sum of
// magnitudes) of the volume trials; [4 grid, 7 grid) per-block max change, volume and grey sums;
// [7 grid, 7 grid + 4) two alternating broadcast cells of sequential sums; then the barrier words.

// Grid-wide deterministic sums of two per-thread values; every block gets the same totals (thread 0 valid).
__device__ void grid_total2(double m0, double m1, const OcArgs& a, int slot, double* sh, bool* ok, double* t0,
                            double* t1) {
  double b0 = block_sum(m0, sh);
  double b1 = block_sum(m1, sh);
  double* part = a.scratch + (size_t)slot * 2 * gridDim.x;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = b0;
    part[gridDim.x + blockIdx.x] = b1;
  }
  if (!grid_sync_bounded(a.bar, a.err, a.max_polls, a.extra)) {
    *ok = false;
    return;
  }
  // warp 0 adds the block partials: lane l takes blocks l, l + 32, ... in order, then a fixed shuffle tree
  // (the same order in every block, so every block gets the same bits)
  double s0 = 0.0, s1 = 0.0;
  if (threadIdx.x < 32) {
    for (unsigned k = threadIdx.x; k < gridDim.x; k += 32) {
      s0 = s0 + ld_volatile(part + k);
      s1 = s1 + ld_volatile(part + gridDim.x + k);
    }
    for (int o = 16; o > 0; o >>= 1) {
      s0 = s0 + __shfl_xor_sync(0xffffffffu, s0, o);
      s1 = s1 + __shfl_xor_sync(0xffffffffu, s1, o);
    }
  }
  *t0 = s0;
  *t1 = s1;
}

// A volume V(lambda) of the bisection: the grid's tree sum, with an error bound against any other order of the
// same terms, or (exact) the sum in the reference's element order.
struct OcVol {
  double v, bound;
  bool exact;
};

__global__ void __launch_bounds__(256) k_oc(OcArgs a, OcParams prm) {
  __shared__ double sh[32];
  __shared__ double bc[4];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool ok = true;
  int slot = 0, cell = 0;
  auto element = [&](int64_t i) -> int64_t { return a.idx ? (int64_t)a.idx[i] : i; };
  auto term = [&](int64_t e, double lam) -> double {
    const double si = a.s[e];
    return si * ((a.pas && a.pas[e]) ? 1.0 : oc_new_rho(a.rho[e], a.dc[e], si, false, lam, prm.move, prm.rho_min));
  };
  // Sum of f(i) over i = 0 .. n-1 in that order (the reference's sequential loops), by warp 0 of block 0: its
  // lanes evaluate 32 consecutive terms, then every lane adds them one by one in index order. The other blocks
  // wait at the grid barrier; the result is broadcast through a scratch cell.
  auto sequential_sum = [&](auto f) -> double {
    double* c = a.scratch + (size_t)7 * gridDim.x + 2 * cell;
    cell ^= 1;
    if (blockIdx.x == 0 && threadIdx.x < 32) {
      double acc = 0.0;
      for (int64_t base = 0; base < a.n; base += 32) {
        const int64_t i = base + threadIdx.x;
        const double t = i < a.n ? f(i) : 0.0;
        const int cnt = (int)min((int64_t)32, a.n - base);
        for (int k = 0; k < cnt; ++k) acc = acc + __shfl_sync(0xffffffffu, t, k);
      }
      if (threadIdx.x == 0) *(volatile double*)c = acc;
    }
    if (!grid_sync_bounded(a.bar, a.err, a.max_polls, a.extra)) {
      ok = false;
      return 0.0;
    }
    return ld_volatile(c);
  };
  // tree depth of a grid total: the per-thread chain, the warp and block steps, the lane-strided block partials
  const double depth = (double)((a.n + stride - 1) / stride) + 5.0 + 8.0 + (double)((gridDim.x + 31) / 32) + 5.0;
  auto volume = [&](double lam) -> OcVol {
    // the thread's elements t0, t0 + stride, ... summed in that order; the loads of 8 of them are issued before
    // their terms are added, so the index -> data load chains overlap
    constexpr int kB = 8;
    double v = 0.0, va = 0.0;
    for (int64_t base = t0; base < a.n; base += kB * stride) {
      double si[kB], rr[kB], dd[kB];
      bool pp[kB];
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        const int64_t i = base + k * stride;
        const int64_t e = i < a.n ? element(i) : 0;
        pp[k] = i < a.n && a.pas && a.pas[e];
        si[k] = i < a.n ? a.s[e] : 0.0;
        rr[k] = i < a.n ? a.rho[e] : 0.0;
        dd[k] = i < a.n ? a.dc[e] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < kB; ++k)
        if (base + k * stride < a.n) {
          const double t = si[k] * (pp[k] ? 1.0 : oc_new_rho(rr[k], dd[k], si[k], false, lam, prm.move, prm.rho_min));
          v = v + t;
          va = va + fabs(t);
        }
    }
    double tv = 0.0, ta = 0.0;
    grid_total2(v, va, a, slot, sh, &ok, &tv, &ta);
    slot ^= 1;
    if (threadIdx.x == 0) {
      bc[0] = tv;
      bc[1] = ta;
    }
    __syncthreads();
    OcVol r;
    r.v = bc[0];
    // |tree - exact| <= gamma_depth sum|t| and |sequential - exact| <= gamma_(n-1) sum|t|, gamma_k = k u / (1 - k u);
    // doubled for the rounding of the computed sum of magnitudes and of the bound itself
    r.bound = 2.0 * ((double)a.n + depth) * 0x1p-53 * bc[1] * 1.0000001;
    r.exact = false;
    __syncthreads();
    return r;
  };
  // the volume at lam in the reference's order, when a decision needs it
  auto make_exact = [&](OcVol& x, double lam) {
    if (x.exact) return;
    x.v = sequential_sum([&](int64_t i) { return term(element(i), lam); });
    x.bound = 0.0;
    x.exact = true;
  };
  // total S (OcOptimizer.cs:28-33): sequential in element order, or the value the caller has cached
  double ts;
  if (prm.total_s >= 0.0) {
    ts = prm.total_s;
  } else if (prm.exact) {
    ts = sequential_sum([&](int64_t i) { return a.s[element(i)]; });
  } else {
    double sv = 0.0;
    for (int64_t i = t0; i < a.n; i += stride) sv = sv + a.s[element(i)];
    double t1 = 0.0;
    grid_total2(sv, 0.0, a, slot, sh, &ok, &ts, &t1);
    slot ^= 1;
    if (threadIdx.x == 0) bc[0] = ts;
    __syncthreads();
    ts = bc[0];
    __syncthreads();
  }
  if (!ok) return;
  const double tv = prm.f * ts;
  // the comparisons of the reference (v < target, v > target, relErr <= tolerance) taken on the tree sum unless
  // it is within its error bound of the threshold; then on the sequential sum (exact mode)
  auto less_than_target = [&](OcVol& x, double lam) -> bool {
    if (prm.exact && !x.exact && fabs(x.v - tv) <= x.bound) make_exact(x, lam);
    return x.v < tv;
  };
  auto greater_than_target = [&](OcVol& x, double lam) -> bool {
    if (prm.exact && !x.exact && fabs(x.v - tv) <= x.bound) make_exact(x, lam);
    return x.v > tv;
  };
  const double denom = maxd(tv, 1e-12);
  auto within_tolerance = [&](OcVol& x, double lam) -> bool {
    if (prm.exact && !x.exact) {
      const double d = fabs(x.v - tv), lim = prm.vol_tol * denom;
      if (fabs(d - lim) <= x.bound + 0x1p-50 * (d + lim)) make_exact(x, lam);
    }
    return fabs(x.v - tv) / denom <= prm.vol_tol;
  };
  const double lg = prm.lambda_guess;
  bool gok = lg > 0.0 && !isinf(lg) && !isnan(lg);
  double l1 = gok ? lg * 0.5 : 1e-12;
  double l2 = gok ? lg * 2.0 : 1e12;
  if (l1 <= 1e-50) l1 = 1e-12;
  if (l2 <= l1) l2 = l1 * 10.0;
  int trials = 0;
  OcVol v1 = volume(l1);
  OcVol v2 = volume(l2);
  trials += 2;
  if (!ok) return;
  int ex = 0;
  while (less_than_target(v1, l1) && l1 > 1e-50 && ex++ < 50) {
    if (!ok) return;
    l2 = l1;
    v2 = v1;
    l1 *= 0.1;
    v1 = volume(l1);
    ++trials;
    if (!ok) return;
  }
  if (!ok) return;
  ex = 0;
  while (greater_than_target(v2, l2) && l2 < 1e50 && ex++ < 50) {
    if (!ok) return;
    l1 = l2;
    v1 = v2;
    l2 *= 10.0;
    v2 = volume(l2);
    ++trials;
    if (!ok) return;
  }
  if (!ok) return;
  double lm = sqrt(l1 * l2);
  for (int st = 0; st < prm.max_bisect; ++st) {
    lm = sqrt(l1 * l2);
    OcVol vm = volume(lm);
    ++trials;
    if (!ok) return;
    const bool done = within_tolerance(vm, lm);
    if (!ok) return;
    if (done) break;
    const bool high = greater_than_target(vm, lm);
    if (!ok) return;
    if (high) l1 = lm;
    else l2 = lm;
    if (fabs(l2 - l1) <= 1e-15 * lm) break;
  }
  // final densities and the iteration metrics (TopologyOptimizer.cs:323-338)
  double mc = 0.0, vs = 0.0, gs = 0.0;
  for (int64_t i = t0; i < a.n; i += stride) {
    int64_t e = element(i);
    bool pas = a.pas && a.pas[e];
    double r = a.rho[e];
    double nr = oc_new_rho(r, a.dc[e], a.s[e], pas, lm, prm.move, prm.rho_min);
    a.rho_new[e] = nr;
    double d = fabs(nr - r);
    if (d > mc) mc = d;
    if (a.rho_phys && !prm.exact) {
      vs = vs + a.rho_phys[e];
      double rb = a.rho_grey[e];
      gs = gs + rb * (1.0 - rb);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_down_sync(0xffffffffu, mc, o);
    if (v > mc) mc = v;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mc;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k)
      if (sh[k] > mc) mc = sh[k];
  }
  double* part = a.scratch + (size_t)4 * gridDim.x;
  double bvs = block_sum(vs, sh);
  double bgs = block_sum(gs, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = mc;
    part[gridDim.x + blockIdx.x] = bvs;
    part[2 * gridDim.x + blockIdx.x] = bgs;
  }
  if (!grid_sync_bounded(a.bar, a.err, a.max_polls, a.extra)) return;
  // exact mode: the volume and grey sums in the reference's element order (:328-335)
  double svol = 0.0, sgrey = 0.0;
  if (prm.exact && a.rho_phys) {
    svol = sequential_sum([&](int64_t i) { return a.rho_phys[element(i)]; });
    sgrey = sequential_sum([&](int64_t i) {
      const double rb = a.rho_grey[element(i)];
      return rb * (1.0 - rb);
    });
    if (!ok) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double m = 0.0, v = 0.0, gg = 0.0;
    for (unsigned k = 0; k < gridDim.x; ++k) {
      double q = ld_volatile(part + k);
      if (q > m) m = q;
      v = v + ld_volatile(part + gridDim.x + k);
      gg = gg + ld_volatile(part + 2 * gridDim.x + k);
    }
    a.out->lambda = lm;
    a.out->max_change = m;
    a.out->vol_sum = prm.exact ? svol : v;
    a.out->grey_sum = prm.exact ? sgrey : gg;
    a.out->total_s = ts;
    a.out->err = 0;
    a.out->trials = trials;
  }
}

int oc_blocks_per_sm(int* out) {
  int b = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_oc, 256, 0);
  if (e != cudaSuccess) return MYCEL_E_DEVICE;
  *out = std::max(1, std::min(b, 2));
  return MYCEL_OK;
}

int launch_oc(mycel_ctx* ctx, int64_t n, const int32_t* d_index, const double* rho, const double* dc, const double* s,
              const uint8_t* passive, double* rho_new, const double* rho_phys_for_metrics,
              const double* rho_tilde_for_grey, const OcParams& prm, double* d_scratch, size_t scratch_doubles,
              OcOut* d_out) {
  const int grid = ctx->oc_grid;  // fixed when the context was created
  if (grid < 1 || oc_scratch_doubles(grid) > scratch_doubles) return MYCEL_E_ARG;
  unsigned int* bar = (unsigned int*)(d_scratch + 7 * (size_t)grid + 4);
  int* err = (int*)(bar + 4);
  if (cudaMemsetAsync(bar, 0, 8 * sizeof(unsigned int), ctx->stream) != cudaSuccess) return MYCEL_E_DEVICE;
  // each wait: about 1 s of polling, plus room for the sequential sums of the exact mode (about 20 ns per term)
  long long polls = ctx->oc_wait_polls > 0 ? ctx->oc_wait_polls : (1ll << 24) + 4 * (long long)n;
  OcArgs a{n, d_index, rho, dc, s, passive, rho_new, rho_phys_for_metrics,
           rho_tilde_for_grey ? rho_tilde_for_grey : rho_phys_for_metrics, d_scratch, bar, err, d_out,
           polls, ctx->oc_wait_unreachable ? 1u : 0u};
  OcParams pp = prm;
  void* args[] = {&a, &pp};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_oc, dim3(grid), dim3(256), args, 0, ctx->stream);
  ctx->launches++;
  if (e != cudaSuccess) return MYCEL_E_DEVICE;
  return MYCEL_OK;
}

// ---------------------------------------------------------------------------------------------------------
// OC update without device allocation.
// Some callers cannot allocate device memory at the time they run the OC step: a host whose device memory is
// reserved in full by another allocator in the same process (a caching allocator or a fixed pool), or a loop
// that must not pay the device-wide synchronisation a cudaMalloc/cudaFree pair can cost. This entry point
// takes the caller's device buffers and keeps the OC kernel's scratch (block partials, barrier words, result)
// in the file-scope array below, which every GPU that loads the library holds until the process exits.
// ---------------------------------------------------------------------------------------------------------
constexpr int kOcNoAllocMaxBlocks = 1024;                                // persistent OC blocks it can serve
constexpr int kOcNoAllocScratch = 8 * kOcNoAllocMaxBlocks + 8;           // partials + barrier words + error flag
constexpr int kOcNoAllocOut = (int)((sizeof(OcOut) + sizeof(double) - 1) / sizeof(double));
static __device__ __align__(256) double g_oc_noalloc[kOcNoAllocScratch + kOcNoAllocOut];  // 65.7 KB

namespace {
std::mutex g_oc_noalloc_mu;
void* g_oc_noalloc_addr[128] = {};  // device address of g_oc_noalloc, per device, filled on first use
}  // namespace

}  // namespace mycel

extern "C" int32_t mycel_oc_update_noalloc(mycel_ctx* ctx, int32_t n, const double* rho, const double* dc,
                                           const double* s, const uint8_t* passive, double* rho_new,
                                           double target_volume_fraction, double move_limit, double rho_min,
                                           double lambda_guess, int32_t max_bisection_steps,
                                           double volume_tolerance, double* lambda_out) {
  using namespace mycel;
  if (!ctx) return set_error(nullptr, MYCEL_E_ARG, "NULL context");
  if (n < 0 || (n > 0 && (!rho || !dc || !s || !rho_new)) || !lambda_out)
    return set_error(ctx, MYCEL_E_ARG, "All spans must have length >= rho.Length.");
  if (ctx->device < 0 || ctx->device >= 128) return set_error(ctx, MYCEL_E_ARG, "device index out of range");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return set_error(ctx, MYCEL_E_DEVICE, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  // set-up, once per device, with that device current: the host-side name of the array is not a device
  // address, so the kernel gets the address the runtime reports for this device
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_oc_noalloc_mu);
    if (!g_oc_noalloc_addr[ctx->device]) {
      e = cudaGetSymbolAddress(&g_oc_noalloc_addr[ctx->device], g_oc_noalloc);
      if (e != cudaSuccess) {
        g_oc_noalloc_addr[ctx->device] = nullptr;
        return set_error(ctx, MYCEL_E_DEVICE, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    base = g_oc_noalloc_addr[ctx->device];
  }
  const int grid = ctx->oc_grid;  // the grid launch_oc uses, fixed when the context was created
  if (oc_scratch_doubles(grid) > (size_t)kOcNoAllocScratch)
    return set_error(ctx, MYCEL_E_ARG, "OC without allocation: this device needs " + std::to_string(grid) +
                                           " persistent blocks, the static scratch holds " +
                                           std::to_string(kOcNoAllocMaxBlocks));
  double* scratch = static_cast<double*>(base);
  OcOut* out = reinterpret_cast<OcOut*>(scratch + kOcNoAllocScratch);
  // the array keeps the previous call's contents: clear the result (launch_oc clears the barrier words)
  e = cudaMemsetAsync(out, 0, sizeof(OcOut), ctx->stream);
  if (e != cudaSuccess) return set_error(ctx, MYCEL_E_DEVICE, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  OcParams prm{target_volume_fraction, move_limit, rho_min, lambda_guess, volume_tolerance, max_bisection_steps, 0};
  if (launch_oc(ctx, n, nullptr, rho, dc, s, passive, rho_new, nullptr, nullptr, prm, scratch, kOcNoAllocScratch,
                out))
    return set_error(ctx, MYCEL_E_DEVICE, std::string("OC kernel launch: ") + cudaGetErrorString(cudaGetLastError()));
  OcOut* h = reinterpret_cast<OcOut*>(ctx->pinned);
  e = cudaMemcpyAsync(h, out, sizeof(OcOut), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return set_error(ctx, MYCEL_E_DEVICE, std::string("OC kernel: ") + cudaGetErrorString(e));
  if (h->trials == 0) return set_error(ctx, MYCEL_E_TIMEOUT, "OC grid barrier timed out");
  *lambda_out = h->lambda;
  return MYCEL_OK;
}

extern "C" int32_t mycel_pow(mycel_ctx* ctx, int64_t n, const double* x, const double* y, int64_t y_len,
                             double* out) {
  using namespace mycel;
  if (!ctx) return set_error(nullptr, MYCEL_E_ARG, "NULL context");
  if (n < 0 || (n > 0 && (!x || !y || !out)) || (n > 0 && y_len != 1 && y_len != n))
    return set_error(ctx, MYCEL_E_ARG, "pow: x and out need n values, y 1 or n");
  if (n == 0) return MYCEL_OK;
  MYCEL_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  double *dx = nullptr, *dy = nullptr, *dout = nullptr;
  MYCEL_CUDA(ctx, cudaMallocAsync((void**)&dx, sizeof(double) * n, st));
  MYCEL_CUDA(ctx, cudaMallocAsync((void**)&dy, sizeof(double) * y_len, st));
  MYCEL_CUDA(ctx, cudaMallocAsync((void**)&dout, sizeof(double) * n, st));
  cudaError_t e = cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, y, sizeof(double) * y_len, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8);
    k_pow<<<blocks, 256, 0, st>>>(n, dx, dy, y_len == 1 ? 1 : 0, dout);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(dx, st);
  cudaFreeAsync(dy, st);
  cudaFreeAsync(dout, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(ctx, MYCEL_E_DEVICE, std::string("pow: ") + cudaGetErrorString(e));
  return MYCEL_OK;
}

// HeavisideProjection.Project / Derivative over host arrays (kernel-level entry points).
static int32_t heaviside_entry(mycel_ctx* ctx, int64_t n, const double* rt, double* out, double beta, double eta,
                               int mode) {
  using namespace mycel;
  if (!ctx) return set_error(nullptr, MYCEL_E_ARG, "NULL context");
  if (n < 0 || (n > 0 && (!rt || !out))) return set_error(ctx, MYCEL_E_ARG, "NULL argument");
  if (n == 0) return MYCEL_OK;
  MYCEL_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  double *din = nullptr, *dout = nullptr;
  MYCEL_CUDA(ctx, cudaMallocAsync((void**)&din, sizeof(double) * n, st));
  MYCEL_CUDA(ctx, cudaMallocAsync((void**)&dout, sizeof(double) * n, st));
  cudaError_t e = cudaMemcpyAsync(din, rt, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    launch_heaviside(ctx, n, nullptr, din, nullptr, dout, beta, eta, mode);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(din, st);
  cudaFreeAsync(dout, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(ctx, MYCEL_E_DEVICE, std::string("Heaviside: ") + cudaGetErrorString(e));
  return MYCEL_OK;
}

extern "C" int32_t mycel_heaviside_project(mycel_ctx* ctx, int64_t n, const double* rho_tilde, double* rho_bar,
                                           double beta, double eta) {
  return heaviside_entry(ctx, n, rho_tilde, rho_bar, beta, eta, 0);
}

extern "C" int32_t mycel_heaviside_derivative(mycel_ctx* ctx, int64_t n, const double* rho_tilde, double* deriv,
                                              double beta, double eta) {
  return heaviside_entry(ctx, n, rho_tilde, deriv, beta, eta, 2);
}
