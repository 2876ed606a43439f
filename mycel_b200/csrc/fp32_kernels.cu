// Mixed-precision form: FP32 inner Jacobi-PCG (K·u and the preconditioner in FP32 with FP32 accumulation)
// inside FP64 iterative refinement. FP64 is kept only for the refinement residual f - K u, the CG alpha/beta
// dot products (FP32 operands, products and sums in FP64), and the accumulated solution u.
//
// Refinement is done by reliable updating: the FP32 CG recurrence runs continuously; whenever its recursive
// residual has dropped by kFlushFactor since the last replacement (or reaches the target), the FP32 correction
// is added to u in FP64, the true residual P(b - A u) is recomputed in FP64 and replaces the FP32 residual, and
// the search direction is kept (beta = rho_new / rho_old), so the Krylov progress is not thrown away.
//
// Per inner iteration two kernels:
//   k_mv32   p_t = z + beta p_{t-1} (on the fly for every gathered node), Ap_t = K p_t, and the FP64 partials of
//            p_t . Ap_t; the last CTA forms alpha.
//   k_xr32   x += alpha p, r -= alpha Ap, z = r invD, FP64 partials of r.r and r.z; the last CTA forms the
//            recursive residual, the replacement/stop triggers and beta.
// Reductions use a fixed CTA decomposition and a fixed-order final sum, so results do not depend on timing.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "internal.h"

namespace mycel {

enum MixStatus : int { MIX_RUNNING = 0, MIX_FLUSH = 1, MIX_BREAKDOWN = 2, MIX_MAXITER = 3, MIX_DONE = 4 };

struct MixState {
  int status;
  int iter;      // inner iterations in total
  int max_iter;
  int first;     // next k_mv32 starts a new direction (p = z)
  double target;     // absolute residual at which to verify convergence (tol * ||P b|| * safety)
  double flush_at;   // absolute recursive residual that triggers a true-residual replacement
  double rho0, alpha, beta, rn, pap;
  double flush_factor;  // a replacement when the recursive residual has dropped by this factor
  unsigned int counter;
  int pmode;  // packed runs: the outer step a right-hand side takes next (0 after a matvec, 1 restart, 2 start)
};

constexpr int kT = 256;
constexpr double kFlushFactor = 1e-1;

// the last of nblk CTAs to arrive (a launch's CTAs, or those of one problem of a packed launch)
__device__ __forceinline__ bool elect_last_n(unsigned int* counter, unsigned nblk) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == nblk - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}
__device__ __forceinline__ bool elect_last32(unsigned int* counter) {
  return elect_last_n(counter, gridDim.x * gridDim.y);
}

// deterministic block sum of a double (result valid in linear thread 0); works for 1-D and 2-D blocks
__device__ __forceinline__ double bsum(double v, double* sh) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (tid == 0)
    for (int k = 0; k < nw; ++k) t += sh[k];
  return t;
}

// deterministic sum of part[0..n) by one warp (lane l takes l, l+32, ...; fixed shuffle tree); all lanes get it
__device__ __forceinline__ double warp_sum_parts(const double* part, unsigned n) {
  int lane = threadIdx.x & 31;
  double s = 0.0;
  for (unsigned q = lane; q < n; q += 32) s += *(const volatile double*)(part + q);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
constexpr long long kMbarSpinLimit = 1ll << 22;
// bounded wait for phase `parity` of an mbarrier; returns false if it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long spin = 0; spin < kMbarSpinLimit; ++spin) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}


// ---------------------------------------------------------------------------------------------------------
// FP32 K p, z-marching shared-memory tiles.
// A CTA owns a TX x TY column of nodes and marches over ZSEG node planes. Three node planes of the input
// (with a one-node halo) and two element planes of E live in shared memory; rows are loaded contiguously.
// Each thread keeps its 27-node neighbourhood in registers and applies the 8 incident elements' KE rows
// (compile-time indices, so KE is read as constant-bank FFMA operands).
// MODE 1 (inner PCG step): the input is p_t = z + beta p_{t-1} formed while loading; owned nodes write p_t;
// the CTA adds p_t . K p_t into an FP64 partial and the last CTA forms alpha.
// Inactive elements carry E = 0, elements outside the grid and halo nodes outside the grid read as 0.
// ---------------------------------------------------------------------------------------------------------
constexpr int TX = 32, TY = 8;
constexpr int PX = TX + 2, PY = TY + 2;  // node plane with halo
constexpr int EX = TX + 1, EY = TY + 1;  // element plane
constexpr int ROWF = 3 * PX;             // floats per node row of a plane (contiguous in global memory)
constexpr int NSLOT = 4;                 // rolling node planes: k-1, k, k+1 in use, k+2 arriving
constexpr int NESLOT = 3;                // rolling element planes: k-1, k in use, k+1 arriving

// Plane loader: warp w copies rows w and w + 8 of a plane (3 * PX contiguous floats each), lane l the offsets
// l, l+32, l+64, l+96 of a row. Everything that does not depend on the plane index is computed once.
struct RowLoad {
  int nrows;         // 1 or 2
  int ly[2];
  int64_t gofs[2];   // global float offset of (row start + lane) at plane 0 (may be negative at i = -1)
  unsigned rowok;    // bit q: row q exists and lies in the grid in y
  unsigned xmask;    // bit r: offset lane + 32 r lies in the grid in x (and < ROWF)
  unsigned own;      // bit 4 * row + r: interior node of an owned row (written back as p_t)
};

template <int MODE>
__global__ void __launch_bounds__(TX * TY, 3) k_mv32(GridDims g, const __grid_constant__ KeF ke,
                                                     const float* __restrict__ xin, const float* __restrict__ z,
                                                     const float* __restrict__ pold, float* __restrict__ pnew,
                                                     float* __restrict__ y, const float* __restrict__ E,
                                                     const uint8_t* __restrict__ nf, int projected, MixState* st,
                                                     double* part, int zseg) {
  __shared__ float4 xs[NSLOT][PY][PX];  // node planes, one float4 per node (w unused)
  __shared__ float es[NESLOT][EY][EX];
  __shared__ double sh[32];
  if (MODE == 1 && st->status != MIX_RUNNING) return;
  const float beta = MODE == 1 ? (float)st->beta : 0.0f;
  const bool first = MODE == 1 ? (st->first != 0) : true;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * zseg;
  const int k1 = min(k0 + zseg, g.nz1);
  const int64_t sy = g.nx1, sz = (int64_t)g.nx1 * g.ny1;
  const int64_t plane_f = (int64_t)g.rp * g.ny1;  // floats per node plane (padded FP32 layout)

  // ---- per-thread load plan (node rows) ----
  RowLoad rl;
  rl.nrows = (ty + 8 < PY) ? 2 : 1;
  rl.xmask = 0;
  rl.own = 0;
  rl.rowok = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    int off = tx + 32 * r;
    int lx = off / 3;
    int i = i0 - 1 + lx;
    if (off < ROWF && i >= 0 && i < g.nx1) rl.xmask |= 1u << r;
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    int ly = ty + 8 * q;
    rl.ly[q] = ly;
    int j = j0 - 1 + ly;
    bool ok = q < rl.nrows && j >= 0 && j < g.ny1;
    rl.gofs[q] = 3 * (int64_t)(i0 - 1) + (int64_t)g.rp * j + tx;
    if (ok) rl.rowok |= 1u << q;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int off = tx + 32 * r, lx = off / 3;
      if (ok && (rl.xmask >> r & 1) && ly >= 1 && ly <= TY && lx >= 1 && lx <= TX) rl.own |= 1u << (4 * q + r);
    }
  }
  // element plane: warp w copies element row w (row 8 by warp 0); lane l the elements l and 32 (lane 0)
  const int erows = (ty == 0) ? 2 : 1;
  int64_t eofs[2];
  unsigned emask = 0;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    int ly = ty + 8 * q;
    int je = j0 - 1 + ly;
    bool ok = q < erows && je >= 0 && je < g.ny;
    eofs[q] = (int64_t)(i0 - 1) + tx + (int64_t)g.nx * je;  // element (i0-1+tx, je) at element plane 0
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int lx = tx + 32 * r, ie = i0 - 1 + lx;
      if (ok && lx < EX && ie >= 0 && ie < g.nx) emask |= 1u << (2 * q + r);
    }
  }
  const int64_t eplane = (int64_t)g.nx * g.ny;

  float pre[2][4];   // prefetched node-plane values (z, or x for MODE 0)
  float prep[2][4];  // prefetched p_{t-1} (MODE 1); p_t = z + beta p_{t-1} is formed at commit time
  float epre[2][2];
  auto fetch = [&](int kk) {
    const bool inz = kk >= 0 && kk < g.nz1;
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        float v = 0.f, w = 0.f;
        if (inz && (rl.rowok >> q & 1) && (rl.xmask >> r & 1)) {
          int64_t idx = rl.gofs[q] + plane_f * kk + 32 * r;
          if (MODE == 1) {
            v = __ldg(z + idx);
            if (!first) w = __ldg(pold + idx);
          } else {
            v = __ldg(xin + idx);
          }
        }
        pre[q][r] = v;
        prep[q][r] = w;
      }
  };
  auto commit = [&](int kk) {
    const int slot = (kk + NSLOT) % NSLOT;
    const bool owned_plane = kk >= k0 && kk < k1;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (q >= rl.nrows) break;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int off = tx + 32 * r;
        const float v = (MODE == 1 && !first) ? fmaf(beta, prep[q][r], pre[q][r]) : pre[q][r];
        if (off < ROWF) reinterpret_cast<float*>(&xs[slot][rl.ly[q]][0])[4 * (off / 3) + off % 3] = v;
        if (MODE == 1 && owned_plane && (rl.own >> (4 * q + r) & 1))
          pnew[rl.gofs[q] + plane_f * kk + 32 * r] = v;
      }
    }
  };
  auto efetch = [&](int ke_) {
    const bool inz = ke_ >= 0 && ke_ < g.nz;
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        float v = 0.f;
        if (inz && (emask >> (2 * q + r) & 1)) v = __ldg(E + eofs[q] + eplane * ke_ + 32 * r);
        epre[q][r] = v;
      }
  };
  auto ecommit = [&](int ke_) {
    const int slot = (ke_ + NESLOT) % NESLOT;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (q >= erows) break;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        int lx = tx + 32 * r;
        if (lx < EX) es[slot][ty + 8 * q][lx] = epre[q][r];
      }
    }
  };

  // prologue: planes k0-1, k0, k0+1 and element planes k0-1, k0 in shared memory; plane k0+2 in flight
  fetch(k0 - 1); commit(k0 - 1);
  fetch(k0); commit(k0);
  fetch(k0 + 1); commit(k0 + 1);
  efetch(k0 - 1); ecommit(k0 - 1);
  efetch(k0); ecommit(k0);
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  const bool mine = i < g.nx1 && j < g.ny1;
  double pap = 0.0;
  for (int k = k0; k < k1; ++k) {
    const bool more = k + 1 < k1;
    if (more) {
      fetch(k + 2);
      efetch(k + 1);
    }
    if (mine) {
      float xn[3][3][3][3];  // [dz][dy][dx][c], offsets -1..+1
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) {
        const int slot = (k - 1 + dz + NSLOT) % NSLOT;
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
            const float4 v4 = xs[slot][ty + dy][tx + dx];
            xn[dz][dy][dx][0] = v4.x;
            xn[dz][dy][dx][1] = v4.y;
            xn[dz][dy][dx][2] = v4.z;
          }
      }
      float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
#pragma unroll
      for (int sz_ = 0; sz_ < 2; ++sz_) {
        const int eslot = (k - 1 + sz_ + NESLOT) % NESLOT;
#pragma unroll
        for (int sy_ = 0; sy_ < 2; ++sy_)
#pragma unroll
          for (int sx_ = 0; sx_ < 2; ++sx_) {
            const float ee = es[eslot][ty + sy_][tx + sx_];
            // this node sits at local (1-sx, 1-sy, 1-sz) of the element
            const int ox = 1 - sx_, oy = 1 - sy_, oz = 1 - sz_;
            const int a = (oy ? (ox ? 2 : 3) : (ox ? 1 : 0)) + 4 * oz;
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
              const int bx = (b == 1 || b == 2 || b == 5 || b == 6) ? 1 : 0;
              const int by = (b == 2 || b == 3 || b == 6 || b == 7) ? 1 : 0;
              const int bz = b >= 4 ? 1 : 0;
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                const float xv = xn[sz_ + bz][sy_ + by][sx_ + bx][c];
                s0 = fmaf(ke.v[(3 * a + 0) * 24 + 3 * b + c], xv, s0);
                s1 = fmaf(ke.v[(3 * a + 1) * 24 + 3 * b + c], xv, s1);
                s2 = fmaf(ke.v[(3 * a + 2) * 24 + 3 * b + c], xv, s2);
              }
            }
            acc0 = fmaf(ee, s0, acc0);
            acc1 = fmaf(ee, s1, acc1);
            acc2 = fmaf(ee, s2, acc2);
          }
      }
      const int64_t n = i + sy * j + sz * k;
      const uint8_t f = projected ? nf[n] : 0;
      const float out[3] = {acc0, acc1, acc2};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float pv = xn[1][1][1][c];
        const float yv = (f & (1 << c)) ? pv : out[c];
        y[plane_f * k + (int64_t)g.rp * j + 3 * i + c] = yv;
        if (MODE == 1) pap += (double)pv * (double)yv;
      }
    }
    if (more) {
      commit(k + 2);   // slot (k+2)%4 held plane k-2: no longer read
      ecommit(k + 1);  // slot (k+1)%3 held element plane k-2
    }
    __syncthreads();
  }
  if (MODE != 1) return;
  double b = bsum(pap, sh);
  const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (tid == 0) part[bid] = b;
  // last-CTA election over the 3-D grid
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(&st->counter, 1u) == nblk - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (tid >= 32) return;
  double s = warp_sum_parts(part, nblk);
  if (tid != 0) return;
  st->counter = 0;
  st->first = 0;
  st->pap = s;
  if (!(s > 0.0) || !isfinite(s)) {
    st->status = MIX_BREAKDOWN;
    return;
  }
  st->alpha = st->rho0 / s;
}

// z-segment length: enough segments that the grid holds about 8 CTAs per SM (the kernel is latency-bound
// with one CTA per SM), at least 2 planes per segment.
static int tile_zseg(const GridDims& g, int num_sms) {
  int64_t txy = (int64_t)((g.nx1 + TX - 1) / TX) * ((g.ny1 + TY - 1) / TY);
  int64_t segs = std::max<int64_t>(1, (8 * (int64_t)num_sms + txy - 1) / txy);
  return (int)std::max<int64_t>(2, (g.nz1 + segs - 1) / segs);
}

static dim3 tile_grid(const GridDims& g, int zseg) {
  return dim3((unsigned)((g.nx1 + TX - 1) / TX), (unsigned)((g.ny1 + TY - 1) / TY), (unsigned)((g.nz1 + zseg - 1) / zseg));
}

// ---------------------------------------------------------------------------------------------------------
// FP32 K p with the factorised cube-element operator (HexOpF, built by build_hexop): per element an 8-point
// Walsh-Hadamard transform of each displacement component, 21 eigenvalue products, 24 products coupling
// pairs of components, and the inverse transform: about 190 flops per element instead of the 1152 of a dense
// 24 x 24 KE product. Results differ from the dense product only by FP32 rounding.
// Element-centric z-marching tiles: a CTA of FX x FY threads computes the FX x FY elements of each element
// plane of its column (thread (l, w) the element (i0 - 1 + l, j0 - 1 + w)) and owns the FOX x FOY nodes
// strictly inside that element tile. A node receives the contributions of its x-neighbour element through a
// warp shuffle and those of its y-neighbour elements through a small shared-memory exchange; the part from
// the element plane below is carried in registers. Node planes with a one-node halo are staged in shared
// memory (two slots, the next-but-one prefetched into registers while the current plane is worked on); each
// plane step has one __syncthreads.
// MODE 1 fuses p_t = z + beta p_{t-1}, the write of p_t and the p.Ap partials, as k_mv32 does.
// ---------------------------------------------------------------------------------------------------------
constexpr int FX = 32, FY = 8;
constexpr int FOX = FX - 1, FOY = FY - 1;  // owned nodes per tile
constexpr int FPY = FY + 1;                // node rows of a staged plane (with halo)

// Packed FP32x2 arithmetic (sm_100): lane .x and lane .y are two independent elements.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.f), a); }  // exact -b
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// 8-point Walsh-Hadamard butterflies over the index bits (x, y, z): afterwards v[p] = sum_a s_p(a) v_a,
// s_p(a) the product over the axes odd in p of (2 a_axis - 1).
__device__ __forceinline__ void wht8x2(float2 (&v)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (!(a & bit)) {
        const float2 lo = v[a], hi = v[a | bit];
        v[a] = f2add(hi, lo);
        v[a | bit] = f2sub(hi, lo);
      }
}

// node values from basis coefficients: per axis (even e, odd o) -> (e - o, e + o)
__device__ __forceinline__ void iwht8x2(float2 (&v)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (!(a & bit)) {
        const float2 e = v[a], o = v[a | bit];
        v[a] = f2sub(e, o);
        v[a | bit] = f2add(e, o);
      }
}

// y = E KE(h) u for two elements at once (lanes .x, .y); u[c][a]: component c at local node
// a = x | y << 1 | z << 2 (bit order, not the reference's local numbering). The outputs of component c are
// handed to sink(c, y_c[8]) as soon as they are formed, which keeps few of them live.
template <class Sink>
__device__ __forceinline__ void hex_apply2(const HexOpF& op, float2 E, float2 (&u)[3][8], Sink&& sink) {
#pragma unroll
  for (int c = 0; c < 3; ++c) wht8x2(u[c]);
  float2 d[2][3], lam[2], mu[2];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int n = 0; n < 3; ++n) d[a][n] = f2mul(E, f2(op.dcl[a][n]));
    lam[a] = f2mul(E, f2(op.lam[a]));
    mu[a] = f2mul(E, f2(op.mu[a]));
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float2 y[8];
    y[0] = f2(0.f);  // rigid translation: no force
#pragma unroll
    for (int p = 1; p < 8; ++p) {
      const int pc = (p >> c) & 1;
      const int n = (p & 1) + ((p >> 1) & 1) + ((p >> 2) & 1) - pc;
      float2 acc = f2mul(d[pc][n], u[c][p]);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (j == c) continue;
        const int k = 3 - c - j;
        const int pj = (p >> j) & 1, pk = (p >> k) & 1;
        const int q = p ^ (1 << c) ^ (1 << j);
        if (pc == 1 && pj == 0) acc = f2fma(lam[pk], u[j][q], acc);
        if (pc == 0 && pj == 1) acc = f2fma(mu[pk], u[j][q], acc);
      }
      y[p] = acc;
    }
    iwht8x2(y);
    sink(c, y);
  }
}

// p.Ap partials of a matvec launch: CTA sum, fixed-order sum of the CTA partials by the last CTA, alpha.
// A launch whose bounded waits gave up has set *err; its last CTA then ends the inner solve as a breakdown.
__device__ __forceinline__ void mv32_finish(double pap, double* sh, MixState* st, double* part, int tid,
                                            const int* err, unsigned nblk, unsigned bid) {
  const double b = bsum(pap, sh);
  if (tid == 0) part[bid] = b;
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(&st->counter, 1u) == nblk - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (tid >= 32) return;
  const double s = warp_sum_parts(part, nblk);
  if (tid != 0) return;
  st->counter = 0;
  st->first = 0;
  st->pap = s;
  if ((err && *(const volatile int*)err) || !(s > 0.0) || !isfinite(s)) {
    st->status = MIX_BREAKDOWN;
    return;
  }
  st->alpha = st->rho0 / s;
}

// TMA (cp.async.bulk.tensor) node-plane loads: the FP32 vectors are 3-D tensors [nz1][ny1][rp] floats; a copy
// brings a [FPY][FBW] box whose x start is rounded down to 16 bytes, and zero-fills what lies outside the grid.
constexpr int FNST = 4;                                     // node-plane stages in flight
constexpr int FBW = 104;                                    // floats per staged node row (>= 99 + 3 of rounding)
constexpr int kFacStageBytes = FPY * FBW * 4;               // bytes landed per array per stage
constexpr int kFacStagePitch = (kFacStageBytes + 127) & ~127;
constexpr size_t fac_smem_bytes(int mode) {
  return (size_t)FNST * kFacStagePitch * (mode == 1 ? 2 : 1) + sizeof(float) * 2 * FY * 9 * FX;
}

__device__ __forceinline__ void tma_load_plane(void* dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// The kernel body, for CTA (bx, by, bz) of a grid of nblk CTAs (linear number bid, x fastest): a launch of
// one matvec (k_mv32f) or one tile of a packed launch (k_mv32f_pk). tm_a / tm_b point at the tensor maps
// (kernel parameters, or a packed launch's table in global memory). Returns 0 when the state is not running
// (nothing done, the mbarriers untouched), 1 after the tile, -1 when a bounded wait gave up (*err set).
// The matvec's pointers and constants: kernel parameters (a launch alone: read from the constant bank) or a
// packed tile's copy in shared memory (read again after each barrier, so they hold no registers across steps).
struct MvArgs {
  const HexOpF* op;
  const CUtensorMap *tm_a, *tm_b;
  float* pnew;
  float* y;
  const float* E;
  const uint8_t* nf;
  MixState* st;
  double* part;
  int* err;
  int projected;
};

template <int MODE, class A>
__device__ __forceinline__ int mv32f_body(const GridDims& g, const A& a, int zseg, int bx, int by, int bz, unsigned nblk,
                                          unsigned bid) {
  MixState* const st = a.st;
  extern __shared__ __align__(128) unsigned char fac_smem[];
  // [FNST] stages of x (MODE 0) or z (MODE 1), then MODE 1: [FNST] stages of p_{t-1}; then y-exchange
  float* yb = reinterpret_cast<float*>(fac_smem + (size_t)FNST * kFacStagePitch * (MODE == 1 ? 2 : 1));
  __shared__ __align__(8) unsigned long long full[FNST];
  __shared__ double sh[32];
  if (st && st->status != MIX_RUNNING) return 0;  // MODE 0 gets a state only inside the multigrid cycle
  const float beta = MODE == 1 ? (float)st->beta : 0.0f;
  const bool two = MODE == 1 && st->first == 0;  // p_t = z + beta p_{t-1} (else p_t = z)
  const int l = threadIdx.x, w = threadIdx.y, tid = w * FX + l;
  const int i0 = bx * FOX, j0 = by * FOY, k0 = bz * zseg;
  const int k1 = min(k0 + zseg, g.nz1);
  const int xs = (3 * (i0 - 1)) & ~3;   // staged row start (floats), 16-byte aligned, may be -4
  const int rem = 3 * (i0 - 1) - xs;    // offset of node i0 - 1 in a staged row
  const uint32_t tx_bytes = (uint32_t)kFacStageBytes * (two ? 2u : 1u);
  // Element planes k0-1 .. k1-1 are taken two per step (the last step may add plane k1, whose nodes are
  // not owned). Node plane k0 - 1 + r ("rel r", r = 0 .. rmax) lives in stage r % FNST; its use of the
  // stage has mbarrier parity (r / FNST) & 1. Step m needs rel 2m (carried), 2m + 1 and 2m + 2.
  const int nsteps = (k1 - k0 + 2) >> 1;
  const int rmax = 2 * nsteps;

  auto plane_a = [&](int sl) { return reinterpret_cast<float*>(fac_smem + (size_t)sl * kFacStagePitch); };
  auto plane_b = [&](int sl) { return reinterpret_cast<float*>(fac_smem + (size_t)(FNST + sl) * kFacStagePitch); };
  auto issue = [&](int r) {  // one thread
    const int sl = r % FNST;
    const uint32_t bar = smem_u32(&full[sl]);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
    tma_load_plane(plane_a(sl), a.tm_a, xs, j0 - 1, k0 - 1 + r, bar);
    if (two) tma_load_plane(plane_b(sl), a.tm_b, xs, j0 - 1, k0 - 1 + r, bar);
  };
  if (tid == 0) {
    for (int q = 0; q < FNST; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int r = 0; r < FNST && r <= rmax; ++r) issue(r);
  bool ok = true;
  auto wait_rel = [&](int r) {
    if (!mbar_wait(smem_u32(&full[r % FNST]), (uint32_t)((r / FNST) & 1))) ok = false;
  };
  // the 4 nodes of this thread's element column in node plane rel r: (x, y) = (0,0), (1,0), (0,1), (1,1);
  // MODE 1 forms p_t = z + beta p_{t-1}
  auto gather4 = [&](int r, float (&v)[4][3]) {
    const int sl = r % FNST;
    const float* a = plane_a(sl);
    const float* b = plane_b(sl);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int o = (w + (q >> 1)) * FBW + rem + 3 * (l + (q & 1));
#pragma unroll
      for (int c = 0; c < 3; ++c) v[q][c] = two ? fmaf(beta, b[o + c], a[o + c]) : a[o + c];
    }
  };

  const int ex = i0 - 1 + l, ey = j0 - 1 + w;
  const bool exy = ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny;
  const int64_t ebase = (int64_t)ex + (int64_t)g.nx * ey, eplane = (int64_t)g.nx * g.ny;
  auto eload = [&](int kk) -> float { return (exy && kk >= 0 && kk < g.nz) ? __ldg(a.E + ebase + eplane * kk) : 0.f; };
  const int nxo = i0 + l, nyo = j0 + w;  // owned node (local node (1, 1) of this thread's elements)
  const bool mine = l < FOX && w < FOY && nxo < g.nx1 && nyo < g.ny1;
  const int64_t nbase = nxo + (int64_t)g.nx1 * nyo;     // node index at plane 0
  const int64_t fbase = (int64_t)g.rp * nyo + 3 * nxo;  // padded FP32 offset at plane 0
  const int64_t fplane = (int64_t)g.rp * g.ny1;
  const int64_t nplane = (int64_t)g.nx1 * g.ny1;
  auto fload = [&](int kk) -> uint8_t {
    return (mine && a.projected && kk >= k0 && kk < k1) ? a.nf[nbase + nplane * kk] : (uint8_t)0;
  };

  wait_rel(0);
  float ub[4][3];
  gather4(0, ub);
  __syncthreads();  // stage of rel 0 is refilled in the first step
  float carry[3] = {0.f, 0.f, 0.f};
  double pap = 0.0;
  float2 e_next = make_float2(eload(k0 - 1), eload(k0));
  uint8_t f_next0 = fload(k0 - 1), f_next1 = fload(k0);
  for (int m = 0; m < nsteps; ++m) {
    const int kk = k0 - 1 + 2 * m;  // element planes kk (lane .x) and kk + 1 (lane .y)
    wait_rel(2 * m + 1);
    wait_rel(2 * m + 2);
    float um[4][3], ut[4][3];
    gather4(2 * m + 1, um);
    gather4(2 * m + 2, ut);
    // stages of rel 2m - 1 and 2m were last read in the previous step (or the prologue); refill them
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
#pragma unroll
      for (int r = 2 * m + 3; r <= 2 * m + 4; ++r)
        if (r >= FNST && r <= rmax) issue(r);
    }
    const float2 e2 = e_next;
    e_next = make_float2(eload(kk + 2), eload(kk + 3));
    const uint8_t f0 = f_next0, f1 = f_next1;
    f_next0 = fload(kk + 2);
    f_next1 = fload(kk + 3);
    if (MODE == 1 && mine) {
      if (kk + 1 >= k0 && kk + 1 < k1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) a.pnew[fbase + fplane * (kk + 1) + c] = um[3][c];
      }
      if (kk + 2 < k1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) a.pnew[fbase + fplane * (kk + 2) + c] = ut[3][c];
      }
    }
    float2 u[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        u[c][b] = make_float2(ub[b][c], um[b][c]);      // local z = 0: planes kk, kk + 1
        u[c][b + 4] = make_float2(um[b][c], ut[b][c]);  // local z = 1: planes kk + 1, kk + 2
      }
    // comb[by][pl][c]: node column ex + 1, node row ey + by, node plane kk + pl, after the x-neighbour's part
    float comb[2][3][3];
    hex_apply2(*a.op, e2, u, [&](int c, float2 (&yc)[8]) {
#pragma unroll
      for (int by = 0; by < 2; ++by) {
        const int a = 2 * by;
        const float s1[3] = {yc[a + 1].x, yc[a + 5].x + yc[a + 1].y, yc[a + 5].y};  // local x = 1
        const float s0[3] = {yc[a].x, yc[a + 4].x + yc[a].y, yc[a + 4].y};          // local x = 0
#pragma unroll
        for (int pl = 0; pl < 3; ++pl) comb[by][pl][c] = s1[pl] + __shfl_down_sync(0xffffffffu, s0[pl], 1);
      }
    });
    // y: the row above adds its local y = 0 sums to this row's local y = 1 sums
    float* ybw = yb + ((m & 1) * FY + w) * 9 * FX + l;
#pragma unroll
    for (int pl = 0; pl < 3; ++pl)
#pragma unroll
      for (int c = 0; c < 3; ++c) ybw[(3 * pl + c) * FX] = comb[0][pl][c];
    __syncthreads();
    if (mine) {
      const float* ybr = yb + ((m & 1) * FY + w + 1) * 9 * FX + l;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float s0 = comb[1][0][c] + ybr[c * FX];
        const float s1 = comb[1][1][c] + ybr[(3 + c) * FX];
        const float s2 = comb[1][2][c] + ybr[(6 + c) * FX];
        if (kk >= k0) {  // node plane kk: the element plane below (carried) + plane kk's bottom faces
          const float pv = ub[3][c];
          const float yo = (f0 >> c & 1) ? pv : carry[c] + s0;
          a.y[fbase + fplane * kk + c] = yo;
          if (MODE == 1) pap += (double)pv * (double)yo;
        }
        if (kk + 1 < k1) {  // node plane kk + 1: complete within this step
          const float pv = um[3][c];
          const float yo = (f1 >> c & 1) ? pv : s1;
          a.y[fbase + fplane * (kk + 1) + c] = yo;
          if (MODE == 1) pap += (double)pv * (double)yo;
        }
        carry[c] = s2;
      }
    }
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) ub[b][c] = ut[b][c];
  }
  // every copy has landed when all waits succeeded: the mbarriers are retired, so a persistent CTA can set
  // them up again for its next tile (after a failed wait a copy may still be in flight: they stay as they are)
  const bool all_ok = __syncthreads_and(ok) != 0;
  if (all_ok && tid == 0)
    for (int q = 0; q < FNST; ++q) asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(&full[q])) : "memory");
  if (!ok && a.err) atomicExch(a.err, 1);
  if (MODE == 1) mv32_finish(pap, sh, a.st, a.part, tid, a.err, nblk, bid);
  return all_ok ? 1 : -1;
}

template <int MODE>
__global__ void __launch_bounds__(FX * FY, 2) k_mv32f(GridDims g, const __grid_constant__ HexOpF op,
                                                      const __grid_constant__ CUtensorMap tm_a,
                                                      const __grid_constant__ CUtensorMap tm_b,
                                                      float* __restrict__ pnew, float* __restrict__ y,
                                                      const float* __restrict__ E, const uint8_t* __restrict__ nf,
                                                      int projected, MixState* st, double* part, int zseg, int* err) {
  const MvArgs a{&op, &tm_a, &tm_b, pnew, y, E, nf, st, part, err, projected};
  mv32f_body<MODE>(g, a, zseg, blockIdx.x, blockIdx.y,
                   blockIdx.z, gridDim.x * gridDim.y * gridDim.z,
                   (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
}

// z-segment length of the factorised kernel: the CTAs of a launch run in ceil(CTAs / resident) waves of
// (segment length + 2) / 2 steps of two element planes (one extra element plane below each segment); pick the segment
// count with the least waves x steps, at least 4 planes per segment.
static int fac_zseg(const GridDims& g, int resident) {
  const int64_t txy = (int64_t)((g.nx1 + FOX - 1) / FOX) * ((g.ny1 + FOY - 1) / FOY);
  const int max_segs = std::max(1, g.nz1 / 4);
  int best_z = g.nz1;
  int64_t best_cost = INT64_MAX;
  for (int segs = 1; segs <= max_segs; ++segs) {
    const int zs = (g.nz1 + segs - 1) / segs;
    const int64_t n = txy * ((g.nz1 + zs - 1) / zs);
    const int64_t cost = ((n + resident - 1) / resident) * ((zs + 2) / 2);  // two element planes per step
    if (cost < best_cost) {
      best_cost = cost;
      best_z = zs;
    }
  }
  return best_z;
}

static dim3 fac_grid(const GridDims& g, int zseg) {
  return dim3((unsigned)((g.nx1 + FOX - 1) / FOX), (unsigned)((g.ny1 + FOY - 1) / FOY),
              (unsigned)((g.nz1 + zseg - 1) / zseg));
}

// ---------------------------------------------------------------------------------------------------------
// FP64 K p with the factorised cube-element operator (fast FP64 form; not bit-exact with the reference's
// colour-ordered product, equal to it up to FP64 rounding). Same tiling as k_mv32f with one element plane
// per step, FP64 node planes by TMA from the padded FP64 layout (row starts rounded down to 16 bytes, boxes
// of FPY x FBW64 doubles), one thread per element, x-neighbour by shuffle, y-neighbour by shared exchange.
// MODE 1 fuses p_t = z + beta p_{t-1}, the write of p_t and the p.Ap partials.
// ---------------------------------------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void wht8s(T (&v)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (!(a & bit)) {
        const T lo = v[a], hi = v[a | bit];
        v[a] = hi + lo;
        v[a | bit] = hi - lo;
      }
}

template <class T>
__device__ __forceinline__ void iwht8s(T (&v)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (!(a & bit)) {
        const T e = v[a], o = v[a | bit];
        v[a] = e - o;
        v[a | bit] = e + o;
      }
}

// y = E KE(h) u for one element in FP64 (same basis and constants as hex_apply2); sink(c, y_c[8])
template <class Sink>
__device__ __forceinline__ void hex_apply64(const HexOpD& op, double E, double (&u)[3][8], Sink&& sink) {
#pragma unroll
  for (int c = 0; c < 3; ++c) wht8s(u[c]);
  double d[2][3], lam[2], mu[2];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int n = 0; n < 3; ++n) d[a][n] = E * op.dcl[a][n];
    lam[a] = E * op.lam[a];
    mu[a] = E * op.mu[a];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double y[8];
    y[0] = 0.0;
#pragma unroll
    for (int p = 1; p < 8; ++p) {
      const int pc = (p >> c) & 1;
      const int n = (p & 1) + ((p >> 1) & 1) + ((p >> 2) & 1) - pc;
      double acc = d[pc][n] * u[c][p];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (j == c) continue;
        const int k = 3 - c - j;
        const int pj = (p >> j) & 1, pk = (p >> k) & 1;
        const int q = p ^ (1 << c) ^ (1 << j);
        if (pc == 1 && pj == 0) acc = fma(lam[pk], u[j][q], acc);
        if (pc == 0 && pj == 1) acc = fma(mu[pk], u[j][q], acc);
      }
      y[p] = acc;
    }
    iwht8s(y);
    sink(c, y);
  }
}

constexpr int FBW64 = 100;                                       // doubles per staged node row (>= 99 + 1)
constexpr int kFac64StageBytes = FPY * FBW64 * 8;
constexpr int kFac64StagePitch = (kFac64StageBytes + 127) & ~127;
constexpr size_t fac64_smem_bytes(int mode) {
  return (size_t)FNST * kFac64StagePitch * (mode == 1 ? 2 : 1) + sizeof(double) * 2 * FY * 6 * FX;
}

template <int MODE>
__global__ void __launch_bounds__(FX * FY, 2) k_mv64f(GridDims g, const __grid_constant__ HexOpD op,
                                                      const __grid_constant__ CUtensorMap tm_a,
                                                      const __grid_constant__ CUtensorMap tm_b,
                                                      double* __restrict__ pnew, double* __restrict__ y,
                                                      const double* __restrict__ E, const uint8_t* __restrict__ nf,
                                                      int projected, MixState* st, double* part, int zseg, int* err) {
  extern __shared__ __align__(128) unsigned char fac_smem[];
  double* yb = reinterpret_cast<double*>(fac_smem + (size_t)FNST * kFac64StagePitch * (MODE == 1 ? 2 : 1));
  __shared__ __align__(8) unsigned long long full[FNST];
  __shared__ double sh[32];
  if (MODE == 1 && st->status != MIX_RUNNING) return;
  const double beta = MODE == 1 ? st->beta : 0.0;
  const bool two = MODE == 1 && st->first == 0;
  const int l = threadIdx.x, w = threadIdx.y, tid = w * FX + l;
  const int i0 = blockIdx.x * FOX, j0 = blockIdx.y * FOY, k0 = blockIdx.z * zseg;
  const int k1 = min(k0 + zseg, g.nz1);
  const int xs = (3 * (i0 - 1)) & ~1;   // staged row start (doubles), 16-byte aligned, may be -4
  const int rem = 3 * (i0 - 1) - xs;    // 0 or 1
  const uint32_t tx_bytes = (uint32_t)kFac64StageBytes * (two ? 2u : 1u);
  auto stage_of = [&](int kk) { return (kk - k0 + 1) % FNST; };
  auto parity_of = [&](int kk) { return (uint32_t)(((kk - k0 + 1) / FNST) & 1); };
  auto plane_a = [&](int sl) { return reinterpret_cast<double*>(fac_smem + (size_t)sl * kFac64StagePitch); };
  auto plane_b = [&](int sl) { return reinterpret_cast<double*>(fac_smem + (size_t)(FNST + sl) * kFac64StagePitch); };
  auto issue = [&](int kk) {  // one thread
    const int sl = stage_of(kk);
    const uint32_t bar = smem_u32(&full[sl]);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx_bytes) : "memory");
    tma_load_plane(plane_a(sl), &tm_a, xs, j0 - 1, kk, bar);
    if (two) tma_load_plane(plane_b(sl), &tm_b, xs, j0 - 1, kk, bar);
  };
  if (tid == 0) {
    for (int q = 0; q < FNST; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int kk = k0 - 1; kk <= min(k0 - 2 + FNST, k1); ++kk) issue(kk);
  bool ok = true;
  auto wait_plane = [&](int kk) {
    if (!mbar_wait(smem_u32(&full[stage_of(kk)]), parity_of(kk))) ok = false;
  };
  auto gather4 = [&](int kk, double (&v)[4][3]) {
    const int sl = stage_of(kk);
    const double* a = plane_a(sl);
    const double* b = plane_b(sl);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int o = (w + (q >> 1)) * FBW64 + rem + 3 * (l + (q & 1));
#pragma unroll
      for (int c = 0; c < 3; ++c) v[q][c] = two ? fma(beta, b[o + c], a[o + c]) : a[o + c];
    }
  };
  const int ex = i0 - 1 + l, ey = j0 - 1 + w;
  const bool exy = ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny;
  const int64_t ebase = (int64_t)ex + (int64_t)g.nx * ey, eplane = (int64_t)g.nx * g.ny;
  auto eload = [&](int kk) -> double { return (exy && kk >= 0 && kk < g.nz) ? __ldg(E + ebase + eplane * kk) : 0.0; };
  const int nxo = i0 + l, nyo = j0 + w;
  const bool mine = l < FOX && w < FOY && nxo < g.nx1 && nyo < g.ny1;
  const int64_t nbase = nxo + (int64_t)g.nx1 * nyo;
  const int64_t fbase = (int64_t)g.rp64 * nyo + 3 * nxo;
  const int64_t fplane = (int64_t)g.rp64 * g.ny1;
  const int64_t nplane = (int64_t)g.nx1 * g.ny1;

  wait_plane(k0 - 1);
  wait_plane(k0);
  double ub[4][3];
  gather4(k0 - 1, ub);
  __syncthreads();  // the stage of plane k0 - 1 is refilled in the first step
  double carry[3] = {0.0, 0.0, 0.0};
  double pap = 0.0;
  double e0 = eload(k0 - 1), e1 = eload(k0);
  uint8_t f_next = (mine && projected && k0 < k1) ? nf[nbase + nplane * k0] : (uint8_t)0;
  for (int kk = k0 - 1; kk < k1; ++kk) {
    wait_plane(kk + 1);
    double ut[4][3];
    gather4(kk + 1, ut);
    if (tid == 0 && kk + FNST <= k1) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue(kk + FNST);
    }
    const double e_cur = e0;
    e0 = e1;
    e1 = eload(kk + 2);
    const bool outp = mine && kk >= k0;
    const uint8_t f = f_next;
    if (outp && projected && kk + 1 < k1) f_next = nf[nbase + nplane * (kk + 1)];
    if (MODE == 1 && mine && kk + 1 >= k0 && kk + 1 < k1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) pnew[fbase + fplane * (kk + 1) + c] = ut[3][c];
    }
    double u[3][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        u[c][b] = ub[b][c];
        u[c][b + 4] = ut[b][c];
      }
    double comb[2][2][3];  // [y][z][c]
    hex_apply64(op, e_cur, u, [&](int c, double (&yc)[8]) {
#pragma unroll
      for (int by = 0; by < 2; ++by)
#pragma unroll
        for (int bz = 0; bz < 2; ++bz) {
          const double nb = __shfl_down_sync(0xffffffffu, yc[2 * by + 4 * bz], 1);
          comb[by][bz][c] = yc[1 + 2 * by + 4 * bz] + nb;
        }
    });
    double* ybw = yb + ((kk & 1) * FY + w) * 6 * FX + l;
#pragma unroll
    for (int bz = 0; bz < 2; ++bz)
#pragma unroll
      for (int c = 0; c < 3; ++c) ybw[(3 * bz + c) * FX] = comb[0][bz][c];
    __syncthreads();
    if (mine) {
      const double* ybr = yb + ((kk & 1) * FY + w + 1) * 6 * FX + l;
      double top[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double bot = comb[1][0][c] + ybr[c * FX];
        top[c] = comb[1][1][c] + ybr[(3 + c) * FX];
        if (outp) {
          const double pv = ub[3][c];
          const double yo = (f >> c & 1) ? pv : carry[c] + bot;
          y[fbase + fplane * kk + c] = yo;
          if (MODE == 1) pap += pv * yo;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) carry[c] = top[c];
    }
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) ub[b][c] = ut[b][c];
  }
  if (!ok && err) atomicExch(err, 1);
  if (MODE == 1)
    mv32_finish(pap, sh, st, part, tid, err, gridDim.x * gridDim.y * gridDim.z,
                (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
}

// z-segment length of the FP64 factorised kernel: one element plane per step
static int fac64_zseg(const GridDims& g, int resident) {
  const int64_t txy = (int64_t)((g.nx1 + FOX - 1) / FOX) * ((g.ny1 + FOY - 1) / FOY);
  const int max_segs = std::max(1, g.nz1 / 4);
  int best_z = g.nz1;
  int64_t best_cost = INT64_MAX;
  for (int segs = 1; segs <= max_segs; ++segs) {
    const int zs = (g.nz1 + segs - 1) / segs;
    const int64_t n = txy * ((g.nz1 + zs - 1) / zs);
    const int64_t cost = ((n + resident - 1) / resident) * (zs + 1);
    if (cost < best_cost) {
      best_cost = cost;
      best_z = zs;
    }
  }
  return best_z;
}

// ---------------------------------------------------------------------------------------------------------
// FP32 K p on the 5th-generation tensor cores (tcgen05, kind::tf32, 3xTF32 for FP32-level products).
// A CTA takes a 16 x 8 tile of elements per element plane (one MMA row per element, M = 128) and owns the
// 15 x 7 nodes strictly inside it; CTAs overlap by one element in x and y. It marches over z: for element
// plane kk it
//   1. gathers each element's 24 DOF values from the two node planes in shared memory, splits them into
//      TF32 hi + lo and writes them into tensor memory (A operand, one TMEM lane per element),
//   2. one thread issues D = A_hi B_hi + A_lo B_hi + A_hi B_lo over the three K-steps (9 MMAs, M128 N32 K8,
//      B = KE^T hi/lo, K-major in shared memory, rows 24-31 zero) and commits them to an mbarrier,
//   3. reads D (24 outputs per element) back with tcgen05.ld, scales it by E_e and stages it in shared memory,
//   4. each owned node adds the bottom outputs of its 4 elements in this plane to the partial sum it carries
//      from the plane below (node plane kk is then complete and written) and starts node plane kk+1 with the
//      top outputs, always in the same order.
// MODE 1 fuses the inner PCG's p update and p.Ap partials exactly as k_mv32 does.
// ---------------------------------------------------------------------------------------------------------
constexpr int CX = 16, CY = 8;          // element tile (M = 128)
constexpr int OX = CX - 1, OY = CY - 1; // owned nodes per tile
constexpr int NX = CX + 1, NY = CY + 1; // node plane of the tile
constexpr int TC_THREADS = 128;
constexpr int TC_TMEM_COLS = 128;       // D: cols 0-31, A_hi: 32-55, A_lo: 64-87


__device__ __forceinline__ uint32_t to_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return r;
}

// K-major, no-swizzle shared-memory matrix descriptor: 8-row core matrices of 16 bytes per row, `lbo` bytes
// between the two 16-byte K halves of a K-step, `sbo` bytes between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;               // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor: D f32, A and B tf32, both K-major, N = 32, M = 128
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t desc_b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(desc_b), "r"(accumulate), "r"(kIdescTf32), "r"(0u));
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n"
               :
               : "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

template <int MODE>
__global__ void __launch_bounds__(TC_THREADS) k_mv32tc(GridDims g, const __grid_constant__ KeTf kt,
                                                      const float* __restrict__ xin, const float* __restrict__ z,
                                                      const float* __restrict__ pold, float* __restrict__ pnew,
                                                      float* __restrict__ y, const float* __restrict__ E,
                                                      const uint8_t* __restrict__ nf, int projected, MixState* st,
                                                      double* part, int zseg, int* err) {
  __shared__ __align__(128) float4 bsm[2][6][32];  // B hi/lo: [K chunk of 4][row n] (16 B per row), K-major
  __shared__ float4 xs[3][NY][NX];                // node planes (w unused)
  __shared__ float dsm[CX * CY][25];              // scaled MMA outputs per element
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ double sh[32];
  __shared__ int fail_sh;
  if (MODE == 1 && st->status != MIX_RUNNING) return;
  const float beta = MODE == 1 ? (float)st->beta : 0.0f;
  const bool first = MODE == 1 ? (st->first != 0) : true;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int ie0 = blockIdx.x * OX - 1, je0 = blockIdx.y * OY - 1;  // element tile origin
  const int k0 = blockIdx.z * zseg, k1 = min(k0 + zseg, g.nz1);
  const int64_t sy = g.nx1, sz = (int64_t)g.nx1 * g.ny1;

  // B operand: row n = output row, K = column of KE (canonical K-major layout, no swizzle)
  for (int q = tid; q < 2 * 6 * 32; q += TC_THREADS) {
    int h = q / (6 * 32), rem = q % (6 * 32), kc = rem / 32, n = rem % 32;
    const float* src = (h ? kt.lo : kt.hi) + n * 24 + 4 * kc;
    bsm[h][kc][n] = make_float4(src[0], src[1], src[2], src[3]);
  }
  if (tid == 0) {
    fail_sh = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&mbar)), "r"(1u) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(smem_u32(&tmem_base_sh)), "r"((uint32_t)TC_TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // B writes visible to the tensor core
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tbase = tmem_base_sh;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;  // this warp's TMEM lanes

  // node plane loader (z + beta p_{t-1} for MODE 1; owned interior nodes of owned planes write p_t)
  auto load_plane = [&](int kk) {
    const int slot = (kk + 3) % 3;
    const bool owned_plane = kk >= k0 && kk < k1;
    for (int q = tid; q < NY * NX * 3; q += TC_THREADS) {
      int c = q % 3, rest = q / 3, lx = rest % NX, ly = rest / NX;
      int i = ie0 + lx, j = je0 + ly;
      float v = 0.f;
      if (kk >= 0 && kk < g.nz1 && i >= 0 && i < g.nx1 && j >= 0 && j < g.ny1) {
        int64_t idx = pidx(g, i, j + (int64_t)g.ny1 * kk, c);
        if (MODE == 1) {
          v = first ? __ldg(z + idx) : fmaf(beta, __ldg(pold + idx), __ldg(z + idx));
          if (owned_plane && lx >= 1 && lx <= OX && ly >= 1 && ly <= OY) pnew[idx] = v;
        } else {
          v = __ldg(xin + idx);
        }
      }
      reinterpret_cast<float*>(&xs[slot][ly][lx])[c] = v;
    }
  };

  // element handled by this thread (one TMEM lane)
  const int ex = tid % CX, ey = tid / CX;
  const int ie = ie0 + ex, je = je0 + ey;
  const bool e_in = ie >= 0 && ie < g.nx && je >= 0 && je < g.ny;
  // owned node handled by this thread (tid < OX * OY)
  const bool owner = tid < OX * OY;
  const int na = 1 + (owner ? tid % OX : 0), nb = 1 + (owner ? tid / OX : 0);
  const int ni = ie0 + na, nj = je0 + nb;
  const bool n_in = owner && ni < g.nx1 && nj < g.ny1;
  float carry[3] = {0.f, 0.f, 0.f};  // top contributions of the plane below
  double pap = 0.0;
  uint32_t phase = 0;
  bool ok = true;

  load_plane(k0 - 1);
  for (int kk = k0 - 1; kk < k1; ++kk) {  // element plane kk couples node planes kk and kk+1
    load_plane(kk + 1);
    __syncthreads();
    // 1. A operand: element DOF values, TF32 hi/lo, into TMEM columns 32.. and 64..
    {
      float ee = 0.f;
      if (e_in && kk >= 0 && kk < g.nz) ee = __ldg(E + ie + (int64_t)g.nx * (je + (int64_t)g.ny * kk));
      uint32_t hi[24], lo[24];
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int bx = (b == 1 || b == 2 || b == 5 || b == 6) ? 1 : 0;
        const int by = (b == 2 || b == 3 || b == 6 || b == 7) ? 1 : 0;
        const int bz = b >= 4 ? 1 : 0;
        const float4 v4 = xs[(kk + bz + 3) % 3][ey + by][ex + bx];
        const float u[3] = {v4.x, v4.y, v4.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float uv = ee != 0.f ? u[c] : 0.f;
          const uint32_t h = to_tf32(uv);
          hi[3 * b + c] = h;
          lo[3 * b + c] = to_tf32(uv - __uint_as_float(h));
        }
      }
      dsm[tid][24] = ee;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        uint32_t vh[8], vl[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          vh[q] = hi[8 * s + q];
          vl[q] = lo[8 * s + q];
        }
        tmem_st8(tbase + lane_base + 32 + 8 * s, vh);
        tmem_st8(tbase + lane_base + 64 + 8 * s, vl);
      }
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    // 2. nine MMAs, one issuing thread, completion on the mbarrier
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t b0 = smem_u32(&bsm[0][0][0]), b1 = smem_u32(&bsm[1][0][0]);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const uint64_t dh = smem_desc(b0 + s * 1024, 512, 128);
        const uint64_t dl = smem_desc(b1 + s * 1024, 512, 128);
        mma_tf32_ts(tbase, tbase + 32 + 8 * s, dh, s > 0 ? 1u : 0u);
        mma_tf32_ts(tbase, tbase + 64 + 8 * s, dh, 1u);
        mma_tf32_ts(tbase, tbase + 32 + 8 * s, dl, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                   ::"r"(smem_u32(&mbar)) : "memory");
    }
    // 3. D back to registers, scaled by E_e, staged for the node gather
    if (!mbar_wait(smem_u32(&mbar), phase)) {
      ok = false;
      fail_sh = 1;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    {
      float d[32];
      tmem_ld32(tbase + lane_base, d);
      const float ee = dsm[tid][24];
#pragma unroll
      for (int r = 0; r < 24; ++r) dsm[tid][r] = d[r] * ee;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (fail_sh) break;
    // 4. owned nodes: bottom outputs finish node plane kk, top outputs start node plane kk+1
    if (owner) {
      float bot[3] = {0.f, 0.f, 0.f}, top[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int sy_ = 0; sy_ < 2; ++sy_)
#pragma unroll
        for (int sx_ = 0; sx_ < 2; ++sx_) {
          const int m = (nb - 1 + sy_) * CX + (na - 1 + sx_);  // element (na-1+sx, nb-1+sy)
          const int ox = 1 - sx_, oy = 1 - sy_;                 // this node's position in that element
          const int a2 = oy ? (ox ? 2 : 3) : (ox ? 1 : 0);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            bot[c] += dsm[m][3 * a2 + c];
            top[c] += dsm[m][3 * (a2 + 4) + c];
          }
        }
      if (kk >= k0 && n_in) {
        const int64_t n = ni + sy * nj + sz * kk;
        const uint8_t f = projected ? nf[n] : 0;
        const float4 pv4 = xs[(kk + 3) % 3][nb][na];
        const float pv[3] = {pv4.x, pv4.y, pv4.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float acc = carry[c] + bot[c];
          const float yv = (f & (1 << c)) ? pv[c] : acc;
          y[pidx(g, ni, nj + (int64_t)g.ny1 * kk, c)] = yv;
          if (MODE == 1) pap += (double)pv[c] * (double)yv;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) carry[c] = top[c];
    }
    __syncthreads();  // dsm and the node plane slot of kk-1 are reused by the next plane
  }
  // release tensor memory
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"((uint32_t)TC_TMEM_COLS)
                 : "memory");
  }
  if (!ok && tid == 0 && err) atomicExch(err, 1);
  if (MODE != 1) return;
  double bsum_v = bsum(pap, sh);
  const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  if (tid == 0) part[bid] = bsum_v;
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(&st->counter, 1u) == nblk - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (tid >= 32) return;
  double s = warp_sum_parts(part, nblk);
  if (tid != 0) return;
  st->counter = 0;
  st->first = 0;
  st->pap = s;
  if (fail_sh || (err && *(volatile int*)err)) {
    st->status = MIX_BREAKDOWN;
    return;
  }
  if (!(s > 0.0) || !isfinite(s)) {
    st->status = MIX_BREAKDOWN;
    return;
  }
  st->alpha = st->rho0 / s;
}

static int tc_zseg(const GridDims& g, int num_sms) {
  int64_t txy = (int64_t)((g.nx1 + OX - 1) / OX) * ((g.ny1 + OY - 1) / OY);
  int64_t segs = std::max<int64_t>(1, (8 * (int64_t)num_sms + txy - 1) / txy);
  return (int)std::max<int64_t>(2, (g.nz1 + segs - 1) / segs);
}

static dim3 tc_grid(const GridDims& g, int zseg) {
  return dim3((unsigned)((g.nx1 + OX - 1) / OX), (unsigned)((g.ny1 + OY - 1) / OY), (unsigned)((g.nz1 + zseg - 1) / zseg));
}

// 20 KB of unused dynamic shared memory keeps the tensor-core kernel at <= 4 CTAs per SM, so the CTAs on an
// SM never ask for more than its 512 TMEM columns (4 x 128).
constexpr int kTcPadSmem = 20 * 1024;

// TMA descriptor of a work vector: 3-D [nz1][ny1][pitch] elements (floats: pitch rp, box [1][FPY][FBW];
// doubles: pitch rp64, box [1][FPY][FBW64]), zero fill outside.
static PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  });
  return encode;
}

static int32_t encode_plane_map(mycel_problem* p, void* base, bool f64, CUtensorMap* out) {
  const PFN_cuTensorMapEncodeTiled encode = tensor_map_encoder();
  if (!encode) return set_error(p->ctx, MYCEL_E_DEVICE, "cuTensorMapEncodeTiled is not available from the driver");
  const GridDims& g = p->g;
  const cuuint64_t pitch = f64 ? (cuuint64_t)g.rp64 : (cuuint64_t)g.rp, es = f64 ? 8 : 4;
  cuuint64_t dims[3] = {pitch, (cuuint64_t)g.ny1, (cuuint64_t)g.nz1};
  cuuint64_t strides[2] = {pitch * es, pitch * g.ny1 * es};
  cuuint32_t box[3] = {(cuuint32_t)(f64 ? FBW64 : FBW), (cuuint32_t)FPY, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(out, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims,
                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(p->ctx, MYCEL_E_DEVICE, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return MYCEL_OK;
}

static const CUtensorMap* tmap_of(mycel_problem* p, const float* ptr) {
  const float* bufs[4] = {p->f_r, p->f_z, p->f_p0, p->f_p1};
  for (int q = 0; q < 4; ++q)
    if (ptr == bufs[q]) return &p->f_tmap[q];
  for (int q = 0; q < p->n_case_tmaps; ++q)
    if (ptr == p->case_tmap_ptr[q]) return p->case_tmap[q];
  return nullptr;
}

static const CUtensorMap* tmap64_of(mycel_problem* p, const double* ptr) {
  const double* bufs[4] = {p->g_r, p->g_z, p->g_p0, p->g_p1};
  for (int q = 0; q < 4; ++q)
    if (ptr == bufs[q]) return &p->g_tmap[q];
  return nullptr;
}

// FP64 factorised matvec launch (fast FP64 form); inputs are mapped FP64 work vectors
template <int MODE>
static void launch_mv64f(mycel_problem* p, cudaStream_t s, const double* xin, const double* z, const double* pold,
                         double* pnew, double* y, int projected, MixState* st, double* part) {
  const GridDims& g = p->g;
  static int occ = 0;
  if (!occ) {
    int o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_mv64f<1>, FX * FY, fac64_smem_bytes(1));
    occ = std::max(1, o);
  }
  const int zs = fac64_zseg(g, occ * p->ctx->num_sms);
  const CUtensorMap* ta = tmap64_of(p, MODE == 1 ? z : xin);
  const CUtensorMap* tb = MODE == 1 ? tmap64_of(p, pold) : ta;
  if (!ta || !tb) {  // internal invariant: inputs are always one of the four mapped work vectors
    std::fprintf(stderr, "mycel: FP64 matvec input is not a mapped work vector\n");
    std::abort();
  }
  const dim3 grid((unsigned)((g.nx1 + FOX - 1) / FOX), (unsigned)((g.ny1 + FOY - 1) / FOY),
                  (unsigned)((g.nz1 + zs - 1) / zs));
  k_mv64f<MODE><<<grid, dim3(FX, FY), fac64_smem_bytes(MODE), s>>>(g, p->hexop64, *ta, *tb, pnew, y, p->d_E,
                                                                     p->d_nflags, projected, st, part, zs, p->d_err);
}

// resident CTAs per SM of the factorised FP32 matvec (same for both modes: same block, registers within bounds);
// it sets the z-segments of a launch, so every launch of a grid (alone or packed) has the same CTA decomposition
static int mv32f_resident_per_sm() {
  static std::once_flag once;
  static int occ = 1;
  std::call_once(once, [] {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_mv32f<1>, FX * FY, fac_smem_bytes(1)) != cudaSuccess) {
      cudaGetLastError();
      o = 1;
    }
    occ = std::max(1, o);
  });
  return occ;
}

// FP32 matvec launch, variant chosen per problem (MYCEL_MV32_*)
template <int MODE>
static void launch_mv32_variant(mycel_problem* p, cudaStream_t s, const float* xin, const float* z, const float* pold,
                                float* pnew, float* y, int projected, MixState* st, double* part) {
  const GridDims& g = p->g;
  if (p->mv32 == MYCEL_MV32_TENSOR) {
    int zs = tc_zseg(g, p->ctx->num_sms);
    k_mv32tc<MODE><<<tc_grid(g, zs), TC_THREADS, kTcPadSmem, s>>>(g, p->ketf, xin, z, pold, pnew, y, p->d_Ef,
                                                                  p->d_nflags, projected, st, part, zs, p->d_err);
  } else if (p->mv32 == MYCEL_MV32_DENSE) {
    int zs = tile_zseg(g, p->ctx->num_sms);
    k_mv32<MODE><<<tile_grid(g, zs), dim3(TX, TY), 0, s>>>(g, p->kef, xin, z, pold, pnew, y, p->d_Ef, p->d_nflags,
                                                           projected, st, part, zs);
  } else {
    int zs = fac_zseg(g, mv32f_resident_per_sm() * p->ctx->num_sms);
    const CUtensorMap* ta = tmap_of(p, MODE == 1 ? z : xin);
    const CUtensorMap* tb = MODE == 1 ? tmap_of(p, pold) : ta;
    if (!ta || !tb) {  // internal invariant: inputs are always one of the four mapped work vectors
      std::fprintf(stderr, "mycel: FP32 matvec input is not a mapped work vector\n");
      std::abort();
    }
    k_mv32f<MODE><<<fac_grid(g, zs), dim3(FX, FY), fac_smem_bytes(MODE), s>>>(
        g, p->hexop, *ta, *tb, pnew, y, p->d_Ef, p->d_nflags, projected, st, part, zs, p->d_err);
  }
}

// Autotuner: on first use, time every variant (K x on the problem's FP32 buffers, after one warm-up launch)
// and keep the factorised one unless another takes under 3/4 of its time; a tensor-core run that reports a
// failed wait is never chosen.
// Variant choices are shared by every problem of the process with the same grid, so a problem's arithmetic
// does not depend on what else was running when it was first timed (first measurement wins).
static std::mutex g_mv32_mu;
static std::map<std::tuple<int, int, int>, int> g_mv32_choice;

static int32_t resolve_mv32(mycel_problem* p) {
  if (p->mv32 > 0) return MYCEL_OK;
  const auto key = std::make_tuple(p->g.nx, p->g.ny, p->g.nz);
  {
    std::lock_guard<std::mutex> lk(g_mv32_mu);
    auto it = g_mv32_choice.find(key);
    if (it != g_mv32_choice.end()) {
      p->mv32 = it->second;
      return MYCEL_OK;
    }
  }
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  MYCEL_CUDA(c, cudaMemsetAsync(p->f_r, 0, sizeof(float) * p->g.n32, s));
  MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int variants[3] = {MYCEL_MV32_FACTORED, MYCEL_MV32_DENSE, MYCEL_MV32_TENSOR};
  float t[3] = {0.f, 0.f, 0.f};
  int herr = 0;
  for (int v = 0; v < 3; ++v) {
    p->mv32 = variants[v];
    (void)cudaGetLastError();
    launch_mv32_variant<0>(p, s, p->f_r, nullptr, nullptr, nullptr, p->f_ap, 1, nullptr, nullptr);
    const cudaError_t le = cudaGetLastError();
    const bool launched = le == cudaSuccess;  // a variant that cannot launch here is skipped, with a warning
    if (!launched)
      std::fprintf(stderr, "mycel: FP32 matvec variant %d not launchable: %s\n", variants[v], cudaGetErrorString(le));
    cudaEventRecord(e0, s);
    for (int r = 0; r < 3; ++r)
      launch_mv32_variant<0>(p, s, p->f_r, nullptr, nullptr, nullptr, p->f_ap, 1, nullptr, nullptr);
    cudaEventRecord(e1, s);
    c->launches += 4;
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      p->mv32 = -1;
      return set_error(c, MYCEL_E_DEVICE, std::string("matvec autotune: ") + cudaGetErrorString(e));
    }
    cudaEventElapsedTime(&t[v], e0, e1);
    if (!launched) t[v] = 1e30f;
    int* herr_p = (int*)((char*)c->pinned + 8192);
    MYCEL_CUDA(c, cudaMemcpyAsync(herr_p, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    herr = *herr_p;
    if (herr) {  // a bounded wait gave up: never choose this variant
      t[v] = 1e30f;
      MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the factorised operator (variants[0]) unless another is clearly faster: timings taken while other work
  // shares the GPU (several jobs at once) scatter by more than the variants differ on small grids
  constexpr float kTuneMargin = 0.75f;
  int best = 0;
  for (int v = 1; v < 3; ++v)
    if (t[v] < kTuneMargin * t[0] && t[v] < t[best]) best = v;
  p->mv32 = variants[best];
  {
    std::lock_guard<std::mutex> lk(g_mv32_mu);
    p->mv32 = g_mv32_choice.emplace(key, p->mv32).first->second;  // another thread may have stored one first
  }
  if (std::getenv("MYCEL_VERBOSE"))
    std::fprintf(stderr, "mycel: FP32 matvec autotune (ms per 3 launches) factored %.4f dense %.4f tensor %.4f -> %d\n",
                 t[0], t[1], t[2], p->mv32);
  return MYCEL_OK;
}

// End of a vector step: CTA sums of r.r and r.z, fixed-order sums by the last CTA, and the inner PCG's scalar
// logic (recursive residual, replacement and stop triggers, beta).
__device__ __forceinline__ void xr_tail(double rr, double rz, MixState* st, double* part, int mode, double* sh) {
  double brr = bsum(rr, sh);
  double brz = bsum(rz, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = brr;
    part[gridDim.x + blockIdx.x] = brz;
  }
  if (!elect_last32(&st->counter)) return;
  if (threadIdx.x >= 32) return;
  double srr = warp_sum_parts(part, gridDim.x);
  double srz = warp_sum_parts(part + gridDim.x, gridDim.x);
  if (threadIdx.x != 0) return;
  st->counter = 0;
  const double rn = sqrt(srr);
  st->rn = rn;
  if (mode == 2) {  // start of a solve
    st->rho0 = srz;
    st->first = 1;
    st->status = (rn <= st->target) ? MIX_FLUSH : MIX_RUNNING;
    st->flush_at = rn * st->flush_factor;
    return;
  }
  if (mode == 1) {  // true residual replaced the recursive one: keep the direction
    if (st->first || !(st->rho0 > 0.0)) {
      st->first = 1;
    } else {
      double beta = srz / st->rho0;
      if (!isfinite(beta) || beta < 0.0) st->first = 1;
      else st->beta = beta;
    }
    st->rho0 = srz;
    st->flush_at = rn * st->flush_factor;
    st->status = MIX_RUNNING;
    return;
  }
  st->iter += 1;
  if (rn <= st->target || rn <= st->flush_at) {
    st->status = MIX_FLUSH;  // rho0 stays rho_k for the beta after the replacement
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

// FP64 vectors of the fast FP64 form (padded layout, n even): the same step as k_xr32
__global__ void __launch_bounds__(kT) k_xr64(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                             double* __restrict__ z, const double* __restrict__ p,
                                             const double* __restrict__ ap, const double* __restrict__ invd,
                                             MixState* st, double* part, int mode) {
  __shared__ double sh[32];
  if (mode == 0 && st->status != MIX_RUNNING) return;
  const double alpha = mode ? 0.0 : st->alpha;
  double rr = 0.0, rz = 0.0;
  const int64_t n2 = n >> 1;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += stride) {
    double2 rv = reinterpret_cast<const double2*>(r)[i];
    const double2 iv = reinterpret_cast<const double2*>(invd)[i];
    if (mode == 0) {
      double2 xv = reinterpret_cast<const double2*>(x)[i];
      const double2 pv = reinterpret_cast<const double2*>(p)[i];
      const double2 av = reinterpret_cast<const double2*>(ap)[i];
      xv.x = fma(alpha, pv.x, xv.x);
      xv.y = fma(alpha, pv.y, xv.y);
      rv.x = fma(-alpha, av.x, rv.x);
      rv.y = fma(-alpha, av.y, rv.y);
      reinterpret_cast<double2*>(x)[i] = xv;
      reinterpret_cast<double2*>(r)[i] = rv;
    }
    const double2 zv = make_double2(rv.x * iv.x, rv.y * iv.y);
    reinterpret_cast<double2*>(z)[i] = zv;
    rr += rv.x * rv.x + rv.y * rv.y;
    rz += rv.x * zv.x + rv.y * zv.y;
  }
  xr_tail(rr, rz, st, part, mode, sh);
}

// x += alpha p, r -= alpha Ap, z = r invD; partials of r.r and r.z (FP64). mode 0: CG step; 1: residual
// replacement (z, rho from the new r; beta = rho_new / rho_old); 2: start (z, rho; next step starts p = z).
__global__ void __launch_bounds__(kT) k_xr32(int64_t n, float* __restrict__ x, float* __restrict__ r,
                                             float* __restrict__ z, const float* __restrict__ p,
                                             const float* __restrict__ ap, const float* __restrict__ invd,
                                             MixState* st, double* part, int mode) {
  __shared__ double sh[32];
  if (mode == 0 && st->status != MIX_RUNNING) return;
  const float alpha = mode ? 0.f : (float)st->alpha;
  double rr = 0.0, rz = 0.0;
  const int64_t n4 = n >> 2;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
    float4 rv = reinterpret_cast<const float4*>(r)[i];
    float4 iv = reinterpret_cast<const float4*>(invd)[i];
    if (mode == 0) {
      float4 xv = reinterpret_cast<const float4*>(x)[i];
      float4 pv = reinterpret_cast<const float4*>(p)[i];
      float4 av = reinterpret_cast<const float4*>(ap)[i];
      xv.x = fmaf(alpha, pv.x, xv.x); xv.y = fmaf(alpha, pv.y, xv.y);
      xv.z = fmaf(alpha, pv.z, xv.z); xv.w = fmaf(alpha, pv.w, xv.w);
      rv.x = fmaf(-alpha, av.x, rv.x); rv.y = fmaf(-alpha, av.y, rv.y);
      rv.z = fmaf(-alpha, av.z, rv.z); rv.w = fmaf(-alpha, av.w, rv.w);
      reinterpret_cast<float4*>(x)[i] = xv;
      reinterpret_cast<float4*>(r)[i] = rv;
    }
    float4 zv = make_float4(rv.x * iv.x, rv.y * iv.y, rv.z * iv.z, rv.w * iv.w);
    reinterpret_cast<float4*>(z)[i] = zv;
    rr += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
    rz += (double)rv.x * zv.x + (double)rv.y * zv.y + (double)rv.z * zv.z + (double)rv.w * zv.w;
  }
  if (blockIdx.x == 0) {  // tail (n not a multiple of 4)
    for (int64_t i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) {
      float rv = r[i];
      if (mode == 0) {
        x[i] = fmaf(alpha, p[i], x[i]);
        rv = fmaf(-alpha, ap[i], rv);
        r[i] = rv;
      }
      float zv = rv * invd[i];
      z[i] = zv;
      rr += (double)rv * rv;
      rz += (double)rv * zv;
    }
  }
  xr_tail(rr, rz, st, part, mode, sh);
}

// Conversions between box-ordered FP64 DOF vectors and the padded FP32 / FP64 layouts walk node rows: row
// q = j + ny1 k holds DOFs [3 nx1 q, 3 nx1 (q + 1)) in the box layout and [pitch q, pitch q + 3 nx1) in the
// padded one (pitch rp for float, rp64 for double). CTA b takes rows b, b + gridDim.x, ...; its threads the
// DOFs of a row.
template <class T>
__device__ __forceinline__ int64_t pad_pitch(const GridDims& g) {
  return sizeof(T) == 4 ? (int64_t)g.rp : (int64_t)g.rp64;
}

// refinement: u += x, x = 0
template <class T>
__global__ void k_flush_u(GridDims g, double* __restrict__ u, T* __restrict__ xw) {
  const int rl = 3 * g.nx1;
  for (int64_t q = blockIdx.x; q < (int64_t)g.ny1 * g.nz1; q += gridDim.x)
    for (int t = threadIdx.x; t < rl; t += blockDim.x) {
      const int64_t f = pad_pitch<T>(g) * q + t;
      u[(int64_t)rl * q + t] += (double)xw[f];
      xw[f] = (T)0;
    }
}

// after A u (padded FP64 layout, factorised FP64 operator): r64 = P(b - A u), r_work = (T) r64, CTA partials of
// r64^2; zero_au clears A u after reading
template <class T>
__global__ void k_resid64p(GridDims g, const uint8_t* __restrict__ nf, const double* __restrict__ b,
                           double* __restrict__ au, T* __restrict__ rw, double* part, int zero_au) {
  __shared__ double sh[32];
  double s = 0.0;
  const int rl = 3 * g.nx1;
  for (int64_t q = blockIdx.x; q < (int64_t)g.ny1 * g.nz1; q += gridDim.x)
    for (int t = threadIdx.x; t < rl; t += blockDim.x) {
      const int64_t i = (int64_t)rl * q + t, a = (int64_t)g.rp64 * q + t;
      const bool con = nf[i / 3] & (1 << (t % 3));
      const double v = con ? 0.0 : (b[i] - au[a]);
      if (zero_au) au[a] = 0.0;
      rw[pad_pitch<T>(g) * q + t] = (T)v;
      s += v * v;
    }
  double bs = bsum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
}

__global__ void k_sum_part(const double* part, int nb, double* out) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  double s = warp_sum_parts(part, (unsigned)nb);
  if (threadIdx.x == 0) *out = s;
}

template <class T>
__global__ void k_to_pad(GridDims g, const double* __restrict__ a, T* __restrict__ b) {
  const int rl = 3 * g.nx1;
  for (int64_t q = blockIdx.x; q < (int64_t)g.ny1 * g.nz1; q += gridDim.x)
    for (int t = threadIdx.x; t < rl; t += blockDim.x) b[pad_pitch<T>(g) * q + t] = (T)a[(int64_t)rl * q + t];
}
template <class T>
__global__ void k_from_pad(GridDims g, const T* __restrict__ a, double* __restrict__ b) {
  const int rl = 3 * g.nx1;
  for (int64_t q = blockIdx.x; q < (int64_t)g.ny1 * g.nz1; q += gridDim.x)
    for (int t = threadIdx.x; t < rl; t += blockDim.x) b[(int64_t)rl * q + t] = (double)a[pad_pitch<T>(g) * q + t];
}

// ---------------------------------------------------------------------------------------------------------
// Geometric multigrid preconditioner (MYCEL_PRECISION_FP64_MG): flexible CG in FP64 on the factorised FP64
// operator, preconditioned by one FP32 V-cycle per iteration.
// Levels: each level halves the element counts of the one above, rounding up (vertex-centred: even fine nodes
// coincide with coarse nodes, odd ones lie midway; with an odd count the last fine element alone forms the last
// coarse element), down to a coarsest level of at most kMgCoarseMax DOFs. Coarse operators are Galerkin
// products built element by element: a coarse element's 24 x 24 matrix is the sum over its (up to 8) fine
// sub-elements s of W_s^T T_s W_s, where T_s is the finer level's element matrix (E_e KE on the voxel grid,
// with the rows and columns of constrained DOFs zeroed) and W_s the trilinear interpolation from the coarse
// element's 8 nodes to the sub-element's 8 nodes. Each coarse level is then stored assembled, as a 27-point
// node stencil of 3 x 3 blocks. Everything is rebuilt from the current E at the start of a solve, unless E is
// unchanged since the last build (the load cases of one stiffness share it).
// Smoothing: damped Jacobi, the same sweeps before and after the coarse correction, so the V-cycle is a
// symmetric operator; the coarsest level is solved by a dense inverse (FP64 Gauss-Jordan in shared memory).
// Outer iteration (FCG with one-term orthogonalisation): alpha = (z, r) / (p, A p) as in PCG, and
// beta = -alpha (z_new, A p) / (z, r), which equals PCG's beta for a fixed SPD preconditioner and stays
// correct when FP32 rounding makes the V-cycle vary slightly from one application to the next.
// Element matrices use the voxel operator's local node order (0,0,0),(1,0,0),(1,1,0),(0,1,0), then the same at
// z = 1, DOF 3 a + c, like KE.
// ---------------------------------------------------------------------------------------------------------
constexpr int kMgMaxLevels = 12;
constexpr int kMgCoarseMax = 144;  // DOFs of the coarsest level (its dense FP64 inverse fits in shared memory)
// Damping of the Jacobi sweeps, per level: omega = kMgOmegaScale / lambda, lambda the largest eigenvalue of
// D^-1 A estimated by power iterations at each set-up (from below, hence the margin to 2: a 25 % low estimate
// still damps every mode). Measured on the bridge: 4/3 -> 47.7, 1.5 -> 49.1, 1.65 -> 50.5 SIMP iter/s.
constexpr float kMgOmegaScale = 1.5f;
constexpr int kMgPowerIters = 8;
// Later set-ups of the same problem start from the previous set-up's eigenvector estimate (the design changes
// little from one solve to the next) and take kMgPowerItersWarm iterations.
constexpr int kMgPowerItersWarm = 3;
constexpr size_t kMgCoarseSmem = (size_t)kMgCoarseMax * kMgCoarseMax * 8 + kMgCoarseMax * 8;

struct MgDims {
  int nx, ny, nz;  // elements per axis (nodes: one more)
};

// Load cases kept apart are advanced together: the coarse-level kernels of one V-cycle take the vectors of up
// to kMgMaxCases cases (the cases share K, so each stencil entry is loaded once per node for all of them).
// Threads are numbered with the case fastest, so the lanes of a node read the same stencil words. Case c's
// vector of a level is p[c]; a single solve is the case set {1 case}.
constexpr int kMgMaxCases = 8;
struct MgPtrs {
  float* p[kMgMaxCases];
};
// (item, case) from a thread number with the case fastest; one case: the number itself (no division). The
// kernels are instantiated for one case (MULTI false: the single solve's code, compile-time case 0) and for
// several.
template <bool MULTI>
__device__ __forceinline__ void mg_item_case(int64_t t, int ncase, int64_t* item, int* c) {
  if (!MULTI || ncase == 1) {
    *item = t;
    *c = 0;
  } else {
    const uint32_t q = (uint32_t)t / (uint32_t)ncase;  // items x cases < 2^32 on every level
    *item = q;
    *c = (int)((uint32_t)t - q * (uint32_t)ncase);
  }
}
__host__ __device__ __forceinline__ MgPtrs mg_one(float* v) {
  MgPtrs r{};
  r.p[0] = v;
  return r;
}

__host__ __device__ __forceinline__ int64_t mg_nn(const MgDims& d) {
  return (int64_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
}
// row stride of a level's stencil array: the node count rounded up to 4 floats, so every row starts on a
// 16-byte boundary (TMA rows); the padding entries stay 0
__host__ __device__ __forceinline__ int64_t mg_ns(const MgDims& d) { return (mg_nn(d) + 3) & ~int64_t(3); }

// coordinates (i, j, k) of entry n of an a x b x . box (nodes or elements) by 32-bit division: every level's
// node count is far below 2^32 (a grid that large would not fit in device memory)
__device__ __forceinline__ void mg_ijk(int64_t n, int a, int b, int* i, int* j, int* k) {
  const uint32_t u = (uint32_t)n, q = u / (uint32_t)a, r = q / (uint32_t)b;
  *i = (int)(u - q * (uint32_t)a);
  *j = (int)(q - r * (uint32_t)b);
  *k = (int)r;
}

// per-axis interpolation weight of coarse node c at fine node f, for a fine axis of n elements
__device__ __forceinline__ float mg_pw(int f, int c, int n) {
  if (!(f & 1)) return c == (f >> 1) ? 1.0f : 0.0f;
  if (f == n) return c == ((n + 1) >> 1) ? 1.0f : 0.0f;  // last node of an odd count
  return (c == (f >> 1) || c == (f >> 1) + 1) ? 0.5f : 0.0f;
}

// local node index from its offsets inside the element, and back
__device__ __forceinline__ int mg_lidx(int bx, int by, int bz) { return 4 * bz + (by ? (bx ? 2 : 3) : bx); }
__device__ __forceinline__ int mg_bx(int a) { return (a ^ (a >> 1)) & 1; }
__device__ __forceinline__ int mg_by(int a) { return (a >> 1) & 1; }
__device__ __forceinline__ int mg_bz(int a) { return a >> 2; }

__device__ __forceinline__ bool mg_running(const MixState* st) { return !st || st->status == MIX_RUNNING; }

// Galerkin element matrices of a coarse level, one CTA per coarse element. FROM_FINE: the finer level is the
// voxel grid (T = E_e KE, masked by the node flags); otherwise its element matrices Kf.
template <bool FROM_FINE>
__global__ void __launch_bounds__(64) k_mg_build(MgDims c, MgDims f, const __grid_constant__ KeF ke,
                                                 const float* __restrict__ Ef, const uint8_t* __restrict__ nf,
                                                 const float* __restrict__ Kf, float* __restrict__ Kc,
                                                 const uint8_t* __restrict__ only) {
  __shared__ float T[576], U[576], W[64];
  __shared__ uint8_t fr[24];
  const int64_t e = blockIdx.x;
  if (only && !only[e]) return;  // done by k_mg_build1
  int ex, ey, ez;
  mg_ijk(e, c.nx, c.ny, &ex, &ey, &ez);
  const int tid = threadIdx.x;
  float acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.f;
  for (int s = 0; s < 8; ++s) {
    const int fx = 2 * ex + (s & 1), fy = 2 * ey + ((s >> 1) & 1), fz = 2 * ez + (s >> 2);
    if (fx >= f.nx || fy >= f.ny || fz >= f.nz) continue;  // uniform over the CTA
    const int64_t fe = fx + (int64_t)f.nx * (fy + (int64_t)f.ny * fz);
    float ee = 1.0f;
    if (FROM_FINE) {
      ee = Ef[fe];
      if (ee == 0.0f) continue;  // inactive element
    }
    {  // W[a][C]: weight of coarse local node C at the sub-element's local node a
      const int a = tid >> 3, C = tid & 7;
      W[tid] = mg_pw(fx + mg_bx(a), ex + mg_bx(C), f.nx) * mg_pw(fy + mg_by(a), ey + mg_by(C), f.ny) *
               mg_pw(fz + mg_bz(a), ez + mg_bz(C), f.nz);
    }
    if (FROM_FINE && tid < 24) {
      const int a = tid / 3, cc = tid % 3;
      const int64_t n = (fx + mg_bx(a)) + (int64_t)(f.nx + 1) * ((fy + mg_by(a)) + (int64_t)(f.ny + 1) * (fz + mg_bz(a)));
      fr[tid] = !(nf[n] & (1 << cc));
    }
    __syncthreads();
    for (int o = tid; o < 576; o += 64) {
      if (FROM_FINE) {
        const int row = o / 24, col = o % 24;
        T[o] = (fr[row] && fr[col]) ? ee * ke.v[o] : 0.0f;
      } else {
        T[o] = Kf[fe * 576 + o];
      }
    }
    __syncthreads();
    // U[(a,c),(C',c')] = sum_b T[(a,c),(b,c')] W[b][C']
    for (int o = tid; o < 576; o += 64) {
      const int row = o / 24, Cp = (o % 24) / 3, cp = o % 3;
      float u = 0.f;
#pragma unroll
      for (int b = 0; b < 8; ++b) u = fmaf(T[row * 24 + 3 * b + cp], W[b * 8 + Cp], u);
      U[o] = u;
    }
    __syncthreads();
    // Kc[(C,c),(C',c')] += sum_a W[a][C] U[(a,c),(C',c')]
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const int o = tid + 64 * k;
      const int C = o / 72, cc = (o / 24) % 3, col = o % 24;
      float v = 0.f;
#pragma unroll
      for (int a = 0; a < 8; ++a) v = fmaf(W[a * 8 + C], U[(3 * a + cc) * 24 + col], v);
      acc[k] += v;
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) Kc[e * 576 + tid + 64 * k] = acc[k];
}

// Level-1 element matrices from the voxel grid, fast path: when all 8 sub-elements of a coarse element exist and
// none of its 27 fine nodes has a constrained DOF, K_c = sum_s E_s G_s with G_s = W_s^T KE W_s (precomputed,
// [8][576]). Other coarse elements (an odd last layer, supports) are marked for k_mg_build<true>. Four coarse
// elements per CTA, 64 threads each.
__global__ void __launch_bounds__(256) k_mg_build1(MgDims c, MgDims f, const float* __restrict__ G,
                                                   const float* __restrict__ Ef, const uint8_t* __restrict__ nf,
                                                   float* __restrict__ Kc, uint8_t* __restrict__ special) {
  __shared__ float Gs[8 * 576];
  __shared__ float Es[4][8];
  __shared__ int sp[4];
  for (int o = threadIdx.x; o < 8 * 576; o += blockDim.x) Gs[o] = G[o];
  const int grp = threadIdx.x >> 6, lt = threadIdx.x & 63;
  const int64_t ne = (int64_t)c.nx * c.ny * c.nz;
  for (int64_t base = (int64_t)blockIdx.x * 4; base < ne; base += (int64_t)gridDim.x * 4) {
    const int64_t e = base + grp;
    const bool valid = e < ne;
    if (lt == 0) sp[grp] = 0;
    __syncthreads();
    if (valid) {
      int ex, ey, ez;
      mg_ijk(e, c.nx, c.ny, &ex, &ey, &ez);
      if (lt < 8) {
        const int fx = 2 * ex + (lt & 1), fy = 2 * ey + ((lt >> 1) & 1), fz = 2 * ez + (lt >> 2);
        if (fx < f.nx && fy < f.ny && fz < f.nz) Es[grp][lt] = Ef[fx + (int64_t)f.nx * (fy + (int64_t)f.ny * fz)];
        else sp[grp] = 1;
      } else if (lt >= 32 && lt < 59) {
        const int q = lt - 32;
        const int i = 2 * ex + q % 3, j = 2 * ey + (q / 3) % 3, k = 2 * ez + q / 9;
        if (i <= f.nx && j <= f.ny && k <= f.nz) {
          const uint8_t fl = nf[i + (int64_t)(f.nx + 1) * (j + (int64_t)(f.ny + 1) * k)];
          if ((fl & (NF_CX | NF_CY | NF_CZ)) && (fl & NF_ACTIVE)) sp[grp] = 1;
        } else {
          sp[grp] = 1;
        }
      }
    }
    __syncthreads();
    if (valid && !sp[grp]) {
      float es[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) es[q] = Es[grp][q];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int o = lt + 64 * k;
        float v = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) v = fmaf(es[q], Gs[q * 576 + o], v);
        Kc[e * 576 + o] = v;
      }
    }
    if (valid && lt == 0) special[e] = (uint8_t)sp[grp];
    __syncthreads();
  }
}

// Assembled 27-point stencil of a level from its element matrices, in symmetric half storage: node n keeps the
// blocks of its neighbours nb = 13 .. 26 (itself and the 13 neighbours later in node order), nb = (dx+1) +
// 3 (dy+1) + 9 (dz+1); S[((nb - 13) * 9 + 3 ci + cj) * ns + n] is the entry (DOF ci of node n, DOF cj of
// neighbour nb). The block of an earlier neighbour m is the transpose of m's block for offset 26 - nb. Also
// 1/diag (0 where the diagonal is 0: DOFs no free fine DOF reaches).
constexpr int kMgHalf = 14;  // stored blocks per node
__global__ void __launch_bounds__(256) k_mg_stencil(MgDims d, const float* __restrict__ K, float* __restrict__ S,
                                                    float* __restrict__ invd) {
  // a thread per (node, row ci): it reads row 3a + ci of each of the node's (up to 8) elements once (24
  // contiguous floats) and adds the entries that belong to the node's own 14 blocks; the elements are taken in
  // ascending index, so every block entry is the same ordered sum as an element-by-element assembly
  const int64_t nn = mg_nn(d);
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= 3 * nn) return;
  const int ci = (int)(t / nn);
  const int64_t n = t - ci * nn;
  const int nx1 = d.nx + 1, ny1 = d.ny + 1;
  int i, j, k;
  mg_ijk(n, nx1, ny1, &i, &j, &k);
  float acc[kMgHalf][3];
#pragma unroll
  for (int h = 0; h < kMgHalf; ++h) acc[h][0] = acc[h][1] = acc[h][2] = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) {  // element (i - ox, j - oy, k - oz), ascending element index
    const int ox = 1 - (q & 1), oy = 1 - ((q >> 1) & 1), oz = 1 - (q >> 2);
    const int ex = i - ox, ey = j - oy, ez = k - oz;
    const bool have = ex >= 0 && ey >= 0 && ez >= 0 && ex < d.nx && ey < d.ny && ez < d.nz;
    const int a = mg_lidx(ox, oy, oz);
    const float* row =
        K + (have ? (ex + (int64_t)d.nx * (ey + (int64_t)d.ny * ez)) * 576 + (3 * a + ci) * 24 : 0);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int dx = mg_bx(b) - ox, dy = mg_by(b) - oy, dz = mg_bz(b) - oz;
      const int nb = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
      if (nb < 13) continue;  // stored (transposed) at the earlier neighbour
#pragma unroll
      for (int cj = 0; cj < 3; ++cj)
        if (have) acc[nb - 13][cj] += row[3 * b + cj];
    }
  }
#pragma unroll
  for (int h = 0; h < kMgHalf; ++h)
#pragma unroll
    for (int cj = 0; cj < 3; ++cj) S[((int64_t)h * 9 + 3 * ci + cj) * mg_ns(d) + n] = acc[h][cj];
  const float dg = ci == 0 ? acc[0][0] : (ci == 1 ? acc[0][1] : acc[0][2]);  // keeps acc in registers
  invd[3 * n + ci] = dg > 0.f ? 1.0f / dg : 0.0f;
}

// Kernels over nodes of the levels below the voxel grid run a thread per DOF: CTAs of 3 x 64 threads, warps
// 0-1 take component 0 of 64 consecutive nodes, warps 2-3 component 1, warps 4-5 component 2 (coalesced loads,
// three times the threads in flight of a thread per node).
constexpr int kMgDofThreads = 192;
constexpr int64_t kMgDofMaxNodes = 65536;  // levels (x cases) up to this many nodes: a thread per DOF
__device__ __forceinline__ int64_t mg_dof_node() { return blockIdx.x * (int64_t)64 + (threadIdx.x & 63); }
__device__ __forceinline__ int mg_dof_comp() { return threadIdx.x >> 6; }
static inline unsigned mg_dof_blocks(int64_t nn) { return (unsigned)((nn + 63) / 64); }

// coarse-level product at node n by gather (ns: the stencil's row stride). mode 0: y = A x; 1: y = x + omega
// invd (r - A x) (one Jacobi sweep); 2: y = r - A x on DOFs with a nonzero diagonal, 0 elsewhere
__device__ __forceinline__ void mg_apply_node(const MgDims& d, int64_t ns, int64_t n, const float* __restrict__ S,
                                              const float* __restrict__ x, const float* __restrict__ r,
                                              const float* __restrict__ invd, float* __restrict__ y, int mode,
                                              float omega) {
  const int nx1 = d.nx + 1, ny1 = d.ny + 1;
  int i, j, k;
  mg_ijk(n, nx1, ny1, &i, &j, &k);
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  // all 27 blocks without branches: a neighbour outside the grid is read at a clamped (valid) node with x
  // taken as 0. Later neighbours' blocks are n's own (row ci at entries 3 ci + cj), earlier ones the transposed
  // blocks stored at the neighbour (row ci at entries 3 cj + ci).
#pragma unroll
  for (int nb = 0; nb < 27; ++nb) {
    const int ui = i + nb % 3 - 1, uj = j + (nb / 3) % 3 - 1, uk = k + nb / 9 - 1;
    const int mi = min(max(ui, 0), d.nx), mj = min(max(uj, 0), d.ny), mk = min(max(uk, 0), d.nz);
    const bool in = mi == ui && mj == uj && mk == uk;
    const int64_t m = mi + (int64_t)nx1 * (mj + (int64_t)ny1 * mk);
    const float x0 = in ? x[3 * m] : 0.f, x1 = in ? x[3 * m + 1] : 0.f, x2 = in ? x[3 * m + 2] : 0.f;
    if (nb >= 13) {
      const float* s = S + (int64_t)(nb - 13) * 9 * ns + n;
      a0 = fmaf(s[0], x0, fmaf(s[ns], x1, fmaf(s[2 * ns], x2, a0)));
      a1 = fmaf(s[3 * ns], x0, fmaf(s[4 * ns], x1, fmaf(s[5 * ns], x2, a1)));
      a2 = fmaf(s[6 * ns], x0, fmaf(s[7 * ns], x1, fmaf(s[8 * ns], x2, a2)));
    } else {
      const float* s = S + (int64_t)(13 - nb) * 9 * ns + m;
      a0 = fmaf(s[0], x0, fmaf(s[3 * ns], x1, fmaf(s[6 * ns], x2, a0)));
      a1 = fmaf(s[ns], x0, fmaf(s[4 * ns], x1, fmaf(s[7 * ns], x2, a1)));
      a2 = fmaf(s[2 * ns], x0, fmaf(s[5 * ns], x1, fmaf(s[8 * ns], x2, a2)));
    }
  }
  const float acc[3] = {a0, a1, a2};
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    const int64_t q = 3 * n + cc;
    if (mode == 0) y[q] = acc[cc];
    else if (mode == 1) y[q] = fmaf(omega * invd[q], r[q] - acc[cc], x[q]);
    else y[q] = invd[q] != 0.0f ? r[q] - acc[cc] : 0.0f;
  }
}

// the same for one row (DOF ci of node n): a third of the loads of a node
__device__ __forceinline__ void mg_apply_row(const MgDims& d, int64_t ns, int64_t n, int ci,
                                             const float* __restrict__ S, const float* __restrict__ x,
                                             const float* __restrict__ r, const float* __restrict__ invd,
                                             float* __restrict__ y, int mode, float omega) {
  const int nx1 = d.nx + 1, ny1 = d.ny + 1;
  int i, j, k;
  mg_ijk(n, nx1, ny1, &i, &j, &k);
  float a = 0.f;
#pragma unroll
  for (int nb = 0; nb < 27; ++nb) {
    const int ui = i + nb % 3 - 1, uj = j + (nb / 3) % 3 - 1, uk = k + nb / 9 - 1;
    const int mi = min(max(ui, 0), d.nx), mj = min(max(uj, 0), d.ny), mk = min(max(uk, 0), d.nz);
    const bool in = mi == ui && mj == uj && mk == uk;
    const int64_t m = mi + (int64_t)nx1 * (mj + (int64_t)ny1 * mk);
    const float x0 = in ? x[3 * m] : 0.f, x1 = in ? x[3 * m + 1] : 0.f, x2 = in ? x[3 * m + 2] : 0.f;
    if (nb >= 13) {
      const float* s = S + ((int64_t)(nb - 13) * 9 + 3 * ci) * ns + n;
      a = fmaf(s[0], x0, fmaf(s[ns], x1, fmaf(s[2 * ns], x2, a)));
    } else {
      const float* s = S + ((int64_t)(13 - nb) * 9 + ci) * ns + m;
      a = fmaf(s[0], x0, fmaf(s[3 * ns], x1, fmaf(s[6 * ns], x2, a)));
    }
  }
  const int64_t q = 3 * n + ci;
  if (mode == 0) y[q] = a;
  else if (mode == 1) y[q] = fmaf(omega * invd[q], r[q] - a, x[q]);
  else y[q] = invd[q] != 0.0f ? r[q] - a : 0.0f;
}

// coarse-level product kernels: a thread per node (large levels: the three rows share their x loads) or a
// thread per DOF (smaller levels: three times the threads in flight); mg_apply_kernel picks by size
// (st: the cases' states, one per case, or null; a case whose state is not running is skipped)
template <bool MULTI>
__global__ void __launch_bounds__(256) k_mg_apply_nodes(MgDims d, const float* __restrict__ S,
                                                        const __grid_constant__ MgPtrs x,
                                                        const __grid_constant__ MgPtrs r,
                                                        const float* __restrict__ invd,
                                                        const __grid_constant__ MgPtrs y, int mode,
                                                        const float* __restrict__ om, const MixState* st, int ncase) {
  const int64_t nn = mg_nn(d);
  int64_t n;
  int c;
  mg_item_case<MULTI>(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, ncase, &n, &c);
  if (n >= nn || !mg_running(st ? st + c : nullptr)) return;
  mg_apply_node(d, mg_ns(d), n, S, x.p[c], r.p[c], invd, y.p[c], mode, mode == 1 ? *om : 0.0f);
}

template <bool MULTI>
__global__ void __launch_bounds__(kMgDofThreads) k_mg_apply(MgDims d, const float* __restrict__ S,
                                                            const __grid_constant__ MgPtrs x,
                                                            const __grid_constant__ MgPtrs r,
                                                            const float* __restrict__ invd,
                                                            const __grid_constant__ MgPtrs y, int mode,
                                                            const float* __restrict__ om, const MixState* st,
                                                            int ncase) {
  const int64_t nn = mg_nn(d);
  int64_t n;  // (node, case) pair, the case fastest
  int c;
  mg_item_case<MULTI>(mg_dof_node(), ncase, &n, &c);
  if (n >= nn || !mg_running(st ? st + c : nullptr)) return;
  mg_apply_row(d, mg_ns(d), n, mg_dof_comp(), S, x.p[c], r.p[c], invd, y.p[c], mode, mode == 1 ? *om : 0.0f);
}

// Coarse-level product of a large level (one case) with the stencil streamed into shared memory by TMA: the
// thread-per-node gather above holds at most a few of its 243 stencil loads in flight and waits on them (load
// latency, not bandwidth, bounds it). Here a CTA takes kS1Nodes consecutive nodes and brings, neighbour by
// neighbour in the gather's order, the 9 stencil rows every thread needs for that neighbour as one 2-D box of
// [9 rows][kS1Box nodes]: the nodes' own rows (nb >= 13), or the transposed rows the earlier neighbour stores
// (nb < 13: the CTA's nodes shifted by the neighbour's offset; the box starts at that node rounded down to 16
// bytes and each thread reads at its remainder). kS1Stages boxes are in flight; a group of kS1Group neighbours
// is released by one CTA barrier. Each product is the same fmaf chain in the same order as mg_apply_node, so
// the results are bit-identical to it: where the neighbour lies outside the grid, x is 0 and the staged value
// (another node's entry, the zero padding or TMA's zero fill) is finite, so its products are signed zeros,
// which leave an accumulator unchanged unless it is -0 (it starts at +0 and reaches -0 only when a partial sum
// underflows to zero from below; then only the sign of that zero could differ from the gather's).
constexpr int kS1Nodes = 252;   // nodes per CTA (+ up to 3 of rounding <= kS1Box)
constexpr int kS1Box = 256;     // staged nodes per row
constexpr int kS1Stages = 6;
constexpr int kS1Group = 3;
constexpr int kS1StageBytes = 9 * kS1Box * 4;
constexpr int kS1Smem = kS1Stages * kS1StageBytes;
static_assert(kS1Stages % kS1Group == 0 && 27 % kS1Group == 0, "stage groups");
static_assert(kS1Nodes % 4 == 0 && kS1Nodes + 3 < kS1Box, "TMA boxes: 16-byte aligned starts cover the CTA");

__global__ void __launch_bounds__(256) k_mg_apply_nodes_tma(MgDims d, const __grid_constant__ CUtensorMap tm,
                                                            const float* __restrict__ x, const float* __restrict__ r,
                                                            const float* __restrict__ invd, float* __restrict__ y,
                                                            int mode, const float* __restrict__ om,
                                                            const MixState* st, int* err) {
  extern __shared__ __align__(128) unsigned char s1_smem[];
  __shared__ __align__(8) unsigned long long full[kS1Stages];
  if (!mg_running(st)) return;  // one case: the same for every CTA
  const int64_t nn = mg_nn(d);
  const int tid = threadIdx.x;
  const int64_t n0 = (int64_t)blockIdx.x * kS1Nodes, n = n0 + tid;
  const int nx1 = d.nx + 1, ny1 = d.ny + 1;
  const int64_t sxy = (int64_t)nx1 * ny1;
  // node whose entries thread 0 uses in block nb
  auto first = [&](int nb) -> int64_t {
    return nb >= 13 ? n0 : n0 + (nb % 3 - 1) + (int64_t)nx1 * ((nb / 3) % 3 - 1) + sxy * (nb / 9 - 1);
  };
  auto issue = [&](int nb) {  // one thread
    const int sl = nb % kS1Stages;
    const uint32_t bar = smem_u32(&full[sl]);
    const int xs = (int)(first(nb) & ~int64_t(3));  // 16-byte aligned start (may be negative: zero fill)
    const int row = nb >= 13 ? (nb - 13) * 9 : (13 - nb) * 9;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"((uint32_t)kS1StageBytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(smem_u32(s1_smem + (size_t)sl * kS1StageBytes)), "l"(reinterpret_cast<uint64_t>(&tm)), "r"(xs), "r"(row),
        "r"(bar)
        : "memory");
  };
  if (tid == 0) {
    for (int q = 0; q < kS1Stages; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  bool ok = true;
  if (tid == 0)
    for (int nb = 0; nb < kS1Stages; ++nb) issue(nb);
  const bool act = tid < kS1Nodes && n < nn;
  const int ts = tid < kS1Nodes ? tid : 0;  // staged column read (threads past kS1Nodes read column 0..3)
  const int64_t nc = act ? n : 0;
  int i, j, k;
  mg_ijk(nc, nx1, ny1, &i, &j, &k);
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
  for (int g = 0; g < 27 / kS1Group; ++g) {
#pragma unroll
    for (int q = 0; q < kS1Group; ++q) {
      const int nb = kS1Group * g + q;
      const int sl = nb % kS1Stages;
      if (!mbar_wait(smem_u32(&full[sl]), (uint32_t)((nb / kS1Stages) & 1))) ok = false;
      const int ui = i + nb % 3 - 1, uj = j + (nb / 3) % 3 - 1, uk = k + nb / 9 - 1;
      const int mi = min(max(ui, 0), d.nx), mj = min(max(uj, 0), d.ny), mk = min(max(uk, 0), d.nz);
      const bool in = act && mi == ui && mj == uj && mk == uk;
      const int64_t m = mi + (int64_t)nx1 * (mj + (int64_t)ny1 * mk);
      const float x0 = in ? x[3 * m] : 0.f, x1 = in ? x[3 * m + 1] : 0.f, x2 = in ? x[3 * m + 2] : 0.f;
      const float* s = reinterpret_cast<const float*>(s1_smem + (size_t)sl * kS1StageBytes) + ts +
                       (int)(first(nb) & 3);
      if (nb >= 13) {
        a0 = fmaf(s[0], x0, fmaf(s[kS1Box], x1, fmaf(s[2 * kS1Box], x2, a0)));
        a1 = fmaf(s[3 * kS1Box], x0, fmaf(s[4 * kS1Box], x1, fmaf(s[5 * kS1Box], x2, a1)));
        a2 = fmaf(s[6 * kS1Box], x0, fmaf(s[7 * kS1Box], x1, fmaf(s[8 * kS1Box], x2, a2)));
      } else {
        a0 = fmaf(s[0], x0, fmaf(s[3 * kS1Box], x1, fmaf(s[6 * kS1Box], x2, a0)));
        a1 = fmaf(s[kS1Box], x0, fmaf(s[4 * kS1Box], x1, fmaf(s[7 * kS1Box], x2, a1)));
        a2 = fmaf(s[2 * kS1Box], x0, fmaf(s[5 * kS1Box], x1, fmaf(s[8 * kS1Box], x2, a2)));
      }
    }
    if (kS1Group * (g + 1) + kS1Stages - kS1Group < 27) {  // a later group reuses these stages
      __syncthreads();
      // a wait that gave up leaves its copy possibly in flight: issue nothing more into the stages
      if (tid == 0 && ok) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
#pragma unroll
        for (int q = 0; q < kS1Group; ++q) {
          const int nb = kS1Group * g + kS1Stages + q;
          if (nb < 27) issue(nb);
        }
      }
    }
  }
  if (!ok && err) atomicExch(err, 1);
  if (!act) return;
  const float acc[3] = {a0, a1, a2};
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    const int64_t q = 3 * n + cc;
    if (mode == 0) y[q] = acc[cc];
    else if (mode == 1) y[q] = fmaf(*om * invd[q], r[q] - acc[cc], x[q]);
    else y[q] = invd[q] != 0.0f ? r[q] - acc[cc] : 0.0f;
  }
}

// a further sweep on the voxel grid (padded FP32 layout, t = A x): x += omega invd (r - t)
__global__ void k_mg_jacobi_fine(int64_t n, const float* __restrict__ r, const float* __restrict__ t,
                                 const float* __restrict__ invd, float* __restrict__ x, const float* __restrict__ om,
                                 const MixState* st) {
  if (!mg_running(st)) return;
  const float omega = *om;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    x[q] = fmaf(omega * invd[q], r[q] - t[q], x[q]);
}

// restriction r_c = W^T res of a level's residual, component cc at coarse node n. PAD: the voxel grid in the
// padded FP32 layout (row pitch pitch), res = r - t; otherwise box layout, res = t. Coarse DOFs with a zero
// diagonal get 0.
template <bool PAD>
__device__ __forceinline__ void mg_restrict_comp(const MgDims& f, int pitch, const float* __restrict__ rf,
                                                 const float* __restrict__ tf, const MgDims& c,
                                                 const float* __restrict__ invdc, float* __restrict__ rc, int64_t n,
                                                 int cc, float* __restrict__ xc, float omega) {
  const int cx1 = c.nx + 1, cy1 = c.ny + 1;
  int I, J, K;
  mg_ijk(n, cx1, cy1, &I, &J, &K);
  const int pi = min(2 * I, f.nx), pj = min(2 * J, f.ny), pk = min(2 * K, f.nz);
  float a = 0.f;
  // the 27 candidate fine nodes around the coarse node's position, without branches: a candidate outside the
  // grid gets weight 0 and a clamped (valid) read
#pragma unroll
  for (int dk = -1; dk <= 1; ++dk) {
    const int k0 = pk + dk, k = min(max(k0, 0), f.nz);
    const float wz = (k0 == k) ? mg_pw(k, K, f.nz) : 0.f;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int j0 = pj + dj, j = min(max(j0, 0), f.ny);
      const float wy = (j0 == j) ? wz * mg_pw(j, J, f.ny) : 0.f;
#pragma unroll
      for (int di = -1; di <= 1; ++di) {
        const int i0 = pi + di, i = min(max(i0, 0), f.nx);
        const float w = (i0 == i) ? wy * mg_pw(i, I, f.nx) : 0.f;
        const int64_t row = j + (int64_t)(f.ny + 1) * k;
        const int64_t b = (PAD ? (int64_t)pitch * row + 3 * i : 3 * (i + (int64_t)(f.nx + 1) * row)) + cc;
        a = fmaf(w, PAD ? rf[b] - tf[b] : tf[b], a);
      }
    }
  }
  const float d = invdc[3 * n + cc], rv = d != 0.f ? a : 0.f;
  rc[3 * n + cc] = rv;
  if (xc) xc[3 * n + cc] = omega * d * rv;  // the coarse level's first Jacobi sweep from x = 0
}


// prolongation x_f += W x_c, component cc at fine node n, on the finer level's free DOFs. PAD: the voxel grid
// (padded FP32 layout, free = node flag bit clear); otherwise box layout, free = nonzero diagonal.
template <bool PAD>
__device__ __forceinline__ void mg_prolong_comp(const MgDims& f, int pitch, const uint8_t* __restrict__ nf,
                                                const float* __restrict__ invdf, float* __restrict__ xf,
                                                const MgDims& c, const float* __restrict__ xc, int64_t n, int cc) {
  const int fx1 = f.nx + 1, fy1 = f.ny + 1;
  int i, j, k;
  mg_ijk(n, fx1, fy1, &i, &j, &k);
  // per axis: two coarse nodes with their weights (the second with weight 0 unless the fine node lies midway)
  int ci[2], cj[2], ck[2];
  float wi[2], wj[2], wk[2];
  auto axis = [](int f_, int n_, int nc_, int* c_, float* ww) {
    const bool mid = (f_ & 1) && f_ != n_;
    c_[0] = ((f_ & 1) && f_ == n_) ? nc_ : (f_ >> 1);
    c_[1] = min(c_[0] + 1, nc_);
    ww[0] = mid ? 0.5f : 1.0f;
    ww[1] = mid ? 0.5f : 0.0f;
  };
  axis(i, f.nx, c.nx, ci, wi);
  axis(j, f.ny, c.ny, cj, wj);
  axis(k, f.nz, c.nz, ck, wk);
  const int cx1 = c.nx + 1, cy1 = c.ny + 1;
  float a = 0.f;
#pragma unroll
  for (int qz = 0; qz < 2; ++qz)
#pragma unroll
    for (int qy = 0; qy < 2; ++qy)
#pragma unroll
      for (int qx = 0; qx < 2; ++qx) {
        const int64_t m = ci[qx] + (int64_t)cx1 * (cj[qy] + (int64_t)cy1 * ck[qz]);
        a = fmaf(wi[qx] * wj[qy] * wk[qz], xc[3 * m + cc], a);
      }
  const bool fr = PAD ? !(nf[n] & (1 << cc)) : (invdf[3 * n + cc] != 0.0f);
  if (fr) xf[(PAD ? (int64_t)pitch * (j + (int64_t)fy1 * k) + 3 * i : 3 * n) + cc] += a;
}

// the same transfers for all three components of a node in one pass (the per-level kernels):
// restriction r_c = W^T res of a level's residual at coarse node n. PAD: the voxel grid in the padded FP32
// layout (row pitch pitch), res = r - t; otherwise box layout, res = t. Coarse DOFs with a zero diagonal get 0.
template <bool PAD>
__device__ __forceinline__ void mg_restrict_node(const MgDims& f, int pitch, const float* __restrict__ rf,
                                                 const float* __restrict__ tf, const MgDims& c,
                                                 const float* __restrict__ invdc, float* __restrict__ rc, int64_t n,
                                                 float* __restrict__ xc, float omega) {
  const int cx1 = c.nx + 1, cy1 = c.ny + 1;
  int I, J, K;
  mg_ijk(n, cx1, cy1, &I, &J, &K);
  const int pi = min(2 * I, f.nx), pj = min(2 * J, f.ny), pk = min(2 * K, f.nz);
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  // the 27 candidate fine nodes around the coarse node's position, without branches: a candidate outside the
  // grid gets weight 0 and a clamped (valid) read
#pragma unroll
  for (int dk = -1; dk <= 1; ++dk) {
    const int k0 = pk + dk, k = min(max(k0, 0), f.nz);
    const float wz = (k0 == k) ? mg_pw(k, K, f.nz) : 0.f;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int j0 = pj + dj, j = min(max(j0, 0), f.ny);
      const float wy = (j0 == j) ? wz * mg_pw(j, J, f.ny) : 0.f;
#pragma unroll
      for (int di = -1; di <= 1; ++di) {
        const int i0 = pi + di, i = min(max(i0, 0), f.nx);
        const float w = (i0 == i) ? wy * mg_pw(i, I, f.nx) : 0.f;
        const int64_t row = j + (int64_t)(f.ny + 1) * k;
        const int64_t b = PAD ? (int64_t)pitch * row + 3 * i : 3 * (i + (int64_t)(f.nx + 1) * row);
        if (PAD) {
          a0 = fmaf(w, rf[b] - tf[b], a0);
          a1 = fmaf(w, rf[b + 1] - tf[b + 1], a1);
          a2 = fmaf(w, rf[b + 2] - tf[b + 2], a2);
        } else {
          a0 = fmaf(w, tf[b], a0);
          a1 = fmaf(w, tf[b + 1], a1);
          a2 = fmaf(w, tf[b + 2], a2);
        }
      }
    }
  }
  const float d0 = invdc[3 * n], d1 = invdc[3 * n + 1], d2 = invdc[3 * n + 2];
  const float r0 = d0 != 0.f ? a0 : 0.f, r1 = d1 != 0.f ? a1 : 0.f, r2 = d2 != 0.f ? a2 : 0.f;
  rc[3 * n] = r0;
  rc[3 * n + 1] = r1;
  rc[3 * n + 2] = r2;
  if (xc) {  // the coarse level's first Jacobi sweep from x = 0: x = omega invd r
    xc[3 * n] = omega * d0 * r0;
    xc[3 * n + 1] = omega * d1 * r1;
    xc[3 * n + 2] = omega * d2 * r2;
  }
}

template <bool PAD, bool MULTI>
__global__ void k_mg_restrict(MgDims f, int pitch, const __grid_constant__ MgPtrs rf, const __grid_constant__ MgPtrs tf,
                              MgDims c, const float* __restrict__ invdc, const __grid_constant__ MgPtrs rc,
                              const MixState* st, const __grid_constant__ MgPtrs xc, int first_sweep,
                              const float* __restrict__ om, int ncase) {
  int64_t n;
  int k;
  mg_item_case<MULTI>(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, ncase, &n, &k);
  if (n >= mg_nn(c) || !mg_running(st ? st + k : nullptr)) return;
  const float omega = first_sweep ? *om : 0.f;
  mg_restrict_node<PAD>(f, pitch, rf.p[k], tf.p[k], c, invdc, rc.p[k], n, first_sweep ? xc.p[k] : nullptr, omega);
}

// prolongation x_f += W x_c at fine node n, on the finer level's free DOFs. PAD: the voxel grid (padded FP32
// layout, free = node flag bit clear); otherwise box layout, free = nonzero diagonal.
template <bool PAD>
__device__ __forceinline__ void mg_prolong_node(const MgDims& f, int pitch, const uint8_t* __restrict__ nf,
                                                const float* __restrict__ invdf, float* __restrict__ xf,
                                                const MgDims& c, const float* __restrict__ xc, int64_t n) {
  const int fx1 = f.nx + 1, fy1 = f.ny + 1;
  int i, j, k;
  mg_ijk(n, fx1, fy1, &i, &j, &k);
  // per axis: two coarse nodes with their weights (the second with weight 0 unless the fine node lies midway)
  int ci[2], cj[2], ck[2];
  float wi[2], wj[2], wk[2];
  auto axis = [](int f_, int n_, int nc_, int* cc, float* ww) {
    const bool mid = (f_ & 1) && f_ != n_;
    cc[0] = ((f_ & 1) && f_ == n_) ? nc_ : (f_ >> 1);
    cc[1] = min(cc[0] + 1, nc_);
    ww[0] = mid ? 0.5f : 1.0f;
    ww[1] = mid ? 0.5f : 0.0f;
  };
  axis(i, f.nx, c.nx, ci, wi);
  axis(j, f.ny, c.ny, cj, wj);
  axis(k, f.nz, c.nz, ck, wk);
  const int cx1 = c.nx + 1, cy1 = c.ny + 1;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
  for (int qz = 0; qz < 2; ++qz)
#pragma unroll
    for (int qy = 0; qy < 2; ++qy)
#pragma unroll
      for (int qx = 0; qx < 2; ++qx) {
        const float w = wi[qx] * wj[qy] * wk[qz];
        const int64_t m = ci[qx] + (int64_t)cx1 * (cj[qy] + (int64_t)cy1 * ck[qz]);
        a0 = fmaf(w, xc[3 * m], a0);
        a1 = fmaf(w, xc[3 * m + 1], a1);
        a2 = fmaf(w, xc[3 * m + 2], a2);
      }
  const float acc[3] = {a0, a1, a2};
  const int64_t b = PAD ? (int64_t)pitch * (j + (int64_t)fy1 * k) + 3 * i : 3 * n;
#pragma unroll
  for (int cc = 0; cc < 3; ++cc) {
    const bool fr = PAD ? !(nf[n] & (1 << cc)) : (invdf[3 * n + cc] != 0.0f);
    if (fr) xf[b + cc] += acc[cc];
  }
}

template <bool PAD, bool MULTI>
__global__ void k_mg_prolong(MgDims f, int pitch, const uint8_t* __restrict__ nf, const float* __restrict__ invdf,
                             const __grid_constant__ MgPtrs xf, MgDims c, const __grid_constant__ MgPtrs xc,
                             const MixState* st, int ncase) {
  int64_t n;
  int k;
  mg_item_case<MULTI>(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, ncase, &n, &k);
  if (n >= mg_nn(f) || !mg_running(st ? st + k : nullptr)) return;
  mg_prolong_node<PAD>(f, pitch, nf, invdf, xf.p[k], c, xc.p[k], n);
}


// coarsest level set-up (one CTA): the dense matrix from the level's stencil, inverted in place by Gauss-Jordan
// elimination without pivoting (SPD) in FP64 shared memory. A pivot that has lost all but 1e-12 of its
// original diagonal (round-off on a nearly singular block) drops its DOF: row and column become 0, as do those
// of DOFs whose diagonal is 0.
__global__ void __launch_bounds__(1024) k_mg_coarse_setup(MgDims d, const float* __restrict__ S,
                                                          double* __restrict__ ainv) {
  extern __shared__ __align__(16) unsigned char mg_smem[];
  const int64_t nn = mg_nn(d), ns = mg_ns(d);
  const int n = (int)(3 * nn);
  double* A = reinterpret_cast<double*>(mg_smem);
  double* dg = A + (size_t)n * n;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nx1 = d.nx + 1, ny1 = d.ny + 1;
  for (int o = tid; o < n * n; o += nt) {
    const int row = o / n, col = o % n;
    const int a = row / 3, ci = row % 3, b = col / 3, cj = col % 3;
    const int dx = b % nx1 - a % nx1, dy = (b / nx1) % ny1 - (a / nx1) % ny1, dz = b / (nx1 * ny1) - a / (nx1 * ny1);
    double v = 0.0;
    if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) {
      const int nb = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
      v = nb >= 13 ? (double)S[((nb - 13) * 9 + 3 * ci + cj) * ns + a] : (double)S[((13 - nb) * 9 + 3 * cj + ci) * ns + b];
    }
    A[o] = v;
  }
  __syncthreads();
  for (int q = tid; q < n; q += nt) {
    dg[q] = A[q * n + q];
    if (!(dg[q] > 0.0)) {  // no free DOF behind it: an identity row for the elimination, zeroed at the end
      dg[q] = 0.0;
      for (int o = 0; o < n; ++o) A[q * n + o] = 0.0;
    }
  }
  __syncthreads();
  for (int q = tid; q < n; q += nt)
    if (dg[q] == 0.0) {
      for (int o = 0; o < n; ++o) A[o * n + q] = 0.0;
      A[q * n + q] = 1.0;
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double piv = A[k * n + k];
    const bool keep = piv > 0.0 && (dg[k] == 0.0 || piv > 1e-12 * dg[k]);
    __syncthreads();
    if (!keep) {
      for (int o = tid; o < n; o += nt) {
        A[k * n + o] = 0.0;
        A[o * n + k] = 0.0;
      }
      __syncthreads();
      continue;
    }
    const double ip = 1.0 / piv;
    for (int i = tid >> 5; i < n; i += nt >> 5) {  // 32 x 32 thread tile: rows by warp, columns by lane
      if (i == k) continue;
      const double f = A[i * n + k] * ip;
      for (int j = tid & 31; j < n; j += 32)
        if (j != k) A[i * n + j] = fma(-f, A[k * n + j], A[i * n + j]);
    }
    __syncthreads();
    for (int o = tid; o < n; o += nt) {
      if (o != k) {
        A[k * n + o] *= ip;
        A[o * n + k] = -A[o * n + k] * ip;
      }
    }
    if (tid == 0) A[k * n + k] = ip;
    __syncthreads();
  }
  for (int o = tid; o < n * n; o += nt) {
    const int i = o / n, j = o % n;
    ainv[o] = (dg[i] == 0.0 || dg[j] == 0.0) ? 0.0 : A[o];
  }
}

// The coarse levels from T down to the coarsest and back in one launch of one thread-block cluster: levels
// this small cost more in separate launches than in work. The cluster's CTAs are co-scheduled, so a cluster
// barrier separates the phases; all vectors stay in global memory (L2).
constexpr int kMgTailCtas = 8, kMgTailThreads = 512;
// levels of at most this many nodes go to the cluster kernel (on the bridge: 12x6x6 and below). Measured on
// the bridge: 2 nodes per cluster thread (8,192, from 24x12x12 down) 45.2 SIMP iter/s, 2,048 47.7, 256 47.2.
constexpr int64_t kMgTailMaxNodes = 2048;

struct MgTailLevel {
  MgDims d;
  int64_t nn;
  const float* S;
  const float* invd;
  float *xa, *xb, *r, *t;  // case 0's vectors; case k's at + k * 3 nn
};
struct MgTail {
  int T, L, sweeps, nc;
  const double* ainv;
  MgTailLevel lv[kMgMaxLevels];
};

// phase barrier of the tail kernel: the cluster's barrier, or the CTA's when it runs as one CTA
__device__ __forceinline__ void mg_cluster_sync(bool one_cta) {
  if (one_cta) {
    __syncthreads();
    return;
  }
  asm volatile("barrier.cluster.arrive.release;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory");
}

// Levels T .. L-1 of the V-cycle for ncase load cases: from r of level T (restricted by the caller) to the
// smoothed correction of level T, left in its xa. Work items are numbered with the case fastest; a case whose
// state is not running is skipped, and the kernel returns at once (every thread alike) when none is.
// Body for the threads gt (of gs) of the cluster (or the single CTA when one_cta) that runs this V-cycle's tail.
template <bool MULTI>
__device__ __forceinline__ void mg_tail_body(const MgTail& tl, const float* __restrict__ om, const MixState* st,
                                             int ncase, int64_t gt, int64_t gs, bool one_cta) {
  bool any = false;
  for (int k = 0; k < ncase; ++k) any = any || mg_running(st ? st + k : nullptr);
  if (!any) return;
  auto live = [&](int k) { return mg_running(st ? st + k : nullptr); };
  float* xc[kMgMaxLevels];
  // a thread per (row, case) where the level's rows fit the cluster's threads, else a thread per (node, case)
  auto apply = [&](const MgTailLevel& v, const float* x, float* y, int mode, float w) {
    const int64_t nd = 3 * v.nn;
    if (3 * v.nn * ncase <= gs) {
      for (int64_t t = gt; t < nd * ncase; t += gs) {
        int64_t it;
        int k;
        mg_item_case<MULTI>(t, ncase, &it, &k);
        if (live(k))
          mg_apply_row(v.d, mg_ns(v.d), it / 3, (int)(it % 3), v.S, x + k * nd, v.r + k * nd, v.invd, y + k * nd,
                       mode, w);
      }
    } else {
      for (int64_t t = gt; t < v.nn * ncase; t += gs) {
        int64_t n;
        int k;
        mg_item_case<MULTI>(t, ncase, &n, &k);
        if (live(k)) mg_apply_node(v.d, mg_ns(v.d), n, v.S, x + k * nd, v.r + k * nd, v.invd, y + k * nd, mode, w);
      }
    }
  };
  for (int l = tl.T; l < tl.L - 1; ++l) {
    const MgTailLevel& v = tl.lv[l];
    const MgTailLevel& cv = tl.lv[l + 1];
    const int64_t nd = 3 * v.nn, cnd = 3 * cv.nn;
    const float w = om[l];
    float *x = v.xa, *o = v.xb;  // x = omega invd r, written with r by the restriction into this level
    for (int k = 1; k < tl.sweeps; ++k) {
      apply(v, x, o, 1, w);
      mg_cluster_sync(one_cta);
      float* tmp = x;
      x = o;
      o = tmp;
    }
    apply(v, x, v.t, 2, 0.0f);
    mg_cluster_sync(one_cta);
    const bool smoothed = l + 1 < tl.L - 1;  // the coarsest level is solved, not smoothed
    const float wc = smoothed ? om[l + 1] : 0.0f;
    for (int64_t q = gt; q < cnd * ncase; q += gs) {
      int64_t it;
      int k;
      mg_item_case<MULTI>(q, ncase, &it, &k);
      if (live(k))
        mg_restrict_comp<false>(v.d, 0, nullptr, v.t + k * nd, cv.d, cv.invd, cv.r + k * cnd, it / 3, (int)(it % 3),
                                smoothed ? cv.xa + k * cnd : nullptr, wc);
    }
    mg_cluster_sync(one_cta);
    xc[l] = x;
  }
  {  // coarsest level: x = A^-1 r, one warp per (row, case)
    const MgTailLevel& v = tl.lv[tl.L - 1];
    const int64_t nd = 3 * v.nn;
    const int lane = threadIdx.x & 31;
    for (int64_t rc = gt >> 5; rc < (int64_t)tl.nc * ncase; rc += gs >> 5) {
      int64_t row;
      int k;
      mg_item_case<MULTI>(rc, ncase, &row, &k);
      if (!live(k)) continue;
      const float* r = v.r + k * nd;
      double acc = 0.0;
      for (int col = lane; col < tl.nc; col += 32) acc = fma(tl.ainv[row * tl.nc + col], (double)r[col], acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) v.xa[k * nd + row] = (float)acc;
    }
    mg_cluster_sync(one_cta);
    xc[tl.L - 1] = v.xa;
  }
  for (int l = tl.L - 2; l >= tl.T; --l) {
    const MgTailLevel& v = tl.lv[l];
    const int64_t nd = 3 * v.nn, cnd = 3 * tl.lv[l + 1].nn;
    const float w = om[l];
    float* x = xc[l];
    float* o = x == v.xa ? v.xb : v.xa;
    for (int64_t q = gt; q < nd * ncase; q += gs) {
      int64_t it;
      int k;
      mg_item_case<MULTI>(q, ncase, &it, &k);
      if (live(k))
        mg_prolong_comp<false>(v.d, 0, nullptr, v.invd, x + k * nd, tl.lv[l + 1].d, xc[l + 1] + k * cnd, it / 3,
                               (int)(it % 3));
    }
    mg_cluster_sync(one_cta);
    for (int k = 0; k < tl.sweeps; ++k) {
      apply(v, x, o, 1, w);
      mg_cluster_sync(one_cta);
      float* tmp = x;
      x = o;
      o = tmp;
    }
    xc[l] = x;
  }
  const MgTailLevel& vt = tl.lv[tl.T];
  if (xc[tl.T] != vt.xa) {
    const int64_t nd = 3 * vt.nn;
    for (int64_t q = gt; q < nd * ncase; q += gs) {
      int64_t it;
      int k;
      mg_item_case<MULTI>(q, ncase, &it, &k);
      if (live(k)) vt.xa[k * nd + it] = xc[tl.T][k * nd + it];
    }
  }
}

template <bool MULTI>
__global__ void __launch_bounds__(kMgTailThreads)
    k_mg_tail(const __grid_constant__ MgTail tl, const float* __restrict__ om, const MixState* st, int ncase) {
  mg_tail_body<MULTI>(tl, om, st, ncase, blockIdx.x * (int64_t)blockDim.x + threadIdx.x,
                      (int64_t)gridDim.x * blockDim.x, gridDim.x == 1);
}

// Outer step, part 1. mode 0: x += alpha p, r -= alpha q (FP64, padded layout), ||r|| against the stop and
// replacement thresholds. All modes: the voxel level's FP32 residual rf = r and its first Jacobi sweep
// xf = omega invd rf (padded FP32 layout).
__global__ void __launch_bounds__(kT) k_mg_enter(GridDims g, double* __restrict__ x, double* __restrict__ r,
                                                 const double* __restrict__ p, const double* __restrict__ q,
                                                 const float* __restrict__ invdf, float* __restrict__ rf,
                                                 float* __restrict__ xf, const float* __restrict__ om, MixState* st,
                                                 double* part, int mode) {
  __shared__ double sh[32];
  if (!mg_running(st)) return;
  const double alpha = st->alpha;
  const float omega = *om;
  const int rl = 3 * g.nx1;
  const int64_t total = (int64_t)g.ny1 * g.nz1 * rl;
  double rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / rl;
    const int t = (int)(i - row * rl);
    const int64_t a = (int64_t)g.rp64 * row + t, b = (int64_t)g.rp * row + t;
    double rv = r[a];
    if (mode == 0) {
      x[a] = fma(alpha, p[a], x[a]);
      rv = fma(-alpha, q[a], rv);
      r[a] = rv;
      rr += rv * rv;
    }
    const float rfv = (float)rv;
    rf[b] = rfv;
    xf[b] = omega * invdf[b] * rfv;
  }
  if (mode != 0) return;
  const double br = bsum(rr, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = br;
  if (!elect_last32(&st->counter)) return;
  if (threadIdx.x >= 32) return;
  const double s = warp_sum_parts(part, gridDim.x);
  if (threadIdx.x != 0) return;
  st->counter = 0;
  const double rn = sqrt(s);
  st->rn = rn;
  st->iter += 1;
  if (rn <= st->target || rn <= st->flush_at) st->status = MIX_FLUSH;
  else if (st->iter >= st->max_iter) st->status = MIX_MAXITER;
}

// End of an outer step (CTA partials of (z, r), (z, A p), (r, r) in b1..b3, valid in thread 0): fixed-order
// sums by the last CTA. mode 0: beta = -alpha (z, A p) / rho, rho = (z, r). mode 1 (after a true-residual
// replacement, direction kept): the same beta, new replacement threshold. mode 2 (start): rho, next direction
// p = z.
__device__ __forceinline__ void mg_exit_tail(double b1, double b2, double b3, MixState* st, double* part, int mode,
                                             unsigned bx, unsigned nb) {
  if (threadIdx.x == 0) {
    part[bx] = b1;
    part[nb + bx] = b2;
    part[2 * nb + bx] = b3;
  }
  if (!elect_last_n(&st->counter, nb)) return;
  if (threadIdx.x >= 32) return;
  const double szr = warp_sum_parts(part, nb);
  const double szq = warp_sum_parts(part + nb, nb);
  const double srr = warp_sum_parts(part + 2 * nb, nb);
  if (threadIdx.x != 0) return;
  st->counter = 0;
  st->pmode = 0;  // the next step follows a matvec
  if (!(szr > 0.0) || !isfinite(szr)) {  // (z, r) > 0 for an SPD preconditioner and r != 0
    st->status = MIX_BREAKDOWN;
    return;
  }
  if (mode != 0) {
    const double rn = sqrt(srr);
    st->rn = rn;
    st->flush_at = rn * st->flush_factor;
  }
  if (mode == 2) {
    st->first = 1;
    st->status = st->rn <= st->target ? MIX_FLUSH : MIX_RUNNING;
  } else if (mode == 1 && (st->iter == 0 || !(st->rho0 > 0.0))) {
    st->first = 1;
  } else {
    const double beta = -st->alpha * szq / st->rho0;
    if (isfinite(beta)) {
      st->beta = beta;
      st->first = 0;
    } else {
      st->first = 1;
    }
  }
  st->rho0 = szr;
}

// Outer step, part 2: the voxel level's last Jacobi sweep written as the FP64 preconditioned residual
// z = xf + omega invd (rf - tf) (tf = A xf), then (z, r), (z, A p) and (r, r) (mg_exit_tail).
__global__ void __launch_bounds__(kT) k_mg_exit(GridDims g, const float* __restrict__ rf, const float* __restrict__ tf,
                                                const float* __restrict__ xf, const float* __restrict__ invdf,
                                                const double* __restrict__ r, const double* __restrict__ q,
                                                double* __restrict__ z, const float* __restrict__ om, MixState* st,
                                                double* part, int mode) {
  __shared__ double sh[32];
  if (!mg_running(st)) return;
  const float omega = *om;
  const int rl = 3 * g.nx1;
  const int64_t total = (int64_t)g.ny1 * g.nz1 * rl;
  double zr = 0.0, zq = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / rl;
    const int t = (int)(i - row * rl);
    const int64_t a = (int64_t)g.rp64 * row + t, b = (int64_t)g.rp * row + t;
    const double zv = (double)fmaf(omega * invdf[b], rf[b] - tf[b], xf[b]);
    const double rv = r[a];
    z[a] = zv;
    zr += zv * rv;
    zq += zv * q[a];
    rr += rv * rv;
  }
  const double b1 = bsum(zr, sh);
  const double b2 = bsum(zq, sh);
  const double b3 = bsum(rr, sh);
  mg_exit_tail(b1, b2, b3, st, part, mode, blockIdx.x, gridDim.x);
}

// The same two parts for the FP32 outer iteration (mixed multigrid form): all vectors in the padded FP32 layout,
// the voxel level's residual is the outer residual r itself and its smoothed correction is built in place in z
// (a mapped matvec input). Dots accumulate in FP64.
// body for CTA bx of nb (a launch, or one unit's share of a packed launch)
__device__ __forceinline__ void mg_enter32_body(int64_t n, float* __restrict__ x, float* __restrict__ r,
                                                const float* __restrict__ p, const float* __restrict__ q,
                                                const float* __restrict__ invd, float* __restrict__ xf,
                                                const float* __restrict__ om, MixState* st, double* part, int mode,
                                                unsigned bx, unsigned nb) {
  __shared__ double sh[32];
  if (!mg_running(st)) return;
  const float alpha = (float)st->alpha;
  const float omega = *om;
  double rr = 0.0;
  const int64_t n4 = n >> 2;  // n is a multiple of 4 (row pitch)
  for (int64_t i = bx * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)nb * blockDim.x) {
    float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 iv = reinterpret_cast<const float4*>(invd)[i];
    if (mode == 0) {
      float4 xv = reinterpret_cast<const float4*>(x)[i];
      const float4 pv = reinterpret_cast<const float4*>(p)[i];
      const float4 qv = reinterpret_cast<const float4*>(q)[i];
      xv.x = fmaf(alpha, pv.x, xv.x); xv.y = fmaf(alpha, pv.y, xv.y);
      xv.z = fmaf(alpha, pv.z, xv.z); xv.w = fmaf(alpha, pv.w, xv.w);
      rv.x = fmaf(-alpha, qv.x, rv.x); rv.y = fmaf(-alpha, qv.y, rv.y);
      rv.z = fmaf(-alpha, qv.z, rv.z); rv.w = fmaf(-alpha, qv.w, rv.w);
      reinterpret_cast<float4*>(x)[i] = xv;
      reinterpret_cast<float4*>(r)[i] = rv;
      rr += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
    }
    reinterpret_cast<float4*>(xf)[i] =
        make_float4(omega * iv.x * rv.x, omega * iv.y * rv.y, omega * iv.z * rv.z, omega * iv.w * rv.w);
  }
  if (mode != 0) return;
  const double br = bsum(rr, sh);
  if (threadIdx.x == 0) part[bx] = br;
  if (!elect_last_n(&st->counter, nb)) return;
  if (threadIdx.x >= 32) return;
  const double s = warp_sum_parts(part, nb);
  if (threadIdx.x != 0) return;
  st->counter = 0;
  const double rn = sqrt(s);
  st->rn = rn;
  st->iter += 1;
  if (rn <= st->target || rn <= st->flush_at) st->status = MIX_FLUSH;
  else if (st->iter >= st->max_iter) st->status = MIX_MAXITER;
}

__global__ void __launch_bounds__(kT) k_mg_enter32(int64_t n, float* __restrict__ x, float* __restrict__ r,
                                                   const float* __restrict__ p, const float* __restrict__ q,
                                                   const float* __restrict__ invd, float* __restrict__ xf,
                                                   const float* __restrict__ om, MixState* st, double* part, int mode) {
  mg_enter32_body(n, x, r, p, q, invd, xf, om, st, part, mode, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ void mg_exit32_body(int64_t n, const float* __restrict__ r, const float* __restrict__ tf,
                                               float* __restrict__ z, const float* __restrict__ invd,
                                               const float* __restrict__ q, const float* __restrict__ om,
                                               MixState* st, double* part, int mode, unsigned bx, unsigned nb) {
  __shared__ double sh[32];
  if (!mg_running(st)) return;
  const float omega = *om;
  double zr = 0.0, zq = 0.0, rr = 0.0;
  const int64_t n4 = n >> 2;
  for (int64_t i = bx * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)nb * blockDim.x) {
    const float4 rv = reinterpret_cast<const float4*>(r)[i];
    const float4 tv = reinterpret_cast<const float4*>(tf)[i];
    const float4 iv = reinterpret_cast<const float4*>(invd)[i];
    const float4 qv = reinterpret_cast<const float4*>(q)[i];
    float4 zv = reinterpret_cast<const float4*>(z)[i];
    zv.x = fmaf(omega * iv.x, rv.x - tv.x, zv.x);
    zv.y = fmaf(omega * iv.y, rv.y - tv.y, zv.y);
    zv.z = fmaf(omega * iv.z, rv.z - tv.z, zv.z);
    zv.w = fmaf(omega * iv.w, rv.w - tv.w, zv.w);
    reinterpret_cast<float4*>(z)[i] = zv;
    zr += (double)zv.x * rv.x + (double)zv.y * rv.y + (double)zv.z * rv.z + (double)zv.w * rv.w;
    zq += (double)zv.x * qv.x + (double)zv.y * qv.y + (double)zv.z * qv.z + (double)zv.w * qv.w;
    rr += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
  }
  const double b1 = bsum(zr, sh);
  const double b2 = bsum(zq, sh);
  const double b3 = bsum(rr, sh);
  mg_exit_tail(b1, b2, b3, st, part, mode, bx, nb);
}

__global__ void __launch_bounds__(kT) k_mg_exit32(int64_t n, const float* __restrict__ r, const float* __restrict__ tf,
                                                  float* __restrict__ z, const float* __restrict__ invd,
                                                  const float* __restrict__ q, const float* __restrict__ om,
                                                  MixState* st, double* part, int mode) {
  mg_exit32_body(n, r, tf, z, invd, q, om, st, part, mode, blockIdx.x, gridDim.x);
}

// Power iteration for lambda_max(D^-1 A) of a level: a fixed pseudo-random start on DOFs with a nonzero
// inverse diagonal, then y = A x, x = D^-1 y / ||D^-1 y||; after the last product lambda ~ ||D^-1 A x||.
__device__ __forceinline__ float mg_start_value(int64_t q) {
  uint32_t h = (uint32_t)q * 2654435761u;
  h ^= h >> 16;
  h *= 2246822519u;
  h ^= h >> 13;
  const float u = (float)(h & 0xffffffu) * (1.0f / 16777216.0f);
  return (h & 0x80000000u) ? -(0.5f + u) : (0.5f + u);
}

__global__ void k_mg_pow_init(int64_t n, const float* __restrict__ invd, float* __restrict__ x) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    x[q] = invd[q] != 0.0f ? mg_start_value(q) : 0.0f;
}

struct MgScratch {
  float omega[kMgMaxLevels];
  float norm;
  unsigned int counter;
};

// ||D^-1 y|| by fixed-order sums into sc->norm; with `omega_out` also that level's damping
__global__ void __launch_bounds__(kT) k_mg_pow_norm(int64_t n, const float* __restrict__ y, const float* __restrict__ invd,
                                                    double* part, MgScratch* sc, float* omega_out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const double v = (double)invd[q] * y[q];
    s += v * v;
  }
  const double b = bsum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = b;
  if (!elect_last32(&sc->counter)) return;
  if (threadIdx.x >= 32) return;
  const double t = warp_sum_parts(part, gridDim.x);
  if (threadIdx.x != 0) return;
  sc->counter = 0;
  const float nrm = (float)sqrt(t);
  sc->norm = nrm;
  if (omega_out) *omega_out = (nrm > 0.0f && isfinite(nrm)) ? kMgOmegaScale / nrm : 0.5f;
}

__global__ void k_mg_pow_scale(int64_t n, const float* __restrict__ y, const float* __restrict__ invd,
                               const MgScratch* __restrict__ sc, float* __restrict__ x) {
  const float inv = 1.0f / fmaxf(sc->norm, 1e-30f);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
    x[q] = invd[q] * y[q] * inv;
}

// grid for the streaming kernels: fixed by n (deterministic reductions), at most 8 CTAs per SM
static int stream_blocks(mycel_problem* p) {
  int64_t want = (p->g.nd / 4 + (int64_t)kT * 4 - 1) / ((int64_t)kT * 4);
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)p->ctx->num_sms * 8));
}

void launch_E_to_f32(mycel_problem* p) {
  (void)p;  // k_update_E writes the FP32 copy of E alongside the FP64 one
}

// FP32 work vectors of the mixed form (padded layout, pads zero) and their TMA descriptors; also grants the
// factorised matvec its shared memory above the 48 KB default (once per process, before any launch or capture)
static int32_t ensure_mixed(mycel_problem* p) {
  static std::once_flag smem_once;
  static cudaError_t smem_err = cudaSuccess;
  std::call_once(smem_once, [] {
    cudaError_t a = cudaFuncSetAttribute(k_mv32f<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac_smem_bytes(0));
    cudaError_t b = cudaFuncSetAttribute(k_mv32f<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac_smem_bytes(1));
    smem_err = a != cudaSuccess ? a : b;
  });
  if (smem_err != cudaSuccess)
    return set_error(p->ctx, MYCEL_E_DEVICE, std::string("matvec shared memory: ") + cudaGetErrorString(smem_err));
  if (p->f_x) return MYCEL_OK;
  const size_t fb = sizeof(float) * (size_t)p->g.n32 + 64;
  cudaError_t e = cudaSuccess;
  float** bufs[] = {&p->f_x, &p->f_r, &p->f_z, &p->f_p0, &p->f_p1, &p->f_ap};
  for (float** b : bufs) {
    if ((e = cudaMallocAsync((void**)b, fb, p->ctx->stream)) != cudaSuccess) break;
    p->device_bytes += (int64_t)fb;
    cudaMemsetAsync(*b, 0, fb, p->ctx->stream);
  }
  if (e != cudaSuccess) return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the mixed-precision workspace");
  float* mapped[4] = {p->f_r, p->f_z, p->f_p0, p->f_p1};
  for (int q = 0; q < 4; ++q) {
    int32_t st = encode_plane_map(p, mapped[q], false, &p->f_tmap[q]);
    if (st) return st;
  }
  return MYCEL_OK;
}

// y = K x (projected: ApplyA form) through the FP32 operator; x and y box-ordered FP64 device vectors
int32_t mixed_apply_k_f64io(mycel_problem* p, const double* x, double* y, int projected) {
  int32_t st = ensure_mixed(p);
  if (st) return st;
  cudaStream_t s = p->ctx->stream;
  k_to_pad<float><<<stream_blocks(p), kT, 0, s>>>(p->g, x, p->f_r);
  launch_mv32_variant<0>(p, s, p->f_r, nullptr, nullptr, nullptr, p->f_ap, projected, nullptr, nullptr);
  k_from_pad<float><<<stream_blocks(p), kT, 0, s>>>(p->g, p->f_ap, y);
  p->ctx->launches += 3;
  return MYCEL_OK;
}

// FP64 work vectors of the fast FP64 form (padded layout, pads zero), their TMA descriptors, and the FP64
// matvec's shared memory above the 48 KB default (once per process, before any launch or capture)
static int32_t ensure_f64f(mycel_problem* p) {
  static std::once_flag smem_once;
  static cudaError_t smem_err = cudaSuccess;
  std::call_once(smem_once, [] {
    cudaError_t a = cudaFuncSetAttribute(k_mv64f<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac64_smem_bytes(0));
    cudaError_t b = cudaFuncSetAttribute(k_mv64f<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac64_smem_bytes(1));
    smem_err = a != cudaSuccess ? a : b;
  });
  if (smem_err != cudaSuccess)
    return set_error(p->ctx, MYCEL_E_DEVICE, std::string("FP64 matvec shared memory: ") + cudaGetErrorString(smem_err));
  if (p->g_x) return MYCEL_OK;
  const size_t fb = sizeof(double) * (size_t)p->g.n64 + 64;
  cudaError_t e = cudaSuccess;
  double** bufs[] = {&p->g_x, &p->g_r, &p->g_z, &p->g_p0, &p->g_p1, &p->g_ap, &p->g_invd};
  for (double** b : bufs) {
    if ((e = cudaMallocAsync((void**)b, fb, p->ctx->stream)) != cudaSuccess) break;
    p->device_bytes += (int64_t)fb;
    cudaMemsetAsync(*b, 0, fb, p->ctx->stream);
  }
  if (e != cudaSuccess) return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the fast FP64 workspace");
  double* mapped[4] = {p->g_r, p->g_z, p->g_p0, p->g_p1};
  for (int q = 0; q < 4; ++q) {
    int32_t st = encode_plane_map(p, mapped[q], true, &p->g_tmap[q]);
    if (st) return st;
  }
  return MYCEL_OK;
}

// y = K x (projected: ApplyA form) through the factorised FP64 operator; x, y box-ordered FP64 device vectors
int32_t fast64_apply_k(mycel_problem* p, const double* x, double* y, int projected) {
  int32_t st = ensure_f64f(p);
  if (st) return st;
  cudaStream_t s = p->ctx->stream;
  k_to_pad<double><<<stream_blocks(p), kT, 0, s>>>(p->g, x, p->g_r);
  launch_mv64f<0>(p, s, p->g_r, nullptr, nullptr, nullptr, p->g_ap, projected, nullptr, nullptr);
  k_from_pad<double><<<stream_blocks(p), kT, 0, s>>>(p->g, p->g_ap, y);
  p->ctx->launches += 3;
  return MYCEL_OK;
}

static MixState* mix_state(mycel_problem* p) { return (MixState*)(p->d_part2 + p->n_part2 - 64); }

__global__ void k_mix_init(MixState* st, double target, int max_iter, double flush_factor) {
  MixState s = {};
  s.status = MIX_RUNNING;
  s.target = target;
  s.max_iter = max_iter;
  s.first = 1;
  s.flush_factor = flush_factor;
  *st = s;
}

__global__ void k_mix_set(MixState* st, int status) { st->status = status; }

// Multigrid hierarchy of a problem (MYCEL_PRECISION_FP64_MG). Level 0 is the voxel grid, whose vectors are the
// mixed form's FP32 work vectors (padded layout): residual f_r, smoothed correction f_p0 (a mapped matvec
// input), its product f_ap. Coarse levels hold box-ordered FP32 vectors and their assembled stencil.
struct MgLevel {
  MgDims d{};
  int64_t nn = 0, nd = 0;
  float *S = nullptr, *invd = nullptr, *xa = nullptr, *xb = nullptr, *r = nullptr, *t = nullptr;
  bool staged = false;  // products of one case by k_mg_apply_nodes_tma through tm_s
  int* err = nullptr;   // the problem's bounded-wait error word
  CUtensorMap tm_s{};   // the stencil as a 2-D tensor [126 rows][ns nodes], boxes of [9][kS1Box]
};

struct MgHier {
  int L = 0;  // levels 0 .. L-1; level L-1 is solved by its dense inverse
  uint64_t setup_version = ~0ull;  // the problem's E version the coarse operators were built from
  MgLevel lv[kMgMaxLevels];
  float* em[2] = {nullptr, nullptr};  // element matrices of alternate coarse levels (rebuilt at each solve)
  float* G = nullptr;                 // [8][576] W_s^T KE W_s of the 8 sub-element positions (level-1 fast path)
  uint8_t* special = nullptr;         // [level-1 elements] built by the general path
  double* ainv = nullptr;
  MgScratch* sc = nullptr;  // per-level damping, power-iteration norm and counter (device)
  // the voxel level's power iteration runs on the context's side stream beside the coarse-level builds: its
  // own norm/counter and block partials, and the fork/join events
  MgScratch* sc0 = nullptr;
  double* part0 = nullptr;
  cudaEvent_t fork_ev = nullptr, stencil_ev = nullptr, join_ev = nullptr;
  int sweeps = 1;
  int per_iter = 0;  // kernel launches per outer iteration
  cudaGraphExec_t graph[2] = {nullptr, nullptr};    // FP64 outer iteration chunks
  int graph_profiled = 0;
  cudaEvent_t ev[2][2] = {};
  cudaGraphExec_t graph32[2] = {nullptr, nullptr};  // FP32 outer iteration chunks (mixed multigrid form)
  int graph32_profiled = 0;
  cudaEvent_t ev32[2][2] = {};
  // live timing of the level-1 residual product (the form's largest coarse-level kernel): event-record nodes
  // around it in the first iteration of each chunk graph, captured only while the context profiles
  cudaEvent_t l1ev[2][2] = {};
  cudaEvent_t* l1_timing = nullptr;  // the pair of the graph being captured (iteration 0 only), else null
  float* f_t = nullptr;  // FP32 outer form: A x of the voxel level's smoothing (padded FP32 layout)
  float* eig[kMgMaxLevels] = {};  // last eigenvector estimate of D^-1 A per smoothed level (warm start)
  bool eig_valid = false;
  int T = 1;             // first level handled by the cluster kernel k_mg_tail
  MgTail tail{};
  bool prefers_f64 = false;  // an FP32 outer solve of this problem stalled: later ones start in FP64
  int ncap = 1;          // load cases the level vectors have room for (case k at + k * nd)
  // load cases solved together (mg_solve_cases): per case the FP32 work vectors x, r, z, p0, p1, ap, t of the
  // voxel level, the TMA descriptors of r, z, p0, p1, one state per case, and the chunk graphs
  struct CaseWork {
    int n = 0;
    float* v[kMgMaxCases][7] = {};
    CUtensorMap tmap[kMgMaxCases][4];
    MixState* st = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_profiled = -1;
    int graph_n = 0;
    int per_chunk = 0;  // kernel launches of one chunk graph
  } cw;
  std::vector<void*> bufs;
};

// Level element counts; 0 when the grid cannot be coarsened to a coarsest level of at most kMgCoarseMax DOFs
// with at least one coarse level.
static int mg_levels(int nx, int ny, int nz, MgDims* out) {
  MgDims d{nx, ny, nz};
  int L = 0;
  out[L++] = d;
  while (L < kMgMaxLevels) {
    if (L >= 2 && 3 * mg_nn(d) <= kMgCoarseMax) break;
    if (d.nx == 1 && d.ny == 1 && d.nz == 1) break;
    d = {(d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2};
    out[L++] = d;
  }
  return (L >= 2 && 3 * mg_nn(out[L - 1]) <= kMgCoarseMax) ? L : 0;
}

int64_t mg_device_bytes(int nx, int ny, int nz, int n_cases, bool cases_together) {
  MgDims lv[kMgMaxLevels];
  const int L = mg_levels(nx, ny, nz, lv);
  if (!L) return 0;
  const int nc = std::min(kMgMaxCases, std::max(1, n_cases));  // level vectors have room for the cases
  int64_t b = 0;
  for (int l = 1; l < L; ++l) b += 4 * (9 * kMgHalf * mg_ns(lv[l]) + (3 + 12 * nc) * mg_nn(lv[l])) + 6 * 64;
  b += sizeof(MgScratch) + 64 + 4 * 8 * 576 + 64 + (int64_t)lv[1].nx * lv[1].ny * lv[1].nz + 64;
  const int64_t rp = (3 * (int64_t)(nx + 1) + 3) & ~int64_t(3);  // FP32 row pitch of the voxel level
  b += 4 * rp * (ny + 1) * (nz + 1) + 64;                         // f_t
  b += 4 * rp * (ny + 1) * (nz + 1) + 64;                         // eigenvector estimate of the voxel level
  for (int l = 1; l < L - 1; ++l) b += 4 * 3 * mg_nn(lv[l]) + 64; // and of the coarse smoothed levels
  b += 4 * 576 * (int64_t)lv[1].nx * lv[1].ny * lv[1].nz + 64;
  if (L > 2) b += 4 * 576 * (int64_t)lv[2].nx * lv[2].ny * lv[2].nz + 64;
  b += 8 * 9 * mg_nn(lv[L - 1]) * mg_nn(lv[L - 1]) + 64;
  if (cases_together && n_cases > 1 && n_cases <= kMgMaxCases)  // the cases' voxel-level vectors and states
    b += (int64_t)n_cases * (7 * (4 * rp * (ny + 1) * (nz + 1) + 64) + (int64_t)sizeof(MixState));
  return b;
}

void mg_release(mycel_problem* p) {
  MgHier* mg = p->mg;
  if (!mg) return;
  for (int k = 0; k < 2; ++k) {
    if (mg->graph[k]) cudaGraphExecDestroy(mg->graph[k]);
    if (mg->graph32[k]) cudaGraphExecDestroy(mg->graph32[k]);
    for (int j = 0; j < 2; ++j) {
      if (mg->ev[k][j]) cudaEventDestroy(mg->ev[k][j]);
      if (mg->ev32[k][j]) cudaEventDestroy(mg->ev32[k][j]);
      if (mg->l1ev[k][j]) cudaEventDestroy(mg->l1ev[k][j]);
    }
    if (mg->cw.graph[k]) cudaGraphExecDestroy(mg->cw.graph[k]);
  }
  for (cudaEvent_t e : {mg->fork_ev, mg->stencil_ev, mg->join_ev})
    if (e) cudaEventDestroy(e);
  p->n_case_tmaps = 0;
  for (void* b : mg->bufs) cudaFreeAsync(b, p->ctx->stream);
  delete mg;
  p->mg = nullptr;
}

static int32_t mg_ensure(mycel_problem* p, bool* available) {
  static std::once_flag smem_once;
  static cudaError_t smem_err = cudaSuccess;
  std::call_once(smem_once, [] {
    smem_err = cudaFuncSetAttribute(k_mg_coarse_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMgCoarseSmem);
    if (smem_err == cudaSuccess)
      smem_err = cudaFuncSetAttribute(k_mg_apply_nodes_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kS1Smem);
    if (smem_err == cudaSuccess)  // four CTAs of 54 KB per SM
      smem_err = cudaFuncSetAttribute(k_mg_apply_nodes_tma, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  });
  if (smem_err != cudaSuccess)
    return set_error(p->ctx, MYCEL_E_DEVICE, std::string("multigrid shared memory: ") + cudaGetErrorString(smem_err));
  *available = false;
  if (p->mg) {
    *available = true;
    return MYCEL_OK;
  }
  MgDims dims[kMgMaxLevels];
  const int L = mg_levels(p->g.nx, p->g.ny, p->g.nz, dims);
  if (!L) return MYCEL_OK;
  MgHier* mg = new MgHier();
  mg->L = L;
  mg->ncap = std::min(kMgMaxCases, std::max(1, (int)p->n_cases));
  if (const char* e = std::getenv("MYCEL_MG_SWEEPS")) mg->sweeps = std::max(1, std::atoi(e));
  cudaStream_t s = p->ctx->stream;
  bool oom = false;
  auto alloc = [&](size_t bytes) -> void* {
    void* ptr = nullptr;
    if (oom || cudaMallocAsync(&ptr, bytes + 64, s) != cudaSuccess) {
      oom = true;
      return nullptr;
    }
    cudaMemsetAsync(ptr, 0, bytes + 64, s);
    p->device_bytes += (int64_t)bytes + 64;
    mg->bufs.push_back(ptr);
    return ptr;
  };
  for (int l = 0; l < L; ++l) {
    MgLevel& v = mg->lv[l];
    v.d = dims[l];
    v.nn = mg_nn(v.d);
    v.nd = 3 * v.nn;
    if (l == 0) continue;
    v.S = (float*)alloc(sizeof(float) * 9 * kMgHalf * mg_ns(v.d));  // zeroed: the row padding stays 0
    v.invd = (float*)alloc(sizeof(float) * v.nd);
    v.err = p->d_err;
    if (v.S && v.nn > kMgDofMaxNodes) {  // the levels whose products run a thread per node
      const PFN_cuTensorMapEncodeTiled encode = tensor_map_encoder();
      cuuint64_t dims[2] = {(cuuint64_t)mg_ns(v.d), (cuuint64_t)(9 * kMgHalf)};
      cuuint64_t strides[1] = {(cuuint64_t)mg_ns(v.d) * 4};
      cuuint32_t box[2] = {(cuuint32_t)kS1Box, 9};
      cuuint32_t estr[2] = {1, 1};
      v.staged = encode && mg_ns(v.d) < (int64_t)INT32_MAX - kS1Box &&
                 encode(&v.tm_s, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, v.S, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    float** vecs[] = {&v.xa, &v.xb, &v.r, &v.t};
    for (float** q : vecs) *q = (float*)alloc(sizeof(float) * v.nd * mg->ncap);
  }
  for (int k = 0; k < 2 && k + 1 < L; ++k) {
    const MgDims& d = mg->lv[k + 1].d;
    mg->em[k] = (float*)alloc(sizeof(float) * 576 * (size_t)d.nx * d.ny * d.nz);
  }
  const int64_t nc = mg->lv[L - 1].nd;
  mg->ainv = (double*)alloc(sizeof(double) * nc * nc);
  mg->sc = (MgScratch*)alloc(sizeof(MgScratch));
  mg->sc0 = (MgScratch*)alloc(sizeof(MgScratch));
  mg->part0 = (double*)alloc(sizeof(double) * 8 * (size_t)p->ctx->num_sms + 64);
  cudaEventCreateWithFlags(&mg->fork_ev, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&mg->stencil_ev, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&mg->join_ev, cudaEventDisableTiming);
  mg->f_t = (float*)alloc(sizeof(float) * (size_t)p->g.n32);
  for (int l = 0; l < L - 1; ++l) mg->eig[l] = (float*)alloc(sizeof(float) * (size_t)(l ? mg->lv[l].nd : p->g.n32));
  mg->G = (float*)alloc(sizeof(float) * 8 * 576);
  mg->special = (uint8_t*)alloc((size_t)dims[1].nx * dims[1].ny * dims[1].nz);
  if (!oom) {  // G_s = W_s^T KE W_s for an interior coarse element (all sub-elements present), in FP64
    auto w1 = [](int f, int c) { return f == 1 ? 0.5 : ((f == 0) == (c == 0) ? 1.0 : 0.0); };
    auto bx = [](int a) { return (a ^ (a >> 1)) & 1; };
    auto by = [](int a) { return (a >> 1) & 1; };
    auto bz = [](int a) { return a >> 2; };
    std::vector<float> G(8 * 576);
    for (int sub = 0; sub < 8; ++sub) {
      const int sx = sub & 1, sy = (sub >> 1) & 1, sz = sub >> 2;
      double W[8][8];
      for (int a = 0; a < 8; ++a)
        for (int C = 0; C < 8; ++C)
          W[a][C] = w1(sx + bx(a), bx(C)) * w1(sy + by(a), by(C)) * w1(sz + bz(a), bz(C));
      for (int row = 0; row < 24; ++row)
        for (int col = 0; col < 24; ++col) {
          const int C = row / 3, cc = row % 3, Cp = col / 3, cp = col % 3;
          double v = 0.0;
          for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) v += W[a][C] * p->ke.v[(3 * a + cc) * 24 + 3 * b + cp] * W[b][Cp];
          G[sub * 576 + row * 24 + col] = (float)v;
        }
    }
    cudaMemcpyAsync(mg->G, G.data(), sizeof(float) * G.size(), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
  }
  {  // the cluster kernel must fit: kMgTailCtas CTAs of kMgTailThreads threads co-resident
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kMgTailCtas);
    cfg.blockDim = dim3(kMgTailThreads);
    cudaLaunchAttribute at{};
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = kMgTailCtas;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    int ncl2 = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_mg_tail<false>, &cfg) != cudaSuccess || nclusters < 1 ||
        cudaOccupancyMaxActiveClusters(&ncl2, k_mg_tail<true>, &cfg) != cudaSuccess || ncl2 < 1) {
      cudaGetLastError();
      return set_error(p->ctx, MYCEL_E_DEVICE, "multigrid: the coarse-level cluster kernel cannot be scheduled");
    }
  }
  // levels T .. L-1 in one cluster launch: T is the first coarse level of at most kMgTailMaxNodes nodes
  mg->T = L - 1;
  for (int l = 1; l < L; ++l)
    if (mg->lv[l].nn <= kMgTailMaxNodes) {
      mg->T = l;
      break;
    }
  mg->tail.T = mg->T;
  mg->tail.L = L;
  mg->tail.sweeps = mg->sweeps;
  mg->tail.nc = (int)nc;
  mg->tail.ainv = mg->ainv;
  for (int l = 1; l < L; ++l) {
    const MgLevel& v = mg->lv[l];
    mg->tail.lv[l] = {v.d, v.nn, v.S, v.invd, v.xa, v.xb, v.r, v.t};
  }
  // launches per outer iteration: matvec, k_mg_enter*, the V-cycle (as issued by mg_vcycle), k_mg_exit*
  const int sw = mg->sweeps, T = mg->T;
  const int cycle = 4 * (sw - 1) + 2 + (T - 1) * (1 + sw) + 1 + (T - 1) * (1 + sw) + 1 + 1;
  mg->per_iter = 3 + cycle;
  p->mg = mg;
  if (oom) return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the multigrid hierarchy");
  *available = true;
  return MYCEL_OK;
}

static unsigned mg_blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

// coarse-level product on the stream: a thread per DOF up to 64k nodes, a thread per node above (measured on
// the bridge: level 2, 31k nodes, 9.6 vs 14.5 us; level 1, 233k nodes, 43 vs 51 us)
// the small levels' kernel: one 8-CTA cluster with cluster barriers between phases (a single CTA with CTA
// barriers was measured slower: 51.9 against 56.6 SIMP iter/s on the bridge)
static int mg_tail_ctas() { return kMgTailCtas; }

static void launch_mg_tail(cudaStream_t s, MgHier* mg, const float* om, const MixState* st, int nc) {
  const int ctas = mg_tail_ctas();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kMgTailThreads);
  cfg.stream = s;
  cudaLaunchAttribute at{};
  at.id = cudaLaunchAttributeClusterDimension;
  at.val.clusterDim.x = ctas;
  at.val.clusterDim.y = 1;
  at.val.clusterDim.z = 1;
  cfg.attrs = &at;
  cfg.numAttrs = ctas > 1 ? 1 : 0;
  if (nc == 1) cudaLaunchKernelEx(&cfg, k_mg_tail<false>, mg->tail, om, st, nc);
  else cudaLaunchKernelEx(&cfg, k_mg_tail<true>, mg->tail, om, st, nc);
}

// case k's vector of a level whose case vectors follow one another (base + k * nd)
static MgPtrs lv_ptrs(float* base, int64_t nd, int n) {
  MgPtrs r{};
  for (int k = 0; k < n; ++k) r.p[k] = base ? base + k * nd : nullptr;
  return r;
}

static void launch_mg_apply(cudaStream_t s, const MgLevel& v, const MgPtrs& x, const MgPtrs& r, const float* invd,
                            const MgPtrs& y, int mode, const float* om, const MixState* st, int nc) {
  if (v.nn * nc <= kMgDofMaxNodes)
    (nc == 1 ? k_mg_apply<false> : k_mg_apply<true>)<<<mg_dof_blocks(v.nn * nc), kMgDofThreads, 0, s>>>(
        v.d, v.S, x, r, invd, y, mode, om, st, nc);
  else if (nc == 1 && v.staged)
    k_mg_apply_nodes_tma<<<(unsigned)((v.nn + kS1Nodes - 1) / kS1Nodes), 256, kS1Smem, s>>>(
        v.d, v.tm_s, x.p[0], r.p[0], invd, y.p[0], mode, om, st, v.err);
  else
    (nc == 1 ? k_mg_apply_nodes<false> : k_mg_apply_nodes<true>)<<<mg_blocks(v.nn * nc), 256, 0, s>>>(
        v.d, v.S, x, r, invd, y, mode, om, st, nc);
}

// The load cases one V-cycle advances: their states (one per case, contiguous) and their voxel-level vectors
// (padded FP32 layout): residual rf, first sweep / correction xf (a mapped matvec input) and tf = A xf.
struct MgRun {
  int n = 1;
  MixState* st = nullptr;
  float* rf[kMgMaxCases] = {};
  float* xf[kMgMaxCases] = {};
  float* tf[kMgMaxCases] = {};
};
static MgPtrs mg_ptrs(float* const (&v)[kMgMaxCases], int n) {
  MgPtrs r{};
  for (int k = 0; k < n; ++k) r.p[k] = v[k];
  return r;
}

// Coarse operators from the current E: Galerkin element matrices level by level, their stencils, and the
// coarsest level's dense inverse.
static void mg_setup(mycel_problem* p) {
  MgHier* mg = p->mg;
  cudaStream_t s = p->ctx->stream, ss = p->ctx->side;
  MgLevel* lv = mg->lv;
  const int sb = stream_blocks(p);
  int nl = 0;
  // power iteration for the damping of level l (all but the coarsest), on stream q
  auto power = [&](int l, cudaStream_t q, MgScratch* sc, double* part) {
    MgLevel& v = lv[l];
    const int64_t n = l ? v.nd : p->g.n32;
    const float* invd = l ? v.invd : p->d_invdf;
    float* x = l ? v.xa : p->f_p0;
    float* y = l ? v.t : p->f_ap;
    const unsigned nb = l ? std::min<unsigned>(mg_blocks(n), (unsigned)sb) : (unsigned)sb;
    if (mg->eig_valid) {
      cudaMemcpyAsync(x, mg->eig[l], sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, q);
    } else {
      k_mg_pow_init<<<nb, 256, 0, q>>>(n, invd, x);
      nl++;
    }
    const int iters = mg->eig_valid ? kMgPowerItersWarm : kMgPowerIters;
    for (int it = 0; it < iters; ++it) {
      if (l) launch_mg_apply(q, v, mg_one(x), mg_one(nullptr), invd, mg_one(y), 0, nullptr, nullptr, 1);
      else launch_mv32_variant<0>(p, q, p->f_p0, nullptr, nullptr, nullptr, p->f_ap, 1, nullptr, nullptr);
      const bool last = it == iters - 1;
      k_mg_pow_norm<<<nb, kT, 0, q>>>(n, y, invd, part, sc, last ? mg->sc->omega + l : nullptr);
      k_mg_pow_scale<<<nb, 256, 0, q>>>(n, y, invd, sc, last ? mg->eig[l] : x);
      nl += 3;
    }
  };
  // the voxel level's power iteration needs only E and the diagonal (ready on s): it runs on the side stream
  // while s builds the coarse levels
  cudaEventRecord(mg->fork_ev, s);
  cudaStreamWaitEvent(ss, mg->fork_ev, 0);
  power(0, ss, mg->sc0, mg->part0);
  const MgDims& d1 = lv[1].d;
  const int64_t ne1 = (int64_t)d1.nx * d1.ny * d1.nz;
  k_mg_build1<<<(unsigned)std::min<int64_t>((ne1 + 3) / 4, 8 * (int64_t)p->ctx->num_sms), 256, 0, s>>>(
      d1, lv[0].d, mg->G, p->d_Ef, p->d_nflags, mg->em[0], mg->special);
  k_mg_build<true><<<(unsigned)ne1, 64, 0, s>>>(d1, lv[0].d, p->kef, p->d_Ef, p->d_nflags, nullptr, mg->em[0],
                                                mg->special);
  k_mg_stencil<<<mg_blocks(3 * lv[1].nn), 256, 0, s>>>(d1, mg->em[0], lv[1].S, lv[1].invd);
  for (int l = 2; l < mg->L; ++l) {
    const MgDims& d = lv[l].d;
    float* src = mg->em[(l - 2) & 1];
    float* dst = mg->em[(l - 1) & 1];
    k_mg_build<false><<<(unsigned)((int64_t)d.nx * d.ny * d.nz), 64, 0, s>>>(d, lv[l - 1].d, p->kef, nullptr,
                                                                           nullptr, src, dst, nullptr);
    k_mg_stencil<<<mg_blocks(3 * lv[l].nn), 256, 0, s>>>(d, dst, lv[l].S, lv[l].invd);
  }
  nl += 2 * (mg->L - 1) + 1;
  // the coarsest level's dense inverse on the side stream too, beside the coarse levels' power iterations
  cudaEventRecord(mg->stencil_ev, s);
  cudaStreamWaitEvent(ss, mg->stencil_ev, 0);
  k_mg_coarse_setup<<<1, 1024, kMgCoarseSmem, ss>>>(lv[mg->L - 1].d, lv[mg->L - 1].S, mg->ainv);
  nl++;
  for (int l = 1; l < mg->L - 1; ++l) power(l, s, mg->sc, p->d_part2);
  cudaEventRecord(mg->join_ev, ss);
  cudaStreamWaitEvent(s, mg->join_ev, 0);
  mg->eig_valid = true;
  p->ctx->launches += nl;
}

// One V-cycle for the cases of R: from each case's voxel-level residual rf and first sweep xf (written by
// k_mg_enter*) up to tf = A xf before the last sweep (done by k_mg_exit*). Voxel-level work runs per case; the
// coarse levels run once for all cases. Returns the kernels launched.
static int mg_vcycle(mycel_problem* p, cudaStream_t s, const MgRun& R) {
  MgHier* mg = p->mg;
  MgLevel* lv = mg->lv;
  const GridDims& g = p->g;
  const float* om = mg->sc->omega;  // device: damping of level l at om + l
  const int sb = stream_blocks(p);
  const int nc = R.n;
  MixState* st = R.st;
  auto cst = [&](int k) { return st ? st + k : nullptr; };
  int nl = 0;
  auto fine_mv = [&](int k) {
    launch_mv32_variant<0>(p, s, R.xf[k], nullptr, nullptr, nullptr, R.tf[k], 1, cst(k), nullptr);
  };
  for (int q = 1; q < mg->sweeps; ++q)
    for (int k = 0; k < nc; ++k) {
      fine_mv(k);
      k_mg_jacobi_fine<<<sb, kT, 0, s>>>(g.n32, R.rf[k], R.tf[k], p->d_invdf, R.xf[k], om, cst(k));
      nl += 2;
    }
  for (int k = 0; k < nc; ++k) fine_mv(k);
  nl += nc;
  // restriction to level 1, with level 1's first sweep (unless level 1 is the coarsest)
  (nc == 1 ? k_mg_restrict<true, false> : k_mg_restrict<true, true>)<<<mg_blocks(lv[1].nn * nc), 256, 0, s>>>(lv[0].d, g.rp, mg_ptrs(R.rf, nc), mg_ptrs(R.tf, nc),
                                                               lv[1].d, lv[1].invd, lv_ptrs(lv[1].r, lv[1].nd, nc), st,
                                                               lv_ptrs(lv[1].xa, lv[1].nd, nc), 1 < mg->L - 1 ? 1 : 0,
                                                               om + 1, nc);
  nl++;
  float* xc[kMgMaxLevels] = {};
  for (int l = 1; l < mg->T; ++l) {
    MgLevel& v = lv[l];
    float *x = v.xa, *o = v.xb;
    const MgPtrs r = lv_ptrs(v.r, v.nd, nc);
    for (int k = 1; k < mg->sweeps; ++k) {
      launch_mg_apply(s, v, lv_ptrs(x, v.nd, nc), r, v.invd, lv_ptrs(o, v.nd, nc), 1, om + l, st, nc);
      std::swap(x, o);
    }
    if (l == 1 && mg->l1_timing) cudaEventRecordWithFlags(mg->l1_timing[0], s, cudaEventRecordExternal);
    launch_mg_apply(s, v, lv_ptrs(x, v.nd, nc), r, v.invd, lv_ptrs(v.t, v.nd, nc), 2, om + l, st, nc);
    if (l == 1 && mg->l1_timing) cudaEventRecordWithFlags(mg->l1_timing[1], s, cudaEventRecordExternal);
    MgLevel& cv = lv[l + 1];
    (nc == 1 ? k_mg_restrict<false, false> : k_mg_restrict<false, true>)<<<mg_blocks(cv.nn * nc), 256, 0, s>>>(v.d, 0, lv_ptrs(nullptr, 0, nc),
                                                               lv_ptrs(v.t, v.nd, nc), cv.d, cv.invd,
                                                               lv_ptrs(cv.r, cv.nd, nc), st,
                                                               lv_ptrs(cv.xa, cv.nd, nc), l + 1 < mg->L - 1 ? 1 : 0,
                                                               om + l + 1, nc);
    xc[l] = x;
    nl += 1 + mg->sweeps;
  }
  launch_mg_tail(s, mg, om, st, nc);
  xc[mg->T] = lv[mg->T].xa;
  nl++;
  for (int l = mg->T - 1; l >= 1; --l) {
    MgLevel& v = lv[l];
    float* x = xc[l];
    float* o = x == v.xa ? v.xb : v.xa;
    (nc == 1 ? k_mg_prolong<false, false> : k_mg_prolong<false, true>)<<<mg_blocks(v.nn * nc), 256, 0, s>>>(v.d, 0, nullptr, v.invd, lv_ptrs(x, v.nd, nc), lv[l + 1].d,
                                                              lv_ptrs(xc[l + 1], lv[l + 1].nd, nc), st, nc);
    const MgPtrs r = lv_ptrs(v.r, v.nd, nc);
    for (int k = 0; k < mg->sweeps; ++k) {
      launch_mg_apply(s, v, lv_ptrs(x, v.nd, nc), r, v.invd, lv_ptrs(o, v.nd, nc), 1, om + l, st, nc);
      std::swap(x, o);
    }
    xc[l] = x;
    nl += 1 + mg->sweeps;
  }
  (nc == 1 ? k_mg_prolong<true, false> : k_mg_prolong<true, true>)<<<mg_blocks(lv[0].nn * nc), 256, 0, s>>>(lv[0].d, g.rp, p->d_nflags, nullptr, mg_ptrs(R.xf, nc),
                                                              lv[1].d, lv_ptrs(xc[1], lv[1].nd, nc), st, nc);
  nl++;
  for (int q = 1; q < mg->sweeps; ++q)
    for (int k = 0; k < nc; ++k) {
      fine_mv(k);
      k_mg_jacobi_fine<<<sb, kT, 0, s>>>(g.n32, R.rf[k], R.tf[k], p->d_invdf, R.xf[k], om, cst(k));
      nl += 2;
    }
  for (int k = 0; k < nc; ++k) fine_mv(k);
  return nl + nc;
}

// The outer step after the matvec (mode 0), or the preconditioned residual after a start (2) or a true-residual
// replacement (1): k_mg_enter*, the V-cycle, k_mg_exit*. FP64 outer iteration: the voxel level works on f_r,
// f_p0, f_ap; FP32 outer iteration: on the outer r (f_r) and z (f_z) and f_t. Returns the kernels launched.
static int launch_mg_step(mycel_problem* p, cudaStream_t s, const void* pcur, int mode, bool f64) {
  MgHier* mg = p->mg;
  MixState* st = mix_state(p);
  const int sb = stream_blocks(p);
  const float* om = mg->sc->omega;
  int nl = 0;
  if (mode == 1) {
    k_mix_set<<<1, 1, 0, s>>>(st, MIX_RUNNING);
    nl++;
  }
  MgRun R;
  R.st = st;
  if (f64) {
    k_mg_enter<<<sb, kT, 0, s>>>(p->g, p->g_x, p->g_r, (const double*)pcur, p->g_ap, p->d_invdf, p->f_r, p->f_p0, om,
                                 st, p->d_part2, mode);
    R.rf[0] = p->f_r;
    R.xf[0] = p->f_p0;
    R.tf[0] = p->f_ap;
    nl += 1 + mg_vcycle(p, s, R);
    k_mg_exit<<<sb, kT, 0, s>>>(p->g, p->f_r, p->f_ap, p->f_p0, p->d_invdf, p->g_r, p->g_ap, p->g_z, om, st,
                                p->d_part2, mode);
  } else {
    k_mg_enter32<<<sb, kT, 0, s>>>(p->g.n32, p->f_x, p->f_r, (const float*)pcur, p->f_ap, p->d_invdf, p->f_z, om, st,
                                   p->d_part2, mode);
    R.rf[0] = p->f_r;
    R.xf[0] = p->f_z;
    R.tf[0] = mg->f_t;
    nl += 1 + mg_vcycle(p, s, R);
    k_mg_exit32<<<sb, kT, 0, s>>>(p->g.n32, p->f_r, mg->f_t, p->f_z, p->d_invdf, p->f_ap, om, st, p->d_part2, mode);
  }
  return nl + 1;
}

// The refined inner PCG runs in one of three forms: FP32 work vectors and the FP32 matvec (mixed form), FP64
// work vectors and the factorised FP64 matvec (fast FP64 form), or the latter preconditioned by a multigrid
// V-cycle (multigrid form). All use the same device state machine.
struct InnerForm {
  bool f64;
  bool mg;
  void *x, *r, *z, *p0, *p1, *ap;
  const void* invd;
  int64_t n;        // padded length
  size_t es;        // element size
  cudaGraphExec_t* graph;
  int* graph_profiled;
  cudaEvent_t (*ev)[2];
  int prof_slot;
  double flush_factor;
  int chunk;     // iterations per graph (even)
  int per_iter;  // kernel launches per iteration
};

static InnerForm inner_form(mycel_problem* p, bool f64) {
  if (f64)
    return {true, false, p->g_x, p->g_r, p->g_z, p->g_p0, p->g_p1, p->g_ap, p->g_invd, p->g.n64, sizeof(double),
            p->pcg64f_graph, &p->pcg64f_graph_profiled, p->prof64f_ev, 2, 1e-4, 16, 2};
  return {false, false, p->f_x, p->f_r, p->f_z, p->f_p0, p->f_p1, p->f_ap, p->d_invdf, p->g.n32, sizeof(float),
          p->pcg32_graph, &p->pcg32_graph_profiled, p->prof_ev, 0, kFlushFactor, 16, 2};
}

// multigrid forms: the fast FP64 form's vectors and matvec (f64), or the mixed form's (FP32, replacement after
// a 1e-3 drop of the recursive residual: a multigrid-preconditioned FP32 recurrence stays close to the true
// residual that far); short chunks, since an iteration past convergence still launches its whole V-cycle
// (whose kernels then return at once)
static InnerForm inner_form_mg(mycel_problem* p, bool f64) {
  MgHier* mg = p->mg;
  if (f64)
    return {true, true, p->g_x, p->g_r, p->g_z, p->g_p0, p->g_p1, p->g_ap, p->g_invd, p->g.n64, sizeof(double),
            mg->graph, &mg->graph_profiled, mg->ev, 2, 1e-4, 2, mg->per_iter};
  return {false, true, p->f_x, p->f_r, p->f_z, p->f_p0, p->f_p1, p->f_ap, p->d_invdf, p->g.n32, sizeof(float),
          mg->graph32, &mg->graph32_profiled, mg->ev32, 0, 1e-3, 2, mg->per_iter};
}

static void launch_inner_mv(mycel_problem* p, const InnerForm& F, cudaStream_t s, void* pold, void* pcur) {
  if (F.f64)
    launch_mv64f<1>(p, s, nullptr, (const double*)F.z, (const double*)pold, (double*)pcur, (double*)F.ap, 1,
                    mix_state(p), p->d_part2);
  else
    launch_mv32_variant<1>(p, s, nullptr, (const float*)F.z, (const float*)pold, (float*)pcur, (float*)F.ap, 1,
                           mix_state(p), p->d_part2);
}

static int launch_inner_xr(mycel_problem* p, const InnerForm& F, cudaStream_t s, void* pcur, int mode) {
  const int sb = stream_blocks(p);
  if (F.mg) return launch_mg_step(p, s, pcur, mode, F.f64);
  if (F.f64)
    k_xr64<<<sb, kT, 0, s>>>(F.n, (double*)F.x, (double*)F.r, (double*)F.z, (const double*)pcur, (const double*)F.ap,
                             (const double*)F.invd, mix_state(p), p->d_part2, mode);
  else
    k_xr32<<<sb, kT, 0, s>>>(F.n, (float*)F.x, (float*)F.r, (float*)F.z, (const float*)pcur, (const float*)F.ap,
                             (const float*)F.invd, mix_state(p), p->d_part2, mode);
  return 1;
}

// Chunk of inner iterations as a graph; p alternates between two buffers (even chunk length, each chunk starts
// from the direction held in p1). When the context profiles, the graph also records events around the chunk's
// first matvec (and, in the multigrid forms, around its first level-1 product), so the kernels are timed where
// they run.
static int32_t capture_inner_graph(mycel_problem* p, const InnerForm& F, int chunk) {
  mycel_ctx* c = p->ctx;
  if (F.graph[0] && *F.graph_profiled == c->profile) return MYCEL_OK;
  for (int k = 0; k < 2; ++k) {
    if (F.graph[k]) cudaGraphExecDestroy(F.graph[k]);
    F.graph[k] = nullptr;
    for (int j = 0; j < 2; ++j)
      if (!F.ev[k][j]) cudaEventCreate(&F.ev[k][j]);
  }
  cudaStream_t s = c->stream;
  int64_t before = c->launches;
  MgHier* mg = F.mg ? p->mg : nullptr;
  if (mg)
    for (int k = 0; k < 2; ++k)
      for (int j = 0; j < 2; ++j)
        if (!mg->l1ev[k][j]) cudaEventCreate(&mg->l1ev[k][j]);
  for (int k = 0; k < 2; ++k) {
    cudaGraph_t graph;
    MYCEL_CUDA(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int t = 0; t < chunk; ++t) {
      void* pcur = (t & 1) ? F.p1 : F.p0;
      void* pprev = (t & 1) ? F.p0 : F.p1;
      if (c->profile && t == 0) {
        // timed in place: event-record nodes around the chunk's first matvec, inside the graph
        cudaEventRecordWithFlags(F.ev[k][0], s, cudaEventRecordExternal);
        launch_inner_mv(p, F, s, pprev, pcur);
        cudaEventRecordWithFlags(F.ev[k][1], s, cudaEventRecordExternal);
      } else {
        launch_inner_mv(p, F, s, pprev, pcur);
      }
      if (mg) mg->l1_timing = (c->profile && t == 0 && mg->T > 1) ? mg->l1ev[k] : nullptr;
      launch_inner_xr(p, F, s, pcur, 0);
      if (mg) mg->l1_timing = nullptr;
    }
    MYCEL_CUDA(c, cudaStreamEndCapture(s, &graph));
    MYCEL_CUDA(c, cudaGraphInstantiate(&F.graph[k], graph, 0));
    cudaGraphDestroy(graph);
  }
  c->launches = before;
  *F.graph_profiled = c->profile;
  return MYCEL_OK;
}

static void launch_inner_chunk(mycel_problem* p, const InnerForm& F, int gi) {
  cudaGraphLaunch(F.graph[gi], p->ctx->stream);
}

// r_work = P(b - A u) in FP64 (then rounded to the form's type), returns ||r|| (synchronises). A u comes from
// the factorised FP64 operator (equal to the reference's product up to FP64 rounding): u goes to g_r (a mapped
// input; the fast FP64 forms' own residual, overwritten here anyway), A u to a vector free at this point (g_x,
// the fast FP64 forms' correction, already added to u and cleared again here; g_ap in the mixed form, whose
// vectors are FP32).
// Issues it and the copy of ||r||^2 to *h (pinned host memory) on the context stream, without waiting.
static int32_t true_residual_issue(mycel_problem* p, const InnerForm& F, const double* d_b, const double* d_u,
                                   double* h) {
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  int sb = stream_blocks(p);
  double* part = p->d_part2;
  double* scal = p->d_part2 + p->n_part2 - 128;
  double* au = F.f64 ? p->g_x : p->g_ap;
  k_to_pad<double><<<sb, kT, 0, s>>>(p->g, d_u, p->g_r);
  launch_mv64f<0>(p, s, p->g_r, nullptr, nullptr, nullptr, au, 1, nullptr, nullptr);
  if (F.f64) k_resid64p<double><<<sb, kT, 0, s>>>(p->g, p->d_nflags, d_b, au, (double*)F.r, part, 1);
  else k_resid64p<float><<<sb, kT, 0, s>>>(p->g, p->d_nflags, d_b, au, (float*)F.r, part, 0);
  k_sum_part<<<1, 32, 0, s>>>(part, sb, scal);
  c->launches += 4;
  MYCEL_CUDA(c, cudaMemcpyAsync(h, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
  return MYCEL_OK;
}

static int32_t true_residual(mycel_problem* p, const InnerForm& F, const double* d_b, const double* d_u, double* rn) {
  mycel_ctx* c = p->ctx;
  double* h = (double*)((char*)c->pinned + 1024);
  int32_t st = true_residual_issue(p, F, d_b, d_u, h);
  if (st) return st;
  MYCEL_CUDA(c, cudaStreamSynchronize(c->stream));
  *rn = std::sqrt(h[0]);
  return MYCEL_OK;
}

struct LoopOut {
  int iterations = 0, flushes = 0;
  double rel = 0.0, rel0 = 0.0;  // relative true residual at the end and at the start of the loop
  bool ok = false, stalled = false;
};

// Refined inner PCG from the current u: the device state machine runs chunks of iterations; whenever the
// recursive residual has dropped by the form's flush factor (or reached the target) the correction is added
// to u in FP64 and the true residual P(b - A u) replaces the recursive one (the direction is kept).
// Convergence is decided on the true residual. watch_stall ends the loop when a cycle stalls (mixed form).
static int32_t refined_loop(mycel_problem* p, const InnerForm& F, const double* d_b, double* d_u, double bnorm,
                            double tol, int max_iter, const volatile int32_t* cancel, bool watch_stall, bool verbose,
                            LoopOut* out) {
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  const int chunk = F.chunk;
  const char* name = F.mg ? "multigrid" : (F.f64 ? "fast FP64" : "mixed");
  MixState* ms = mix_state(p);
  int32_t st;
  if (F.f64) {
    k_to_pad<double><<<stream_blocks(p), kT, 0, s>>>(p->g, p->d_invd, p->g_invd);
    c->launches++;
  }
  if ((st = capture_inner_graph(p, F, chunk))) return st;
  double rn = 0.0;
  if ((st = true_residual(p, F, d_b, d_u, &rn))) return st;
  out->rel = out->rel0 = rn / bnorm;
  out->ok = out->rel <= tol;
  if (out->ok) return MYCEL_OK;
  MixState* slot[2] = {(MixState*)((char*)c->pinned + 2048), (MixState*)((char*)c->pinned + 3072)};
  cudaEvent_t evs[2];
  cudaEventCreateWithFlags(&evs[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&evs[1], cudaEventDisableTiming);
  struct EvGuard { cudaEvent_t* e; ~EvGuard() { cudaEventDestroy(e[0]); cudaEventDestroy(e[1]); } } evg{evs};
  cudaMemsetAsync(F.x, 0, F.es * F.n, s);
  k_mix_init<<<1, 1, 0, s>>>(ms, 0.5 * tol * bnorm, max_iter, F.flush_factor);
  c->launches += 1 + launch_inner_xr(p, F, s, F.p0, 2);
  int64_t launched = 0;
  const int64_t cap = (int64_t)max_iter + 64 * chunk + 4096;
  int iter_at_resume = 0;
  // stall watch: each refinement cycle gains log10(1/flush factor) orders of the true residual. CG's later
  // orders cost more than its first ones, so a cycle counts as stalled (FP32 CG on a badly conditioned system)
  // only once it has run longer than 3x all earlier cycles together, and at least 2000 iterations. A multigrid
  // form gains its orders in tens of iterations: there the floor is 300, and it also bounds the first cycle.
  const int64_t stall_floor = F.mg ? 300 : 2000;
  int64_t cycle_limit = F.mg ? stall_floor : INT64_MAX;
  for (;;) {
    // pipeline: chunk k is queued while the status after chunk k-1 is read
    int64_t k = 0;
    int status = MIX_RUNNING;
    for (;; ++k) {
      if (cancel && *cancel) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
      }
      if (launched > cap) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_TIMEOUT, "inner PCG device state did not reach a final status");
      }
      int gi = (int)(k & 1);
      launch_inner_chunk(p, F, gi);
      MYCEL_CUDA(c, cudaGetLastError());
      launched += chunk;
      c->launches += (int64_t)F.per_iter * chunk;
      MYCEL_CUDA(c, cudaMemcpyAsync(slot[gi], ms, sizeof(MixState), cudaMemcpyDeviceToHost, s));
      MYCEL_CUDA(c, cudaEventRecord(evs[gi], s));
      if (k == 0) continue;
      int pi = (int)((k - 1) & 1);
      MYCEL_CUDA(c, cudaEventSynchronize(evs[pi]));
      status = slot[pi]->status;
      if (status != MIX_RUNNING) break;
      if (watch_stall && slot[pi]->iter - iter_at_resume > cycle_limit) {
        out->stalled = true;
        k_mix_set<<<1, 1, 0, s>>>(ms, MIX_FLUSH);  // the queued chunk and what follows skip their work
        c->launches++;
        break;
      }
      if (c->profile) {  // every iteration of chunk k-1 ran: its first matvec is a full launch
        float ms_ = 0.f;
        if (cudaEventElapsedTime(&ms_, F.ev[pi][0], F.ev[pi][1]) == cudaSuccess) {
          c->prof_ms[F.prof_slot] += ms_;
          c->prof_n[F.prof_slot] += 1;
          c->prof_nodes[F.prof_slot] += p->g.nn;
          c->prof_elems[F.prof_slot] += p->n_active;
        }
        if (F.mg && p->mg->T > 1 &&
            cudaEventElapsedTime(&ms_, p->mg->l1ev[pi][0], p->mg->l1ev[pi][1]) == cudaSuccess) {
          c->prof_ms[3] += ms_;
          c->prof_n[3] += 1;
          c->prof_nodes[3] += p->mg->lv[1].nn;
        }
      }
    }
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    MixState* h = slot[0];
    MYCEL_CUDA(c, cudaMemcpyAsync(h, ms, sizeof(MixState), cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    out->iterations = h->iter;
    status = h->status;
    // the latest direction is in p{(m-1)&1} after m iterations since the chunks restarted
    int m = out->iterations - iter_at_resume;
    if (m > 0 && (m & 1)) MYCEL_CUDA(c, cudaMemcpyAsync(F.p1, F.p0, F.es * F.n, cudaMemcpyDeviceToDevice, s));
    // reliable update: u += x; r = P(b - A u) in FP64
    if (F.f64) k_flush_u<double><<<stream_blocks(p), kT, 0, s>>>(p->g, d_u, (double*)F.x);
    else k_flush_u<float><<<stream_blocks(p), kT, 0, s>>>(p->g, d_u, (float*)F.x);
    c->launches++;
    ++out->flushes;
    if ((st = true_residual(p, F, d_b, d_u, &rn))) return st;
    out->rel = rn / bnorm;
    if (verbose)
      std::fprintf(stderr, "mycel: %s refinement %d: inner %d, status %d, recursive %.3e, true %.3e (tol %.1e)\n", name,
                   out->flushes, out->iterations, status, h->rn / bnorm, out->rel, tol);
    if (out->rel <= tol) {
      out->ok = true;
      break;
    }
    cycle_limit = std::max<int64_t>(stall_floor, 3 * (int64_t)out->iterations);
    if (out->stalled || status != MIX_FLUSH || out->iterations >= max_iter) break;
    c->launches += launch_inner_xr(p, F, s, F.p0, 1);
    iter_at_resume = out->iterations;
  }
  return MYCEL_OK;
}

// Refined solve of A u = b (A = P K P + I - P) to ||P(b - A u)|| / ||P b|| <= tol, measured in FP64.
// MYCEL_PRECISION_MIXED: FP32 inner PCG; if it stalls, breaks down or runs out of iterations the solve goes on
// in the fast FP64 form from the refined u, and finally (should that fail too) in the plain FP64 PCG.
// MYCEL_PRECISION_FP64_FACTORED: the fast FP64 form, then the plain FP64 PCG if it does not converge.
// MYCEL_PRECISION_FP64_MG: the multigrid form (where the grid coarsens), then as MYCEL_PRECISION_FP64_FACTORED.
// MYCEL_PRECISION_MIXED_MG: the multigrid form with FP32 outer iteration and FP64 refinement, then as
// MYCEL_PRECISION_FP64_MG.
int32_t refined_solve_entry(mycel_problem* p, const double* d_b, const int32_t* d_nz, int32_t n_nz, double* d_u,
                            double tol, int max_iter, const volatile int32_t* cancel, int precision,
                            mycel_pcg_result* res) {
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
  const bool mixed = precision == MYCEL_PRECISION_MIXED;
  const bool mgp = precision == MYCEL_PRECISION_FP64_MG || precision == MYCEL_PRECISION_MIXED_MG;
  if ((mixed || mgp) && (st = ensure_mixed(p))) return st;
  if ((st = ensure_f64f(p))) return st;  // every refined form measures its true residual with the FP64 operator
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
  // project u and ||P b|| (same kernels as the FP64 path)
  cudaMemsetAsync(p->d_state, 0, sizeof(PcgState), s);
  launch_project_x(p, d_u, &p->d_state->nonzero_x);
  launch_pcg_bnorm(p);
  PcgState* hs = (PcgState*)c->pinned;
  MYCEL_CUDA(c, cudaMemcpyAsync(hs, p->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  const double bnorm = hs->bnorm;
  if (bnorm <= 1e-30) {
    MYCEL_CUDA(c, cudaMemsetAsync(d_u, 0, sizeof(double) * p->g.nd, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    res->converged = 1;
    std::snprintf(res->message, sizeof res->message, "RHS is zero. Solution is zero.");
    return MYCEL_OK;
  }
  const bool verbose = std::getenv("MYCEL_VERBOSE") != nullptr;
  MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));  // bounded-wait failures of this solve only
  LoopOut l32, l64, lmg, lmg32;
  bool ok = false;
  double rel = 0.0;
  bool ran_mg = false;
  if (mgp) {
    bool avail = false;
    if ((st = resolve_mv32(p)) || (st = mg_ensure(p, &avail))) return st;
    if (avail) {
      ran_mg = true;
      if (p->mg->setup_version != p->e_version) {  // solves on an unchanged E (load cases) share the set-up
        mg_setup(p);
        p->mg->setup_version = p->e_version;
      }
      // MYCEL_PRECISION_MIXED_MG: the FP32 outer iteration first (unless one of this problem's solves stalled
      // in it), then the FP64 outer iteration from the refined u
      if (precision == MYCEL_PRECISION_MIXED_MG && !p->mg->prefers_f64) {
        if ((st = refined_loop(p, inner_form_mg(p, false), d_b, d_u, bnorm, tol, max_iter, cancel, true, verbose,
                               &lmg32)))
          return st;
        ok = lmg32.ok;
        rel = lmg32.rel;
        if (lmg32.stalled) p->mg->prefers_f64 = true;
        if (!ok && verbose)
          std::fprintf(stderr, "mycel: FP32 multigrid solve %s after %d iterations (%.3e); FP64 multigrid next\n",
                       lmg32.stalled ? "stalled" : "not converged", lmg32.iterations, lmg32.rel);
      }
      if (!ok) {
        const int budget = lmg32.iterations ? std::max(max_iter - lmg32.iterations, max_iter / 2) : max_iter;
        if ((st = refined_loop(p, inner_form_mg(p, true), d_b, d_u, bnorm, tol, budget, cancel, false, verbose, &lmg)))
          return st;
        ok = lmg.ok;
        rel = lmg.rel;
      }
      if (ok && lmg.iterations + lmg32.iterations == 0 && lmg.flushes + lmg32.flushes == 0)
        std::snprintf(res->message, sizeof res->message, "Initial guess already converged.");
    }
  }
  // Which inner form a mixed solve starts in. Once a mixed solve of a problem has stalled (its designs have
  // become badly conditioned, which in a SIMP run does not go away), its later mixed solves start in the fast
  // FP64 form. Otherwise the FP32 form runs unless the last solves showed it needing more than kCost64 times the
  // fast FP64 form's iterations per decade of residual (kCost64: the cost of a fast FP64 iteration relative to
  // an FP32 one); the second solve of a problem probes the fast FP64 form, and every 16th solve re-probes the
  // form not in use. The choice rests on iteration counts only, so it is the same whatever else runs.
  constexpr double kCost64 = 1.5;
  bool use32 = true;
  if (mixed && !p->mixed_prefers_f64f) {
    const int n = p->mix_solves++;
    if (p->it32_per_dec > 0.0 && p->it64_per_dec > 0.0) use32 = p->it32_per_dec <= kCost64 * p->it64_per_dec;
    if (n == 1) use32 = false;
    else if (n >= 16 && n % 16 == 0) use32 = !use32;
  }
  const bool run32 = mixed && !p->mixed_prefers_f64f && use32;
  if (run32) {
    if ((st = resolve_mv32(p))) return st;
    if ((st = refined_loop(p, inner_form(p, false), d_b, d_u, bnorm, tol, max_iter, cancel, true, verbose, &l32)))
      return st;
    ok = l32.ok;
    rel = l32.rel;
    if (l32.stalled) p->mixed_prefers_f64f = true;
    if (ok && l32.iterations > 0 && l32.rel0 > l32.rel)
      p->it32_per_dec = l32.iterations / std::max(0.1, std::log10(l32.rel0 / l32.rel));
    if (ok && l32.iterations == 0 && l32.flushes == 0)
      std::snprintf(res->message, sizeof res->message, "Initial guess already converged.");
  }
  int remaining = std::max(1, max_iter - l32.iterations);
  if (!ok && ran_mg && verbose)
    std::fprintf(stderr, "mycel: multigrid solve not converged after %d iterations (%.3e); fast FP64 form next\n",
                 lmg.iterations, lmg.rel);
  if (!ok) {
    if ((st = ensure_f64f(p))) return st;
    MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
    if ((st = refined_loop(p, inner_form(p, true), d_b, d_u, bnorm, tol, run32 ? std::max(remaining, max_iter / 2)
                                                                             : max_iter,
                           cancel, false, verbose, &l64)))
      return st;
    ok = l64.ok;
    rel = l64.rel;
    if (mixed && !run32 && ok && l64.iterations > 0 && l64.rel0 > l64.rel)
      p->it64_per_dec = l64.iterations / std::max(0.1, std::log10(l64.rel0 / l64.rel));
    if (verbose && run32)
      std::fprintf(stderr, "mycel: mixed solve went on in fast FP64 (%s after %d inner iterations): %d iterations, %.3e\n",
                   l32.stalled ? "stalled" : "not converged", l32.iterations, l64.iterations, rel);
    if (!run32 && !ran_mg && ok && l64.iterations == 0 && l64.flushes == 0)
      std::snprintf(res->message, sizeof res->message, "Initial guess already converged.");
  }
  int plain_iter = 0;
  if (!ok) {
    mycel_pcg_result r64;
    if ((st = pcg_solve_fp64(p, d_b, d_nz, n_nz, d_u, tol, max_iter, cancel, &r64))) return st;
    plain_iter = r64.iterations;
    ok = r64.converged != 0;
    rel = r64.final_residual;
    if (verbose) std::fprintf(stderr, "mycel: solve finished by the plain FP64 PCG: %d iterations, %.3e\n", plain_iter, rel);
  }
  if (mixed) {
    res->inner_iterations = l32.iterations;
    res->fallback_iterations = l64.iterations + plain_iter;
  } else if (precision == MYCEL_PRECISION_MIXED_MG) {
    res->inner_iterations = lmg32.iterations;
    res->fallback_iterations = lmg.iterations + l64.iterations + plain_iter;
  } else if (mgp) {
    res->inner_iterations = lmg.iterations;
    res->fallback_iterations = l64.iterations + plain_iter;
  } else {
    res->inner_iterations = l64.iterations;
    res->fallback_iterations = plain_iter;
  }
  res->iterations = res->inner_iterations + res->fallback_iterations;
  res->refinement_steps = l32.flushes + l64.flushes + lmg.flushes + lmg32.flushes;
  res->final_residual = rel;
  res->converged = ok ? 1 : 0;
  if (!ok)
    std::snprintf(res->message, sizeof res->message,
                  "PCG reached maximum iterations without converging. Is the model not sufficiently constrained?");
  res->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return MYCEL_OK;
}

// ---------------------------------------------------------------------------------------------------------
// Load cases kept apart, solved together (mixed multigrid form). The cases share K: their outer FP32
// flexible CG iterations run side by side in the same chunk graphs, each with its own state (alpha, beta,
// residual, status), and one V-cycle serves all of them: the voxel-level products run per case, the coarse
// levels (restriction, stencil products, the cluster kernel, prolongation) once for all cases, loading each
// stencil entry once per node. Every case's arithmetic is that of its solve alone.
// A round runs the chunks until no case is running (each has reached its true-residual replacement point or a
// final state); then every case is refined in FP64 (u += x, r = P(b - A u)) and those not yet converged
// restart together. A case that stalls, breaks down or runs out of iterations is finished afterwards, alone,
// by refined_solve_entry from its refined u (FP64 multigrid, then the fast FP64 and plain forms).
// ---------------------------------------------------------------------------------------------------------
static int32_t mg_ensure_cases(mycel_problem* p, int n) {
  MgHier* mg = p->mg;
  auto& cw = mg->cw;
  if (cw.n >= n) return MYCEL_OK;
  if (cw.n > 0 || n > mg->ncap) return set_error(p->ctx, MYCEL_E_ARG, "multigrid case workspace: too many cases");
  cudaStream_t s = p->ctx->stream;
  const size_t fb = sizeof(float) * (size_t)p->g.n32 + 64;
  for (int k = 0; k < n; ++k)
    for (int q = 0; q < 7; ++q) {
      void* b = nullptr;
      if (cudaMallocAsync(&b, fb, s) != cudaSuccess)
        return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the load cases' multigrid workspace");
      cudaMemsetAsync(b, 0, fb, s);
      p->device_bytes += (int64_t)fb;
      mg->bufs.push_back(b);
      cw.v[k][q] = (float*)b;
    }
  void* st = nullptr;
  if (cudaMallocAsync(&st, sizeof(MixState) * n, s) != cudaSuccess)
    return set_error(p->ctx, MYCEL_E_OOM, "out of device memory for the load cases' multigrid workspace");
  cudaMemsetAsync(st, 0, sizeof(MixState) * n, s);
  p->device_bytes += (int64_t)(sizeof(MixState) * n);
  mg->bufs.push_back(st);
  cw.st = (MixState*)st;
  for (int k = 0; k < n; ++k)
    for (int q = 0; q < 4; ++q) {  // r, z, p0, p1 are matvec inputs
      int32_t e = encode_plane_map(p, cw.v[k][1 + q], false, &cw.tmap[k][q]);
      if (e) return e;
      p->case_tmap_ptr[p->n_case_tmaps] = cw.v[k][1 + q];
      p->case_tmap[p->n_case_tmaps] = &cw.tmap[k][q];
      p->n_case_tmaps++;
    }
  cw.n = n;
  return MYCEL_OK;
}

// vector q of case k: 0 x, 1 r, 2 z, 3 p0, 4 p1, 5 ap, 6 t
static float* cwv(MgHier* mg, int k, int q) { return mg->cw.v[k][q]; }

// One outer step of every case (mode 0: after the matvec; 1: after a replacement; 2: start): k_mg_enter32 per
// case, one V-cycle for all, k_mg_exit32 per case. Returns the kernels launched.
static int launch_mg_step_cases(mycel_problem* p, cudaStream_t s, int n, const int* pcur_sel, int mode) {
  MgHier* mg = p->mg;
  const int sb = stream_blocks(p);
  const float* om = mg->sc->omega;
  MgRun R;
  R.n = n;
  R.st = mg->cw.st;
  int nl = 0;
  for (int k = 0; k < n; ++k) {
    float* pcur = cwv(mg, k, 3 + pcur_sel[k]);
    k_mg_enter32<<<sb, kT, 0, s>>>(p->g.n32, cwv(mg, k, 0), cwv(mg, k, 1), pcur, cwv(mg, k, 5), p->d_invdf,
                                   cwv(mg, k, 2), om, R.st + k, p->d_part2, mode);
    R.rf[k] = cwv(mg, k, 1);
    R.xf[k] = cwv(mg, k, 2);
    R.tf[k] = cwv(mg, k, 6);
    nl++;
  }
  nl += mg_vcycle(p, s, R);
  for (int k = 0; k < n; ++k) {
    k_mg_exit32<<<sb, kT, 0, s>>>(p->g.n32, cwv(mg, k, 1), cwv(mg, k, 6), cwv(mg, k, 2), p->d_invdf, cwv(mg, k, 5), om,
                                  R.st + k, p->d_part2, mode);
    nl++;
  }
  return nl;
}

// chunk graphs of the cases (two iterations each; p alternates between p0 and p1 as in the single solve)
static int32_t capture_cases_graph(mycel_problem* p, int n) {
  mycel_ctx* c = p->ctx;
  MgHier* mg = p->mg;
  auto& cw = mg->cw;
  if (cw.graph[0] && cw.graph_profiled == c->profile && cw.graph_n == n) return MYCEL_OK;
  for (int k = 0; k < 2; ++k) {
    if (cw.graph[k]) cudaGraphExecDestroy(cw.graph[k]);
    cw.graph[k] = nullptr;
  }
  cudaStream_t s = c->stream;
  const int64_t before = c->launches;
  for (int g = 0; g < 2; ++g) {
    cudaGraph_t graph;
    MYCEL_CUDA(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int nl = 0;
    for (int t = 0; t < 2; ++t) {
      int sel[kMgMaxCases];
      for (int k = 0; k < n; ++k) {
        float* pcur = cwv(mg, k, (t & 1) ? 4 : 3);
        float* pprev = cwv(mg, k, (t & 1) ? 3 : 4);
        launch_mv32_variant<1>(p, s, nullptr, cwv(mg, k, 2), pprev, pcur, cwv(mg, k, 5), 1, cw.st + k, p->d_part2);
        sel[k] = t & 1;
        nl++;
      }
      nl += launch_mg_step_cases(p, s, n, sel, 0);
    }
    cw.per_chunk = nl;
    MYCEL_CUDA(c, cudaStreamEndCapture(s, &graph));
    MYCEL_CUDA(c, cudaGraphInstantiate(&cw.graph[g], graph, 0));
    cudaGraphDestroy(graph);
  }
  c->launches = before;
  cw.graph_profiled = c->profile;
  cw.graph_n = n;
  return MYCEL_OK;
}

__global__ void k_mix_set_if(MixState* st, int from, int to) {
  if (st->status == from) st->status = to;
}

// Device time of one launch of a solver kernel, measured in place: `reps` launches back to back in one CUDA
// graph (as the chunk graphs issue them), bracketed by CUDA events on the context stream after a warm-up
// launch of the same graph. which 0: the FP32 outer matvec k_mv32f (MODE 1: p = z + beta p_old, K p, p.Ap)
// on the problem's FP32 work vectors with a scratch state; 3: the multigrid level-1 residual product
// (r - A x on level 1). Uses only work vectors that hold nothing between solves.
int32_t kernel_bench(mycel_problem* p, int which, int reps, double* avg_us) {
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  int32_t st = MYCEL_OK;
  if (reps < 1 || (which != 0 && which != 3)) return set_error(c, MYCEL_E_ARG, "kernel_bench: which / reps");
  if ((st = ensure_pcg_workspace(p)) || (st = ensure_mixed(p)) || (st = resolve_mv32(p))) return st;
  MgHier* mg = nullptr;
  if (which == 3) {
    bool avail = false;
    if ((st = mg_ensure(p, &avail))) return st;
    if (!avail || p->mg->T <= 1) return set_error(c, MYCEL_E_ARG, "kernel_bench: no multigrid level 1 on the whole GPU");
    mg = p->mg;
    if (mg->setup_version != p->e_version) {
      mg_setup(p);
      mg->setup_version = p->e_version;
    }
  }
  MixState* ms = nullptr;
  MYCEL_CUDA(c, cudaMallocAsync((void**)&ms, sizeof(MixState), s));
  struct Free {
    MixState* m; cudaStream_t s;
    ~Free() { cudaFreeAsync(m, s); }
  } fr{ms, s};
  const unsigned sb = (unsigned)stream_blocks(p);
  if (which == 0) {  // nonzero directions on the free DOFs, a running state
    k_mg_pow_init<<<sb, 256, 0, s>>>(p->g.n32, p->d_invdf, p->f_z);
    k_mg_pow_init<<<sb, 256, 0, s>>>(p->g.n32, p->d_invdf, p->f_p1);
    k_mix_init<<<1, 1, 0, s>>>(ms, 0.0, INT32_MAX, 1e-3);
  } else {
    const MgLevel& v = mg->lv[1];
    k_mg_pow_init<<<std::min<unsigned>(mg_blocks(v.nd), sb), 256, 0, s>>>(v.nd, v.invd, v.xa);
    k_mg_pow_init<<<std::min<unsigned>(mg_blocks(v.nd), sb), 256, 0, s>>>(v.nd, v.invd, v.r);
  }
  cudaGraph_t graph;
  cudaGraphExec_t exec = nullptr;
  MYCEL_CUDA(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < reps; ++k) {
    if (which == 0) {
      float* pcur = (k & 1) ? p->f_p1 : p->f_p0;
      float* pold = (k & 1) ? p->f_p0 : p->f_p1;
      launch_mv32_variant<1>(p, s, nullptr, p->f_z, pold, pcur, p->f_ap, 1, ms, p->d_part2);
    } else {
      const MgLevel& v = mg->lv[1];
      launch_mg_apply(s, v, mg_one(v.xa), mg_one(v.r), v.invd, mg_one(v.t), 2, nullptr, nullptr, 1);
    }
  }
  MYCEL_CUDA(c, cudaStreamEndCapture(s, &graph));
  cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return set_error(c, MYCEL_E_DEVICE, std::string("kernel_bench: ") + cudaGetErrorString(e));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaGraphLaunch(exec, s);  // warm-up
  cudaEventRecord(e0, s);
  cudaGraphLaunch(exec, s);
  cudaEventRecord(e1, s);
  e = cudaEventSynchronize(e1);
  float ms_ = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(exec);
  c->launches += 2 * (int64_t)reps + 3;
  if (e != cudaSuccess) return set_error(c, MYCEL_E_DEVICE, std::string("kernel_bench: ") + cudaGetErrorString(e));
  *avg_us = 1000.0 * ms_ / reps;
  return MYCEL_OK;
}

bool cases_together_enabled() {
  const char* e = std::getenv("MYCEL_CASES_TOGETHER");  // "0": one case after another (for comparisons)
  return !(e && e[0] == '0');
}

int32_t mg_solve_cases(mycel_problem* p, int ncase, double* d_u, double tol, int max_iter,
                       const volatile int32_t* cancel, mycel_pcg_result* res) {
  mycel_ctx* c = p->ctx;
  cudaStream_t s = c->stream;
  auto t0 = std::chrono::steady_clock::now();
  const int64_t nd = p->g.nd;
  for (int k = 0; k < ncase; ++k) std::memset(res + k, 0, sizeof(mycel_pcg_result));
  if (p->n_active_fixed < 6)
    return set_error(c, MYCEL_E_UNDERCONSTRAINED,
                     "Model has fewer than 6 unique fixed DOFs on active nodes (found " +
                         std::to_string(p->n_active_fixed) +
                         "). At least 6 fixed DOFs are required to prevent rigid body modes in 3D.");
  if (ncase < 1 || ncase > kMgMaxCases) return set_error(c, MYCEL_E_ARG, "batched multigrid solve: case count");
  int32_t st = ensure_pcg_workspace(p);
  if (st || (st = ensure_mixed(p)) || (st = ensure_f64f(p))) return st;
  bool avail = false;
  if ((st = resolve_mv32(p)) || (st = mg_ensure(p, &avail))) return st;
  auto solve_alone = [&](int k, int budget, int precision) -> int32_t {
    const double* b = p->d_case_b + (int64_t)k * nd;
    const int32_t* nz = p->d_case_nz + p->case_nz_off[2 * k + 1];
    return refined_solve_entry(p, b, nz, p->case_nz_cnt[2 * k + 1], d_u + k * nd, tol, budget, cancel, precision,
                               res + k);
  };
  if (!avail || p->mg->prefers_f64 || ncase > p->mg->ncap) {  // no batched form here: one case after another
    for (int k = 0; k < ncase; ++k)
      if ((st = solve_alone(k, max_iter, MYCEL_PRECISION_MIXED_MG))) return st;
    return MYCEL_OK;
  }
  MgHier* mg = p->mg;
  if ((st = mg_ensure_cases(p, ncase))) return st;
  // per case: project u, ||P b||, the true residual; cases with a zero right-hand side or already converged
  // take no part
  double bnorm[kMgMaxCases] = {}, rel[kMgMaxCases] = {};
  bool active[kMgMaxCases] = {}, ok[kMgMaxCases] = {}, stalled[kMgMaxCases] = {};
  int iters[kMgMaxCases] = {}, flushes[kMgMaxCases] = {}, resume[kMgMaxCases] = {};
  double* saved_b = p->d_b;
  int32_t* saved_nz = p->d_bnz;
  int32_t saved_n = p->n_bnz;
  struct Restore {
    mycel_problem* p; double* b; int32_t* nz; int32_t n;
    ~Restore() { p->d_b = b; p->d_bnz = nz; p->n_bnz = n; }
  } restore{p, saved_b, saved_nz, saved_n};
  auto bind = [&](int k) {
    p->d_b = p->d_case_b + (int64_t)k * nd;
    p->d_bnz = p->d_case_nz + p->case_nz_off[2 * k + 1];
    p->n_bnz = p->case_nz_cnt[2 * k + 1];
  };
  auto form = [&](int k) {  // the single-solve form with case k's vectors (for the true residual)
    InnerForm F = inner_form_mg(p, false);
    F.x = cwv(mg, k, 0);
    F.r = cwv(mg, k, 1);
    F.z = cwv(mg, k, 2);
    F.p0 = cwv(mg, k, 3);
    F.p1 = cwv(mg, k, 4);
    F.ap = cwv(mg, k, 5);
    return F;
  };
  MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
  // one stiffness: the hierarchy is rebuilt when E has changed, once for all cases
  if (mg->setup_version != p->e_version) {
    mg_setup(p);
    mg->setup_version = p->e_version;
  }
  PcgState* hs = (PcgState*)c->pinned;
  int nact = 0;
  for (int k = 0; k < ncase; ++k) {
    bind(k);
    double* u = d_u + k * nd;
    cudaMemsetAsync(p->d_state, 0, sizeof(PcgState), s);
    launch_project_x(p, u, &p->d_state->nonzero_x);
    launch_pcg_bnorm(p);
    MYCEL_CUDA(c, cudaMemcpyAsync(hs, p->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    bnorm[k] = hs->bnorm;
    if (bnorm[k] <= 1e-30) {
      MYCEL_CUDA(c, cudaMemsetAsync(u, 0, sizeof(double) * nd, s));
      res[k].converged = 1;
      std::snprintf(res[k].message, sizeof res[k].message, "RHS is zero. Solution is zero.");
      ok[k] = true;
      continue;
    }
    double rn = 0.0;
    if ((st = true_residual(p, form(k), p->d_b, u, &rn))) return st;
    rel[k] = rn / bnorm[k];
    if (rel[k] <= tol) {
      ok[k] = true;
      std::snprintf(res[k].message, sizeof res[k].message, "Initial guess already converged.");
      continue;
    }
    cudaMemsetAsync(cwv(mg, k, 0), 0, sizeof(float) * (size_t)p->g.n32, s);
    k_mix_init<<<1, 1, 0, s>>>(mg->cw.st + k, 0.5 * tol * bnorm[k], max_iter, 1e-3);
    c->launches++;
    active[k] = true;
    ++nact;
  }
  for (int k = 0; k < ncase; ++k)
    if (!active[k]) {  // not running: every batched kernel skips the case
      k_mix_set<<<1, 1, 0, s>>>(mg->cw.st + k, MIX_DONE);
      c->launches++;
    }
  if (nact > 0) {
    if ((st = capture_cases_graph(p, ncase))) return st;
    int sel[kMgMaxCases] = {};
    c->launches += launch_mg_step_cases(p, s, ncase, sel, 2);
  }
  MixState* slot[2] = {(MixState*)((char*)c->pinned + 2048), (MixState*)((char*)c->pinned + 2048 + 2048)};
  static_assert(sizeof(MixState) * kMgMaxCases <= 2048, "pinned state slots");
  cudaEvent_t evs[2];
  cudaEventCreateWithFlags(&evs[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&evs[1], cudaEventDisableTiming);
  struct EvGuard { cudaEvent_t* e; ~EvGuard() { cudaEventDestroy(e[0]); cudaEventDestroy(e[1]); } } evg{evs};
  const int64_t stall_floor = 300;
  int64_t cycle_limit[kMgMaxCases];
  for (int k = 0; k < ncase; ++k) cycle_limit[k] = stall_floor;
  const int64_t cap = (int64_t)max_iter + 64 * 2 + 4096;
  int64_t launched = 0;
  while (nact > 0) {
    // chunks until no case runs (pipelined: chunk k is queued while the states after chunk k-1 are read)
    for (int64_t k = 0;; ++k) {
      if (cancel && *cancel) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
      }
      if (launched > cap) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_TIMEOUT, "batched inner PCG device state did not reach a final status");
      }
      const int gi = (int)(k & 1);
      cudaGraphLaunch(mg->cw.graph[gi], s);
      MYCEL_CUDA(c, cudaGetLastError());
      launched += 2;
      c->launches += mg->cw.per_chunk;
      MYCEL_CUDA(c, cudaMemcpyAsync(slot[gi], mg->cw.st, sizeof(MixState) * ncase, cudaMemcpyDeviceToHost, s));
      MYCEL_CUDA(c, cudaEventRecord(evs[gi], s));
      if (k == 0) continue;
      const int pi = (int)((k - 1) & 1);
      MYCEL_CUDA(c, cudaEventSynchronize(evs[pi]));
      bool running = false;
      for (int q = 0; q < ncase; ++q) {
        if (!active[q] || slot[pi][q].status != MIX_RUNNING) continue;
        if (slot[pi][q].iter - resume[q] > cycle_limit[q]) {  // stalled: stop it (the queued chunk skips it)
          stalled[q] = true;
          k_mix_set_if<<<1, 1, 0, s>>>(mg->cw.st + q, MIX_RUNNING, MIX_FLUSH);
          c->launches++;
          continue;
        }
        running = true;
      }
      if (!running) break;
    }
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    MixState* h = slot[0];
    MYCEL_CUDA(c, cudaMemcpyAsync(h, mg->cw.st, sizeof(MixState) * ncase, cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    bool restart = false;
    for (int k = 0; k < ncase; ++k) {
      if (!active[k]) continue;
      bind(k);
      const int status = h[k].status;
      iters[k] = h[k].iter;
      const int m = iters[k] - resume[k];
      if (m > 0 && (m & 1))
        MYCEL_CUDA(c, cudaMemcpyAsync(cwv(mg, k, 4), cwv(mg, k, 3), sizeof(float) * (size_t)p->g.n32,
                                      cudaMemcpyDeviceToDevice, s));
      k_flush_u<float><<<stream_blocks(p), kT, 0, s>>>(p->g, d_u + k * nd, cwv(mg, k, 0));
      c->launches++;
      ++flushes[k];
      double rn = 0.0;
      if ((st = true_residual(p, form(k), p->d_b, d_u + k * nd, &rn))) return st;
      rel[k] = rn / bnorm[k];
      cycle_limit[k] = std::max<int64_t>(stall_floor, 3 * (int64_t)iters[k]);
      if (rel[k] <= tol) {
        ok[k] = true;
        active[k] = false;
        --nact;
        k_mix_set<<<1, 1, 0, s>>>(mg->cw.st + k, MIX_DONE);
        c->launches++;
      } else if (stalled[k] || status != MIX_FLUSH || iters[k] >= max_iter) {
        active[k] = false;  // finished alone below
        --nact;
        k_mix_set<<<1, 1, 0, s>>>(mg->cw.st + k, MIX_DONE);
        c->launches++;
      } else {
        k_mix_set<<<1, 1, 0, s>>>(mg->cw.st + k, MIX_RUNNING);
        c->launches++;
        resume[k] = iters[k];
        restart = true;
      }
    }
    if (!restart) break;
    // the restarting cases' preconditioned residual after the replacement (the others are not running)
    int sel[kMgMaxCases] = {};
    c->launches += launch_mg_step_cases(p, s, ncase, sel, 1);
  }
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  for (int k = 0; k < ncase; ++k) {
    if (res[k].message[0] && ok[k]) {  // zero right-hand side or converged at the start
      res[k].elapsed_ms = ms;
      continue;
    }
    if (!ok[k]) {  // finished alone from the refined u, as a single solve goes on after its FP32 iteration
      if (stalled[k]) mg->prefers_f64 = true;
      const int budget = std::max(max_iter - iters[k], max_iter / 2);
      if ((st = solve_alone(k, budget, MYCEL_PRECISION_FP64_MG))) return st;
      mycel_pcg_result& r = res[k];
      r.fallback_iterations = r.iterations;
      r.inner_iterations = iters[k];
      r.iterations += iters[k];
      r.refinement_steps += flushes[k];
      continue;
    }
    res[k].inner_iterations = iters[k];
    res[k].iterations = iters[k];
    res[k].refinement_steps = flushes[k];
    res[k].final_residual = rel[k];
    res[k].converged = 1;
    res[k].elapsed_ms = ms;
  }
  return MYCEL_OK;
}

// ---------------------------------------------------------------------------------------------------------
// Packed solves: the FP32 outer iterations of the mixed multigrid form for many problems (and for the load
// cases of each) advance together, every kernel of an outer iteration one launch for all of them. A packed
// launch splits its CTAs between entries (one per right-hand side at the voxel level, one per problem on the
// coarse levels) through a table in device memory: entry e owns the CTAs [starts[e], starts[e + 1]) and holds
// the arguments its launch alone would take, and runs the same kernel body with its CTA number within its
// share. Each share has the CTA decomposition of the launch alone, so every reduction sums the same partials
// in the same order and each right-hand side gets the bits of its solve alone. Problems with different level
// counts are aligned by level index: the step of level l covers the problems whose V-cycle launches level l
// separately (above its cluster kernel). Rounds as for the load cases of one problem (mg_solve_cases): chunks
// of two outer iterations run until no right-hand side is running; then each is refined in FP64 and those not
// converged restart together. A right-hand side that stalls, breaks down or runs out of iterations is
// finished alone from its refined u, as a single solve goes on after its FP32 outer iteration.
// ---------------------------------------------------------------------------------------------------------
// A packed solve runs the factorised FP32 matvec: a problem whose variant the autotuner chose (not the
// caller) goes over to it, with its captured solver graphs dropped (they hold the other variant's launches).
// Its later solves alone then use it too, so alone and packed it computes the same.
static void pack_matvec(mycel_problem* p) {
  if (p->tune_mv32 != 0 || p->mv32 == MYCEL_MV32_FACTORED) return;
  p->mv32 = MYCEL_MV32_FACTORED;
  for (int k = 0; k < 2; ++k) {
    if (p->pcg32_graph[k]) cudaGraphExecDestroy(p->pcg32_graph[k]);
    p->pcg32_graph[k] = nullptr;
    if (MgHier* mg = p->mg) {
      if (mg->graph[k]) cudaGraphExecDestroy(mg->graph[k]);
      if (mg->graph32[k]) cudaGraphExecDestroy(mg->graph32[k]);
      if (mg->cw.graph[k]) cudaGraphExecDestroy(mg->cw.graph[k]);
      mg->graph[k] = mg->graph32[k] = mg->cw.graph[k] = nullptr;
    }
  }
}

constexpr int kPkMaxUnits = 1024;
constexpr int kPkStall = 100;  // state op: a running right-hand side's cycle stalled (replacement point)

// Work lists: a packed launch's CTAs of one entry alone become work items (entry << kPkLbBits | CTA number);
// at the start of each outer iteration k_pk_compact lists the items of the entries whose right-hand sides are
// still running, and the launch's persistent CTAs take the listed items in turn, so the entries that are done
// cost nothing.
constexpr int kPkLbBits = 22;
constexpr unsigned kPkLbMask = (1u << kPkLbBits) - 1;
static_assert(kPkMaxUnits <= (1 << (32 - kPkLbBits)), "entry index field of a work item");

struct PkList {             // the work list of one packed launch
  int n;                    // entries
  const unsigned* starts;   // [n + 1] first CTA of each entry (its launch alone's CTAs), then the total
  MixState* const* est;     // [n] the entry's first state (its cases' states follow)
  const int* enc;           // [n] states of the entry
  unsigned* items;          // [total] listed work items
  unsigned* count;          // items listed
  int after_matvec;         // list only right-hand sides whose next step follows a matvec (pmode 0)
};

// one CTA per list: the running entries' items, in entry order
__global__ void __launch_bounds__(1024) k_pk_compact(const PkList* __restrict__ lists) {
  const PkList& L = lists[blockIdx.x];
  __shared__ unsigned off[kPkMaxUnits + 1];
  __shared__ unsigned char run[kPkMaxUnits];
  for (int e = threadIdx.x; e < L.n; e += blockDim.x) {
    bool r = false;
    for (int k = 0; k < L.enc[e]; ++k)
      r = r || (L.est[e][k].status == MIX_RUNNING && (!L.after_matvec || L.est[e][k].pmode == 0));
    run[e] = r ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int e = 0; e < L.n; ++e) {
      off[e] = acc;
      if (run[e]) acc += L.starts[e + 1] - L.starts[e];
    }
    *L.count = acc;
  }
  __syncthreads();
  for (int e = 0; e < L.n; ++e) {
    if (!run[e]) continue;
    const unsigned nb = L.starts[e + 1] - L.starts[e], o = off[e];
    for (unsigned j = threadIdx.x; j < nb; j += blockDim.x) L.items[o + j] = ((unsigned)e << kPkLbBits) | j;
  }
}

struct alignas(64) PkMv {  // one FP32 matvec (k_mv32f) of a right-hand side
  CUtensorMap ta, tb;
  GridDims g;
  HexOpF op;
  float* pnew;
  float* y;
  const float* E;
  const uint8_t* nf;
  MixState* st;
  double* part;
  int* err;
  int projected, zseg;
  unsigned gx, gy, gz;
};

template <int MODE>
__global__ void __launch_bounds__(FX * FY, 2) k_mv32f_pk(const PkMv* __restrict__ tab, const unsigned* __restrict__ items,
                                                         const unsigned* __restrict__ count) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    __syncthreads();  // the previous tile is done with the shared memory
    const unsigned code = items[w];
    const PkMv* m = tab + (code >> kPkLbBits);
    const unsigned lb = code & kPkLbMask;
    const unsigned gx = m->gx, gy = m->gy;
    __shared__ MvArgs sa;
    __shared__ HexOpF sop;
    __shared__ GridDims sg;
    if (threadIdx.x == 0 && threadIdx.y == 0) {  // the thread that issues the copies; maps written before launch
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&m->ta) : "memory");
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&m->tb) : "memory");
      sop = m->op;
      sg = m->g;
      sa = MvArgs{&sop, &m->ta, &m->tb, m->pnew, m->y, m->E, m->nf, m->st, m->part, m->err, m->projected};
    }
    __syncthreads();
    const int r = mv32f_body<MODE>(sg, sa, m->zseg, (int)(lb % gx), (int)((lb / gx) % gy), (int)(lb / (gx * gy)),
                                   gx * gy * m->gz, lb);
    if (r < 0) break;  // a copy may still be in flight into this CTA's shared memory (uniform: the CTA's result)
  }
}

struct PkVec {  // k_mg_enter32 / k_mg_exit32 of a right-hand side
  int64_t n;
  float *x, *r, *p, *q, *z, *t;
  const float* invd;
  const float* om;
  MixState* st;
  double* part;
  unsigned nb;
};

__global__ void __launch_bounds__(kT) k_mg_enter32_pk(const PkVec* __restrict__ tab, const unsigned* __restrict__ items,
                                                      const unsigned* __restrict__ count, int mode) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    __syncthreads();
    const unsigned code = items[w];
    const PkVec& a = tab[code >> kPkLbBits];
    const int md = mode >= 0 ? mode : *(const volatile int*)&a.st->pmode;
    mg_enter32_body(a.n, a.x, a.r, a.p, a.q, a.invd, a.z, a.om, a.st, a.part, md, code & kPkLbMask, a.nb);
  }
}

__global__ void __launch_bounds__(kT) k_mg_exit32_pk(const PkVec* __restrict__ tab, const unsigned* __restrict__ items,
                                                     const unsigned* __restrict__ count, int mode) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    __syncthreads();
    const unsigned code = items[w];
    const PkVec& a = tab[code >> kPkLbBits];
    const int md = mode >= 0 ? mode : *(const volatile int*)&a.st->pmode;
    mg_exit32_body(a.n, a.r, a.t, a.z, a.invd, a.q, a.om, a.st, a.part, md, code & kPkLbMask, a.nb);
  }
}

struct PkApply {  // a coarse-level product of a problem (all its cases)
  MgDims d;
  const float* S;
  MgPtrs x, r, y;
  const float* invd;
  const float* om;
  const MixState* st;
  int ncase;
};

template <bool MULTI>
__global__ void __launch_bounds__(256) k_mg_apply_nodes_pk(const PkApply* __restrict__ tab,
                                                           const unsigned* __restrict__ items,
                                                           const unsigned* __restrict__ count, int mode) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    const unsigned code = items[w];
    const PkApply& a = tab[code >> kPkLbBits];
    const int64_t nn = mg_nn(a.d);
    int64_t q;
    int c;
    mg_item_case<MULTI>((int64_t)(code & kPkLbMask) * blockDim.x + threadIdx.x, a.ncase, &q, &c);
    if (q >= nn || !mg_running(a.st ? a.st + c : nullptr)) continue;
    mg_apply_node(a.d, mg_ns(a.d), q, a.S, a.x.p[c], a.r.p[c], a.invd, a.y.p[c], mode, mode == 1 ? *a.om : 0.0f);
  }
}

template <bool MULTI>
__global__ void __launch_bounds__(kMgDofThreads) k_mg_apply_pk(const PkApply* __restrict__ tab,
                                                               const unsigned* __restrict__ items,
                                                               const unsigned* __restrict__ count, int mode) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    const unsigned code = items[w];
    const PkApply& a = tab[code >> kPkLbBits];
    const int64_t nn = mg_nn(a.d);
    int64_t q;
    int c;
    mg_item_case<MULTI>((int64_t)(code & kPkLbMask) * 64 + (threadIdx.x & 63), a.ncase, &q, &c);
    if (q >= nn || !mg_running(a.st ? a.st + c : nullptr)) continue;
    mg_apply_row(a.d, mg_ns(a.d), q, (int)(threadIdx.x >> 6), a.S, a.x.p[c], a.r.p[c], a.invd, a.y.p[c], mode,
                 mode == 1 ? *a.om : 0.0f);
  }
}

struct PkRestrict {  // restriction of a problem's level to the next coarser one (all its cases)
  MgDims f, c;
  int pitch, first_sweep, ncase;
  MgPtrs rf, tf, rc, xc;
  const float* invdc;
  const MixState* st;
  const float* om;
};

template <bool PAD, bool MULTI>
__global__ void k_mg_restrict_pk(const PkRestrict* __restrict__ tab,
                                                        const unsigned* __restrict__ items,
                                                        const unsigned* __restrict__ count) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    const unsigned code = items[w];
    const PkRestrict& a = tab[code >> kPkLbBits];
    int64_t q;
    int k;
    mg_item_case<MULTI>((int64_t)(code & kPkLbMask) * blockDim.x + threadIdx.x, a.ncase, &q, &k);
    if (q >= mg_nn(a.c) || !mg_running(a.st ? a.st + k : nullptr)) continue;
    const float omega = a.first_sweep ? *a.om : 0.f;
    mg_restrict_node<PAD>(a.f, a.pitch, a.rf.p[k], a.tf.p[k], a.c, a.invdc, a.rc.p[k], q,
                          a.first_sweep ? a.xc.p[k] : nullptr, omega);
  }
}

struct PkProlong {  // prolongation of a problem's level to the next finer one (all its cases)
  MgDims f, c;
  int pitch, ncase;
  const uint8_t* nf;
  const float* invdf;
  MgPtrs xf, xc;
  const MixState* st;
};

template <bool PAD, bool MULTI>
__global__ void k_mg_prolong_pk(const PkProlong* __restrict__ tab,
                                                       const unsigned* __restrict__ items,
                                                       const unsigned* __restrict__ count) {
  const unsigned cnt = *count;
  for (unsigned w = blockIdx.x; w < cnt; w += gridDim.x) {
    const unsigned code = items[w];
    const PkProlong& a = tab[code >> kPkLbBits];
    int64_t q;
    int k;
    mg_item_case<MULTI>((int64_t)(code & kPkLbMask) * blockDim.x + threadIdx.x, a.ncase, &q, &k);
    if (q >= mg_nn(a.f) || !mg_running(a.st ? a.st + k : nullptr)) continue;
    mg_prolong_node<PAD>(a.f, a.pitch, a.nf, a.invdf, a.xf.p[k], a.c, a.xc.p[k], q);
  }
}

struct PkTail {  // the cluster kernel of a problem's V-cycle (all its cases); one cluster per entry
  MgTail tl;
  const float* om;
  const MixState* st;
  int ncase;
};

template <bool MULTI>
__global__ void __launch_bounds__(kMgTailThreads) k_mg_tail_pk(const PkTail* __restrict__ tab) {
  const PkTail& t = tab[blockIdx.x / kMgTailCtas];
  mg_tail_body<MULTI>(t.tl, t.om, t.st, t.ncase, (int64_t)(blockIdx.x % kMgTailCtas) * blockDim.x + threadIdx.x,
                      (int64_t)kMgTailCtas * blockDim.x, false);
}

// state ops of the right-hand sides (a kernel parameter, so the host may rewrite its copy at once): -1 none,
// kPkStall FLUSH if running, else the new status
struct PkOps {
  int n;
  signed char op[kPkMaxUnits];
};
constexpr int kPkRestart = 101;  // state op: running again, next step a restart (after a replacement)
__global__ void k_pk_set(MixState* const* __restrict__ sts, const __grid_constant__ PkOps o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= o.n || o.op[i] < 0) return;
  MixState* st = sts[i];
  if (o.op[i] == kPkStall) {
    if (st->status == MIX_RUNNING) st->status = MIX_FLUSH;
  } else if (o.op[i] == kPkRestart) {
    st->status = MIX_RUNNING;
    st->pmode = 1;
  } else {
    st->status = o.op[i];
  }
}
__global__ void k_pk_gather(MixState* const* __restrict__ sts, int n, MixState* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = *sts[i];
}
struct PkInit {
  double target;
  int max_iter;
  int op;  // 0: left as it is, 1: a new solve (k_mix_init, next step the start), 2: set done
};
// k_mix_init of the right-hand sides that start a solve (flush factor of the FP32 multigrid form)
__global__ void k_pk_init(MixState* const* __restrict__ sts, const PkInit* __restrict__ in, int n, double flush) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || in[i].op == 0) return;
  if (in[i].op == 2) {
    sts[i]->status = MIX_DONE;
    return;
  }
  MixState s = {};
  s.status = MIX_RUNNING;
  s.target = in[i].target;
  s.max_iter = in[i].max_iter;
  s.first = 1;
  s.flush_factor = flush;
  s.pmode = 2;
  *sts[i] = s;
}

enum PkKind : int { PK_MV0, PK_MV1, PK_ENTER, PK_EXIT, PK_APPLY_DOF, PK_APPLY_NODE, PK_RESTRICT, PK_PROLONG, PK_TAIL };

struct PkLaunch {
  int kind;
  bool pad, multi;
  int mode;  // apply: 1 sweep, 2 residual (enter / exit take the step's mode)
  size_t tab, starts, est, enc, items, count;  // byte offsets in the plan's device arena
  int n;
  unsigned blocks;  // work items when every entry runs (its launches alone's CTAs)
  unsigned grid;    // persistent CTAs of the launch
};

// A right-hand side of a packed solve: its voxel-level FP32 vectors, state, RHS and solution.
struct PkUnit {
  mycel_problem* p;
  int job, k;  // k: load case, -1 the problem's single right-hand side
  float *x, *r, *z, *p0, *p1, *ap, *t;
  const CUtensorMap *tz, *tp0, *tp1;
  MixState* st;
  double* part;
  const double* b;
  const int32_t* bnz;
  int32_t nbnz;
  double* u;
};

struct PackPlan {
  std::vector<uint64_t> key;
  void* arena_alloc = nullptr;
  void* arena = nullptr;        // device tables (128-byte aligned inside arena_alloc)
  size_t arena_bytes = 0;
  int nu = 0;
  MixState** d_sts = nullptr;   // [nu] state pointers (in the arena)
  MixState* d_states = nullptr; // [nu] gathered states
  PkInit* d_init = nullptr;     // [nu]
  std::vector<PkLaunch> mv1[2], enter[2], exitl, vcycle;
  // work lists compacted together at the start of an outer iteration (t = 0, 1) and of a start / restart
  size_t grp_iter[2] = {0, 0}, grp_step = 0;
  int n_iter[2] = {0, 0}, n_step = 0;
  cudaGraphExec_t chunk = nullptr;
  int per_chunk = 0;
};

// packed-solve workspace of a context: the plan of the latest set of right-hand sides and pinned host slots
struct PackWork {
  PackPlan plan;
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  std::vector<void*> part_bufs;  // per-unit partial-sum buffers of the plan (device)
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

static void pk_release_plan(mycel_ctx* c, PackWork* w) {
  PackPlan& P = w->plan;
  if (P.chunk) cudaGraphExecDestroy(P.chunk);
  if (P.arena_alloc) cudaFreeAsync(P.arena_alloc, c->stream);
  for (void* b : w->part_bufs) cudaFreeAsync(b, c->stream);
  w->part_bufs.clear();
  P = PackPlan();
}

void pack_release(mycel_ctx* c) {
  PackWork* w = (PackWork*)c->pack;
  if (!w) return;
  pk_release_plan(c, w);
  if (w->pinned) cudaFreeHost(w->pinned);
  for (cudaEvent_t e : w->ev)
    if (e) cudaEventDestroy(e);
  delete w;
  c->pack = nullptr;
}

// host-side table builder: entries of one packed launch, 64-byte aligned, then their CTA starts
struct PkBuilder {
  std::vector<unsigned char> host;
  bool overflow = false;
  size_t put(const void* src, size_t bytes, size_t align) {
    size_t off = (host.size() + align - 1) & ~(align - 1);
    host.resize(off + bytes);
    std::memcpy(host.data() + off, src, bytes);
    return off;
  }
  template <class T>
  void add(std::vector<PkLaunch>& out, int kind, bool pad, bool multi, int mode, const std::vector<T>& ents,
           const std::vector<unsigned>& nblk, const std::vector<std::pair<MixState*, int>>& es) {
    if (ents.empty()) return;
    PkLaunch L{};
    L.kind = kind;
    L.pad = pad;
    L.multi = multi;
    L.mode = mode;
    L.n = (int)ents.size();
    L.tab = put(ents.data(), sizeof(T) * ents.size(), 64);
    std::vector<unsigned> st(ents.size() + 1);
    std::vector<MixState*> ep(ents.size());
    std::vector<int> ec(ents.size());
    unsigned acc = 0;
    for (size_t e = 0; e < ents.size(); ++e) {
      st[e] = acc;
      acc += nblk[e];
      if (nblk[e] > kPkLbMask) overflow = true;  // a work item holds the CTA number in kPkLbBits bits
      ep[e] = es[e].first;
      ec[e] = es[e].second;
    }
    st[ents.size()] = acc;
    L.blocks = acc;
    L.starts = put(st.data(), sizeof(unsigned) * st.size(), 16);
    L.est = put(ep.data(), sizeof(MixState*) * ep.size(), 16);
    L.enc = put(ec.data(), sizeof(int) * ec.size(), 16);
    std::vector<unsigned> zero(acc + 1, 0u);
    L.items = put(zero.data(), sizeof(unsigned) * acc, 16);
    L.count = put(zero.data(), sizeof(unsigned), 16);
    out.push_back(L);
  }
};

// resident CTAs per SM of a packed kernel (its persistent grid: this times the SMs, at most its work items)
static int pk_resident(int kind, bool pad, bool multi) {
  static std::mutex mu;
  static std::map<int, int> memo;
  const int key = kind * 4 + (pad ? 2 : 0) + (multi ? 1 : 0);
  std::lock_guard<std::mutex> lk(mu);
  auto it = memo.find(key);
  if (it != memo.end()) return it->second;
  int o = 0;
  cudaError_t e = cudaSuccess;
  switch (kind) {
    case PK_MV0: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_mv32f_pk<0>, FX * FY, fac_smem_bytes(0)); break;
    case PK_MV1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_mv32f_pk<1>, FX * FY, fac_smem_bytes(1)); break;
    case PK_ENTER: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_mg_enter32_pk, kT, 0); break;
    case PK_EXIT: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_mg_exit32_pk, kT, 0); break;
    case PK_APPLY_DOF:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, multi ? k_mg_apply_pk<true> : k_mg_apply_pk<false>,
                                                        kMgDofThreads, 0);
      break;
    case PK_APPLY_NODE:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &o, multi ? k_mg_apply_nodes_pk<true> : k_mg_apply_nodes_pk<false>, 256, 0);
      break;
    case PK_RESTRICT:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &o, pad ? (multi ? k_mg_restrict_pk<true, true> : k_mg_restrict_pk<true, false>)
                  : (multi ? k_mg_restrict_pk<false, true> : k_mg_restrict_pk<false, false>), 256, 0);
      break;
    case PK_PROLONG:
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &o, pad ? (multi ? k_mg_prolong_pk<true, true> : k_mg_prolong_pk<true, false>)
                  : (multi ? k_mg_prolong_pk<false, true> : k_mg_prolong_pk<false, false>), 256, 0);
      break;
    default: o = 1;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    o = 1;
  }
  o = std::max(1, o);
  memo[key] = o;
  return o;
}

static void pk_issue(const PackPlan& P, const PkLaunch& L, cudaStream_t s, int step_mode) {
  const char* base = (const char*)P.arena;
  const void* tab = base + L.tab;
  const unsigned* it = (const unsigned*)(base + L.items);
  const unsigned* cn = (const unsigned*)(base + L.count);
  const unsigned g = L.grid;
  switch (L.kind) {
    case PK_MV0:
      k_mv32f_pk<0><<<g, dim3(FX, FY), fac_smem_bytes(0), s>>>((const PkMv*)tab, it, cn);
      break;
    case PK_MV1:
      k_mv32f_pk<1><<<g, dim3(FX, FY), fac_smem_bytes(1), s>>>((const PkMv*)tab, it, cn);
      break;
    case PK_ENTER:
      k_mg_enter32_pk<<<g, kT, 0, s>>>((const PkVec*)tab, it, cn, step_mode);
      break;
    case PK_EXIT:
      k_mg_exit32_pk<<<g, kT, 0, s>>>((const PkVec*)tab, it, cn, step_mode);
      break;
    case PK_APPLY_DOF:
      (L.multi ? k_mg_apply_pk<true> : k_mg_apply_pk<false>)<<<g, kMgDofThreads, 0, s>>>((const PkApply*)tab, it, cn,
                                                                                         L.mode);
      break;
    case PK_APPLY_NODE:
      (L.multi ? k_mg_apply_nodes_pk<true> : k_mg_apply_nodes_pk<false>)<<<g, 256, 0, s>>>((const PkApply*)tab, it,
                                                                                           cn, L.mode);
      break;
    case PK_RESTRICT: {
      auto k = L.pad ? (L.multi ? k_mg_restrict_pk<true, true> : k_mg_restrict_pk<true, false>)
                     : (L.multi ? k_mg_restrict_pk<false, true> : k_mg_restrict_pk<false, false>);
      k<<<g, 256, 0, s>>>((const PkRestrict*)tab, it, cn);
      break;
    }
    case PK_PROLONG: {
      auto k = L.pad ? (L.multi ? k_mg_prolong_pk<true, true> : k_mg_prolong_pk<true, false>)
                     : (L.multi ? k_mg_prolong_pk<false, true> : k_mg_prolong_pk<false, false>);
      k<<<g, 256, 0, s>>>((const PkProlong*)tab, it, cn);
      break;
    }
    case PK_TAIL: {  // one cluster per problem (not listed: a done problem's cluster returns at once)
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(kMgTailCtas * L.n));
      cfg.blockDim = dim3(kMgTailThreads);
      cfg.stream = s;
      cudaLaunchAttribute at{};
      at.id = cudaLaunchAttributeClusterDimension;
      at.val.clusterDim.x = kMgTailCtas;
      at.val.clusterDim.y = 1;
      at.val.clusterDim.z = 1;
      cfg.attrs = &at;
      cfg.numAttrs = 1;
      if (L.multi) cudaLaunchKernelEx(&cfg, k_mg_tail_pk<true>, (const PkTail*)tab);
      else cudaLaunchKernelEx(&cfg, k_mg_tail_pk<false>, (const PkTail*)tab);
      break;
    }
  }
}

// the work lists of a group, compacted on the device (one CTA per list)
static void pk_compact(const PackPlan& P, cudaStream_t s, size_t grp, int n) {
  if (n > 0) k_pk_compact<<<n, 1024, 0, s>>>((const PkList*)((const char*)P.arena + grp));
}

// one outer step of every unit (mode 0: after the matvec, pcur p0 (sel 0) or p1; 1: after a replacement;
// 2: start): k_mg_enter32, the V-cycle, k_mg_exit32, all packed. Returns the launches.
static int pk_step(const PackPlan& P, cudaStream_t s, int mode, int sel) {
  for (const PkLaunch& L : P.enter[sel]) pk_issue(P, L, s, mode);
  for (const PkLaunch& L : P.vcycle) pk_issue(P, L, s, mode);
  for (const PkLaunch& L : P.exitl) pk_issue(P, L, s, mode);
  return (int)(P.enter[sel].size() + P.vcycle.size() + P.exitl.size());
}

// a start (mode 2) or restart (mode 1) step of the units that run, their lists compacted first
static int pk_restart(const PackPlan& P, cudaStream_t s, int mode) {
  pk_compact(P, s, P.grp_step, P.n_step);
  return 1 + pk_step(P, s, mode, 0);
}

// Builds the packed launches of the units (grouped by problem: the units of a problem with load cases are its
// cases 0 .. n-1, in order) and the chunk graph, with the arguments, grids and level order that mg_vcycle,
// launch_mg_step and launch_mv32_variant issue for each problem alone.
static int32_t pk_build(mycel_ctx* c, PackWork* w, std::vector<PkUnit>& units, const std::vector<uint64_t>& key) {
  cudaStream_t s = c->stream;
  pk_release_plan(c, w);
  PackPlan& P = w->plan;
  const int nu = (int)units.size();
  // per-unit partial sums: the matvec's CTA partials and 3 per stream block of k_mg_exit32
  for (PkUnit& u : units) {
    const GridDims& g = u.p->g;
    const int zs = fac_zseg(g, mv32f_resident_per_sm() * c->num_sms);
    const dim3 gr = fac_grid(g, zs);
    const size_t need = std::max<size_t>((size_t)gr.x * gr.y * gr.z, 3 * (size_t)stream_blocks(u.p)) + 64;
    void* b = nullptr;
    if (cudaMallocAsync(&b, sizeof(double) * need, s) != cudaSuccess)
      return set_error(c, MYCEL_E_OOM, "out of device memory for the packed solve's partial sums");
    w->part_bufs.push_back(b);
    u.part = (double*)b;
  }
  PkBuilder B;
  std::vector<MixState*> sts(nu);
  for (int i = 0; i < nu; ++i) sts[i] = units[i].st;
  const size_t o_sts = B.put(sts.data(), sizeof(MixState*) * nu, 64);
  std::vector<MixState> zs_(nu);
  std::memset(zs_.data(), 0, sizeof(MixState) * nu);
  const size_t o_states = B.put(zs_.data(), sizeof(MixState) * nu, 64);
  std::vector<PkInit> ini(nu);
  const size_t o_init = B.put(ini.data(), sizeof(PkInit) * nu, 64);
  auto mv_entry = [&](const PkUnit& u, const CUtensorMap* ta, const CUtensorMap* tb, float* pnew, float* y,
                      MixState* st, double* part, unsigned* nb) {
    mycel_problem* p = u.p;
    PkMv m;
    std::memset(&m, 0, sizeof m);
    m.ta = *ta;
    m.tb = *tb;
    m.g = p->g;
    m.op = p->hexop;
    m.pnew = pnew;
    m.y = y;
    m.E = p->d_Ef;
    m.nf = p->d_nflags;
    m.st = st;
    m.part = part;
    m.err = p->d_err;
    m.projected = 1;
    m.zseg = fac_zseg(p->g, mv32f_resident_per_sm() * c->num_sms);
    const dim3 gr = fac_grid(p->g, m.zseg);
    m.gx = gr.x;
    m.gy = gr.y;
    m.gz = gr.z;
    *nb = gr.x * gr.y * gr.z;
    return m;
  };
  for (int t = 0; t < 2; ++t) {  // outer K p: t = 0 p0 = z + beta p1, t = 1 p1 = z + beta p0
    std::vector<PkMv> e;
    std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
    for (const PkUnit& u : units) {
      unsigned n_ = 0;
      e.push_back(mv_entry(u, u.tz, t ? u.tp0 : u.tp1, t ? u.p1 : u.p0, u.ap, u.st, u.part, &n_));
      nb.push_back(n_);
      es.push_back({u.st, 1});
    }
    B.add(P.mv1[t], PK_MV1, false, false, 1, e, nb, es);
  }
  for (int sel = 0; sel < 2; ++sel) {
    std::vector<PkVec> e;
    std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
    for (const PkUnit& u : units) {
      PkVec v{};
      v.n = u.p->g.n32;
      v.x = u.x;
      v.r = u.r;
      v.p = sel ? u.p1 : u.p0;
      v.q = u.ap;
      v.z = u.z;
      v.t = u.t;
      v.invd = u.p->d_invdf;
      v.om = u.p->mg->sc->omega;
      v.st = u.st;
      v.part = u.part;
      v.nb = (unsigned)stream_blocks(u.p);
      e.push_back(v);
      nb.push_back(v.nb);
      es.push_back({u.st, 1});
    }
    B.add(P.enter[sel], PK_ENTER, false, false, 0, e, nb, es);
    if (sel == 0) B.add(P.exitl, PK_EXIT, false, false, 0, e, nb, es);
  }
  struct Prob {  // a problem: its first unit and case count
    mycel_problem* p;
    int u0, nc;
    const MixState* st;
  };
  std::vector<Prob> probs;
  for (int i = 0; i < nu;) {
    int j = i;
    while (j < nu && units[j].p == units[i].p) ++j;
    probs.push_back({units[i].p, i, j - i, units[i].st});
    i = j;
  }
  auto fine_mv = [&]() {  // t = A z at the voxel level, every unit (MODE 0)
    std::vector<PkMv> e;
    std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
    for (const PkUnit& u : units) {
      unsigned n_ = 0;
      e.push_back(mv_entry(u, u.tz, u.tz, nullptr, u.t, u.st, nullptr, &n_));
      nb.push_back(n_);
      es.push_back({u.st, 1});
    }
    B.add(P.vcycle, PK_MV0, false, false, 0, e, nb, es);
  };
  auto unit_ptrs = [&](const Prob& q, int which) {  // voxel-level vectors of a problem's units: r, t or z
    MgPtrs r{};
    for (int k = 0; k < q.nc; ++k) {
      const PkUnit& u = units[q.u0 + k];
      r.p[k] = which == 0 ? u.r : (which == 1 ? u.t : u.z);
    }
    return r;
  };
  int maxT = 1;
  for (const Prob& q : probs) maxT = std::max(maxT, q.p->mg->T);
  std::vector<std::vector<float*>> xc(probs.size(), std::vector<float*>(kMgMaxLevels, nullptr));
  fine_mv();
  for (int multi = 0; multi < 2; ++multi) {  // voxel grid -> level 1, with level 1's first sweep
    std::vector<PkRestrict> e;
    std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
    for (const Prob& q : probs) {
      if ((q.nc > 1) != (multi == 1)) continue;
      MgHier* mg = q.p->mg;
      const MgLevel& v1 = mg->lv[1];
      PkRestrict a{};
      a.f = mg->lv[0].d;
      a.pitch = q.p->g.rp;
      a.rf = unit_ptrs(q, 0);
      a.tf = unit_ptrs(q, 1);
      a.c = v1.d;
      a.invdc = v1.invd;
      a.rc = lv_ptrs(v1.r, v1.nd, q.nc);
      a.st = q.st;
      a.xc = lv_ptrs(v1.xa, v1.nd, q.nc);
      a.first_sweep = 1 < mg->L - 1 ? 1 : 0;
      a.om = mg->sc->omega + 1;
      a.ncase = q.nc;
      e.push_back(a);
      nb.push_back(mg_blocks(v1.nn * q.nc));
      es.push_back({const_cast<MixState*>(q.st), q.nc});
    }
    B.add(P.vcycle, PK_RESTRICT, true, multi == 1, 0, e, nb, es);
  }
  auto applies = [&](int l, bool down) {  // level l's product of every problem that smooths it separately
    for (int node = 0; node < 2; ++node)
      for (int multi = 0; multi < 2; ++multi) {
        std::vector<PkApply> e;
        std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
        for (size_t qi = 0; qi < probs.size(); ++qi) {
          const Prob& q = probs[qi];
          MgHier* mg = q.p->mg;
          if (l >= mg->T || (q.nc > 1) != (multi == 1)) continue;
          const MgLevel& v = mg->lv[l];
          const bool is_node = !(v.nn * q.nc <= kMgDofMaxNodes);
          if (is_node != (node == 1)) continue;
          PkApply a{};
          a.d = v.d;
          a.S = v.S;
          a.invd = v.invd;
          a.r = lv_ptrs(v.r, v.nd, q.nc);
          a.x = lv_ptrs(v.xa, v.nd, q.nc);                  // down: the restriction's first sweep; up: prolonged
          a.y = lv_ptrs(down ? v.t : v.xb, v.nd, q.nc);      // down: r - A x; up: one sweep into xb
          a.om = mg->sc->omega + l;
          a.st = q.st;
          a.ncase = q.nc;
          e.push_back(a);
          nb.push_back(node ? mg_blocks(v.nn * q.nc) : mg_dof_blocks(v.nn * q.nc));
          es.push_back({const_cast<MixState*>(q.st), q.nc});
        }
        B.add(P.vcycle, node ? PK_APPLY_NODE : PK_APPLY_DOF, false, multi == 1, down ? 2 : 1, e, nb, es);
      }
  };
  for (int l = 1; l < maxT; ++l) {
    applies(l, true);
    for (int multi = 0; multi < 2; ++multi) {  // level l -> l + 1
      std::vector<PkRestrict> e;
      std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
      for (size_t qi = 0; qi < probs.size(); ++qi) {
        const Prob& q = probs[qi];
        MgHier* mg = q.p->mg;
        if (l >= mg->T || (q.nc > 1) != (multi == 1)) continue;
        const MgLevel& v = mg->lv[l];
        const MgLevel& cv = mg->lv[l + 1];
        PkRestrict a{};
        a.f = v.d;
        a.pitch = 0;
        a.rf = lv_ptrs(nullptr, 0, q.nc);
        a.tf = lv_ptrs(v.t, v.nd, q.nc);
        a.c = cv.d;
        a.invdc = cv.invd;
        a.rc = lv_ptrs(cv.r, cv.nd, q.nc);
        a.st = q.st;
        a.xc = lv_ptrs(cv.xa, cv.nd, q.nc);
        a.first_sweep = l + 1 < mg->L - 1 ? 1 : 0;
        a.om = mg->sc->omega + l + 1;
        a.ncase = q.nc;
        e.push_back(a);
        nb.push_back(mg_blocks(cv.nn * q.nc));
        es.push_back({const_cast<MixState*>(q.st), q.nc});
        xc[qi][l] = v.xa;
      }
      B.add(P.vcycle, PK_RESTRICT, false, multi == 1, 0, e, nb, es);
    }
  }
  for (int multi = 0; multi < 2; ++multi) {  // the cluster kernels
    std::vector<PkTail> e;
    std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
    for (size_t qi = 0; qi < probs.size(); ++qi) {
      const Prob& q = probs[qi];
      if ((q.nc > 1) != (multi == 1)) continue;
      MgHier* mg = q.p->mg;
      PkTail t{};
      t.tl = mg->tail;
      t.om = mg->sc->omega;
      t.st = q.st;
      t.ncase = q.nc;
      e.push_back(t);
      nb.push_back(kMgTailCtas);
      es.push_back({const_cast<MixState*>(q.st), q.nc});
      xc[qi][mg->T] = mg->lv[mg->T].xa;
    }
    B.add(P.vcycle, PK_TAIL, false, multi == 1, 0, e, nb, es);
  }
  for (int l = maxT - 1; l >= 1; --l) {
    for (int multi = 0; multi < 2; ++multi) {  // level l + 1 -> l, into xa (the downward sweep's vector)
      std::vector<PkProlong> e;
      std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
      for (size_t qi = 0; qi < probs.size(); ++qi) {
        const Prob& q = probs[qi];
        MgHier* mg = q.p->mg;
        if (l >= mg->T || (q.nc > 1) != (multi == 1)) continue;
        const MgLevel& v = mg->lv[l];
        PkProlong a{};
        a.f = v.d;
        a.pitch = 0;
        a.nf = nullptr;
        a.invdf = v.invd;
        a.xf = lv_ptrs(xc[qi][l], v.nd, q.nc);
        a.c = mg->lv[l + 1].d;
        a.xc = lv_ptrs(xc[qi][l + 1], mg->lv[l + 1].nd, q.nc);
        a.st = q.st;
        a.ncase = q.nc;
        e.push_back(a);
        nb.push_back(mg_blocks(v.nn * q.nc));
        es.push_back({const_cast<MixState*>(q.st), q.nc});
      }
      B.add(P.vcycle, PK_PROLONG, false, multi == 1, 0, e, nb, es);
    }
    applies(l, false);
    for (size_t qi = 0; qi < probs.size(); ++qi)
      if (l < probs[qi].p->mg->T) xc[qi][l] = probs[qi].p->mg->lv[l].xb;  // one sweep: xa -> xb
  }
  for (int multi = 0; multi < 2; ++multi) {  // level 1 -> voxel grid, into each unit's z
    std::vector<PkProlong> e;
    std::vector<unsigned> nb;
    std::vector<std::pair<MixState*, int>> es;
    for (size_t qi = 0; qi < probs.size(); ++qi) {
      const Prob& q = probs[qi];
      if ((q.nc > 1) != (multi == 1)) continue;
      MgHier* mg = q.p->mg;
      PkProlong a{};
      a.f = mg->lv[0].d;
      a.pitch = q.p->g.rp;
      a.nf = q.p->d_nflags;
      a.invdf = nullptr;
      a.xf = unit_ptrs(q, 2);
      a.c = mg->lv[1].d;
      a.xc = lv_ptrs(xc[qi][1], mg->lv[1].nd, q.nc);
      a.st = q.st;
      a.ncase = q.nc;
      e.push_back(a);
      nb.push_back(mg_blocks(mg->lv[0].nn * q.nc));
      es.push_back({const_cast<MixState*>(q.st), q.nc});
    }
    B.add(P.vcycle, PK_PROLONG, true, multi == 1, 0, e, nb, es);
  }
  fine_mv();
  if (B.overflow) return set_error(c, MYCEL_E_ARG, "packed solve: a problem's launch has too many CTAs for a work item");
  // persistent grids: the resident CTAs, at most the work items (the cluster kernels are not persistent)
  for (std::vector<PkLaunch>* v : {&P.mv1[0], &P.mv1[1], &P.enter[0], &P.enter[1], &P.exitl, &P.vcycle})
    for (PkLaunch& L : *v)
      if (L.kind != PK_TAIL)
        L.grid = std::max(1u, std::min<unsigned>(L.blocks, (unsigned)(pk_resident(L.kind, L.pad, L.multi) * c->num_sms)));
  // work-list groups, written once the arena's address is known
  std::vector<const PkLaunch*> gi[2], gs;
  auto listed = [](std::vector<const PkLaunch*>& g, const std::vector<PkLaunch>& v) {
    for (const PkLaunch& L : v)
      if (L.kind != PK_TAIL) g.push_back(&L);
  };
  for (int t = 0; t < 2; ++t) {
    listed(gi[t], P.mv1[t]);
    listed(gi[t], P.enter[t]);
    listed(gi[t], P.vcycle);
    listed(gi[t], P.exitl);
  }
  listed(gs, P.enter[0]);
  listed(gs, P.vcycle);
  listed(gs, P.exitl);
  auto reserve = [&](const std::vector<const PkLaunch*>& g) {
    std::vector<PkList> z(g.size());
    std::memset(z.data(), 0, sizeof(PkList) * z.size());
    return B.put(z.data(), sizeof(PkList) * z.size(), 64);
  };
  for (int t = 0; t < 2; ++t) {
    P.grp_iter[t] = reserve(gi[t]);
    P.n_iter[t] = (int)gi[t].size();
  }
  P.grp_step = reserve(gs);
  P.n_step = (int)gs.size();
  P.arena_bytes = B.host.size();
  MYCEL_CUDA(c, cudaMallocAsync(&P.arena_alloc, P.arena_bytes + 128, s));
  P.arena = (void*)(((uintptr_t)P.arena_alloc + 127) & ~(uintptr_t)127);  // tensor maps: 64-byte aligned
  char* base = (char*)P.arena;
  auto fill = [&](size_t off, const std::vector<const PkLaunch*>& g) {
    for (size_t k = 0; k < g.size(); ++k) {
      const PkLaunch& L = *g[k];
      PkList h{L.n, (const unsigned*)(base + L.starts), (MixState* const*)(base + L.est), (const int*)(base + L.enc),
               (unsigned*)(base + L.items), (unsigned*)(base + L.count), L.kind == PK_MV1 ? 1 : 0};
      std::memcpy(B.host.data() + off + k * sizeof(PkList), &h, sizeof h);
    }
  };
  for (int t = 0; t < 2; ++t) fill(P.grp_iter[t], gi[t]);
  fill(P.grp_step, gs);
  MYCEL_CUDA(c, cudaMemcpyAsync(P.arena, B.host.data(), P.arena_bytes, cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  P.nu = nu;
  P.d_sts = (MixState**)(base + o_sts);
  P.d_states = (MixState*)(base + o_states);
  P.d_init = (PkInit*)(base + o_init);
  P.key = key;
  // chunk graph: two outer iterations of every unit (each starting with its work lists), then the states
  // gathered for one copy
  cudaGraph_t graph;
  MYCEL_CUDA(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int nl = 0;
  for (int t = 0; t < 2; ++t) {
    pk_compact(P, s, P.grp_iter[t], P.n_iter[t]);
    for (const PkLaunch& L : P.mv1[t]) pk_issue(P, L, s, 0);
    // the step each right-hand side takes next: 0 after its matvec; a (re)start of a packed run (1, 2) in the
    // first slot, whose matvec list left it out
    nl += 1 + (int)P.mv1[t].size() + pk_step(P, s, -1, t);
  }
  k_pk_gather<<<(nu + 127) / 128, 128, 0, s>>>(P.d_sts, nu, P.d_states);
  nl++;
  MYCEL_CUDA(c, cudaStreamEndCapture(s, &graph));
  cudaError_t ge = cudaGraphInstantiate(&P.chunk, graph, 0);
  cudaGraphDestroy(graph);
  if (ge != cudaSuccess) return set_error(c, MYCEL_E_DEVICE, std::string("packed chunk graph: ") + cudaGetErrorString(ge));
  P.per_chunk = nl;
  return MYCEL_OK;
}

static int32_t pk_set(mycel_ctx* c, const PackPlan& P, const std::vector<signed char>& op) {
  PkOps o;
  o.n = P.nu;
  std::memset(o.op, -1, sizeof o.op);
  for (int i = 0; i < P.nu; ++i) o.op[i] = op[i];
  k_pk_set<<<(P.nu + 127) / 128, 128, 0, c->stream>>>(P.d_sts, o);
  c->launches++;
  MYCEL_CUDA(c, cudaGetLastError());
  return MYCEL_OK;
}

// The right-hand sides of one problem: its single solve's vectors (ncase 1) or its load cases' (0 .. ncase-1)
static void pk_add_units(mycel_problem* p, int job, int ncase, double* d_u, std::vector<PkUnit>* out) {
  MgHier* mg = p->mg;
  const int64_t nd = p->g.nd;
  for (int k = 0; k < ncase; ++k) {
    PkUnit u{};
    u.p = p;
    u.job = job;
    if (ncase == 1) {
      u.k = -1;
      u.x = p->f_x; u.r = p->f_r; u.z = p->f_z; u.p0 = p->f_p0; u.p1 = p->f_p1; u.ap = p->f_ap; u.t = mg->f_t;
      u.tz = &p->f_tmap[1];
      u.tp0 = &p->f_tmap[2];
      u.tp1 = &p->f_tmap[3];
      u.st = mix_state(p);
      u.b = p->d_b;
      u.bnz = p->d_bnz;
      u.nbnz = p->n_bnz;
      u.u = d_u;
    } else {
      u.k = k;
      u.x = cwv(mg, k, 0); u.r = cwv(mg, k, 1); u.z = cwv(mg, k, 2); u.p0 = cwv(mg, k, 3); u.p1 = cwv(mg, k, 4);
      u.ap = cwv(mg, k, 5); u.t = cwv(mg, k, 6);
      u.tz = &mg->cw.tmap[k][1];
      u.tp0 = &mg->cw.tmap[k][2];
      u.tp1 = &mg->cw.tmap[k][3];
      u.st = mg->cw.st + k;
      u.b = p->d_case_b + (int64_t)k * nd;
      u.bnz = p->d_case_nz + p->case_nz_off[2 * k + 1];
      u.nbnz = p->case_nz_cnt[2 * k + 1];
      u.u = d_u + (int64_t)k * nd;
    }
    out->push_back(u);
  }
}

int32_t mg_solve_packed(mycel_ctx* c, int njobs, PackJob* jobs, const volatile int32_t* cancel) {
  cudaStream_t s = c->stream;
  auto t0 = std::chrono::steady_clock::now();
  int32_t st = MYCEL_OK;
  static std::once_flag smem_once;  // the packed matvec's shared memory above the 48 KB default
  static cudaError_t smem_err = cudaSuccess;
  std::call_once(smem_once, [] {
    cudaError_t a = cudaFuncSetAttribute(k_mv32f_pk<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac_smem_bytes(0));
    cudaError_t b = cudaFuncSetAttribute(k_mv32f_pk<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac_smem_bytes(1));
    smem_err = a != cudaSuccess ? a : b;
  });
  if (smem_err != cudaSuccess)
    return set_error(c, MYCEL_E_DEVICE, std::string("packed matvec shared memory: ") + cudaGetErrorString(smem_err));
  const bool verbose = std::getenv("MYCEL_VERBOSE") != nullptr;
  auto tp = std::chrono::steady_clock::now();
  auto lap = [&](const char* what, int extra) {
    if (!verbose) return;
    cudaStreamSynchronize(s);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "mycel: packed %s %.3f ms (%d)\n", what,
                 std::chrono::duration<double, std::milli>(now - tp).count(), extra);
    tp = now;
  };
  std::vector<PkUnit> units;
  std::vector<char> packed(njobs, 0);
  std::vector<mycel_problem*> need_setup;
  // eligibility; the others are solved alone here, in job order
  for (int j = 0; j < njobs; ++j) {
    PackJob& J = jobs[j];
    mycel_problem* p = J.p;
    for (int k = 0; k < J.ncase; ++k) std::memset(J.res + k, 0, sizeof(mycel_pcg_result));
    if (p->ctx != c) return set_error(c, MYCEL_E_ARG, "packed solve: every problem must belong to the context");
    if (p->n_active_fixed < 6)
      return set_error(c, MYCEL_E_UNDERCONSTRAINED,
                       "Model has fewer than 6 unique fixed DOFs on active nodes (found " +
                           std::to_string(p->n_active_fixed) +
                           "). At least 6 fixed DOFs are required to prevent rigid body modes in 3D.");
    if (J.ncase < 1 || J.ncase > kMgMaxCases) return set_error(c, MYCEL_E_ARG, "packed solve: case count");
    if ((st = ensure_pcg_workspace(p)) || (st = ensure_mixed(p)) || (st = ensure_f64f(p))) return st;
    if (J.ncase > 1 && (st = ensure_cases(p))) return st;
    bool avail = false;
    if ((st = resolve_mv32(p)) || (st = mg_ensure(p, &avail))) return st;
    if (avail) pack_matvec(p);
    bool ok = avail && !p->mg->prefers_f64 && p->mg->sweeps == 1 && p->mv32 == MYCEL_MV32_FACTORED &&
              (J.ncase == 1 || J.ncase <= p->mg->ncap) && (int)units.size() + J.ncase <= kPkMaxUnits;
    for (int i = 0; i < j && ok; ++i) ok = !(packed[i] && jobs[i].p == p);  // one job per problem
    if (ok && J.ncase > 1 && (st = mg_ensure_cases(p, J.ncase))) return st;
    if (!ok) {
      if (J.ncase == 1)
        st = refined_solve_entry(p, p->d_b, p->d_bnz, p->n_bnz, J.d_u, J.tol, J.max_iter, cancel,
                                 MYCEL_PRECISION_MIXED_MG, J.res);
      else
        st = mg_solve_cases(p, J.ncase, J.d_u, J.tol, J.max_iter, cancel, J.res);
      if (st) return st;
      continue;
    }
    packed[j] = 1;
    MgHier* mg = p->mg;
    MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
    if (mg->setup_version != p->e_version) need_setup.push_back(p);
    pk_add_units(p, j, J.ncase, J.d_u, &units);
  }
  // the coarse operators of the packed problems, rebuilt from their new E side by side on the fan's streams
  if (!need_setup.empty()) {
    if ((st = fan_begin(c))) return st;
    for (size_t q = 0; q < need_setup.size(); ++q) {
      fan_use(c, (int)q);
      mg_setup(need_setup[q]);
      need_setup[q]->mg->setup_version = need_setup[q]->e_version;
    }
    fan_end(c);
  }
  const int nu = (int)units.size();
  lap("set-up and unpacked jobs", nu);
  if (nu == 0) return MYCEL_OK;
  if (!c->pack) c->pack = new PackWork();
  PackWork* w = (PackWork*)c->pack;
  const size_t pin_need = (size_t)nu * (2 * sizeof(MixState) + 2 * sizeof(double) + sizeof(PkInit)) + 4096;
  if (w->pinned_bytes < pin_need) {
    if (w->pinned) cudaFreeHost(w->pinned);
    w->pinned = nullptr;
    w->pinned_bytes = 0;
    MYCEL_CUDA(c, cudaMallocHost(&w->pinned, pin_need));
    w->pinned_bytes = pin_need;
  }
  for (int q = 0; q < 2; ++q)
    if (!w->ev[q]) MYCEL_CUDA(c, cudaEventCreateWithFlags(&w->ev[q], cudaEventDisableTiming));
  MixState* slot[2] = {(MixState*)w->pinned, (MixState*)w->pinned + nu};
  double* h_bn = (double*)(slot[1] + nu);
  double* h_rn2 = h_bn + nu;
  PkInit* h_init = (PkInit*)(h_rn2 + nu);
  // the plan of this set of right-hand sides (rebuilt when the set changes)
  std::vector<uint64_t> key;
  for (const PkUnit& u : units) {
    key.push_back(u.p->serial);
    key.push_back((uint64_t)(int64_t)u.k);
  }
  if (w->plan.key != key || !w->plan.chunk) {
    if ((st = pk_build(c, w, units, key))) return st;
  } else {
    for (int i = 0; i < nu; ++i) units[i].part = (double*)w->part_bufs[i];
  }
  PackPlan& P = w->plan;
  lap("plan", P.per_chunk);
  c->packed_rhs += nu;
  struct Saved {
    mycel_problem* p;
    double* b;
    int32_t* nz;
    int32_t n;
  };
  std::vector<Saved> saved;
  for (const PkUnit& u : units)
    if (saved.empty() || saved.back().p != u.p) saved.push_back({u.p, u.p->d_b, u.p->d_bnz, u.p->n_bnz});
  struct RestoreAll {
    std::vector<Saved>* v;
    ~RestoreAll() {
      for (Saved& r : *v) r.p->d_b = r.b, r.p->d_bnz = r.nz, r.p->n_bnz = r.n;
    }
  } restore_all{&saved};
  auto bind = [&](const PkUnit& u) {
    u.p->d_b = const_cast<double*>(u.b);
    u.p->d_bnz = const_cast<int32_t*>(u.bnz);
    u.p->n_bnz = u.nbnz;
  };
  auto form = [&](const PkUnit& u) {
    InnerForm F = inner_form_mg(u.p, false);
    F.x = u.x; F.r = u.r; F.z = u.z; F.p0 = u.p0; F.p1 = u.p1; F.ap = u.ap;
    return F;
  };
  // per unit: project u, ||P b||, the true residual (one wait for all)
  for (int i = 0; i < nu; ++i) {
    const PkUnit& u = units[i];
    mycel_problem* p = u.p;
    bind(u);
    cudaMemsetAsync(p->d_state, 0, sizeof(PcgState), s);
    launch_project_x(p, u.u, &p->d_state->nonzero_x);
    launch_pcg_bnorm(p);
    MYCEL_CUDA(c, cudaMemcpyAsync(h_bn + i, &p->d_state->bnorm, sizeof(double), cudaMemcpyDeviceToHost, s));
    if ((st = true_residual_issue(p, form(u), u.b, u.u, h_rn2 + i))) return st;
  }
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  std::vector<double> bnorm(nu), rel(nu);
  std::vector<char> active(nu, 0), ok(nu, 0), stalled(nu, 0), msg(nu, 0);
  std::vector<int> iters(nu, 0), flushes(nu, 0), resume(nu, 0);
  std::vector<int64_t> cycle_limit(nu, 300);
  const int64_t stall_floor = 300;
  int nact = 0;
  int64_t cap = 0;
  for (int i = 0; i < nu; ++i) {
    const PkUnit& u = units[i];
    PackJob& J = jobs[u.job];
    mycel_pcg_result& r = J.res[u.k < 0 ? 0 : u.k];
    bnorm[i] = h_bn[i];
    h_init[i] = PkInit{0.0, 0, 2};
    if (bnorm[i] <= 1e-30) {
      MYCEL_CUDA(c, cudaMemsetAsync(u.u, 0, sizeof(double) * u.p->g.nd, s));
      r.converged = 1;
      std::snprintf(r.message, sizeof r.message, "RHS is zero. Solution is zero.");
      ok[i] = msg[i] = 1;
      continue;
    }
    rel[i] = std::sqrt(h_rn2[i]) / bnorm[i];
    if (rel[i] <= J.tol) {
      ok[i] = msg[i] = 1;
      r.converged = 1;
      r.final_residual = rel[i];
      std::snprintf(r.message, sizeof r.message, "Initial guess already converged.");
      continue;
    }
    MYCEL_CUDA(c, cudaMemsetAsync(u.x, 0, sizeof(float) * (size_t)u.p->g.n32, s));
    h_init[i] = PkInit{0.5 * J.tol * bnorm[i], J.max_iter, 1};
    active[i] = 1;
    ++nact;
    cap = std::max<int64_t>(cap, (int64_t)J.max_iter + 64 * 2 + 4096);
  }
  MYCEL_CUDA(c, cudaMemcpyAsync(P.d_init, h_init, sizeof(PkInit) * nu, cudaMemcpyHostToDevice, s));
  k_pk_init<<<(nu + 127) / 128, 128, 0, s>>>(P.d_sts, P.d_init, nu, 1e-3);
  c->launches++;
  if (nact > 0) c->launches += pk_restart(P, s, 2);
  lap("initial residuals and start", nact);
  int64_t launched = 0;
  int rounds = 0;
  std::vector<signed char> op(nu, -1);
  while (nact > 0) {
    for (int64_t k = 0;; ++k) {  // chunk k is queued while the states after chunk k-1 are read
      if (cancel && *cancel) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
      }
      if (launched > cap) {
        cudaStreamSynchronize(s);
        return set_error(c, MYCEL_E_TIMEOUT, "packed inner PCG device state did not reach a final status");
      }
      const int gi = (int)(k & 1);
      MYCEL_CUDA(c, cudaGraphLaunch(P.chunk, s));
      launched += 2;
      c->launches += P.per_chunk;
      MYCEL_CUDA(c, cudaMemcpyAsync(slot[gi], P.d_states, sizeof(MixState) * nu, cudaMemcpyDeviceToHost, s));
      MYCEL_CUDA(c, cudaEventRecord(w->ev[gi], s));
      if (k == 0) continue;
      const int pi = (int)((k - 1) & 1);
      MYCEL_CUDA(c, cudaEventSynchronize(w->ev[pi]));
      bool running = false, any_stall = false;
      std::fill(op.begin(), op.end(), (signed char)-1);
      for (int q = 0; q < nu; ++q) {
        if (!active[q] || slot[pi][q].status != MIX_RUNNING) continue;
        if (slot[pi][q].iter - resume[q] > cycle_limit[q]) {  // stalled: stop it (the queued chunk skips it)
          stalled[q] = 1;
          op[q] = kPkStall;
          any_stall = true;
          continue;
        }
        running = true;
      }
      if (any_stall && (st = pk_set(c, P, op))) return st;
      if (!running) break;
    }
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    MixState* h = slot[0];
    k_pk_gather<<<(nu + 127) / 128, 128, 0, s>>>(P.d_sts, nu, P.d_states);  // the live states
    c->launches++;
    MYCEL_CUDA(c, cudaMemcpyAsync(h, P.d_states, sizeof(MixState) * nu, cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    std::vector<int> status(nu, MIX_DONE);
    for (int i = 0; i < nu; ++i) {
      if (!active[i]) continue;
      const PkUnit& u = units[i];
      status[i] = h[i].status;
      iters[i] = h[i].iter;
      const int m = iters[i] - resume[i];
      if (m > 0 && (m & 1))
        MYCEL_CUDA(c, cudaMemcpyAsync(u.p1, u.p0, sizeof(float) * (size_t)u.p->g.n32, cudaMemcpyDeviceToDevice, s));
      k_flush_u<float><<<stream_blocks(u.p), kT, 0, s>>>(u.p->g, u.u, u.x);
      c->launches++;
      ++flushes[i];
      if ((st = true_residual_issue(u.p, form(u), u.b, u.u, h_rn2 + i))) return st;
    }
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    bool restart = false;
    std::fill(op.begin(), op.end(), (signed char)-1);
    for (int i = 0; i < nu; ++i) {
      if (!active[i]) continue;
      const PackJob& J = jobs[units[i].job];
      rel[i] = std::sqrt(h_rn2[i]) / bnorm[i];
      cycle_limit[i] = std::max<int64_t>(stall_floor, 3 * (int64_t)iters[i]);
      if (rel[i] <= J.tol) {
        ok[i] = 1;
        active[i] = 0;
        --nact;
        op[i] = MIX_DONE;
      } else if (stalled[i] || status[i] != MIX_FLUSH || iters[i] >= J.max_iter) {
        active[i] = 0;  // finished alone below
        --nact;
        op[i] = MIX_DONE;
      } else {
        op[i] = MIX_RUNNING;
        resume[i] = iters[i];
        restart = true;
      }
    }
    if ((st = pk_set(c, P, op))) return st;
    lap("round", (int)launched);
    ++rounds;
    if (!restart) break;
    c->launches += pk_restart(P, s, 1);  // the restarting units' preconditioned residual (the others skip)
  }
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  for (int i = 0; i < nu; ++i) {
    const PkUnit& u = units[i];
    PackJob& J = jobs[u.job];
    mycel_pcg_result& r = J.res[u.k < 0 ? 0 : u.k];
    if (msg[i]) {  // zero right-hand side or converged at the start
      r.elapsed_ms = ms;
      continue;
    }
    if (!ok[i]) {  // finished alone from the refined u, as the solve alone goes on after its FP32 iteration
      if (stalled[i]) u.p->mg->prefers_f64 = true;
      const int budget = (u.k < 0 && iters[i] == 0) ? J.max_iter : std::max(J.max_iter - iters[i], J.max_iter / 2);
      if ((st = refined_solve_entry(u.p, u.b, u.bnz, u.nbnz, u.u, J.tol, budget, cancel, MYCEL_PRECISION_FP64_MG, &r)))
        return st;
      r.fallback_iterations = r.iterations;
      r.inner_iterations = iters[i];
      r.iterations += iters[i];
      r.refinement_steps += flushes[i];
      continue;
    }
    r.inner_iterations = iters[i];
    r.iterations = iters[i];
    r.refinement_steps = flushes[i];
    r.final_residual = rel[i];
    r.converged = 1;
    r.elapsed_ms = ms;
  }
  lap("finished alone", rounds);
  if (verbose) {
    std::vector<int> it(iters);
    std::sort(it.begin(), it.end());
    int64_t sum = 0;
    for (int v : it) sum += v;
    std::fprintf(stderr, "mycel: packed outer iterations per right-hand side min %d median %d max %d sum %lld, "
                 "lockstep %lld, rounds %d\n", it.front(), it[it.size() / 2], it.back(), (long long)sum,
                 (long long)launched, rounds);
  }
  return MYCEL_OK;
}

// ---------------------------------------------------------------------------------------------------------
// Asynchronous packed runs (mycel_simp_run_many): the right-hand sides of several problems stay in one packed
// plan for a whole optimisation, and each problem's solves start and end on their own. Every chunk of outer
// iterations advances the right-hand sides that are running; one that stops (replacement point, breakdown,
// iteration limit) is refined in FP64 right after that chunk and restarts with the next one (its restart step
// then runs inside the chunk: the step mode is per right-hand side), so no right-hand side waits for another
// and a problem whose solve has ended goes on to its next SIMP iteration while the others still solve.
// A (re)started right-hand side takes its first matvec in the chunk's second slot (its restart step fills the
// first), so after m outer iterations its latest direction is in p1 when m is odd: it is copied to p0, where
// the next restart's first matvec reads it. Per right-hand side the arithmetic is that of its solve alone.
// ---------------------------------------------------------------------------------------------------------
struct PackRun {
  mycel_ctx* c = nullptr;
  std::vector<PkUnit> units;
  std::vector<mycel_problem*> jp;
  std::vector<int> ju0, jnc;
  std::vector<std::chrono::steady_clock::time_point> jt0;
  // per right-hand side: 0 idle, 1 start issued, 2 running, 3 stopped (refinement issued), 4 converged,
  // 5 finished alone, 6 done at the start (zero right-hand side or converged already)
  std::vector<char> state, stalled, stall_pending;
  std::vector<int> iters, flushes, resume, stop_status, max_iter;
  std::vector<int64_t> cycle_limit;
  std::vector<double> bnorm, rel, tol;
  std::vector<mycel_pcg_result> res;
  double *h_bn = nullptr, *h_rn2 = nullptr;
  MixState* h_st = nullptr;
  PkInit* h_init = nullptr;
};

void pkr_close(PackRun* r) { delete r; }

int32_t pkr_open(mycel_ctx* c, const std::vector<PackRunJob>& jobs, PackRun** out, std::vector<char>* packed) {
  *out = nullptr;
  packed->assign(jobs.size(), 0);
  cudaStream_t s = c->stream;
  int32_t st = MYCEL_OK;
  static std::once_flag smem_once;
  static cudaError_t smem_err = cudaSuccess;
  std::call_once(smem_once, [] {
    cudaError_t a = cudaFuncSetAttribute(k_mv32f_pk<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac_smem_bytes(0));
    cudaError_t b = cudaFuncSetAttribute(k_mv32f_pk<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fac_smem_bytes(1));
    smem_err = a != cudaSuccess ? a : b;
  });
  if (smem_err != cudaSuccess)
    return set_error(c, MYCEL_E_DEVICE, std::string("packed matvec shared memory: ") + cudaGetErrorString(smem_err));
  PackRun* r = new PackRun();
  r->c = c;
  struct Del { PackRun** r; ~Del() { if (*r) delete *r; } } del{&r};
  for (size_t j = 0; j < jobs.size(); ++j) {
    mycel_problem* p = jobs[j].p;
    const int nc = jobs[j].ncase;
    if (nc == 0) {  // not in the mixed multigrid form: stepped alone by the caller
      r->jp.push_back(nullptr);
      r->ju0.push_back((int)r->units.size());
      r->jnc.push_back(0);
      continue;
    }
    if (p->ctx != c) return set_error(c, MYCEL_E_ARG, "packed run: every problem must belong to the context");
    for (size_t i = 0; i < j; ++i)
      if (jobs[i].p == p) return set_error(c, MYCEL_E_ARG, "packed run: one job per problem");
    if (p->n_active_fixed < 6 || nc < 1 || nc > kMgMaxCases)
      return set_error(c, MYCEL_E_ARG, "packed run: a problem the packed form cannot take");
    if ((st = ensure_pcg_workspace(p)) || (st = ensure_mixed(p)) || (st = ensure_f64f(p))) return st;
    if (nc > 1 && (st = ensure_cases(p))) return st;
    bool avail = false;
    if ((st = resolve_mv32(p)) || (st = mg_ensure(p, &avail))) return st;
    if (avail) pack_matvec(p);
    if (!avail || p->mg->prefers_f64 || p->mg->sweeps != 1 || p->mv32 != MYCEL_MV32_FACTORED ||
        (nc > 1 && nc > p->mg->ncap) || (int)r->units.size() + nc > kPkMaxUnits) {
      r->jp.push_back(nullptr);  // stepped alone by the caller
      r->ju0.push_back((int)r->units.size());
      r->jnc.push_back(0);
      continue;
    }
    if (nc > 1 && (st = mg_ensure_cases(p, nc))) return st;
    (*packed)[j] = 1;
    r->jp.push_back(p);
    r->ju0.push_back((int)r->units.size());
    r->jnc.push_back(nc);
    pk_add_units(p, (int)j, nc, jobs[j].d_u, &r->units);
  }
  const int nu = (int)r->units.size();
  if (nu == 0) return set_error(c, MYCEL_E_ARG, "packed run: no problem the packed form can take");
  r->jt0.resize(jobs.size());
  r->state.assign(nu, 0);
  r->stalled.assign(nu, 0);
  r->stall_pending.assign(nu, 0);
  r->iters.assign(nu, 0);
  r->flushes.assign(nu, 0);
  r->resume.assign(nu, 0);
  r->stop_status.assign(nu, MIX_DONE);
  r->max_iter.assign(nu, 0);
  r->cycle_limit.assign(nu, 300);
  r->bnorm.assign(nu, 0.0);
  r->rel.assign(nu, 0.0);
  r->tol.assign(nu, 0.0);
  r->res.assign(nu, mycel_pcg_result{});
  if (!c->pack) c->pack = new PackWork();
  PackWork* w = (PackWork*)c->pack;
  const size_t pin_need = (size_t)nu * (2 * sizeof(MixState) + 2 * sizeof(double) + sizeof(PkInit)) + 4096;
  if (w->pinned_bytes < pin_need) {
    if (w->pinned) cudaFreeHost(w->pinned);
    w->pinned = nullptr;
    w->pinned_bytes = 0;
    MYCEL_CUDA(c, cudaMallocHost(&w->pinned, pin_need));
    w->pinned_bytes = pin_need;
  }
  r->h_st = (MixState*)w->pinned;
  r->h_bn = (double*)(r->h_st + 2 * nu);
  r->h_rn2 = r->h_bn + nu;
  r->h_init = (PkInit*)(r->h_rn2 + nu);
  std::vector<uint64_t> key;
  for (const PkUnit& u : r->units) {
    key.push_back(u.p->serial);
    key.push_back((uint64_t)(int64_t)u.k);
  }
  if (w->plan.key != key || !w->plan.chunk) {
    if ((st = pk_build(c, w, r->units, key))) return st;
  } else {
    for (int i = 0; i < nu; ++i) r->units[i].part = (double*)w->part_bufs[i];
  }
  for (int i = 0; i < nu; ++i) r->h_init[i] = PkInit{0.0, 0, 2};  // nothing runs until its start
  MYCEL_CUDA(c, cudaMemcpyAsync(w->plan.d_init, r->h_init, sizeof(PkInit) * nu, cudaMemcpyHostToDevice, s));
  k_pk_init<<<(nu + 127) / 128, 128, 0, s>>>(w->plan.d_sts, w->plan.d_init, nu, 1e-3);
  c->launches++;
  MYCEL_CUDA(c, cudaStreamSynchronize(s));
  *out = r;
  r = nullptr;
  return MYCEL_OK;
}

static InnerForm pkr_form(const PkUnit& u) {
  InnerForm F = inner_form_mg(u.p, false);
  F.x = u.x; F.r = u.r; F.z = u.z; F.p0 = u.p0; F.p1 = u.p1; F.ap = u.ap;
  return F;
}

// the start of job j's next solve on the context stream: its coarse operators (when E has changed), then per
// right-hand side the projection of u, ||P b|| and the true residual, copied to pinned memory
int32_t pkr_begin(PackRun* r, int j, double tol, int max_iter) {
  mycel_ctx* c = r->c;
  cudaStream_t s = c->stream;
  mycel_problem* p = r->jp[j];
  int32_t st = MYCEL_OK;
  r->jt0[j] = std::chrono::steady_clock::now();
  MYCEL_CUDA(c, cudaMemsetAsync(p->d_err, 0, sizeof(int), s));
  if (p->mg->setup_version != p->e_version) {
    mg_setup(p);
    p->mg->setup_version = p->e_version;
  }
  double* sb = p->d_b;
  int32_t* snz = p->d_bnz;
  const int32_t sn = p->n_bnz;
  for (int i = r->ju0[j]; i < r->ju0[j] + r->jnc[j]; ++i) {
    const PkUnit& u = r->units[i];
    p->d_b = const_cast<double*>(u.b);
    p->d_bnz = const_cast<int32_t*>(u.bnz);
    p->n_bnz = u.nbnz;
    cudaMemsetAsync(p->d_state, 0, sizeof(PcgState), s);
    launch_project_x(p, u.u, &p->d_state->nonzero_x);
    launch_pcg_bnorm(p);
    st = cudaMemcpyAsync(r->h_bn + i, &p->d_state->bnorm, sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess
             ? true_residual_issue(p, pkr_form(u), u.b, u.u, r->h_rn2 + i)
             : set_error(c, MYCEL_E_DEVICE, "packed run: read-back of ||P b||");
    r->tol[i] = tol;
    r->max_iter[i] = max_iter;
    r->state[i] = 1;
    c->packed_rhs++;
    r->res[i] = mycel_pcg_result{};
    if (st) break;
  }
  p->d_b = sb;
  p->d_bnz = snz;
  p->n_bnz = sn;
  return st;
}

// after a synchronisation: the started right-hand sides run, or are done at once
int32_t pkr_after_begin(PackRun* r) {
  mycel_ctx* c = r->c;
  cudaStream_t s = c->stream;
  const int nu = (int)r->units.size();
  bool any = false;
  for (int i = 0; i < nu; ++i) {
    r->h_init[i] = PkInit{0.0, 0, 0};
    if (r->state[i] != 1) continue;
    const PkUnit& u = r->units[i];
    mycel_pcg_result& res = r->res[i];
    r->bnorm[i] = r->h_bn[i];
    r->iters[i] = r->flushes[i] = r->resume[i] = 0;
    r->cycle_limit[i] = 300;
    r->stalled[i] = r->stall_pending[i] = 0;
    if (r->bnorm[i] <= 1e-30) {
      MYCEL_CUDA(c, cudaMemsetAsync(u.u, 0, sizeof(double) * u.p->g.nd, s));
      res.converged = 1;
      std::snprintf(res.message, sizeof res.message, "RHS is zero. Solution is zero.");
      r->state[i] = 6;
      continue;
    }
    r->rel[i] = std::sqrt(r->h_rn2[i]) / r->bnorm[i];
    if (r->rel[i] <= r->tol[i]) {
      res.converged = 1;
      res.final_residual = r->rel[i];
      std::snprintf(res.message, sizeof res.message, "Initial guess already converged.");
      r->state[i] = 6;
      continue;
    }
    MYCEL_CUDA(c, cudaMemsetAsync(u.x, 0, sizeof(float) * (size_t)u.p->g.n32, s));
    r->h_init[i] = PkInit{0.5 * r->tol[i] * r->bnorm[i], r->max_iter[i], 1};
    r->state[i] = 2;
    any = true;
  }
  if (!any) return MYCEL_OK;
  PackPlan& P = ((PackWork*)c->pack)->plan;
  MYCEL_CUDA(c, cudaMemcpyAsync(P.d_init, r->h_init, sizeof(PkInit) * nu, cudaMemcpyHostToDevice, s));
  k_pk_init<<<(nu + 127) / 128, 128, 0, s>>>(P.d_sts, P.d_init, nu, 1e-3);
  c->launches++;
  MYCEL_CUDA(c, cudaGetLastError());
  return MYCEL_OK;
}

// k_mix_init of one job's right-hand sides (kernel parameters: the host may start other jobs at once)
struct PkInitJob {
  int n;
  MixState* st[kMgMaxCases];
  double target[kMgMaxCases];
  int max_iter[kMgMaxCases];
};
__global__ void k_pk_init_job(const __grid_constant__ PkInitJob J, double flush) {
  const int i = threadIdx.x;
  if (i >= J.n || !J.st[i]) return;
  MixState s = {};
  s.status = MIX_RUNNING;
  s.target = J.target[i];
  s.max_iter = J.max_iter[i];
  s.first = 1;
  s.flush_factor = flush;
  s.pmode = 2;
  *J.st[i] = s;
}

int32_t pkr_after_begin_job(PackRun* r, int j) {
  mycel_ctx* c = r->c;
  cudaStream_t s = c->stream;
  PkInitJob J{};
  J.n = r->jnc[j];
  bool any = false;
  for (int q = 0; q < r->jnc[j]; ++q) {
    const int i = r->ju0[j] + q;
    J.st[q] = nullptr;
    if (r->state[i] != 1) continue;
    const PkUnit& u = r->units[i];
    mycel_pcg_result& res = r->res[i];
    r->bnorm[i] = r->h_bn[i];
    r->iters[i] = r->flushes[i] = r->resume[i] = 0;
    r->cycle_limit[i] = 300;
    r->stalled[i] = r->stall_pending[i] = 0;
    if (r->bnorm[i] <= 1e-30) {
      MYCEL_CUDA(c, cudaMemsetAsync(u.u, 0, sizeof(double) * u.p->g.nd, s));
      res.converged = 1;
      std::snprintf(res.message, sizeof res.message, "RHS is zero. Solution is zero.");
      r->state[i] = 6;
      continue;
    }
    r->rel[i] = std::sqrt(r->h_rn2[i]) / r->bnorm[i];
    if (r->rel[i] <= r->tol[i]) {
      res.converged = 1;
      res.final_residual = r->rel[i];
      std::snprintf(res.message, sizeof res.message, "Initial guess already converged.");
      r->state[i] = 6;
      continue;
    }
    MYCEL_CUDA(c, cudaMemsetAsync(u.x, 0, sizeof(float) * (size_t)u.p->g.n32, s));
    J.st[q] = u.st;
    J.target[q] = 0.5 * r->tol[i] * r->bnorm[i];
    J.max_iter[q] = r->max_iter[i];
    r->state[i] = 2;
    any = true;
  }
  if (!any) return MYCEL_OK;
  k_pk_init_job<<<1, 32, 0, s>>>(J, 1e-3);
  c->launches++;
  MYCEL_CUDA(c, cudaGetLastError());
  return MYCEL_OK;
}

bool pkr_running(const PackRun* r) {
  for (char v : r->state)
    if (v == 2) return true;
  return false;
}

// One chunk of every running right-hand side (synchronised); the stopped ones are refined and restarted (or
// end); the jobs whose solves have ended are appended to ended (their results: pkr_result).
int32_t pkr_advance(PackRun* r, const volatile int32_t* cancel, std::vector<int>* ended) {
  mycel_ctx* c = r->c;
  cudaStream_t s = c->stream;
  const int nu = (int)r->units.size();
  PackWork* w = (PackWork*)c->pack;
  PackPlan& P = w->plan;
  int32_t st = MYCEL_OK;
  if (cancel && *cancel) return set_error(c, MYCEL_E_CANCELLED, "The operation was canceled.");
  std::vector<signed char> op(nu, -1);
  bool any_op = false, any_stop = false;
  if (pkr_running(r)) {
    MYCEL_CUDA(c, cudaGraphLaunch(P.chunk, s));
    c->launches += P.per_chunk;
    MYCEL_CUDA(c, cudaMemcpyAsync(r->h_st, P.d_states, sizeof(MixState) * nu, cudaMemcpyDeviceToHost, s));
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    for (int i = 0; i < nu; ++i) {
      if (r->state[i] != 2) continue;
      const MixState& m = r->h_st[i];
      bool stop = m.status != MIX_RUNNING && m.pmode == 0;  // a restart set after this chunk's copy reads pmode 1
      if (!stop) {
        if (r->stall_pending[i]) {  // the chunk after the one that showed the stall ran: stop it
          r->stalled[i] = 1;
          op[i] = kPkStall;
          any_op = stop = true;
        } else if (m.iter - r->resume[i] > r->cycle_limit[i] || (int64_t)m.iter > (int64_t)r->max_iter[i] + 4096) {
          r->stall_pending[i] = 1;
        }
      }
      if (!stop) continue;
      r->iters[i] = m.iter;
      r->stop_status[i] = r->stalled[i] ? MIX_FLUSH : m.status;
      r->state[i] = 3;
      any_stop = true;
    }
    if (any_op && (st = pk_set(c, P, op))) return st;
    for (int i = 0; i < nu; ++i) {
      if (r->state[i] != 3) continue;
      const PkUnit& u = r->units[i];
      const int mm = r->iters[i] - r->resume[i];
      if (mm > 0 && (mm & 1))
        MYCEL_CUDA(c, cudaMemcpyAsync(u.p0, u.p1, sizeof(float) * (size_t)u.p->g.n32, cudaMemcpyDeviceToDevice, s));
      k_flush_u<float><<<stream_blocks(u.p), kT, 0, s>>>(u.p->g, u.u, u.x);
      c->launches++;
      ++r->flushes[i];
      if ((st = true_residual_issue(u.p, pkr_form(u), u.b, u.u, r->h_rn2 + i))) return st;
    }
  }
  if (any_stop) {
    MYCEL_CUDA(c, cudaStreamSynchronize(s));
    std::fill(op.begin(), op.end(), (signed char)-1);
    for (int i = 0; i < nu; ++i) {
      if (r->state[i] != 3) continue;
      r->rel[i] = std::sqrt(r->h_rn2[i]) / r->bnorm[i];
      r->cycle_limit[i] = std::max<int64_t>(300, 3 * (int64_t)r->iters[i]);
      if (r->rel[i] <= r->tol[i]) {
        op[i] = MIX_DONE;
        r->state[i] = 4;
      } else if (r->stalled[i] || r->stop_status[i] != MIX_FLUSH || r->iters[i] >= r->max_iter[i]) {
        op[i] = MIX_DONE;
        r->state[i] = 5;  // finished alone below
      } else {
        op[i] = kPkRestart;
        r->resume[i] = r->iters[i];
        r->stall_pending[i] = 0;
        r->state[i] = 2;
      }
    }
    if ((st = pk_set(c, P, op))) return st;
  }
  for (size_t j = 0; j < r->jp.size(); ++j) {
    if (!r->jp[j]) continue;
    bool live = false, over = true;
    for (int i = r->ju0[j]; i < r->ju0[j] + r->jnc[j]; ++i) {
      live = live || r->state[i] != 0;
      over = over && (r->state[i] >= 4);
    }
    if (!live || !over) continue;
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r->jt0[j]).count();
    for (int i = r->ju0[j]; i < r->ju0[j] + r->jnc[j]; ++i) {
      const PkUnit& u = r->units[i];
      mycel_pcg_result& res = r->res[i];
      if (r->state[i] == 6) {
        res.elapsed_ms = ms;
      } else if (r->state[i] == 5) {  // from the refined u, as the solve alone goes on after its FP32 iteration
        if (r->stalled[i]) u.p->mg->prefers_f64 = true;
        const int mx = r->max_iter[i];
        const int budget = (u.k < 0 && r->iters[i] == 0) ? mx : std::max(mx - r->iters[i], mx / 2);
        if ((st = refined_solve_entry(u.p, u.b, u.bnz, u.nbnz, u.u, r->tol[i], budget, cancel, MYCEL_PRECISION_FP64_MG,
                                      &res)))
          return st;
        res.fallback_iterations = res.iterations;
        res.inner_iterations = r->iters[i];
        res.iterations += r->iters[i];
        res.refinement_steps += r->flushes[i];
        std::vector<signed char> done_op(nu, -1);  // the solve alone used the same state: no chunk may take it
        done_op[i] = MIX_DONE;
        if ((st = pk_set(c, P, done_op))) return st;
      } else {
        res.inner_iterations = r->iters[i];
        res.iterations = r->iters[i];
        res.refinement_steps = r->flushes[i];
        res.final_residual = r->rel[i];
        res.converged = 1;
        res.elapsed_ms = ms;
      }
      r->state[i] = 0;
    }
    ended->push_back((int)j);
  }
  return MYCEL_OK;
}

const mycel_pcg_result* pkr_results(const PackRun* r, int j) { return r->res.data() + r->ju0[j]; }

int32_t mixed_solve_entry(mycel_problem* p, const double* d_b, const int32_t* d_nz, int32_t n_nz, double* d_u,
                          double tol, int max_iter, const volatile int32_t* cancel, mycel_pcg_result* res) {
  return refined_solve_entry(p, d_b, d_nz, n_nz, d_u, tol, max_iter, cancel, MYCEL_PRECISION_MIXED, res);
}

}  // namespace mycel
