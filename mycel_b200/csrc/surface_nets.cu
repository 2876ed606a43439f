// Iso-surface of a density field by constrained Surface Nets, on the device: the port of
// SurfaceNetsExtractor.Extract (src/Mycel.Core/PostProcessing/SurfaceNetsExtractor.cs:31-312), with the same
// vertices, triangles and orders as the reference's sequential code.
//
//   k_sn_pad       the 1-voxel zero-padded copy of the density and its threshold mask (:48-78)
//   k_sn_detect    counts face saddles and corner kisses of the current mask (a pass that finds none changes
//                  nothing, so the common case skips the next kernel)
//   k_sn_compose   MakeWellComposed (:352-435): the reference resolves saddles and kisses in one sequential
//                  lexicographic sweep per pass, each resolution changing the voxels the later checks read.
//                  A check at (px, py, pz) touches only the voxels (px..px+1, py..py+1, pz..pz+1), so two
//                  checks interact only if their positions differ by at most 1 per axis; with
//                  t = px + 2 py + 4 pz every such earlier position has a smaller t and no two positions of
//                  the same t interact. Running the checks wavefront by wavefront in t therefore gives the
//                  sequential result exactly. One thread-block cluster runs all wavefronts of all passes,
//                  with a cluster barrier between wavefronts (its CTAs are co-scheduled).
//   k_sn_cells     one vertex per dual cell with mixed corners (:89-179), the reference's float arithmetic
//                  with every operation rounded (no contraction)
//   k_sn_scan_*    deterministic exclusive prefix sums (vertex numbers in cell order; quad slots in edge order)
//   k_sn_quads     two triangles per sign-changing grid edge, X then Y then Z edges in the reference's loop
//                  orders, split along the shorter diagonal (EmitQuad :314-346)
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "internal.h"

struct mycel_mesh {
  std::vector<float> positions;  // 3 per vertex
  std::vector<int32_t> indices;  // 3 per triangle
  int32_t passes = 0;            // well-composedness passes
  int64_t changes = 0;           // saddle / corner-kiss resolutions
};

namespace mycel {
namespace {

struct SnGrid {
  int nx, ny, nz;
  int64_t sy, sz;  // padded strides
};

__device__ __forceinline__ bool sn_saddle(uint8_t* s, float* rho, float thr, int64_t i00, int64_t i10, int64_t i01,
                                          int64_t i11) {
  const bool s00 = s[i00], s10 = s[i10], s01 = s[i01], s11 = s[i11];
  if (!(s00 == s11 && s10 == s01 && s00 != s10)) return false;
  const int64_t a = s00 ? i10 : i00, b = s00 ? i01 : i11;  // the two empty voxels of the diagonal pair
  const int64_t pick = rho[a] >= rho[b] ? a : b;
  s[pick] = 1;
  if (rho[pick] < thr) rho[pick] = thr;
  return true;
}

__device__ __forceinline__ bool sn_kiss(uint8_t* s, float* rho, float thr, int64_t dA, int64_t dB, int64_t a1,
                                        int64_t a2, int64_t a3, int64_t b1, int64_t b2, int64_t b3) {
  if (!(s[dA] && s[dB])) return false;
  const bool linked = (s[a1] && (s[b1] || s[b2])) || (s[a2] && (s[b1] || s[b3])) || (s[a3] && (s[b2] || s[b3]));
  if (linked) return false;
  s[a1] = 1;
  s[b1] = 1;
  if (rho[a1] < thr) rho[a1] = thr;
  if (rho[b1] < thr) rho[b1] = thr;
  return true;
}

// the three face checks at (x, y, z), in the reference's order (XY, XZ, YZ); returns the resolutions made
__device__ __forceinline__ int sn_faces(const SnGrid& g, uint8_t* s, float* rho, float thr, int64_t x, int64_t y,
                                        int64_t z) {
  const int64_t b = x + y * g.sy + z * g.sz;
  int n = 0;
  if (x < g.nx && y < g.ny && sn_saddle(s, rho, thr, b, b + 1, b + g.sy, b + g.sy + 1)) n++;
  if (x < g.nx && z < g.nz && sn_saddle(s, rho, thr, b, b + 1, b + g.sz, b + g.sz + 1)) n++;
  if (y < g.ny && z < g.nz && sn_saddle(s, rho, thr, b, b + g.sy, b + g.sz, b + g.sz + g.sy)) n++;
  return n;
}

// the corner-kiss check of the 2x2x2 cube at (x, y, z): the first of its four diagonals that needs it
__device__ __forceinline__ int sn_cube(const SnGrid& g, uint8_t* s, float* rho, float thr, int64_t x, int64_t y,
                                       int64_t z) {
  const int64_t c000 = x + y * g.sy + z * g.sz, c100 = c000 + 1, c010 = c000 + g.sy, c110 = c010 + 1;
  const int64_t c001 = c000 + g.sz, c101 = c001 + 1, c011 = c001 + g.sy, c111 = c011 + 1;
  return (sn_kiss(s, rho, thr, c000, c111, c100, c010, c001, c110, c101, c011) ||
          sn_kiss(s, rho, thr, c100, c011, c000, c110, c101, c010, c001, c111) ||
          sn_kiss(s, rho, thr, c010, c101, c000, c110, c011, c100, c001, c111) ||
          sn_kiss(s, rho, thr, c001, c110, c000, c101, c011, c100, c010, c111))
             ? 1
             : 0;
}

__global__ void k_sn_pad(SnGrid g, const float* __restrict__ in, float thr, float* __restrict__ rho,
                         uint8_t* __restrict__ s) {
  const int64_t P = g.sz * (g.nz + 2);
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t z = p / g.sz, y = (p / g.sy) % (g.ny + 2), x = p % g.sy;
    float v = 0.0f;
    if (x >= 1 && x <= g.nx && y >= 1 && y <= g.ny && z >= 1 && z <= g.nz)
      v = in[(x - 1) + (int64_t)g.nx * ((y - 1) + (int64_t)g.ny * (z - 1))];
    rho[p] = v;
    s[p] = v >= thr;
  }
}

// candidates in the current mask (read only): saddle faces and cubes whose kiss check would resolve
__global__ void k_sn_detect(SnGrid g, const uint8_t* __restrict__ s, unsigned long long* count) {
  const int64_t N = (int64_t)g.nx * g.ny * g.nz;
  unsigned long long c = 0;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = 1 + q % g.nx, y = 1 + (q / g.nx) % g.ny, z = 1 + q / ((int64_t)g.nx * g.ny);
    const int64_t b = x + y * g.sy + z * g.sz;
    auto sad = [&](int64_t i00, int64_t i10, int64_t i01, int64_t i11) {
      return s[i00] == s[i11] && s[i10] == s[i01] && s[i00] != s[i10];
    };
    if (x < g.nx && y < g.ny && sad(b, b + 1, b + g.sy, b + g.sy + 1)) c++;
    if (x < g.nx && z < g.nz && sad(b, b + 1, b + g.sz, b + g.sz + 1)) c++;
    if (y < g.ny && z < g.nz && sad(b, b + g.sy, b + g.sz, b + g.sz + g.sy)) c++;
    if (x < g.nx && y < g.ny && z < g.nz) {
      const int64_t c000 = b, c100 = b + 1, c010 = b + g.sy, c110 = c010 + 1;
      const int64_t c001 = b + g.sz, c101 = c001 + 1, c011 = c001 + g.sy, c111 = c011 + 1;
      auto kiss = [&](int64_t dA, int64_t dB, int64_t a1, int64_t a2, int64_t a3, int64_t b1, int64_t b2,
                      int64_t b3) {
        return s[dA] && s[dB] &&
               !((s[a1] && (s[b1] || s[b2])) || (s[a2] && (s[b1] || s[b3])) || (s[a3] && (s[b2] || s[b3])));
      };
      if (kiss(c000, c111, c100, c010, c001, c110, c101, c011) || kiss(c100, c011, c000, c110, c101, c010, c001, c111) ||
          kiss(c010, c101, c000, c110, c011, c100, c001, c111) || kiss(c001, c110, c000, c101, c011, c100, c010, c111))
        c++;
    }
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

constexpr int kSnCtas = 8, kSnThreads = 1024;

__device__ __forceinline__ void sn_cluster_sync() {
  asm volatile("barrier.cluster.arrive.release;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory");
}

// MakeWellComposed: passes until one changes nothing (at most 8). flags[k] collects "pass k changed"
// (zeroed by the caller); out[0] = passes run, out[1] = resolutions made.
__global__ void __cluster_dims__(kSnCtas, 1, 1) __launch_bounds__(kSnThreads)
    k_sn_compose(SnGrid g, uint8_t* s, float* rho, float thr, int* flags, long long* out) {
  __shared__ int cta_changes;
  const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, gs = (int64_t)gridDim.x * blockDim.x;
  const int64_t pairs = (int64_t)g.ny * g.nz;
  long long mine = 0;
  int pass = 0;
  for (; pass < 8; ++pass) {
    if (threadIdx.x == 0) cta_changes = 0;
    __syncthreads();
    int local = 0;
    // face checks at x in [1, nx], y in [1, ny], z in [1, nz], wavefront t = x + 2y + 4z
    for (int64_t t = 7; t <= (int64_t)g.nx + 2 * g.ny + 4 * g.nz; ++t) {
      for (int64_t q = gt; q < pairs; q += gs) {
        const int64_t y = 1 + q % g.ny, z = 1 + q / g.ny, x = t - 2 * y - 4 * z;
        if (x >= 1 && x <= g.nx) local += sn_faces(g, s, rho, thr, x, y, z);
      }
      sn_cluster_sync();
    }
    // corner-kiss checks at x in [1, nx-1], y in [1, ny-1], z in [1, nz-1]
    if (g.nx > 1 && g.ny > 1 && g.nz > 1) {
      const int64_t kp = (int64_t)(g.ny - 1) * (g.nz - 1);
      for (int64_t t = 7; t <= (int64_t)(g.nx - 1) + 2 * (g.ny - 1) + 4 * (g.nz - 1); ++t) {
        for (int64_t q = gt; q < kp; q += gs) {
          const int64_t y = 1 + q % (g.ny - 1), z = 1 + q / (g.ny - 1), x = t - 2 * y - 4 * z;
          if (x >= 1 && x <= g.nx - 1) local += sn_cube(g, s, rho, thr, x, y, z);
        }
        sn_cluster_sync();
      }
    }
    mine += local;
    if (local) atomicAdd(&cta_changes, local);
    __syncthreads();
    if (threadIdx.x == 0 && cta_changes) atomicOr(&flags[pass], 1);
    sn_cluster_sync();
    const int changed = *(volatile int*)&flags[pass];
    if (!changed) break;
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd((unsigned long long*)&out[1], (unsigned long long)mine);
  if (gt == 0) out[0] = pass < 8 ? pass + 1 : 8;
}

// one vertex per dual cell with mixed corners: flag[c] = 1 and its world position in tmp[3c..3c+2]
__global__ void k_sn_cells(SnGrid g, const float* __restrict__ rho, const uint8_t* __restrict__ s, float thr,
                           float h, float ox, float oy, float oz, int32_t* __restrict__ flag, float* __restrict__ tmp) {
  const int64_t CX = g.nx + 1, CY = g.ny + 1, C = CX * CY * (g.nz + 1);
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cx = c % CX, cy = (c / CX) % CY, cz = c / (CX * CY);
    float cr[8];
    bool cs[8];
    int mask = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int64_t p = (cx + (k & 1)) + g.sy * (cy + ((k >> 1) & 1)) + g.sz * (cz + (k >> 2));
      cr[k] = rho[p];
      cs[k] = s[p];
      if (cs[k]) mask |= 1 << k;
    }
    if (mask == 0 || mask == 255) {
      flag[c] = 0;
      continue;
    }
    // the 12 cube edges in the reference's order: 4 x-directed, 4 y-directed, 4 z-directed
    const int ea[12] = {0, 2, 4, 6, 0, 1, 4, 5, 0, 1, 2, 3};
    const int eb[12] = {1, 3, 5, 7, 2, 3, 6, 7, 4, 5, 6, 7};
    float sx = 0.f, sy = 0.f, sz = 0.f;
    int cnt = 0;
#pragma unroll
    for (int e = 0; e < 12; ++e) {
      const int a = ea[e], b = eb[e];
      if (cs[a] == cs[b]) continue;
      const float va = cr[a], vb = cr[b];
      const float den = __fsub_rn(vb, va);
      float al = 0.5f;
      if (fabsf(den) > 1e-12f) {
        al = __fdiv_rn(__fsub_rn(thr, va), den);
        al = al < 0.05f ? 0.05f : (al > 0.95f ? 0.95f : al);
      }
      const float ax = (a & 1) - 0.5f, ay = ((a >> 1) & 1) - 0.5f, az = (a >> 2) - 0.5f;
      const float bx = (b & 1) - 0.5f, by = ((b >> 1) & 1) - 0.5f, bz = (b >> 2) - 0.5f;
      sx = __fadd_rn(sx, __fadd_rn(ax, __fmul_rn(al, __fsub_rn(bx, ax))));
      sy = __fadd_rn(sy, __fadd_rn(ay, __fmul_rn(al, __fsub_rn(by, ay))));
      sz = __fadd_rn(sz, __fadd_rn(az, __fmul_rn(al, __fsub_rn(bz, az))));
      cnt++;
    }
    float lx = 0.f, ly = 0.f, lz = 0.f;
    if (cnt > 0) {
      const float fc = (float)cnt;
      lx = __fdiv_rn(sx, fc);
      ly = __fdiv_rn(sy, fc);
      lz = __fdiv_rn(sz, fc);
    }
    flag[c] = 1;
    tmp[3 * c] = __fadd_rn(ox, __fmul_rn(__fadd_rn((float)cx, lx), h));
    tmp[3 * c + 1] = __fadd_rn(oy, __fmul_rn(__fadd_rn((float)cy, ly), h));
    tmp[3 * c + 2] = __fadd_rn(oz, __fmul_rn(__fadd_rn((float)cz, lz), h));
  }
}

// Exclusive prefix sum of int32 flags in place (deterministic): blocks of 1024 scan themselves and store their
// totals, one CTA scans the totals, then every block adds its offset. total receives the sum.
constexpr int kScanBlock = 1024;

__device__ __forceinline__ int32_t sn_block_exclusive(int32_t v, int32_t* warp_tot, int32_t* block_total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    int32_t t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
    int32_t ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t u = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += u;
    }
    if (lane < (int)(blockDim.x >> 5)) warp_tot[lane] = ti - t;
    if (lane == 31) *block_total = ti;
  }
  __syncthreads();
  return inc - v + warp_tot[w];
}

__global__ void __launch_bounds__(kScanBlock) k_sn_scan_blocks(int32_t* __restrict__ a, int64_t n,
                                                              int32_t* __restrict__ sums) {
  __shared__ int32_t wt[32];
  __shared__ int32_t bt;
  const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  const int32_t v = i < n ? a[i] : 0;
  const int32_t ex = sn_block_exclusive(v, wt, &bt);
  if (i < n) a[i] = ex;
  if (threadIdx.x == 0) sums[blockIdx.x] = bt;
}

__global__ void __launch_bounds__(kScanBlock) k_sn_scan_sums(int32_t* __restrict__ sums, int64_t nb,
                                                            long long* __restrict__ total) {
  __shared__ int32_t wt[32];
  __shared__ int32_t bt;
  long long carry = 0;
  for (int64_t base = 0; base < nb; base += kScanBlock) {
    const int64_t i = base + threadIdx.x;
    const int32_t v = i < nb ? sums[i] : 0;
    const int32_t ex = sn_block_exclusive(v, wt, &bt);
    if (i < nb) sums[i] = (int32_t)(carry + ex);
    carry += bt;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_sn_scan_add(int32_t* __restrict__ a, int64_t n, const int32_t* __restrict__ sums) {
  const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  if (i < n) a[i] += sums[blockIdx.x];
}

// vertex numbers: vidx[c] = number of the cell's vertex or -1; positions compacted in cell order
__global__ void k_sn_compact(int64_t C, const int32_t* __restrict__ flag_in, const int32_t* __restrict__ ex,
                             const float* __restrict__ tmp, int32_t* __restrict__ vidx, float* __restrict__ pos) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
    if (flag_in[c]) {
      const int32_t v = ex[c];
      vidx[c] = v;
      pos[3 * (int64_t)v] = tmp[3 * c];
      pos[3 * (int64_t)v + 1] = tmp[3 * c + 1];
      pos[3 * (int64_t)v + 2] = tmp[3 * c + 2];
    } else {
      vidx[c] = -1;
    }
  }
}

// Grid edge e in the reference's emission order: x-directed edges (z in [1,nz], y in [1,ny], x in [0,nx]), then
// y-directed (z in [1,nz], y in [0,ny], x in [1,nx]), then z-directed (z in [0,nz], y in [1,ny], x in [1,nx]).
// Gives the two padded voxels and the four cells (v0..v3 before any flip) of the edge.
struct SnEdge {
  int64_t p0, p1;
  int64_t c[4];
};

__device__ __forceinline__ SnEdge sn_edge(const SnGrid& g, int64_t e) {
  const int64_t nx = g.nx, ny = g.ny, nz = g.nz, CX = nx + 1, CY = ny + 1;
  const int64_t EX = nz * ny * (nx + 1), EY = nz * (ny + 1) * nx;
  auto cell = [&](int64_t x, int64_t y, int64_t z) { return x + CX * (y + CY * z); };
  SnEdge r;
  if (e < EX) {
    const int64_t x = e % (nx + 1), y = 1 + (e / (nx + 1)) % ny, z = 1 + e / ((nx + 1) * ny);
    r.p0 = x + y * g.sy + z * g.sz;
    r.p1 = r.p0 + 1;
    r.c[0] = cell(x, y - 1, z - 1);
    r.c[1] = cell(x, y, z - 1);
    r.c[2] = cell(x, y, z);
    r.c[3] = cell(x, y - 1, z);
  } else if (e < EX + EY) {
    const int64_t f = e - EX;
    const int64_t x = 1 + f % nx, y = (f / nx) % (ny + 1), z = 1 + f / (nx * (ny + 1));
    r.p0 = x + y * g.sy + z * g.sz;
    r.p1 = r.p0 + g.sy;
    r.c[0] = cell(x - 1, y, z - 1);
    r.c[1] = cell(x - 1, y, z);
    r.c[2] = cell(x, y, z);
    r.c[3] = cell(x, y, z - 1);
  } else {
    const int64_t f = e - EX - EY;
    const int64_t x = 1 + f % nx, y = 1 + (f / nx) % ny, z = f / (nx * ny);
    r.p0 = x + y * g.sy + z * g.sz;
    r.p1 = r.p0 + g.sz;
    r.c[0] = cell(x - 1, y - 1, z);
    r.c[1] = cell(x, y - 1, z);
    r.c[2] = cell(x, y, z);
    r.c[3] = cell(x - 1, y, z);
  }
  return r;
}

__global__ void k_sn_edge_flags(SnGrid g, int64_t E, const uint8_t* __restrict__ s, const int32_t* __restrict__ vidx,
                                int32_t* __restrict__ flag) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const SnEdge r = sn_edge(g, e);
    const bool emit = s[r.p0] != s[r.p1] && vidx[r.c[0]] >= 0 && vidx[r.c[1]] >= 0 && vidx[r.c[2]] >= 0 &&
                      vidx[r.c[3]] >= 0;
    flag[e] = emit ? 1 : 0;
  }
}

__device__ __forceinline__ float sn_d2(const float* __restrict__ pos, int32_t i, int32_t j) {
  const float dx = __fsub_rn(pos[3 * (int64_t)i], pos[3 * (int64_t)j]);
  const float dy = __fsub_rn(pos[3 * (int64_t)i + 1], pos[3 * (int64_t)j + 1]);
  const float dz = __fsub_rn(pos[3 * (int64_t)i + 2], pos[3 * (int64_t)j + 2]);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// flag_in: emit flags (before the scan), slot: their exclusive prefix sums (quad numbers)
__global__ void k_sn_quads(SnGrid g, int64_t E, const uint8_t* __restrict__ s, const int32_t* __restrict__ vidx,
                           const float* __restrict__ pos, const int32_t* __restrict__ slot,
                           int32_t* __restrict__ idx) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const SnEdge r = sn_edge(g, e);
    if (s[r.p0] == s[r.p1]) continue;
    int32_t v0 = vidx[r.c[0]], v1 = vidx[r.c[1]], v2 = vidx[r.c[2]], v3 = vidx[r.c[3]];
    if (v0 < 0 || v1 < 0 || v2 < 0 || v3 < 0) continue;
    if (!s[r.p0]) {  // flip: the solid side is the edge's far voxel
      const int32_t t = v1;
      v1 = v3;
      v3 = t;
    }
    int32_t* o = idx + 6 * (int64_t)slot[e];
    if (sn_d2(pos, v0, v2) <= sn_d2(pos, v1, v3)) {
      o[0] = v0; o[1] = v1; o[2] = v2; o[3] = v0; o[4] = v2; o[5] = v3;
    } else {
      o[0] = v0; o[1] = v1; o[2] = v3; o[3] = v1; o[4] = v2; o[5] = v3;
    }
  }
}

// ---- TaubinSmoother.Smooth (PostProcessing/TaubinSmoother.cs:15-134) ----
// Neighbour lists: each triangle adds (i1, i2) to i0, (i2, i0) to i1, (i0, i1) to i2 (slots taken with atomics;
// the order does not matter because each list is then sorted), then sorted and de-duplicated per vertex, the
// vertex itself dropped except as the first entry, as in the reference.
__global__ void k_tb_check(int64_t ni, const int32_t* __restrict__ idx, int64_t nv, int* bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ni; i += (int64_t)gridDim.x * blockDim.x)
    if (idx[i] < 0 || idx[i] >= nv) *bad = 1;
}

__global__ void k_tb_degree(int64_t nt, const int32_t* __restrict__ idx, int32_t* deg) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
    atomicAdd(&deg[idx[3 * t]], 2);
    atomicAdd(&deg[idx[3 * t + 1]], 2);
    atomicAdd(&deg[idx[3 * t + 2]], 2);
  }
}

__global__ void k_tb_fill(int64_t nt, const int32_t* __restrict__ idx, int32_t* cursor, int32_t* __restrict__ nb) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = idx[3 * t], b = idx[3 * t + 1], c = idx[3 * t + 2];
    int32_t k = atomicAdd(&cursor[a], 2);
    nb[k] = b; nb[k + 1] = c;
    k = atomicAdd(&cursor[b], 2);
    nb[k] = c; nb[k + 1] = a;
    k = atomicAdd(&cursor[c], 2);
    nb[k] = a; nb[k + 1] = b;
  }
}

// sort (insertion: lists are short) and de-duplicate each vertex's list in place; cnt[v] = unique count
__global__ void k_tb_sort(int64_t nv, const int32_t* __restrict__ off, const int32_t* __restrict__ deg,
                          int32_t* __restrict__ nb, int32_t* __restrict__ cnt) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t s0 = off[v], len = deg[v];
    if (len == 0) {
      cnt[v] = 0;
      continue;
    }
    int32_t* l = nb + s0;
    for (int32_t i = 1; i < len; ++i) {
      const int32_t x = l[i];
      int32_t j = i - 1;
      while (j >= 0 && l[j] > x) {
        l[j + 1] = l[j];
        --j;
      }
      l[j + 1] = x;
    }
    int32_t d = 1;
    for (int32_t k = 1; k < len; ++k)
      if (l[k] != l[d - 1] && l[k] != (int32_t)v) l[d++] = l[k];
    cnt[v] = d;
  }
}

// dst[v] = p + (factor / count) * sum over the sorted neighbours q of (q - p), every operation rounded
__global__ void k_tb_step(int64_t nv, const float* __restrict__ src, float* __restrict__ dst,
                          const int32_t* __restrict__ off, const int32_t* __restrict__ cnt,
                          const int32_t* __restrict__ nb, float factor) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const float px = src[3 * v], py = src[3 * v + 1], pz = src[3 * v + 2];
    const int32_t c = cnt[v];
    if (c == 0) {
      dst[3 * v] = px; dst[3 * v + 1] = py; dst[3 * v + 2] = pz;
      continue;
    }
    const int32_t* l = nb + off[v];
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int32_t k = 0; k < c; ++k) {
      const int64_t q = l[k];
      sx = __fadd_rn(sx, __fsub_rn(src[3 * q], px));
      sy = __fadd_rn(sy, __fsub_rn(src[3 * q + 1], py));
      sz = __fadd_rn(sz, __fsub_rn(src[3 * q + 2], pz));
    }
    const float w = __fdiv_rn(factor, (float)c);
    dst[3 * v] = __fadd_rn(px, __fmul_rn(w, sx));
    dst[3 * v + 1] = __fadd_rn(py, __fmul_rn(w, sy));
    dst[3 * v + 2] = __fadd_rn(pz, __fmul_rn(w, sz));
  }
}

int sn_grid_blocks(int64_t n, int num_sms) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms * 16));
}

// exclusive scan of n int32 flags in place; *total (device) receives their sum
int32_t sn_scan(mycel_ctx* c, int32_t* a, int64_t n, int32_t* sums, long long* total) {
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  k_sn_scan_blocks<<<(unsigned)nb, kScanBlock, 0, c->stream>>>(a, n, sums);
  k_sn_scan_sums<<<1, kScanBlock, 0, c->stream>>>(sums, nb, total);
  k_sn_scan_add<<<(unsigned)nb, kScanBlock, 0, c->stream>>>(a, n, sums);
  c->launches += 3;
  MYCEL_CUDA(c, cudaGetLastError());
  return MYCEL_OK;
}

}  // namespace
}  // namespace mycel

using namespace mycel;

namespace mycel {
// The extraction from a density already in device memory (d_density: nx*ny*nz floats, box order), or from
// host memory (h_density, copied in first).
int32_t surface_nets_core(mycel_ctx* ctx, int32_t nx, int32_t ny, int32_t nz, float h, const float* origin,
                          const float* h_density, const float* d_density, float threshold, mycel_mesh** out) {
  *out = nullptr;
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t CX = nx + 1, CY = ny + 1, CZ = nz + 1, C = CX * CY * CZ;
  const int64_t P = (int64_t)(nx + 2) * (ny + 2) * (nz + 2);
  const int64_t E = (int64_t)nz * ny * (nx + 1) + (int64_t)nz * (ny + 1) * nx + (int64_t)(nz + 1) * ny * nx;
  if (C >= INT32_MAX / 8 || E >= INT32_MAX / 8)
    return set_error(ctx, MYCEL_E_ARG, "grid too large for the iso-surface (cell or edge count beyond 2^28)");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const SnGrid g{nx, ny, nz, (int64_t)nx + 2, (int64_t)(nx + 2) * (ny + 2)};
  // device work space, freed in stream order at the end
  std::vector<void*> bufs;
  bool oom = false;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (oom || cudaMallocAsync(&p, bytes + 16, s) != cudaSuccess) {
      oom = true;
      return nullptr;
    }
    bufs.push_back(p);
    return p;
  };
  struct Free {
    std::vector<void*>* b;
    cudaStream_t s;
    ~Free() {
      for (void* p : *b) cudaFreeAsync(p, s);
    }
  } guard{&bufs, s};
  float* d_in = h_density ? (float*)alloc(sizeof(float) * n) : const_cast<float*>(d_density);
  float* d_rho = (float*)alloc(sizeof(float) * P);
  uint8_t* d_s = (uint8_t*)alloc(P);
  int32_t* d_cflag = (int32_t*)alloc(sizeof(int32_t) * C);
  int32_t* d_cex = (int32_t*)alloc(sizeof(int32_t) * C);
  int32_t* d_vidx = (int32_t*)alloc(sizeof(int32_t) * C);
  float* d_tmp = (float*)alloc(sizeof(float) * 3 * C);
  float* d_pos = (float*)alloc(sizeof(float) * 3 * C);
  int32_t* d_eflag = (int32_t*)alloc(sizeof(int32_t) * E);
  int32_t* d_eslot = (int32_t*)alloc(sizeof(int32_t) * E);
  int32_t* d_sums = (int32_t*)alloc(sizeof(int32_t) * ((std::max(C, E) + kScanBlock - 1) / kScanBlock + 1));
  long long* d_scal = (long long*)alloc(sizeof(long long) * 8);  // [0] candidates, [1..2] passes/changes, [3..4] totals
  int* d_flags = (int*)alloc(sizeof(int) * 8);
  if (oom) return set_error(ctx, MYCEL_E_OOM, "out of device memory for the iso-surface");
  long long* h_scal = (long long*)ctx->pinned;  // at least 64 bytes of pinned scratch
  if (h_density) MYCEL_CUDA(ctx, cudaMemcpyAsync(d_in, h_density, sizeof(float) * n, cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(ctx, cudaMemsetAsync(d_scal, 0, sizeof(long long) * 8, s));
  MYCEL_CUDA(ctx, cudaMemsetAsync(d_flags, 0, sizeof(int) * 8, s));
  const int nsm = ctx->num_sms;
  k_sn_pad<<<sn_grid_blocks(P, nsm), 256, 0, s>>>(g, d_in, threshold, d_rho, d_s);
  k_sn_detect<<<sn_grid_blocks(n, nsm), 256, 0, s>>>(g, d_s, (unsigned long long*)d_scal);
  ctx->launches += 2;
  MYCEL_CUDA(ctx, cudaMemcpyAsync(h_scal, d_scal, sizeof(long long), cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(ctx, cudaStreamSynchronize(s));
  mycel_mesh* m = new mycel_mesh();
  struct MeshGuard {
    mycel_mesh** m;
    ~MeshGuard() {
      if (*m) delete *m;
    }
  } mguard{&m};
  if (h_scal[0] > 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kSnCtas);
    cfg.blockDim = dim3(kSnThreads);
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_sn_compose, &cfg) != cudaSuccess || nclusters < 1) {
      cudaGetLastError();
      return set_error(ctx, MYCEL_E_DEVICE, "iso-surface: the well-composedness cluster kernel cannot be scheduled");
    }
    k_sn_compose<<<kSnCtas, kSnThreads, 0, s>>>(g, d_s, d_rho, threshold, d_flags, d_scal + 1);
    ctx->launches++;
    MYCEL_CUDA(ctx, cudaGetLastError());
  }
  k_sn_cells<<<sn_grid_blocks(C, nsm), 256, 0, s>>>(g, d_rho, d_s, threshold, h, origin[0], origin[1], origin[2],
                                                    d_cflag, d_tmp);
  MYCEL_CUDA(ctx, cudaMemcpyAsync(d_cex, d_cflag, sizeof(int32_t) * C, cudaMemcpyDeviceToDevice, s));
  ctx->launches++;
  if (int32_t st = sn_scan(ctx, d_cex, C, d_sums, d_scal + 3)) return st;
  k_sn_compact<<<sn_grid_blocks(C, nsm), 256, 0, s>>>(C, d_cflag, d_cex, d_tmp, d_vidx, d_pos);
  k_sn_edge_flags<<<sn_grid_blocks(E, nsm), 256, 0, s>>>(g, E, d_s, d_vidx, d_eflag);
  MYCEL_CUDA(ctx, cudaMemcpyAsync(d_eslot, d_eflag, sizeof(int32_t) * E, cudaMemcpyDeviceToDevice, s));
  ctx->launches += 2;
  if (int32_t st = sn_scan(ctx, d_eslot, E, d_sums, d_scal + 4)) return st;
  MYCEL_CUDA(ctx, cudaMemcpyAsync(h_scal, d_scal, sizeof(long long) * 8, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(ctx, cudaStreamSynchronize(s));
  const long long nv = h_scal[3], nq = h_scal[4];
  m->passes = h_scal[0] > 0 ? (int32_t)h_scal[1] : 1;
  m->changes = h_scal[2];
  if (nv > 0) {
    int32_t* d_idx = (int32_t*)alloc(sizeof(int32_t) * 6 * std::max<long long>(nq, 1));
    if (oom) return set_error(ctx, MYCEL_E_OOM, "out of device memory for the iso-surface");
    k_sn_quads<<<sn_grid_blocks(E, nsm), 256, 0, s>>>(g, E, d_s, d_vidx, d_pos, d_eslot, d_idx);
    ctx->launches++;
    m->positions.resize((size_t)(3 * nv));
    m->indices.resize((size_t)(6 * nq));
    MYCEL_CUDA(ctx, cudaMemcpyAsync(m->positions.data(), d_pos, sizeof(float) * 3 * nv, cudaMemcpyDeviceToHost, s));
    if (nq > 0)
      MYCEL_CUDA(ctx, cudaMemcpyAsync(m->indices.data(), d_idx, sizeof(int32_t) * 6 * nq, cudaMemcpyDeviceToHost, s));
  }
  MYCEL_CUDA(ctx, cudaStreamSynchronize(s));
  MYCEL_CUDA(ctx, cudaGetLastError());
  *out = m;
  m = nullptr;
  return MYCEL_OK;
}
}  // namespace mycel

extern "C" int32_t mycel_surface_nets(mycel_ctx* ctx, int32_t nx, int32_t ny, int32_t nz, float h, const float* origin,
                                      const float* density, int64_t density_len, float threshold, mycel_mesh** out) {
  if (!ctx || !density || !origin || !out) return set_error(ctx, MYCEL_E_ARG, "NULL argument");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1) return set_error(ctx, MYCEL_E_ARG, "Grid dimensions must be positive.");
  const int64_t n = (int64_t)nx * ny * nz;
  if (density_len < n)
    return set_error(ctx, MYCEL_E_ARG, "physicalDensity length (" + std::to_string(density_len) +
                                           ") is smaller than grid element count (" + std::to_string(n) + ").");
  return surface_nets_core(ctx, nx, ny, nz, h, origin, density, nullptr, threshold, out);
}

extern "C" int32_t mycel_mesh_info(const mycel_mesh* m, int64_t* n_vertices, int64_t* n_indices, int32_t* passes,
                                   int64_t* changes) {
  if (!m) return MYCEL_E_ARG;
  if (n_vertices) *n_vertices = (int64_t)(m->positions.size() / 3);
  if (n_indices) *n_indices = (int64_t)m->indices.size();
  if (passes) *passes = m->passes;
  if (changes) *changes = m->changes;
  return MYCEL_OK;
}

extern "C" int32_t mycel_mesh_copy(const mycel_mesh* m, float* positions, int32_t* indices) {
  if (!m) return MYCEL_E_ARG;
  if (positions && !m->positions.empty()) std::copy(m->positions.begin(), m->positions.end(), positions);
  if (indices && !m->indices.empty()) std::copy(m->indices.begin(), m->indices.end(), indices);
  return MYCEL_OK;
}

extern "C" void mycel_mesh_destroy(mycel_mesh* m) { delete m; }

extern "C" int32_t mycel_taubin_smooth(mycel_ctx* ctx, float* positions, int64_t n_vertices, const int32_t* indices,
                                       int64_t n_indices, int32_t iterations, float lambda, float mu) {
  if (!ctx || (!positions && n_vertices) || (!indices && n_indices)) return set_error(ctx, MYCEL_E_ARG, "NULL argument");
  if (n_vertices < 0 || n_indices < 0 || n_indices % 3) return set_error(ctx, MYCEL_E_ARG, "indices must hold whole triangles");
  if (iterations <= 0 || n_vertices == 0 || n_indices == 0) return MYCEL_OK;  // the mesh is returned unchanged
  if (n_indices >= INT32_MAX / 2 || n_vertices >= INT32_MAX)
    return set_error(ctx, MYCEL_E_ARG, "mesh too large for the smoother (index count beyond 2^30)");
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const int64_t nv = n_vertices, ni = n_indices, nt = ni / 3;
  std::vector<void*> bufs;
  bool oom = false;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (oom || cudaMallocAsync(&p, bytes + 16, s) != cudaSuccess) {
      oom = true;
      return nullptr;
    }
    bufs.push_back(p);
    return p;
  };
  struct Free {
    std::vector<void*>* b;
    cudaStream_t s;
    ~Free() {
      for (void* p : *b) cudaFreeAsync(p, s);
    }
  } guard{&bufs, s};
  int32_t* d_idx = (int32_t*)alloc(sizeof(int32_t) * ni);
  float* d_a = (float*)alloc(sizeof(float) * 3 * nv);
  float* d_b = (float*)alloc(sizeof(float) * 3 * nv);
  int32_t* d_deg = (int32_t*)alloc(sizeof(int32_t) * nv);
  int32_t* d_off = (int32_t*)alloc(sizeof(int32_t) * nv);
  int32_t* d_cur = (int32_t*)alloc(sizeof(int32_t) * nv);
  int32_t* d_cnt = (int32_t*)alloc(sizeof(int32_t) * nv);
  int32_t* d_nb = (int32_t*)alloc(sizeof(int32_t) * 2 * ni);
  int32_t* d_sums = (int32_t*)alloc(sizeof(int32_t) * ((nv + kScanBlock - 1) / kScanBlock + 1));
  long long* d_tot = (long long*)alloc(sizeof(long long) * 2);
  int* d_bad = (int*)alloc(sizeof(int));
  if (oom) return set_error(ctx, MYCEL_E_OOM, "out of device memory for the mesh smoother");
  int* h_bad = (int*)ctx->pinned;
  const int nsm = ctx->num_sms;
  MYCEL_CUDA(ctx, cudaMemcpyAsync(d_idx, indices, sizeof(int32_t) * ni, cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(ctx, cudaMemcpyAsync(d_a, positions, sizeof(float) * 3 * nv, cudaMemcpyHostToDevice, s));
  MYCEL_CUDA(ctx, cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  MYCEL_CUDA(ctx, cudaMemsetAsync(d_deg, 0, sizeof(int32_t) * nv, s));
  k_tb_check<<<sn_grid_blocks(ni, nsm), 256, 0, s>>>(ni, d_idx, nv, d_bad);
  MYCEL_CUDA(ctx, cudaMemcpyAsync(h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->launches++;
  if (*h_bad) return set_error(ctx, MYCEL_E_ARG, "triangle index out of range of the vertex array");
  k_tb_degree<<<sn_grid_blocks(nt, nsm), 256, 0, s>>>(nt, d_idx, d_deg);
  MYCEL_CUDA(ctx, cudaMemcpyAsync(d_off, d_deg, sizeof(int32_t) * nv, cudaMemcpyDeviceToDevice, s));
  ctx->launches++;
  if (int32_t st = sn_scan(ctx, d_off, nv, d_sums, d_tot)) return st;
  MYCEL_CUDA(ctx, cudaMemcpyAsync(d_cur, d_off, sizeof(int32_t) * nv, cudaMemcpyDeviceToDevice, s));
  k_tb_fill<<<sn_grid_blocks(nt, nsm), 256, 0, s>>>(nt, d_idx, d_cur, d_nb);
  k_tb_sort<<<sn_grid_blocks(nv, nsm), 256, 0, s>>>(nv, d_off, d_deg, d_nb, d_cnt);
  ctx->launches += 2;
  for (int it = 0; it < iterations; ++it) {
    k_tb_step<<<sn_grid_blocks(nv, nsm), 256, 0, s>>>(nv, d_a, d_b, d_off, d_cnt, d_nb, lambda);
    k_tb_step<<<sn_grid_blocks(nv, nsm), 256, 0, s>>>(nv, d_b, d_a, d_off, d_cnt, d_nb, mu);
    ctx->launches += 2;
  }
  MYCEL_CUDA(ctx, cudaGetLastError());
  MYCEL_CUDA(ctx, cudaMemcpyAsync(positions, d_a, sizeof(float) * 3 * nv, cudaMemcpyDeviceToHost, s));
  MYCEL_CUDA(ctx, cudaStreamSynchronize(s));
  return MYCEL_OK;
}
