// Device helpers shared by the kernels: element-type tables computed on the
// fly, periodic images, reductions.
#pragma once

#include <cuda_runtime.h>

#include "ctx.cuh"

namespace cacb200 {

// Grid for a kernel that strides over a count known only on the device:
// enough blocks to fill the 148 SMs several times over, no more than the
// capacity `n_max` needs.
inline int stride_grid(long n_max, int threads) {
  long b = (n_max + threads - 1) / threads;
  if (b > 148L * 16) b = 148L * 16;
  return (int)(b < 1 ? 1 : b);
}

inline BoxD make_box(const Ctx &c) {
  BoxD b;
  for (int d = 0; d < 3; d++) {
    b.lo[d] = c.boxlo[d];
    b.hi[d] = c.boxhi[d];
    b.L[d] = c.prd[d];
  }
  return b;
}

// Hex node n sits at natural corner (xi, eta, zeta) in {0,1}^3 with the
// reference's numbering (element_vec_cac.cpp:1740-1770):
// 0 (0,0,0) 1 (1,0,0) 2 (1,1,0) 3 (0,1,0) 4 (0,0,1) 5 (1,0,1) 6 (1,1,1) 7 (0,1,1)
__host__ __device__ __forceinline__ int node_xi(int n) { return (n == 1 || n == 2 || n == 5 || n == 6); }
__host__ __device__ __forceinline__ int node_eta(int n) { return (n == 2 || n == 3 || n == 6 || n == 7); }
__host__ __device__ __forceinline__ int node_zeta(int n) { return n >= 4; }
__host__ __device__ __forceinline__ int corner_node(int xi, int eta, int zeta) {
  return zeta * 4 + (eta ? (xi ? 2 : 3) : (xi ? 1 : 0));
}

// Gauss cell g = (i*2 + j)*2 + k at lattice indices {0, 8} (setup_integration_point,
// element_vec_cac.cpp:2484-2553): its lattice site and node.
__host__ __device__ __forceinline__ int gauss_site(int g) {
  return ((g >> 2) & 1) * 8 * NC * NC + ((g >> 1) & 1) * 8 * NC + (g & 1) * 8;
}
__host__ __device__ __forceinline__ int gauss_node(int g) {
  return corner_node((g >> 2) & 1, (g >> 1) & 1, g & 1);
}
__host__ __device__ __forceinline__ int node_gauss(int n) {
  return node_xi(n) * 4 + node_eta(n) * 2 + node_zeta(n);
}
// lattice site u -> Gauss cell index, or -1 when u is not a corner
__host__ __device__ __forceinline__ int site_gauss(int u) {
  int i = u / (NC * NC), j = (u / NC) % NC, k = u % NC;
  if ((i != 0 && i != NC - 1) || (j != 0 && j != NC - 1) || (k != 0 && k != NC - 1)) return -1;
  return ((i ? 1 : 0) * 2 + (j ? 1 : 0)) * 2 + (k ? 1 : 0);
}

// Trilinear shape function of node n at lattice site u
// (Element::shape_function Hex, element.cpp:2988-2997, at px = 0.25 i - 1).
// Every factor is a multiple of 1/4 in [0, 2], so the product is exact in
// binary64 and equals the reference's table entry bit for bit.
__host__ __device__ __forceinline__ double shape_val(int u, int n) {
  int i = u / (NC * NC), j = (u / NC) % NC, k = u % NC;
  double px = 0.25 * i - 1.0, py = 0.25 * j - 1.0, pz = 0.25 * k - 1.0;
  double a = node_xi(n) ? (1 + px) : (1 - px);
  double b = node_eta(n) ? (1 + py) : (1 - py);
  double c = node_zeta(n) ? (1 + pz) : (1 - pz);
  return 0.125 * a * b * c;
}

__host__ __device__ __forceinline__ int img_code(int sx, int sy, int sz) {
  return (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
}
__host__ __device__ __forceinline__ void img_decode(int code, int &sx, int &sy, int &sz) {
  sx = code % 3 - 1;
  sy = (code / 3) % 3 - 1;
  sz = code / 9 - 1;
}

// 256-bit loads through the read-only path (sm_100 and later; the address
// must be 32-byte aligned).  One instruction brings a whole 32-byte record,
// so a scattered gather costs one L1 wavefront per record instead of two.
// Only for data that no thread of the same kernel writes, apart from fields
// the reader ignores.
__device__ __forceinline__ double4 ldg256(const double4 *p) {
  double4 r;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
      : "l"(p));
  return r;
}
__device__ __forceinline__ void ldg256(const float4 *p, float4 &a, float4 &b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block reduction of NV doubles into out[blockIdx.x * NV + k].
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&vals)[NV], double *out) {
  __shared__ double sh[32][NV];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) vals[k] = warp_sum(vals[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) sh[warp][k] = vals[k];
  __syncthreads();
  if (warp == 0) {
    int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double v = lane < nw ? sh[lane][k] : 0.0;
      v = warp_sum(v);
      if (lane == 0) out[blockIdx.x * NV + k] = v;
    }
  }
}

// SM-local runs: work cut into nrun runs (of list slots, of cells), with SM
// s owning runs [s*nrun/nsm, (s+1)*nrun/nsm), so that the blocks resident on
// one SM work on neighbouring runs (cell-sorted: neighbouring space) and find
// their neighbours' data in the SM's L1, instead of the hardware's spread of
// consecutive blocks over all SMs.  A persistent block takes runs from a
// range's counter (cleared before the launch), its own SM's range first;
// once that is exhausted, warp 0 scans the other ranges 32 at a time for one
// with runs left.  Counters only grow, so a range seen exhausted stays so and
// the scan ends; every run is taken exactly once.  Returns the run, or -1
// when none is left.  v: the block's current range (shared), initially
// sm_id() % nsm.  Every thread of the block calls it.
__device__ __forceinline__ int sm_id() {
  unsigned s;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
  return (int)s;
}

__device__ __forceinline__ int sm_run(int *cnt, int nsm, int nrun, int &v) {
  __shared__ int got;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    auto lo = [&](int u) { return (int)((long)u * nrun / nsm); };
    int cur = v, res = -1;
    for (;;) {
      int k = 0;
      if (lane == 0) k = atomicAdd(cnt + cur, 1);
      k = __shfl_sync(0xffffffffu, k, 0);
      if (lo(cur) + k < lo(cur + 1)) {
        res = lo(cur) + k;
        break;
      }
      int found = -1;
      for (int base = 1; base <= nsm && found < 0; base += 32) {
        const int u = (cur + base + lane) % nsm;
        const bool left = base + lane <= nsm && lo(u) + *(volatile int *)(cnt + u) < lo(u + 1);
        const unsigned b = __ballot_sync(0xffffffffu, left);
        if (b) found = (cur + base + __ffs(b) - 1) % nsm;
      }
      if (found < 0) break;
      cur = found;
    }
    if (lane == 0) {
      got = res;
      v = cur;
    }
  }
  __syncthreads();
  return got;
}

// PrefixRule (ctx.cuh) for list site i (site-table index) of replica rep:
// does it walk the rest of its list?  The sum is rounded up.
__device__ __forceinline__ bool walk_rest(const PrefixRule &p, int i, int rep) {
  if (!p.inner_ok[rep]) return true;
  const float d = i < p.na ? p.disp[i] : p.edisp[(i - p.na) / NG];
  return __fadd_ru(d, __uint_as_float(p.dmax[rep])) > p.lim;
}

}  // namespace cacb200
