// Plane split of a small level over a cluster of CTAs, shared by the
// cluster kernels of the coarsest levels (cg_cluster.cuh, bottom_cluster.cuh):
// interior planes 2 .. nz-1 go to kCgCtas CTAs in order, at most
// kCgMaxPlanes each.
#pragma once

#include "pmg_common.cuh"

namespace pmg {

constexpr int kCgCtas = 8;        // CTAs of the cluster
constexpr int kCgThreads = 512;   // threads per CTA, one point each
constexpr int kCgMaxPlanes = 2;   // interior planes per CTA
constexpr int kCgMaxN = 17;       // points per axis (incl. shell)

// first interior plane of CTA c (planes 2 .. nz-1 split evenly)
__host__ __device__ inline int cg_plane_lo(int c, int nz) {
  return 2 + (c * (nz - 2)) / kCgCtas;
}

// CTA holding interior plane k
__host__ __device__ inline int cg_plane_owner(int k, int nz) {
  int c = 0;
  while (c + 1 < kCgCtas && cg_plane_lo(c + 1, nz) <= k)
    ++c;
  return c;
}

// Sum of v over the CTA, in every thread (warp sums, then the warps in
// order); sh holds 32 doubles.
__device__ __forceinline__ double cg_block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int w = 0; w < nw; ++w)
    t += sh[w];
  return t;
}

} // namespace pmg
