// Eight-colour Gauss-Seidel on the 27-point operator (Vgsrb27x,
// pmgc/gsd.cc:114-212) with each tile's iterate planes staged by the tensor
// memory accelerator: the float levels of the mixed path between the
// one-launch bottom levels and the finest level.
//
// The sweep is gs27_tiled.cuh's: one launch per plane parity, one CTA per
// TT x TT tile of a plane (TT 32, 16 or 8 by the level's size, as there), four sub-colour steps with a recomputed halo of
// 3 - t points in step t, ping-pong buffers and the reference's per-point
// arithmetic (sums27 order), so the bits are the same. The x planes k - 1,
// k, k + 1 over the tile and its halo arrive as three tensor-map boxes on
// one mbarrier (transaction bytes) instead of one 4-byte cp.async per point
// with its index arithmetic; the couplings are read per point from global
// memory as before. The tensor maps cover this GPU's own arrays (no
// multicast).
//
// Staging the operator as well (27 boxes per tile: 114 KB, one CTA per SM
// with two stages, persistent) was built and measured slower: 69 against
// 41 us per launch at 129^3 (ncu: 12.5% of the warp slots active, issue
// 15%), because a tile step has only ~200 points of work and the boxes
// leave room for one tile in flight per stage.
//
// The arrays' rows are padded to a 16-byte multiple (Dims::px) because a
// tensor map's strides must be: 129 floats a row becomes 132. A box starts
// at the 16-byte boundary at or below the tile's halo (x coordinate
// 32 bx - 4, a multiple of four floats); coordinates before the array or
// past its last point (the map's extent is nx, not px) read as zero, which
// no update uses. A box is (TT + 12) x (TT + 8) floats, so the tensor maps
// of a level are made for its tile edge.
#pragma once

#include <cuda.h>

#include "gs27_tiled.cuh"

namespace pmg {

// box of a TT x TT tile: rows of TT + 12 floats (a 16-byte multiple, from
// the 16-byte boundary below the halo), TT + 8 rows
template <int TT> struct TmaBox {
  static constexpr int BX = TT + 12, BY = TT + 8, SIZE = BX * BY;
  static constexpr unsigned BYTES = 3 * SIZE * sizeof(float); // 3 planes
};
// mbarrier polls before the stage counts as lost: about 0.1 s, some 10^4
// times the longest real wait
constexpr long kTmaMaxPolls = 1L << 20;

// Tensor maps of the two iterate buffers in the roles of the launch.
struct alignas(64) Gs27TmaMaps {
  CUtensorMap own, nb;
};

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(
                   smem_addr(bar)),
               "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar,
                                               unsigned bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
          smem_addr(bar)),
      "r"(bytes)
      : "memory");
}
// true once the phase with this parity has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar,
                                              unsigned parity) {
  unsigned done;
  asm volatile("{\n"
               ".reg .pred p;\n"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               "selp.u32 %0, 1, 0, p;\n"
               "}\n"
               : "=r"(done)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return done != 0;
}
// bounded wait: false if the phase did not complete within kTmaMaxPolls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  for (long n = 0; n < kTmaMaxPolls; ++n) {
    if (mbar_try_wait(bar, parity))
      return true;
    if (n > 64)
      __nanosleep(64);
  }
  return false;
}
// one box of a 3-D tensor map into shared memory, completing on bar
__device__ __forceinline__ void tma_load_3d(float *dst, const CUtensorMap *map,
                                            int x, int y, int z,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx"
      "::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// One plane-parity phase on TT x TT tiles (gs27_phase_kernel with the x
// planes staged by three tensor-map boxes). err: set to 1 when the stage
// did not arrive within the bounded wait (the block then waits once more,
// also bounded, for its copies and returns). extra_tx: bytes expected on
// top of the boxes' (0; a test sets it so that every wait runs out).
template <int TT>
__global__ void __launch_bounds__(Gs27Tile<TT>::THREADS, 2048 /
                                  Gs27Tile<TT>::THREADS)
    gs27_tma_kernel(const __grid_constant__ Gs27TmaMaps maps, Dims d,
                    Op14<float> A, const float *__restrict__ fc, float *out,
                    int kfirst, int order, int *err, unsigned extra_tx) {
  constexpr int W = TmaBox<TT>::BX, NT = Gs27Tile<TT>::THREADS;
  constexpr int kBox = TmaBox<TT>::SIZE;
  __shared__ __align__(128) float xs[3 * kBox];
  __shared__ uint64_t bar;
  const int ti0 = 2 + blockIdx.x * TT, tj0 = 2 + blockIdx.y * TT;
  const int k = kfirst + 2 * blockIdx.z;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // box origin (0-based): x at the 16-byte boundary ti0 - 6, y five rows
    // above the tile (the 4-point halo starts at tj0 - 4, 1-based)
    const int cx = ti0 - 6, cy = tj0 - 5, z = k - 1;
    mbar_expect_tx(&bar, TmaBox<TT>::BYTES + extra_tx);
    tma_load_3d(xs, &maps.nb, cx, cy, z - 1, &bar);
    tma_load_3d(xs + kBox, &maps.own, cx, cy, z, &bar);
    tma_load_3d(xs + 2 * kBox, &maps.nb, cx, cy, z + 1, &bar);
  }
  const bool ok = mbar_wait(&bar, 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicOr(err, 1);
      (void)mbar_wait(&bar, 0); // the copies land before the block leaves
    }
    return;
  }
  // box column c holds 1-based i = ti0 - 5 + c, row r holds j = tj0 - 4 + r;
  // gs27_step_at's origin is (ti0 - 4, tj0 - 4): one column on
  float *xc = xs + kBox + 1;
  gs27_step_at<float, TT, W, kBox, 3>(d, A, nullptr, fc, xc, ti0, tj0, k,
                                      order);
  __syncthreads();
  gs27_step_at<float, TT, W, kBox, 2>(d, A, nullptr, fc, xc, ti0, tj0, k,
                                      order);
  __syncthreads();
  gs27_step_at<float, TT, W, kBox, 1>(d, A, nullptr, fc, xc, ti0, tj0, k,
                                      order);
  __syncthreads();
  gs27_step_at<float, TT, W, kBox, 0>(d, A, nullptr, fc, xc, ti0, tj0, k,
                                      order);
  __syncthreads();
  const int i_max = d.nx - 1, j_max = d.ny - 1;
#pragma unroll
  for (int m = 0; m < (TT * TT + NT - 1) / NT; ++m) {
    const int q = threadIdx.x + m * NT;
    const int jj = q / TT, ii = q - jj * TT;
    const int i = ti0 + ii, j = tj0 + jj;
    if (q < TT * TT && i <= i_max && j <= j_max)
      out[d.at(i, j, k)] = xc[(i - (ti0 - 4)) + W * (j - (tj0 - 4))];
  }
}

} // namespace pmg
