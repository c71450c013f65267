// Eight-colour Gauss-Seidel on the 27-point operator (Vgsrb27x,
// pmgc/gsd.cc:114-212) with each tile's iterate planes staged by the tensor
// memory accelerator: the float levels of the mixed path between the
// one-launch bottom levels and the finest level.
//
// The sweep is gs27_tiled.cuh's: one launch per plane parity, one CTA per
// tile of a plane, four sub-colour steps with a recomputed halo of 3 - t
// points in step t, ping-pong buffers and the reference's per-point
// arithmetic (sums27 order), so the bits are the same. Two things differ:
//
// - The tiles are TI x TJ = 2 TT x TT / 2 (TT 32, the size class of levels
//   from 97 points per axis), so one sub-colour row of a tile is TT + H
//   points and a warp's points lie along one row. The couplings are read from copies of
//   the level's fourteen arrays split by the parity of i (CoefSplit): the
//   points of a sub-colour row and each of their 26 couplings are
//   consecutive floats, where the reference layout puts them two apart and
//   leaves half of every sector unused.
// - The x planes k - 1, k, k + 1 over the tile and its halo arrive as three
//   tensor-map boxes on one mbarrier (transaction bytes); each box row is
//   then split by column parity in place, so the neighbours that a warp's
//   points read in shared memory are consecutive words (no bank conflicts
//   between the even and odd columns). The tensor maps cover this GPU's own
//   arrays (no multicast).
//
// Levels of the 16 and 8 size classes (65^3 and 33^3 of pb257) use
// gs27_tma_square_kernel: TT x TT tiles, the couplings in the level's own
// layout, the staged rows as they arrive.
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
// TI bx - 4, a multiple of four floats); coordinates before the array or
// past its last point (the map's extent is nx, not px) read as zero, which
// no update uses. A box is (TI + 12) x (TJ + 8) floats, so the tensor maps
// of a level are made for its tile edge.
#pragma once

#include <cuda.h>

#include "gs27_tiled.cuh"

namespace pmg {

// box of a tile of size class TT: TI = 2 TT columns, TJ = TT / 2 rows; box
// rows of TI + 12 floats (a 16-byte multiple, from the 16-byte boundary below
// the halo; even, so a row splits into two halves of HB), TJ + 8 rows. The
// three planes' boxes lie PS floats apart in shared memory: a tensor copy's
// destination must be 128-byte aligned, and SIZE is not always a multiple
// of 32 floats (336 for TT = 8).
template <int TT> struct TmaBox {
  static constexpr int TI = 2 * TT, TJ = TT / 2;
  static constexpr int BX = TI + 12, BY = TJ + 8, SIZE = BX * BY,
                       HB = BX / 2, PS = (SIZE + 31) & ~31;
  static constexpr unsigned BYTES = 3 * SIZE * sizeof(float); // 3 planes
  static_assert(BX % 4 == 0 && BX % 2 == 0,
                "box rows must be a 16-byte multiple and even");
  static_assert(PS * sizeof(float) % 128 == 0,
                "box destinations must be 128-byte aligned");
};

// box of a TT x TT tile (gs27_tma_square_kernel): rows of TT + 12 floats
// (a 16-byte multiple, from the 16-byte boundary below the halo), TT + 8
// rows; SIZE is a multiple of 32 floats for TT = 8, 16, 32
template <int TT> struct TmaSqBox {
  static constexpr int BX = TT + 12, BY = TT + 8, SIZE = BX * BY;
  static constexpr unsigned BYTES = 3 * SIZE * sizeof(float); // 3 planes
  static_assert(SIZE * sizeof(float) % 128 == 0,
                "box destinations must be 128-byte aligned");
};

// The i-parity split layout of a padded float level's coupling copies: row
// (j, k) holds the even i at [0, hx) and the odd i at [hx, 2 hx), entry i >> 1
// (i = 1 .. nx, 1-based as Dims). hx is a multiple of 4 floats (16 bytes):
// 68 for 129 points, where a sector multiple (72) would read 6% more.
struct CoefSplit {
  int hx, ny;
  __host__ __device__ static CoefSplit of(const Dims &d) {
    return CoefSplit{(((d.nx >> 1) + 1) + 3) & ~3, d.ny};
  }
  __host__ __device__ int row() const { return 2 * hx; }
  __host__ __device__ int plane() const { return 2 * hx * ny; }
  __host__ __device__ long count(int nz) const { return (long)plane() * nz; }
  __host__ __device__ int at(int i, int j, int k) const {
    return ((k - 1) * ny + (j - 1)) * 2 * hx + (i & 1) * hx + (i >> 1);
  }
};

// Copies the fourteen couplings of a padded float level (rows d.px apart)
// into the split layout, every point of the array (shell included).
__global__ void coef_split_kernel(Dims d, CoefSplit cs, Op14<float> A,
                                  Op14W<float> out) {
  const long n = (long)d.nx * d.ny * d.nz;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % d.nx) + 1;
    const long r = t / d.nx;
    const int j = (int)(r % d.ny) + 1, k = (int)(r / d.ny) + 1;
    const int src = d.at(i, j, k), dst = cs.at(i, j, k);
#pragma unroll
    for (int q = 0; q < 14; ++q)
      out.a[q][dst] = A.a[q][src];
  }
}

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
// bulk copy of `bytes` (a multiple of 16) from 16-byte aligned global
// memory into shared memory, completing on bar
__device__ __forceinline__ void bulk_load(void *dst, const void *src,
                                          unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx"
               "::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Sub-colour step S (points (i, j) with i % 2 = S & 1, j % 2 = S >> 1) with
// halo H of a TI x TJ tile: a fixed NUX x NUY grid of the points within H of
// the tile, clipped to the interior. xk: the staged plane k with its rows
// split by column parity (column c of a box row at (c & 1) HB + (c >> 1));
// column c holds i = ti0 - 5 + c, row r holds j = tj0 - 4 + r; planes k - 1
// and k + 1 at xk -/+ PS. The couplings come from the split copies (cs),
// the right-hand side from fc (rows d.px apart). ti0 and tj0 are even.
template <int TT, int S, int H>
__device__ __forceinline__ void gs27_split_step(const Dims &d,
                                                const CoefSplit &cs,
                                                const Op14<float> &A,
                                                const float *__restrict__ fc,
                                                float *xk, int ti0, int tj0,
                                                int k) {
  using B = TmaBox<TT>;
  constexpr int NT = Gs27Tile<TT>::THREADS;
  constexpr int NUX = B::TI / 2 + H, NUY = B::TJ / 2 + H, NQ = NUX * NUY;
  constexpr int PI = S & 1, PJ = S >> 1;
  // first point of the sub-colour at or after ti0 - H (tj0 - H)
  constexpr int IA = -H + ((PI + H) & 1), JA = -H + ((PJ + H) & 1);
  // shared memory: column c = i - ti0 + 5 has parity 1 - PI; its
  // neighbours i + 1 and i - 1 are in the other half
  constexpr int PC = 1 - PI;
  constexpr int XO = (1 - 2 * PC) * B::HB;
  constexpr int XE = XO + PC, XW = XO + PC - 1, XN = B::BX;
  // split couplings: i + 1 and i - 1 in the other half, rows R, planes Z
  const int co = (1 - 2 * PI) * cs.hx;
  const int ce = co + PI, cw = co + PI - 1;
  const int R = cs.row(), Z = cs.plane();
  const int i_max = d.nx - 1, j_max = d.ny - 1;
  const float *const *a = A.a;
#pragma unroll
  for (int m = 0; m < (NQ + NT - 1) / NT; ++m) {
    const int q = threadIdx.x + m * NT;
    const int v = q / NUX, u = q - v * NUX;
    const int i = ti0 + IA + 2 * u, j = tj0 + JA + 2 * v;
    if (q < NQ && i >= 2 && i <= i_max && j >= 2 && j <= j_max) {
      const int c = i - ti0 + 5;
      const int sidx = (j - tj0 + 4) * B::BX + PC * B::HB + (c >> 1);
      const int p = cs.at(i, j, k);
      Gs27Point<float> g;
      g.a[0] = a[kON][p];
      g.a[1] = a[kON][p - R];
      g.a[2] = a[kOE][p];
      g.a[3] = a[kOE][p + cw];
      g.a[4] = a[kONE][p];
      g.a[5] = a[kONW][p];
      g.a[6] = a[kONW][p + ce - R];
      g.a[7] = a[kONE][p + cw - R];
      g.a[8] = a[kUC][p];
      g.a[9] = a[kUN][p];
      g.a[10] = a[kUS][p];
      g.a[11] = a[kUE][p];
      g.a[12] = a[kUW][p];
      g.a[13] = a[kUNE][p];
      g.a[14] = a[kUNW][p];
      g.a[15] = a[kUSE][p];
      g.a[16] = a[kUSW][p];
      g.a[17] = a[kUC][p - Z];
      g.a[18] = a[kUS][p + R - Z];
      g.a[19] = a[kUN][p - R - Z];
      g.a[20] = a[kUW][p + ce - Z];
      g.a[21] = a[kUE][p + cw - Z];
      g.a[22] = a[kUSW][p + ce + R - Z];
      g.a[23] = a[kUSE][p + cw + R - Z];
      g.a[24] = a[kUNW][p + ce - R - Z];
      g.a[25] = a[kUNE][p + cw - R - Z];
      g.f = fc[d.at(i, j, k)];
      g.d = a[kOC][p] + 0.f; // gs27_load's oC + cc with no cc
      const float *xc = xk + sidx, *xd = xc - B::PS, *xu = xc + B::PS;
      // gs27_update's sums with the split neighbour offsets
      const float tO = g.a[0] * xc[XN] + g.a[1] * xc[-XN] + g.a[2] * xc[XE] +
                       g.a[3] * xc[XW] + g.a[4] * xc[XE + XN] +
                       g.a[5] * xc[XW + XN] + g.a[6] * xc[XE - XN] +
                       g.a[7] * xc[XW - XN];
      const float tU = g.a[8] * xu[0] + g.a[9] * xu[XN] + g.a[10] * xu[-XN] +
                       g.a[11] * xu[XE] + g.a[12] * xu[XW] +
                       g.a[13] * xu[XE + XN] + g.a[14] * xu[XW + XN] +
                       g.a[15] * xu[XE - XN] + g.a[16] * xu[XW - XN];
      const float tD = g.a[17] * xd[0] + g.a[18] * xd[XN] +
                       g.a[19] * xd[-XN] + g.a[20] * xd[XE] +
                       g.a[21] * xd[XW] + g.a[22] * xd[XE + XN] +
                       g.a[23] * xd[XW + XN] + g.a[24] * xd[XE - XN] +
                       g.a[25] * xd[XW - XN];
      xk[sidx] = (g.f + (tO + tU + tD)) / g.d;
    }
  }
}

// One plane-parity phase on TI x TJ tiles, the sub-colours in forward order
// (0, 1, 2, 3: the mixed path's pre- and post-smoothing both sweep forward).
// err: set to 1 when the stage did not arrive within the bounded wait (the
// block then waits once more, also bounded, for its copies and returns).
// extra_tx: bytes expected on top of the boxes' (0; a test sets it so that
// every wait runs out).
template <int TT>
__global__ void __launch_bounds__(Gs27Tile<TT>::THREADS, 2048 /
                                  Gs27Tile<TT>::THREADS)
    gs27_tma_kernel(const __grid_constant__ Gs27TmaMaps maps, Dims d,
                    CoefSplit cs, Op14<float> A, const float *__restrict__ fc,
                    float *out, int kfirst, int *err, unsigned extra_tx) {
  using B = TmaBox<TT>;
  constexpr int NT = Gs27Tile<TT>::THREADS;
  __shared__ __align__(128) float xs[3 * B::PS];
  __shared__ uint64_t bar;
  const int ti0 = 2 + blockIdx.x * B::TI, tj0 = 2 + blockIdx.y * B::TJ;
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
    mbar_expect_tx(&bar, B::BYTES + extra_tx);
    tma_load_3d(xs, &maps.nb, cx, cy, z - 1, &bar);
    tma_load_3d(xs + B::PS, &maps.own, cx, cy, z, &bar);
    tma_load_3d(xs + 2 * B::PS, &maps.nb, cx, cy, z + 1, &bar);
  }
  const bool ok = mbar_wait(&bar, 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicOr(err, 1);
      (void)mbar_wait(&bar, 0); // the copies land before the block leaves
    }
    return;
  }
  // split every box row by column parity, in place: a warp holds a row in
  // registers, then writes column c to (c & 1) HB + (c >> 1)
  {
    constexpr int NW = NT / 32, PER = (B::BX + 31) / 32;
    const int lane = threadIdx.x & 31;
    for (int row = threadIdx.x >> 5; row < 3 * B::BY; row += NW) {
      const int pl = row / B::BY;
      float *r = xs + pl * B::PS + (row - pl * B::BY) * B::BX;
      float t[PER];
#pragma unroll
      for (int e = 0; e < PER; ++e) {
        const int c = lane + 32 * e;
        t[e] = c < B::BX ? r[c] : 0.f;
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < PER; ++e) {
        const int c = lane + 32 * e;
        if (c < B::BX)
          r[(c & 1) * B::HB + (c >> 1)] = t[e];
      }
    }
  }
  __syncthreads();
  float *xk = xs + B::PS;
  gs27_split_step<TT, 0, 3>(d, cs, A, fc, xk, ti0, tj0, k);
  __syncthreads();
  gs27_split_step<TT, 1, 2>(d, cs, A, fc, xk, ti0, tj0, k);
  __syncthreads();
  gs27_split_step<TT, 2, 1>(d, cs, A, fc, xk, ti0, tj0, k);
  __syncthreads();
  gs27_split_step<TT, 3, 0>(d, cs, A, fc, xk, ti0, tj0, k);
  __syncthreads();
  const int i_max = d.nx - 1, j_max = d.ny - 1;
#pragma unroll
  for (int m = 0; m < (B::TI * B::TJ + NT - 1) / NT; ++m) {
    const int q = threadIdx.x + m * NT;
    const int jj = q / B::TI, ii = q - jj * B::TI;
    const int i = ti0 + ii, j = tj0 + jj, c = ii + 5;
    if (q < B::TI * B::TJ && i <= i_max && j <= j_max)
      out[d.at(i, j, k)] =
          xk[(jj + 4) * B::BX + (c & 1) * B::HB + (c >> 1)];
  }
}

// One plane-parity phase on TT x TT tiles (gs27_phase_kernel with the x
// planes staged by three tensor-map boxes, the couplings read in the
// level's own layout): the 16 and 8 tile classes, where the wide tiles'
// extra rows (a second round of loads in the first step at TT = 16) and the
// row split cost more than the split reads save (ncu, cold cache: 10.5
// against 13.9 us per launch at 65^3, 8.1 against 9.5 at 33^3). err and
// extra_tx as gs27_tma_kernel's.
template <int TT>
__global__ void __launch_bounds__(Gs27Tile<TT>::THREADS, 2048 /
                                  Gs27Tile<TT>::THREADS)
    gs27_tma_square_kernel(const __grid_constant__ Gs27TmaMaps maps, Dims d,
                           Op14<float> A, const float *__restrict__ fc,
                           float *out, int kfirst, int order, int *err,
                           unsigned extra_tx) {
  constexpr int W = TmaSqBox<TT>::BX, NT = Gs27Tile<TT>::THREADS;
  constexpr int kBox = TmaSqBox<TT>::SIZE;
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
    mbar_expect_tx(&bar, TmaSqBox<TT>::BYTES + extra_tx);
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
