// Eight-colour Gauss-Seidel on the 27-point operator in two launches per
// sweep instead of eight.
//
// The reference visits colours c = (i%2) + 2(j%2) + 4(k%2) in order 0..7
// (7..0 with iadjoint), one parallel launch per colour (Vgsrb27x,
// pmgc/gsd.cc:160-210). Colours 0-3 live on even planes, 4-7 on odd planes,
// so a sweep is: every plane of the first parity (neighbour planes still
// old), then every plane of the second parity (neighbour planes already
// new); inside a plane the four sub-colours s = (i%2) + 2(j%2) follow one
// another. Each CTA takes one 32x32 tile of one plane, stages the x values of
// planes k-1, k, k+1 over the tile plus a 4-point halo in shared memory and
// runs the four sub-colour steps there; step t also recomputes its
// sub-colour on a halo of 3 - t points so that the next steps find new
// values at the tile edge without talking to other CTAs. Coefficients are
// read from global memory (each once per computed point). The x planes are
// staged with cp.async (zero fill off the array), and every sub-colour step
// walks a fixed (TT/2 + h)^2 grid of its points, so the slot-to-point map is
// compile-time arithmetic.
//
// Reads and writes go to different buffers (ping-pong): the first-parity
// launch reads `cur` and writes the first-parity planes of `alt`; the
// second-parity launch reads its own planes from `cur` and the neighbour
// planes from `alt`, and writes `alt`. No CTA can therefore see a value that
// another CTA has already advanced, and the new state is all in `alt`.
// The per-point arithmetic is the reference's (sums27 order), so the result
// is bit-identical to the colour-by-colour sweep.
#pragma once

#include "stencil_kernels.cuh"

namespace pmg {

constexpr int kH27 = 4; // staged halo
// tile edges the launcher can use (x and y); threads per CTA by tile
constexpr int kGs27Tiles[3] = {8, 16, 32};
template <int TT> struct Gs27Tile {
  static constexpr int W = TT + 2 * kH27;
  static constexpr int THREADS = TT >= 32 ? 256 : TT >= 16 ? 128 : 64;
};

// The couplings, right-hand side and diagonal of one point; loaded in full
// before any of it is used (fewer live registers than interleaving the loads
// with the sums).
template <typename T> struct Gs27Point {
  T a[26]; // sums27's couplings in its order: tO (8), tU (9), tD (9)
  T f, d;  // right-hand side, diagonal (oC + cc)
};

template <typename T>
__device__ __forceinline__ void gs27_load(const Op14<T> &A, const T *cc,
                                          const T *fc, int p, int sy, int sz,
                                          Gs27Point<T> &c) {
  const T *const *a = A.a;
  c.a[0] = a[kON][p];
  c.a[1] = a[kON][p - sy];
  c.a[2] = a[kOE][p];
  c.a[3] = a[kOE][p - 1];
  c.a[4] = a[kONE][p];
  c.a[5] = a[kONW][p];
  c.a[6] = a[kONW][p + 1 - sy];
  c.a[7] = a[kONE][p - 1 - sy];
  c.a[8] = a[kUC][p];
  c.a[9] = a[kUN][p];
  c.a[10] = a[kUS][p];
  c.a[11] = a[kUE][p];
  c.a[12] = a[kUW][p];
  c.a[13] = a[kUNE][p];
  c.a[14] = a[kUNW][p];
  c.a[15] = a[kUSE][p];
  c.a[16] = a[kUSW][p];
  c.a[17] = a[kUC][p - sz];
  c.a[18] = a[kUS][p + sy - sz];
  c.a[19] = a[kUN][p - sy - sz];
  c.a[20] = a[kUW][p + 1 - sz];
  c.a[21] = a[kUE][p - 1 - sz];
  c.a[22] = a[kUSW][p + 1 + sy - sz];
  c.a[23] = a[kUSE][p - 1 + sy - sz];
  c.a[24] = a[kUNW][p + 1 - sy - sz];
  c.a[25] = a[kUNE][p - 1 - sy - sz];
  c.f = fc[p];
  c.d = a[kOC][p] + (cc ? cc[p] : T(0));
}

// The new value from x staged around the point (xc: plane k, xd: k-1, xu:
// k+1, rows w apart): (f + (tO + tU + tD)) / (oC + cc), sums27's order.
template <typename T, int w>
__device__ __forceinline__ T gs27_update(const Gs27Point<T> &c, const T *xc,
                                         const T *xd, const T *xu) {
  const T tO = c.a[0] * xc[w] + c.a[1] * xc[-w] + c.a[2] * xc[1] +
               c.a[3] * xc[-1] + c.a[4] * xc[1 + w] + c.a[5] * xc[-1 + w] +
               c.a[6] * xc[1 - w] + c.a[7] * xc[-1 - w];
  const T tU = c.a[8] * xu[0] + c.a[9] * xu[w] + c.a[10] * xu[-w] +
               c.a[11] * xu[1] + c.a[12] * xu[-1] + c.a[13] * xu[1 + w] +
               c.a[14] * xu[-1 + w] + c.a[15] * xu[1 - w] +
               c.a[16] * xu[-1 - w];
  const T tD = c.a[17] * xd[0] + c.a[18] * xd[w] + c.a[19] * xd[-w] +
               c.a[20] * xd[1] + c.a[21] * xd[-1] + c.a[22] * xd[1 + w] +
               c.a[23] * xd[-1 + w] + c.a[24] * xd[1 - w] +
               c.a[25] * xd[-1 - w];
  return (c.f + (tO + tU + tD)) / c.d;
}

// Sub-colour step with halo H (step 3 - H of the phase): the points of the
// step's sub-colour within H of the tile, a fixed NU x NU grid of them
// clipped to the interior. xk: the staged plane k, its entry 0 at
// (ti0 - 4, tj0 - 4), rows W apart; planes k - 1 and k + 1 at xk -/+ PS.
template <typename T, int TT, int W, int PS, int H>
__device__ __forceinline__ void gs27_step_at(const Dims &d, const Op14<T> &A,
                                             const T *cc, const T *fc, T *xk,
                                             int ti0, int tj0, int k,
                                             int order) {
  constexpr int NT = Gs27Tile<TT>::THREADS;
  constexpr int NU = TT / 2 + H, NQ = NU * NU;
  const int sy = d.sy(), sz = d.sz();
  const int s = (order >> (2 * (3 - H))) & 3;
  const int pi = s & 1, pj = s >> 1;
  // first point of the sub-colour at or after ti0 - H (tj0 - H)
  const int ia = ti0 - H + ((pi - (ti0 - H)) & 1);
  const int ja = tj0 - H + ((pj - (tj0 - H)) & 1);
  const int i_lo = ti0 - kH27, j_lo = tj0 - kH27;
  const int i_max = d.nx - 1, j_max = d.ny - 1;
#pragma unroll
  for (int m = 0; m < (NQ + NT - 1) / NT; ++m) {
    const int q = threadIdx.x + m * NT;
    const int v = q / NU, u = q - v * NU;
    const int i = ia + 2 * u, j = ja + 2 * v;
    if (q < NQ && i >= 2 && i <= i_max && j >= 2 && j <= j_max) {
      const int sidx = (i - i_lo) + W * (j - j_lo);
      Gs27Point<T> c;
      gs27_load(A, cc, fc, d.at(i, j, k), sy, sz, c);
      xk[sidx] =
          gs27_update<T, W>(c, &xk[sidx], &xk[sidx - PS], &xk[sidx + PS]);
    }
  }
}

// gs27_step_at on the staged planes of gs27_phase_kernel (W x W each, plane
// k - 1 first)
template <typename T, int TT, int H>
__device__ __forceinline__ void gs27_step(const Dims &d, const Op14<T> &A,
                                          const T *cc, const T *fc, T *xs,
                                          int ti0, int tj0, int k,
                                          int order) {
  constexpr int W = Gs27Tile<TT>::W;
  gs27_step_at<T, TT, W, W * W, H>(d, A, cc, fc, xs + W * W, ti0, tj0, k,
                                   order);
}

// One parity phase on TT x TT tiles. kfirst: first plane of the parity (2 or
// 3); order: the four sub-colours in visiting order, 2 bits each (step t in
// bits 2t..2t+1).
template <typename T, int TT>
__global__ void __launch_bounds__(Gs27Tile<TT>::THREADS)
    gs27_phase_kernel(Dims d, Op14<T> A, const T *__restrict__ cc,
                      const T *__restrict__ fc, const T *__restrict__ own,
                      const T *nb, T *out, int kfirst, int order) {
  constexpr int W = Gs27Tile<TT>::W, NT = Gs27Tile<TT>::THREADS;
  // planes k-1 (nb), k (own), k+1 (nb), W x W points each
  __shared__ __align__(16) T xs[3 * W * W];
  const int ti0 = 2 + blockIdx.x * TT, tj0 = 2 + blockIdx.y * TT;
  const int k = kfirst + 2 * blockIdx.z;
  const int i_lo = ti0 - kH27, j_lo = tj0 - kH27;

  // points off the array are never read by an update and are set to zero
  for (int q = threadIdx.x; q < 3 * W * W; q += NT) {
    const int pl = q / (W * W), rem = q - pl * (W * W);
    const int jj = rem / W, ii = rem - jj * W;
    const int i = i_lo + ii, j = j_lo + jj;
    const bool in = i >= 1 && i <= d.nx && j >= 1 && j <= d.ny;
    const T *src = (pl == 1 ? own : nb) + (in ? d.at(i, j, k - 1 + pl) : 0);
    cp_async_zfill<sizeof(T)>(&xs[q], src, in);
  }
  cp_async_wait_all();
  __syncthreads();
  gs27_step<T, TT, 3>(d, A, cc, fc, xs, ti0, tj0, k, order);
  __syncthreads();
  gs27_step<T, TT, 2>(d, A, cc, fc, xs, ti0, tj0, k, order);
  __syncthreads();
  gs27_step<T, TT, 1>(d, A, cc, fc, xs, ti0, tj0, k, order);
  __syncthreads();
  gs27_step<T, TT, 0>(d, A, cc, fc, xs, ti0, tj0, k, order);
  __syncthreads();

  // write the tile's interior points of plane k
  const int i_max = d.nx - 1, j_max = d.ny - 1;
#pragma unroll
  for (int m = 0; m < (TT * TT + NT - 1) / NT; ++m) {
    const int q = threadIdx.x + m * NT;
    const int jj = q / TT, ii = q - jj * TT;
    const int i = ti0 + ii, j = tj0 + jj;
    if (q < TT * TT && i <= i_max && j <= j_max)
      out[d.at(i, j, k)] = xs[W * W + (i - i_lo) + W * (j - j_lo)];
  }
}

template <typename T, int TT>
void launch_gs27_phase(const Dims &d, const Op14<T> &A, const T *cc,
                       const T *fc, const T *own, const T *nb, T *out,
                       int kfirst, int order, int planes, cudaStream_t s) {
  const unsigned tx = (unsigned)((d.nx - 2 + TT - 1) / TT);
  const unsigned ty = (unsigned)((d.ny - 2 + TT - 1) / TT);
  gs27_phase_kernel<T, TT>
      <<<dim3(tx, ty, (unsigned)planes), Gs27Tile<TT>::THREADS, 0, s>>>(
          d, A, cc, fc, own, nb, out, kfirst, order);
}

// Tile edge for a level: the tuned choice when pmg_build_hierarchy measured
// one for this grid and element size (gs27_tune), else by size. Every tile
// gives bit-identical results; only the speed differs.
int gs27_tile_for(const Dims &d, int esize);
// the edge used when nothing was measured: 32 from 97 points per axis, 16
// from 49, else 8
int gs27_tile_by_size(const Dims &d);
// whether pmg_build_hierarchy measures tile edges (pmg_set_autotune mode 1)
bool gs27_autotune_on();

// nsweeps eight-colour sweeps starting from x in `cur`, ping-ponging with
// `alt` (whose shell must equal cur's). Returns the buffer holding the
// result through *result. tile 0 picks gs27_tile_for.
template <typename T>
int launch_gs27_pp(const Dims &d, const Op14<T> &A, const T *cc, const T *fc,
                   T *cur, T *alt, int nsweeps, int iadjoint, int zero_init,
                   cudaStream_t s, T **result, int tile = 0) {
  if (zero_init)
    PMG_CUDA_TRY(cudaMemsetAsync(cur, 0, sizeof(T) * d.count(), s));
  if (tile == 0)
    tile = gs27_tile_for(d, (int)sizeof(T));
  // visiting order of the colours c = sub + 4 * kpar
  const int first_par = iadjoint ? 1 : 0;
  const int order = iadjoint ? (3 | 2 << 2 | 1 << 4 | 0 << 6)
                             : (0 | 1 << 2 | 2 << 4 | 3 << 6);
  for (int sw = 0; sw < nsweeps; ++sw) {
    for (int ph = 0; ph < 2; ++ph) {
      const int par = ph == 0 ? first_par : 1 - first_par;
      const int kfirst = par == 0 ? 2 : 3;
      const int planes = kfirst > d.nz - 1 ? 0 : (d.nz - 1 - kfirst) / 2 + 1;
      if (planes == 0)
        continue;
      const T *nb = ph == 0 ? cur : alt;
      if (tile == 8)
        launch_gs27_phase<T, 8>(d, A, cc, fc, cur, nb, alt, kfirst, order,
                                planes, s);
      else if (tile == 16)
        launch_gs27_phase<T, 16>(d, A, cc, fc, cur, nb, alt, kfirst, order,
                                 planes, s);
      else
        launch_gs27_phase<T, 32>(d, A, cc, fc, cur, nb, alt, kfirst, order,
                                 planes, s);
    }
    T *t = cur;
    cur = alt;
    alt = t;
  }
  PMG_LAUNCH_CHECK();
  *result = cur;
  return PMG_OK;
}

// Measures every tile edge on a level (two sweeps each, CUDA events, best of
// three) and records the fastest for gs27_tile_for; the size rule's edge
// is kept unless another is more than 10% faster. x and alt are scratch
// iterates of the level (same shell); synchronises the stream.
template <typename T>
int gs27_tune(const Dims &d, const Op14<T> &A, const T *fc, T *x, T *alt,
              cudaStream_t s);
void gs27_tile_record(const Dims &d, int esize, int tile);
bool gs27_tile_known(const Dims &d, int esize);

} // namespace pmg
