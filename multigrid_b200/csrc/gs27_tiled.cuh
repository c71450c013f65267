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
// read from global memory (each once per computed point).
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

template <typename T, int w>
__device__ __forceinline__ void sums27_tile(const Op14<T> &A, int p, int sy,
                                            int sz, const T *xc, const T *xd,
                                            const T *xu, T &tO, T &tU,
                                            T &tD) {
  const T *const *a = A.a;
  tO = a[kON][p] * xc[w] + a[kON][p - sy] * xc[-w] + a[kOE][p] * xc[1] +
       a[kOE][p - 1] * xc[-1] + a[kONE][p] * xc[1 + w] +
       a[kONW][p] * xc[-1 + w] + a[kONW][p + 1 - sy] * xc[1 - w] +
       a[kONE][p - 1 - sy] * xc[-1 - w];
  tU = a[kUC][p] * xu[0] + a[kUN][p] * xu[w] + a[kUS][p] * xu[-w] +
       a[kUE][p] * xu[1] + a[kUW][p] * xu[-1] + a[kUNE][p] * xu[1 + w] +
       a[kUNW][p] * xu[-1 + w] + a[kUSE][p] * xu[1 - w] +
       a[kUSW][p] * xu[-1 - w];
  tD = a[kUC][p - sz] * xd[0] + a[kUS][p + sy - sz] * xd[w] +
       a[kUN][p - sy - sz] * xd[-w] + a[kUW][p + 1 - sz] * xd[1] +
       a[kUE][p - 1 - sz] * xd[-1] + a[kUSW][p + 1 + sy - sz] * xd[1 + w] +
       a[kUSE][p - 1 + sy - sz] * xd[-1 + w] +
       a[kUNW][p + 1 - sy - sz] * xd[1 - w] +
       a[kUNE][p - 1 - sy - sz] * xd[-1 - w];
}

// One parity phase on TT x TT tiles. kfirst: first plane of the parity (2 or
// 3); order: the four sub-colours in visiting order, 2 bits each (step t in
// bits 2t..2t+1).
template <typename T, int TT>
__global__ void __launch_bounds__(Gs27Tile<TT>::THREADS)
    gs27_phase_kernel(Dims d, Op14<T> A, const T *__restrict__ cc,
                      const T *__restrict__ fc, const T *__restrict__ own,
                      const T *nb, T *out, int kfirst, int order) {
  constexpr int kT27 = TT, kW27 = Gs27Tile<TT>::W;
  __shared__ T xs[3][kW27 * kW27];
  const int ti0 = 2 + blockIdx.x * kT27;
  const int tj0 = 2 + blockIdx.y * kT27;
  const int k = kfirst + 2 * blockIdx.z;
  const int sy = d.sy(), sz = d.sz();
  const int i_lo = ti0 - kH27, j_lo = tj0 - kH27;

  // stage planes k-1 (nb), k (own), k+1 (nb); points off the array are
  // never read by an update and are set to zero
  for (int q = threadIdx.x; q < 3 * kW27 * kW27; q += blockDim.x) {
    const int pl = q / (kW27 * kW27);
    const int rem = q - pl * kW27 * kW27;
    const int jj = rem / kW27, ii = rem - jj * kW27;
    const int i = i_lo + ii, j = j_lo + jj, kk = k - 1 + pl;
    T v = T(0);
    if (i >= 1 && i <= d.nx && j >= 1 && j <= d.ny) {
      const int g = d.at(i, j, kk);
      v = pl == 1 ? own[g] : nb[g];
    }
    xs[pl][rem] = v;
  }
  __syncthreads();

  const int i_max = d.nx - 1, j_max = d.ny - 1;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int s = (order >> (2 * t)) & 3;
    const int h = 3 - t;
    const int pi = s & 1, pj = (s >> 1) & 1;
    // region of this step, clipped to the interior, first point of parity
    int ia = max(ti0 - h, 2), ib = min(ti0 + kT27 - 1 + h, i_max);
    int ja = max(tj0 - h, 2), jb = min(tj0 + kT27 - 1 + h, j_max);
    ia += (pi - ia) & 1;
    ja += (pj - ja) & 1;
    const int ni = ib >= ia ? (ib - ia) / 2 + 1 : 0;
    const int nj = jb >= ja ? (jb - ja) / 2 + 1 : 0;
    for (int q = threadIdx.x; q < ni * nj; q += blockDim.x) {
      const int qj = q / ni;
      const int i = ia + 2 * (q - qj * ni), j = ja + 2 * qj;
      const int p = d.at(i, j, k);
      const int sidx = (i - i_lo) + kW27 * (j - j_lo);
      T tO, tU, tD;
      sums27_tile<T, kW27>(A, p, sy, sz, &xs[1][sidx], &xs[0][sidx],
                           &xs[2][sidx], tO, tU, tD);
      const T c = cc ? cc[p] : T(0);
      xs[1][sidx] = (fc[p] + (tO + tU + tD)) / (A.a[kOC][p] + c);
    }
    __syncthreads();
  }

  // write the tile's interior points of plane k
  for (int q = threadIdx.x; q < kT27 * kT27; q += blockDim.x) {
    const int jj = q / kT27, ii = q - jj * kT27;
    const int i = ti0 + ii, j = tj0 + jj;
    if (i <= i_max && j <= j_max)
      out[d.at(i, j, k)] = xs[1][(i - i_lo) + kW27 * (j - j_lo)];
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
// three) and records the fastest for gs27_tile_for. x and alt are scratch
// iterates of the level (same shell); synchronises the stream.
template <typename T>
int gs27_tune(const Dims &d, const Op14<T> &A, const T *fc, T *x, T *alt,
              cudaStream_t s);
void gs27_tile_record(const Dims &d, int esize, int tile);
bool gs27_tile_known(const Dims &d, int esize);

} // namespace pmg
