// Red-black Gauss-Seidel on the 7-point operator, NS sweeps (two colours
// each) in one launch.
//
// The reference runs one parallel launch per colour (Vgsrb7x,
// pmgc/gsd.cc:81-110): every launch streams all coefficients. Here a CTA owns
// a TX x TY tile of (x, y) and a chunk [k0, k1] of planes and walks it as a
// wavefront: at step t it loads plane t + 2NS, then brings plane t+2NS-1-h to
// half-sweep level h for h = 0 .. 2NS-1 (level h updates the colour of
// half-sweep h from its six neighbours at level h-1), and plane t is final.
// Planes live in a rolling window of 2NS+2 planes in shared memory, updated in
// place: an update at level h only reads the other colour, which its
// neighbour planes hold at level h-1 or h. Level h is computed on an in-plane
// and k halo of 2NS-1-h points around the CTA's core so that the final
// values need nothing from other CTAs; the redundant halo work is the price
// of one pass over memory for NS sweeps instead of 2 NS passes.
//
// The launch reads x from `in` and writes the core points to `out` (a
// different buffer with the same shell), so no CTA ever reads a value that
// another CTA has already advanced. Per-point arithmetic is the reference's,
// so the result is bit-identical to NS reference sweeps.
#pragma once

#include "stencil_kernels.cuh"

namespace pmg {

template <typename T> struct Gs7Tile;
template <> struct Gs7Tile<float> {
  static constexpr int TX = 64, TY = 16;
};
template <> struct Gs7Tile<double> {
  static constexpr int TX = 32, TY = 16;
};

template <typename T, int NS>
__global__ void __launch_bounds__(256)
    gs7_fused_kernel(Dims d, const T *__restrict__ oC,
                     const T *__restrict__ cc, const T *__restrict__ fc,
                     const T *__restrict__ oE, const T *__restrict__ oN,
                     const T *__restrict__ uC, const T *__restrict__ in,
                     T *__restrict__ out, int chunk, int iadjoint,
                     int zero_init) {
  constexpr int TX = Gs7Tile<T>::TX, TY = Gs7Tile<T>::TY;
  constexpr int HL = 2 * NS;          // staged halo
  constexpr int W = TX + 2 * HL, H = TY + 2 * HL;
  constexpr int NP = 2 * NS + 2;      // planes in the window
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *win = reinterpret_cast<T *>(smem_raw); // [NP][H][W]

  const int ti0 = 2 + blockIdx.x * TX, tj0 = 2 + blockIdx.y * TY;
  const int k0 = 2 + blockIdx.z * chunk;
  const int k1 = min(k0 + chunk - 1, d.nz - 1);
  const int i_lo = ti0 - HL, j_lo = tj0 - HL;
  const int sy = d.sy(), sz = d.sz();
  const int imax = d.nx - 1, jmax = d.ny - 1, kmax = d.nz - 1;

  auto slot = [&](int p) { return ((p % NP) + NP) % NP; };
  auto load_plane = [&](int p) {
    if (p < 1 || p > d.nz)
      return;
    T *dst = win + slot(p) * (W * H);
    for (int q = threadIdx.x; q < W * H; q += blockDim.x) {
      const int jj = q / W, ii = q - jj * W;
      const int i = i_lo + ii, j = j_lo + jj;
      T v = T(0);
      if (i >= 1 && i <= d.nx && j >= 1 && j <= d.ny)
        v = in[d.at(i, j, p)];
      dst[q] = v;
    }
  };

  const int t_first = k0 - 2 * (2 * NS - 1);
  load_plane(k0 - HL);
  load_plane(k0 - HL + 1);
  for (int t = t_first; t <= k1; ++t) {
    if (t + HL <= k1 + HL)
      load_plane(t + HL);
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2 * NS; ++h) {
      const int e = 2 * NS - 1 - h; // halo of this level
      const int p = t + 2 * NS - 1 - h;
      if (p >= max(k0 - e, 2) && p <= min(k1 + e, kmax)) {
        const int c = h & 1;
        const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
        const T keep = (zero_init && h == 0) ? T(0) : T(1);
        const int ia = max(ti0 - e, 2), ib = min(ti0 + TX - 1 + e, imax);
        const int ja = max(tj0 - e, 2), jb = min(tj0 + TY - 1 + e, jmax);
        const int nj = jb - ja + 1;
        // points of the colour: in row j the first i has parity of
        // want - j - p
        const int ni2 = (ib - ia + 2) / 2;
        T *xc = win + slot(p) * (W * H);
        const T *xd = win + slot(p - 1) * (W * H);
        const T *xu = win + slot(p + 1) * (W * H);
        for (int q = threadIdx.x; q < ni2 * nj; q += blockDim.x) {
          const int qj = q / ni2;
          const int j = ja + qj;
          const int i = ia + ((want - ia - j - p) & 1) + 2 * (q - qj * ni2);
          if (i > ib || nj <= 0)
            continue;
          const int g = d.at(i, j, p);
          const int s = (i - i_lo) + W * (j - j_lo);
          const T sum = oN[g] * xc[s + W] + oN[g - sy] * xc[s - W] +
                        oE[g] * xc[s + 1] + oE[g - 1] * xc[s - 1] +
                        uC[g - sz] * xd[s] + uC[g] * xu[s];
          const T ccv = cc ? cc[g] : T(0);
          xc[s] = (fc[g] + keep * sum) / (oC[g] + ccv);
        }
      }
      __syncthreads();
    }
    // plane t is final: write the core
    if (t >= k0) {
      const T *xc = win + slot(t) * (W * H);
      for (int q = threadIdx.x; q < TX * TY; q += blockDim.x) {
        const int jj = q / TX, ii = q - jj * TX;
        const int i = ti0 + ii, j = tj0 + jj;
        if (i <= imax && j <= jmax)
          out[d.at(i, j, t)] = xc[(i - i_lo) + W * (j - j_lo)];
      }
    }
  }
}

template <typename T, int NS> constexpr size_t gs7_fused_smem() {
  constexpr int TX = Gs7Tile<T>::TX, TY = Gs7Tile<T>::TY;
  return sizeof(T) * (2 * NS + 2) * (TX + 4 * NS) * (TY + 4 * NS);
}

// Chunk of planes per CTA: enough CTAs to cover the GPU about twice.
inline int gs7_chunk(const Dims &d, int tx, int ty) {
  const long tiles = (long)((d.nx - 2 + tx - 1) / tx) *
                     ((d.ny - 2 + ty - 1) / ty);
  const int planes = d.nz - 2;
  long want_chunks = (2 * 148 + tiles - 1) / tiles;
  if (want_chunks < 1)
    want_chunks = 1;
  int chunk = (int)((planes + want_chunks - 1) / want_chunks);
  return chunk < 8 ? (planes < 8 ? planes : 8) : chunk;
}

// nsweeps red-black sweeps from `cur`, ping-ponging with `alt` (same shell);
// *result gets the buffer holding the final iterate.
template <typename T>
int launch_gs7_fused(const Dims &d, const T *oC, const T *cc, const T *fc,
                     const T *oE, const T *oN, const T *uC, T *cur, T *alt,
                     int nsweeps, int iadjoint, int zero_init, cudaStream_t s,
                     T **result) {
  constexpr int TX = Gs7Tile<T>::TX, TY = Gs7Tile<T>::TY;
  static bool configured = false;
  if (!configured) {
    PMG_CUDA_TRY(cudaFuncSetAttribute(
        gs7_fused_kernel<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)gs7_fused_smem<T, 2>()));
    PMG_CUDA_TRY(cudaFuncSetAttribute(
        gs7_fused_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)gs7_fused_smem<T, 1>()));
    configured = true;
  }
  const int chunk = gs7_chunk(d, TX, TY);
  const dim3 grid((d.nx - 2 + TX - 1) / TX, (d.ny - 2 + TY - 1) / TY,
                  (d.nz - 2 + chunk - 1) / chunk);
  int left = nsweeps;
  while (left > 0) {
    if (left >= 2) {
      gs7_fused_kernel<T, 2><<<grid, 256, gs7_fused_smem<T, 2>(), s>>>(
          d, oC, cc, fc, oE, oN, uC, cur, alt, chunk, iadjoint, zero_init);
      left -= 2;
    } else {
      gs7_fused_kernel<T, 1><<<grid, 256, gs7_fused_smem<T, 1>(), s>>>(
          d, oC, cc, fc, oE, oN, uC, cur, alt, chunk, iadjoint, zero_init);
      left -= 1;
    }
    zero_init = 0;
    T *t = cur;
    cur = alt;
    alt = t;
  }
  PMG_LAUNCH_CHECK();
  *result = cur;
  return PMG_OK;
}

} // namespace pmg
