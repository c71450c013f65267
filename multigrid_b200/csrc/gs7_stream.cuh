// One red-black sweep of the 7-point operator per launch, both colours in
// one pass over the arrays (Vgsrb7x, pmgc/gsd.cc:61-111, one iteration).
//
// The reference runs one launch per colour, so every sweep streams the
// coefficients twice. Here a CTA owns a TXC x TY tile of (i, j) columns and a
// chunk [k0, k1] of planes and marches up the planes as a wavefront: step t
// updates the first colour of plane t+1 over the tile plus a one-point ring
// (so the tile edge sees new values without talking to other CTAs) and then
// the second colour of plane t, which is then final and written out. Every
// thread owns a pair of adjacent columns (i, i+1) -- one point of each colour
// per plane -- and keeps its columns' values in registers: x for planes
// t-1 .. t+2 and the coefficients of planes t and t+1, while the loads of
// plane t+2 (coefficients) and t+3 (x) are in flight. Only the values other
// threads need (x, oE, oN of the plane) go through shared memory, in a ring
// of three plane slots, so a step needs a single barrier. The chunk's edge
// plane k0-1 gets its first colour recomputed locally.
//
// Threads cover the tile plus a two-point ring (the first colour of the
// one-point ring reads one point further out); the launch reads x from `in`
// and writes the tile cores to `out` (same shell), so no CTA reads a value
// another CTA has already advanced. Per-point arithmetic is
// gs7_color_kernel's: the result is bit-identical to one reference sweep.
#pragma once

#include <type_traits>

#include "stencil_kernels.cuh"

namespace pmg {

template <typename T> struct Gs7StreamShape;
// core tile (TXC x TY); the CTA is (TXC + 4) / 2 x (TY + 4) threads
template <> struct Gs7StreamShape<float> {
  static constexpr int TXC = 60, TY = 12;
};
template <> struct Gs7StreamShape<double> {
  static constexpr int TXC = 28, TY = 12;
};

template <typename T, int TXC, int TY>
__global__ void __launch_bounds__(((TXC + 4) / 2) * (TY + 4))
    gs7_stream_kernel(Dims d, const T *__restrict__ oC,
                      const T *__restrict__ oE, const T *__restrict__ oN,
                      const T *__restrict__ uC, const T *__restrict__ fc,
                      const T *__restrict__ in, T *__restrict__ out,
                      int chunk, int want_first, T keep) {
  constexpr int PW = (TXC + 4) / 2; // column pairs per row
  constexpr int W = TXC + 4, H = TY + 4;
  constexpr int SLOT = W * H;
  // three plane slots of x, oE, oN
  __shared__ T sx[3][SLOT], se[3][SLOT], sn[3][SLOT];

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ti0 = 2 + blockIdx.x * TXC, tj0 = 2 + blockIdx.y * TY;
  const int k0 = 2 + blockIdx.z * chunk;
  const int k1 = min(k0 + chunk - 1, d.nz - 1);
  const int imax = d.nx - 1, jmax = d.ny - 1, kmax = d.nz - 1;
  const int want_second = 1 - want_first;
  const int sz = d.sz();

  // the thread's columns: i = ia, ia + 1 at row j; smem offsets sa, sa + 1
  const int ia = ti0 - 2 + 2 * tx, j = tj0 - 2 + ty;
  const int sa = 2 * tx + W * ty;
  const bool in_a = ia >= 1 && ia <= d.nx && j >= 1 && j <= d.ny;
  const bool in_b = ia + 1 >= 1 && ia + 1 <= d.nx && j >= 1 && j <= d.ny;
  const int ga = in_a ? d.at(ia, j, 1) : 0;
  const int gb = in_b ? d.at(ia + 1, j, 1) : 0;
  // which of the two columns computes in each phase (ring / core)
  const bool ring_j = j >= tj0 - 1 && j <= tj0 + TY && j >= 2 && j <= jmax;
  const bool core_j = j >= tj0 && j < tj0 + TY && j <= jmax;
  auto ring_i = [&](int i) {
    return i >= ti0 - 1 && i <= ti0 + TXC && i >= 2 && i <= imax;
  };
  auto core_i = [&](int i) { return i >= ti0 && i < ti0 + TXC && i <= imax; };

  auto ld = [&](const T *a, int g, bool ok, int p) -> T {
    return (ok && p >= 1 && p <= d.nz) ? a[(long)(p - 1) * sz + g] : T(0);
  };

  // registers: [0] column a, [1] column b
  T xm1[2], x0[2], xp1[2], xp2[2], xp3[2];
  T c0[2], f0[2], e0[2], n0[2], u0[2];      // plane t
  T c1[2], f1[2], e1[2], n1[2], u1[2];      // plane t+1
  T c2[2], f2[2], e2[2], n2[2], u2[2];      // plane t+2 (in flight)
  T um1[2];                                 // uC of plane t-1
  const int t_first = k0 - 2;
  {
    const int p = t_first;
    const bool ok[2] = {in_a, in_b};
    const int g[2] = {ga, gb};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      xm1[c] = T(0);
      x0[c] = ld(in, g[c], ok[c], p);
      xp1[c] = ld(in, g[c], ok[c], p + 1);
      xp2[c] = ld(in, g[c], ok[c], p + 2);
      xp3[c] = ld(in, g[c], ok[c], p + 3);
      um1[c] = ld(uC, g[c], ok[c], p - 1);
      c0[c] = ld(oC, g[c], ok[c], p);
      f0[c] = ld(fc, g[c], ok[c], p);
      e0[c] = ld(oE, g[c], ok[c], p);
      n0[c] = ld(oN, g[c], ok[c], p);
      u0[c] = ld(uC, g[c], ok[c], p);
      c1[c] = ld(oC, g[c], ok[c], p + 1);
      f1[c] = ld(fc, g[c], ok[c], p + 1);
      e1[c] = ld(oE, g[c], ok[c], p + 1);
      n1[c] = ld(oN, g[c], ok[c], p + 1);
      u1[c] = ld(uC, g[c], ok[c], p + 1);
      c2[c] = ld(oC, g[c], ok[c], p + 2);
      f2[c] = ld(fc, g[c], ok[c], p + 2);
      e2[c] = ld(oE, g[c], ok[c], p + 2);
      n2[c] = ld(oN, g[c], ok[c], p + 2);
      u2[c] = ld(uC, g[c], ok[c], p + 2);
    }
    // plane t in its slot (old x, oE, oN) for the first step's second
    // colour, which does not run at t = k0 - 2: nothing to stage
  }
  for (int t = t_first; t <= k1; ++t) {
    const int s0 = (t - t_first) % 3, s1 = (t - t_first + 1) % 3;
    // stage plane t+1: old x and the couplings other columns read
    sx[s1][sa] = xp1[0];
    sx[s1][sa + 1] = xp1[1];
    se[s1][sa] = e1[0];
    se[s1][sa + 1] = e1[1];
    sn[s1][sa] = n1[0];
    sn[s1][sa + 1] = n1[1];
    // loads for the next steps: x of plane t+4, coefficients of plane t+3
    T xl[2], cl[2], fl[2], el[2], nl[2], ul[2];
    {
      const bool ok[2] = {in_a, in_b};
      const int g[2] = {ga, gb};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        xl[c] = ld(in, g[c], ok[c], t + 4);
        cl[c] = ld(oC, g[c], ok[c], t + 3);
        fl[c] = ld(fc, g[c], ok[c], t + 3);
        el[c] = ld(oE, g[c], ok[c], t + 3);
        nl[c] = ld(oN, g[c], ok[c], t + 3);
        ul[c] = ld(uC, g[c], ok[c], t + 3);
      }
    }
    __syncthreads();
    // first colour of plane t+1 (tile + ring), then the second colour of
    // plane t (core); both in the same column of the pair
    const int p1 = t + 1;
    const int cc = (want_first - ia - j - p1) & 1;
    auto update = [&](auto col) {
      constexpr int c = decltype(col)::value;
      const int s = sa + c;
      if (p1 >= 2 && p1 <= kmax && ring_j && ring_i(ia + c)) {
        const T *X = sx[s1], *E = se[s1], *N = sn[s1];
        const T sum = N[s] * X[s + W] + N[s - W] * X[s - W] +
                      E[s] * X[s + 1] + E[s - 1] * X[s - 1] +
                      u0[c] * x0[c] + u1[c] * xp2[c];
        const T v = (f1[c] + keep * sum) / (c1[c] + T(0));
        xp1[c] = v;
        sx[s1][s] = v;
      }
      if (t >= k0 && t <= kmax && core_j && core_i(ia + c)) {
        const T *X = sx[s0], *E = se[s0], *N = sn[s0];
        const T sum = N[s] * X[s + W] + N[s - W] * X[s - W] +
                      E[s] * X[s + 1] + E[s - 1] * X[s - 1] +
                      um1[c] * xm1[c] + u0[c] * xp1[c];
        x0[c] = (f0[c] + sum) / (c0[c] + T(0));
      }
    };
    if (cc)
      update(std::integral_constant<int, 1>());
    else
      update(std::integral_constant<int, 0>());
    // plane t is final on the core
    if (t >= k0 && t <= kmax && core_j) {
      if (core_i(ia))
        out[(long)(t - 1) * sz + ga] = x0[0];
      if (core_i(ia + 1))
        out[(long)(t - 1) * sz + gb] = x0[1];
    }
    // shift the planes
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      xm1[c] = x0[c];
      x0[c] = xp1[c];
      xp1[c] = xp2[c];
      xp2[c] = xp3[c];
      xp3[c] = xl[c];
      um1[c] = u0[c];
      c0[c] = c1[c]; f0[c] = f1[c]; e0[c] = e1[c]; n0[c] = n1[c];
      u0[c] = u1[c];
      c1[c] = c2[c]; f1[c] = f2[c]; e1[c] = e2[c]; n1[c] = n2[c];
      u1[c] = u2[c];
      c2[c] = cl[c]; f2[c] = fl[c]; e2[c] = el[c]; n2[c] = nl[c];
      u2[c] = ul[c];
    }
  }
}

// Planes per CTA: about one wave of CTAs (blocks_per_sm resident per SM).
inline int gs7_stream_chunk(const Dims &d, int txc, int ty,
                            int blocks_per_sm) {
  const long tiles = (long)((d.nx - 2 + txc - 1) / txc) *
                     ((d.ny - 2 + ty - 1) / ty);
  const int planes = d.nz - 2;
  long chunks = (blocks_per_sm * 148L) / (tiles > 0 ? tiles : 1);
  if (chunks < 1)
    chunks = 1;
  const int chunk = (int)((planes + chunks - 1) / chunks);
  return chunk < 8 ? (planes < 8 ? planes : 8) : chunk;
}

// nsweeps red-black sweeps (Vgsrb7x with cc = 0) from `cur`, ping-ponging
// with `alt` (same shell); *result gets the buffer holding the final
// iterate. zero_init drops the old values in the first colour of the first
// sweep (the reference's zero_initialize).
template <typename T>
int launch_gs7_stream(const Dims &d, const T *oC, const T *fc, const T *oE,
                      const T *oN, const T *uC, T *cur, T *alt, int nsweeps,
                      int iadjoint, int zero_init, cudaStream_t s,
                      T **result) {
  constexpr int TXC = Gs7StreamShape<T>::TXC, TY = Gs7StreamShape<T>::TY;
  const dim3 block((TXC + 4) / 2, TY + 4);
  int per_sm = 0;
  PMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, gs7_stream_kernel<T, TXC, TY>, block.x * block.y, 0));
  const int chunk = gs7_stream_chunk(d, TXC, TY, per_sm > 0 ? per_sm : 1);
  const dim3 grid((d.nx - 2 + TXC - 1) / TXC, (d.ny - 2 + TY - 1) / TY,
                  (d.nz - 2 + chunk - 1) / chunk);
  const int want_first = iadjoint; // (1 - iad) * 0 + iad * 1
  for (int sw = 0; sw < nsweeps; ++sw) {
    const T keep = (sw == 0 && zero_init) ? T(0) : T(1);
    gs7_stream_kernel<T, TXC, TY><<<grid, block, 0, s>>>(
        d, oC, oE, oN, uC, fc, cur, alt, chunk, want_first, keep);
    T *t = cur;
    cur = alt;
    alt = t;
  }
  PMG_LAUNCH_CHECK();
  *result = cur;
  return PMG_OK;
}

} // namespace pmg
