// One red-black sweep of the 7-point operator per launch, both colours in
// one pass over the arrays (Vgsrb7x, pmgc/gsd.cc:61-111, one iteration).
//
// The reference runs one launch per colour, so every sweep streams the
// coefficients twice. Here a CTA owns a TXC x TY tile of (i, j) columns and a
// chunk [k0, k1] of planes and marches up the planes as a wavefront: step t
// updates the first colour of plane t+1 over the tile plus a one-point ring
// (so the tile edge sees new values without talking to other CTAs) and then
// the second colour of plane t, which is then final and written out.
//
// Every plane of the six arrays (x, oC, oE, oN, uC, f) over the tile plus a
// two-point ring is staged in a ring of shared-memory stages by cp.async
// copies issued D planes ahead, so the loads of a plane are in flight for two
// steps before they are needed and the updates only read shared memory. Each
// thread owns a pair of adjacent columns (i, i+1) -- one point of each colour
// per plane -- and copies and updates its own pair: every lane works in both
// colour phases, and a step needs a single barrier. (Bulk tensor copies
// would need a 16-byte row pitch; the reference layout has rows of
// 4*(2^k+1) bytes.) The chunk's edge plane k0-1 gets its first colour
// recomputed locally.
//
// The launch reads x from `in` and writes the tile cores to `out` (same
// shell), so no CTA reads a value another CTA has already advanced.
// Per-point arithmetic is gs7_color_kernel's: the result is bit-identical to
// one reference sweep.
#pragma once

#include "stencil_kernels.cuh"

namespace pmg {

__device__ __forceinline__ void ring_cp_async(unsigned s, const float *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(g));
}
__device__ __forceinline__ void ring_cp_async(unsigned s, const double *g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(g));
}
__device__ __forceinline__ void ring_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N> __device__ __forceinline__ void ring_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// core tile TXC x TY (TXC even), D planes of prefetch
template <typename T, int TXC_, int TY_, int D_> struct Gs7RingShape {
  using type = T;
  static constexpr int TXC = TXC_, TY = TY_, D = D_;
  static constexpr int W = TXC + 4, H = TY + 4, SLOT = W * H, NARR = 6;
  static constexpr int S = D + 3; // stages: planes t-1 .. t+D in use
  static constexpr int THREADS = (W / 2) * H;
  static constexpr size_t bytes() {
    return sizeof(T) * (size_t)S * NARR * SLOT;
  }
  static_assert(TXC % 2 == 0 && D >= 2, "bad ring shape");
};

template <typename T> struct Gs7RingDefault;
template <> struct Gs7RingDefault<float> {
  using shape = Gs7RingShape<float, 60, 8, 3>;
};
template <> struct Gs7RingDefault<double> {
  using shape = Gs7RingShape<double, 28, 12, 3>;
};

template <class C>
__global__ void __launch_bounds__(C::THREADS)
    gs7_ring_kernel(Dims d, const typename C::type *__restrict__ oC,
                    const typename C::type *__restrict__ oE,
                    const typename C::type *__restrict__ oN,
                    const typename C::type *__restrict__ uC,
                    const typename C::type *__restrict__ fc,
                    const typename C::type *__restrict__ in,
                    typename C::type *__restrict__ out, int chunk,
                    int want_first, typename C::type keep) {
  using T = typename C::type;
  constexpr int TXC = C::TXC, TY = C::TY, W = C::W, SLOT = C::SLOT;
  constexpr int NARR = C::NARR, S = C::S, D = C::D;
  // array order inside a stage: 0 x, 1 oC, 2 oE, 3 oN, 4 uC, 5 f
  extern __shared__ __align__(16) unsigned char ring_raw[];
  T *ring = reinterpret_cast<T *>(ring_raw);
  const unsigned ring_s = (unsigned)__cvta_generic_to_shared(ring);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ti0 = 2 + blockIdx.x * TXC, tj0 = 2 + blockIdx.y * TY;
  const int k0 = 2 + blockIdx.z * chunk;
  const int k1 = min(k0 + chunk - 1, d.nz - 1);
  const int imax = d.nx - 1, jmax = d.ny - 1, kmax = d.nz - 1;
  const int sz = d.sz();
  const int p_first = k0 - 2, p_last = k1 + 2;

  const int ia = ti0 - 2 + 2 * tx, j = tj0 - 2 + ty;
  const int sa = 2 * tx + W * ty;
  const bool in_j = j >= 1 && j <= d.ny;
  const bool in_a = in_j && ia >= 1 && ia <= d.nx;
  const bool in_b = in_j && ia + 1 >= 1 && ia + 1 <= d.nx;
  const int ga = in_a ? d.at(ia, j, 1) : 0;
  const int gb = in_b ? d.at(ia + 1, j, 1) : 0;
  const bool ring_j = j >= tj0 - 1 && j <= tj0 + TY && j >= 2 && j <= jmax;
  const bool core_j = j >= tj0 && j < tj0 + TY && j <= jmax;

  auto stage = [&](int p) { return (p - p_first) % S; };
  auto issue = [&](int p) {
    if (p <= p_last) {
      const int st = stage(p);
      T *base = ring + st * NARR * SLOT + sa;
      const unsigned sbase =
          ring_s + (unsigned)((st * NARR * SLOT + sa) * sizeof(T));
      const bool plane_in = p >= 1 && p <= d.nz;
      const long off = (long)(p - 1) * sz;
      const T *src[NARR] = {in, oC, oE, oN, uC, fc};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const bool ok = plane_in && (c ? in_b : in_a);
        const long g = off + (c ? gb : ga);
#pragma unroll
        for (int a = 0; a < NARR; ++a) {
          if (ok)
            ring_cp_async(sbase + (unsigned)((a * SLOT + c) * sizeof(T)),
                          src[a] + g);
          else
            base[a * SLOT + c] = T(0);
        }
      }
    }
    ring_commit();
  };

  const int t_first = k0 - 2;
#pragma unroll 1
  for (int u = 0; u < D; ++u)
    issue(p_first + u);
#pragma unroll 1
  for (int t = t_first; t <= k1; ++t) {
    issue(t + D);
    ring_wait<D - 2>(); // this thread's copies of planes up to t+2 landed
    __syncthreads();    // ... and everyone's
    const int p1 = t + 1;
    // the pair's column whose point of plane t+1 has the first colour: its
    // point of plane t has the second colour; the other column's point of
    // plane t has the first colour (updated in the previous step)
    const int c = (want_first - ia - j - p1) & 1;
    const int s = sa + c, so = sa + 1 - c;
    const int i = ia + c, io = ia + 1 - c;
    const long gc = (long)(t - 1) * sz + (c ? gb : ga);
    const long go = (long)(t - 1) * sz + (c ? ga : gb);
    T *X0 = ring + stage(t) * NARR * SLOT;
    T *X1 = ring + stage(p1) * NARR * SLOT;
    // first colour of plane t+1 over the tile and its one-point ring
    if (p1 >= 2 && p1 <= kmax && ring_j && i >= ti0 - 1 && i <= ti0 + TXC &&
        i >= 2 &&
        i <= imax) {
      const T *X2 = ring + stage(t + 2) * NARR * SLOT;
      const T *E = X1 + 2 * SLOT, *N = X1 + 3 * SLOT;
      const T sum = N[s] * X1[s + W] + N[s - W] * X1[s - W] +
                    E[s] * X1[s + 1] + E[s - 1] * X1[s - 1] +
                    X0[4 * SLOT + s] * X0[s] + X1[4 * SLOT + s] * X2[s];
      X1[s] = (X1[5 * SLOT + s] + keep * sum) / (X1[SLOT + s] + T(0));
    }
    if (t >= k0 && core_j) {
      // second colour of plane t on the core; plane t is then final there
      if (i >= ti0 && i < ti0 + TXC && i <= imax) {
        const T *Xm = ring + stage(t - 1) * NARR * SLOT;
        const T *E = X0 + 2 * SLOT, *N = X0 + 3 * SLOT;
        const T sum = N[s] * X0[s + W] + N[s - W] * X0[s - W] +
                      E[s] * X0[s + 1] + E[s - 1] * X0[s - 1] +
                      Xm[4 * SLOT + s] * Xm[s] + X0[4 * SLOT + s] * X1[s];
        out[gc] = (X0[5 * SLOT + s] + sum) / (X0[SLOT + s] + T(0));
      }
      if (io >= ti0 && io < ti0 + TXC && io <= imax)
        out[go] = X0[so];
    }
  }
  ring_wait<0>();
}

// Planes per CTA: about one wave of CTAs (blocks_per_sm resident per SM).
inline int gs7_ring_chunk(const Dims &d, int txc, int ty, int blocks_per_sm,
                          int sms) {
  const long tiles = (long)((d.nx - 2 + txc - 1) / txc) *
                     ((d.ny - 2 + ty - 1) / ty);
  const int planes = d.nz - 2;
  long chunks = ((long)blocks_per_sm * sms) / (tiles > 0 ? tiles : 1);
  if (chunks < 1)
    chunks = 1;
  const int chunk = (int)((planes + chunks - 1) / chunks);
  return chunk < 8 ? (planes < 8 ? planes : 8) : chunk;
}

// nsweeps sweeps (Vgsrb7x with cc = 0) from `cur`, ping-ponging with `alt`
// (same shell); *result gets the buffer holding the final iterate.
// zero_init drops the old values in the first colour of the first sweep.
template <class C>
int launch_gs7_ring_shape(const Dims &d, const typename C::type *oC,
                          const typename C::type *fc,
                          const typename C::type *oE,
                          const typename C::type *oN,
                          const typename C::type *uC, typename C::type *cur,
                          typename C::type *alt, int nsweeps, int iadjoint,
                          int zero_init, cudaStream_t s,
                          typename C::type **result) {
  using T = typename C::type;
  static int per_sm = 0, sms = 0;
  if (!per_sm) {
    PMG_CUDA_TRY(cudaFuncSetAttribute(
        gs7_ring_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)C::bytes()));
    PMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, gs7_ring_kernel<C>, C::THREADS, C::bytes()));
    int dev = 0;
    PMG_CUDA_TRY(cudaGetDevice(&dev));
    PMG_CUDA_TRY(
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1)
      per_sm = 1;
  }
  const int chunk = gs7_ring_chunk(d, C::TXC, C::TY, per_sm, sms);
  const dim3 grid((d.nx - 2 + C::TXC - 1) / C::TXC,
                  (d.ny - 2 + C::TY - 1) / C::TY,
                  (d.nz - 2 + chunk - 1) / chunk);
  const dim3 block(C::W / 2, C::H);
  for (int sw = 0; sw < nsweeps; ++sw) {
    const T keep = (sw == 0 && zero_init) ? T(0) : T(1);
    gs7_ring_kernel<C><<<grid, block, C::bytes(), s>>>(
        d, oC, oE, oN, uC, fc, cur, alt, chunk, iadjoint, keep);
    T *t = cur;
    cur = alt;
    alt = t;
  }
  PMG_LAUNCH_CHECK();
  *result = cur;
  return PMG_OK;
}

template <typename T>
int launch_gs7_ring(const Dims &d, const T *oC, const T *fc, const T *oE,
                    const T *oN, const T *uC, T *cur, T *alt, int nsweeps,
                    int iadjoint, int zero_init, cudaStream_t s, T **result) {
  return launch_gs7_ring_shape<typename Gs7RingDefault<T>::shape>(
      d, oC, fc, oE, oN, uC, cur, alt, nsweeps, iadjoint, zero_init, s,
      result);
}

} // namespace pmg
