// Colour-split layout of the mixed path's finest-level float arrays.
//
// In the reference layout a red-black colour pass touches every other point
// of a row, so it streams whole cache sectors of every array it reads: one
// sweep moves about twice the bytes it needs. The mixed path owns its float
// copies of the finest operator, right-hand side and correction, so it keeps
// them with every row split by the parity of i-1: points with even i-1 first,
// then those with odd i-1. One colour of a row is then a contiguous run, and
// a colour pass reads only its own half of oC and f and the other colour's
// half of x (it still needs both halves of oE, oN, uC: the couplings to the
// west, south and lower neighbours are stored at those neighbours). Per sweep
// that is 10 arrays' worth of traffic instead of about 13.5.
//
// Only the arrays of the finest float level use this layout; the kernels
// here read and write them, converting at the boundaries (the double
// residual, the prolongation's correction, the refinement update). The
// per-point arithmetic is the reference-layout kernels', so results are
// bit-identical.
#pragma once

#include "launch.cuh"

namespace pmg {

struct Split {
  int nx, ny, nz, hx; // hx = (nx + 1) / 2: entries of the even half
  __host__ __device__ static Split of(const Dims &d) {
    return Split{d.nx, d.ny, d.nz, (d.nx + 1) / 2};
  }
  __host__ __device__ int row(int j, int k) const {
    return ((k - 1) * ny + (j - 1)) * nx;
  }
  // split index of (i, j, k)
  __host__ __device__ int at(int i, int j, int k) const {
    const int q = i - 1;
    return row(j, k) + (q >> 1) + (q & 1) * hx;
  }
  // split index of the reference-layout linear index g
  __host__ __device__ int of_linear(int g) const {
    const int r = g / nx, q = g - r * nx;
    return r * nx + (q >> 1) + (q & 1) * hx;
  }
};

// dst (split) = (Tout) src (reference layout), every entry
template <typename Tin, typename Tout>
__global__ void to_split_kernel(Dims d, const Tin *__restrict__ src,
                                Tout *__restrict__ dst) {
  const Split sp = Split::of(d);
  const long n = d.count();
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n;
       g += (long)gridDim.x * blockDim.x)
    dst[sp.of_linear((int)g)] = (Tout)src[g];
}

// dst (reference layout) = (Tout) src (split), every entry
template <typename Tin, typename Tout>
__global__ void from_split_kernel(Dims d, const Tin *__restrict__ src,
                                  Tout *__restrict__ dst) {
  const Split sp = Split::of(d);
  const long n = d.count();
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n;
       g += (long)gridDim.x * blockDim.x)
    dst[g] = (Tout)src[sp.of_linear((int)g)];
}

// x64 (reference layout) += (double) e32 (split) on the interior
__global__ void add_correction_split_kernel(Dims d, double *__restrict__ x,
                                            const float *__restrict__ e);

// Neighbour offsets of the point at split index s with q = i - 1 of parity
// qp: west and east (the other half), north/south (one row), up/down (one
// plane).
struct SplitNb {
  int w, e, n, s, u, dn;
};
__device__ __forceinline__ SplitNb split_nb(const Split &sp, int s, int qp) {
  SplitNb nb;
  // even q: west (q-1) and east (q+1) sit at q/2 - 1 and q/2 of the odd half;
  // odd q: at (q-1)/2 and (q+1)/2 of the even half
  nb.w = qp ? s - sp.hx : s + sp.hx - 1;
  nb.e = qp ? s - sp.hx + 1 : s + sp.hx;
  nb.n = s + sp.nx;
  nb.s = s - sp.nx;
  nb.u = s + sp.nx * sp.ny;
  nb.dn = s - sp.nx * sp.ny;
  return nb;
}

// One colour of the red-black sweep (gs7_color_kernel) on split arrays: the
// points of a row with (i + j + k) % 2 == want are one contiguous run. One
// thread per point; blockIdx.z is the plane.
template <typename T>
__global__ void __launch_bounds__(256)
    gs7_split_color_kernel(Dims d, const T *__restrict__ oC,
                           const T *__restrict__ fc, const T *__restrict__ oE,
                           const T *__restrict__ oN, const T *__restrict__ uC,
                           T *x, int want, T keep) {
  const Split sp = Split::of(d);
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (j > d.ny - 1)
    return;
  const int i = 2 + ((2 + j + k + want) & 1) +
                2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i > d.nx - 1)
    return;
  const int qp = (i - 1) & 1;
  const int p = sp.at(i, j, k);
  const SplitNb nb = split_nb(sp, p, qp);
  const T s = oN[p] * x[nb.n] + oN[nb.s] * x[nb.s] + oE[p] * x[nb.e] +
              oE[nb.w] * x[nb.w] + uC[nb.dn] * x[nb.dn] + uC[p] * x[nb.u];
  x[p] = (fc[p] + keep * s) / (oC[p] + T(0));
}

// itmax red-black sweeps on split arrays (Vgsrb7x semantics, cc = 0)
template <typename T>
int launch_gs7_split(const Dims &d, const T *oC, const T *fc, const T *oE,
                     const T *oN, const T *uC, T *x, int itmax, int iadjoint,
                     int zero_init, cudaStream_t s) {
  for (int it = 0; it < itmax; ++it)
    for (int c = 0; c <= 1; ++c) {
      const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
      const T keep = zero_init ? T(0) : T(1);
      gs7_split_color_kernel<T><<<gs7_grid(d), interior_block(), 0, s>>>(
          d, oC, fc, oE, oN, uC, x, want, keep);
      zero_init = 0;
    }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// r (reference layout) = f - A x with f, x and the 7-point operator split
// (defect_kernel<7>, the class's map order)
template <typename T>
__global__ void __launch_bounds__(256)
    defect7_split_kernel(Dims d, const T *__restrict__ oC,
                         const T *__restrict__ oE, const T *__restrict__ oN,
                         const T *__restrict__ uC, const T *__restrict__ f,
                         const T *__restrict__ x, T *__restrict__ r) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const Split sp = Split::of(d);
  const int p = sp.at(t.i, t.j, t.k);
  const SplitNb nb = split_nb(sp, p, (t.i - 1) & 1);
  const T ax = -oN[p] * x[nb.n] - oN[nb.s] * x[nb.s] - oE[p] * x[nb.e] -
               oE[nb.w] * x[nb.w] - uC[nb.dn] * x[nb.dn] - uC[p] * x[nb.u] +
               (oC[p] + T(0)) * x[p];
  r[d.at(t.i, t.j, t.k)] = f[p] - ax;
}

} // namespace pmg
