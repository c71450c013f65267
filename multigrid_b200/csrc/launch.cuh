// Launch shapes and host launchers shared by the C-ABI wrappers and the
// solver. All launchers are asynchronous on the given stream and return a
// pmg_status (launch errors only).
#pragma once

#include "stencil_kernels.cuh"

namespace pmg {

inline unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

// Interior kernels: one thread per interior point, block 32 x 8, one plane
// per blockIdx.z.
inline dim3 interior_block() { return dim3(32, 8, 1); }
inline dim3 interior_grid(const Dims &d) {
  return dim3(cdiv(d.nx - 2, 32), cdiv(d.ny - 2, 8), (unsigned)(d.nz - 2));
}
// Reductions: one thread per interior column, 8 planes per block.
inline dim3 reduce_grid(const Dims &d) {
  return dim3(cdiv(d.nx - 2, 32), cdiv(d.ny - 2, 8), cdiv(d.nz - 2, 8));
}
// The damping reduction on coarse levels: fewer planes per block on smaller
// levels, so that they still launch enough blocks (33^3 with 8 planes per
// block is 16 blocks).
inline int lambda_planes(const Dims &d) {
  const int n = d.nx < d.ny ? d.nx : d.ny;
  return n >= 97 ? 4 : n >= 49 ? 2 : 1;
}
inline dim3 lambda_grid(const Dims &d) {
  return dim3(cdiv(d.nx - 2, 32), cdiv(d.ny - 2, 8),
              cdiv(d.nz - 2, lambda_planes(d)));
}
// Interpolation: one thread per coarse cell (ii,jj,kk) in [1, n_c-1]^3.
inline dim3 interp_grid(const Dims &dc) {
  return dim3(cdiv(dc.nx - 1, 32), cdiv(dc.ny - 1, 8), (unsigned)(dc.nz - 1));
}
// Red-black colour: half of each row.
inline dim3 gs7_grid(const Dims &d) {
  return dim3(cdiv(cdiv(d.nx - 2, 2), 32), cdiv(d.ny - 2, 8),
              (unsigned)(d.nz - 2));
}
// Eight-colour: half of each axis.
inline dim3 gs27_block() { return dim3(32, 4, 1); }
inline dim3 gs27_grid(const Dims &d) {
  return dim3(cdiv(cdiv(d.nx - 2, 2), 32), cdiv(cdiv(d.ny - 2, 2), 4),
              cdiv(d.nz - 2, 2));
}
inline unsigned flat_grid(long n) {
  const long b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

// itmax red-black sweeps (Vgsrb7x semantics).
template <typename T>
int launch_gs7(const Dims &d, const T *oC, const T *cc, const T *fc,
               const T *oE, const T *oN, const T *uC, T *x, int itmax,
               int iadjoint, int zero_init, cudaStream_t s) {
  for (int it = 0; it < itmax; ++it)
    for (int c = 0; c <= 1; ++c) {
      const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
      const T keep = zero_init ? T(0) : T(1);
      gs7_color_kernel<T><<<gs7_grid(d), interior_block(), 0, s>>>(
          d, oC, cc, fc, oE, oN, uC, x, want, keep);
      zero_init = 0;
    }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// itmax eight-colour sweeps (Vgsrb27x semantics).
template <typename T>
int launch_gs27(const Dims &d, const Op14<T> &A, const T *cc, const T *fc,
                T *x, int itmax, int iadjoint, int zero_init, cudaStream_t s) {
  if (zero_init)
    PMG_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(T) * d.count(), s));
  for (int it = 0; it < itmax; ++it)
    for (int c = 0; c < 8; ++c) {
      const int want = c * (1 - iadjoint) + iadjoint * (7 - c);
      gs27_color_kernel<T><<<gs27_grid(d), gs27_block(), 0, s>>>(d, A, cc, fc,
                                                                 x, want);
    }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// Prolongation / Galerkin builders (pmg_build.cu). P32 / out32 (all null:
// none) also receive the float copies of the interior entries written.
// P32 / out32 (optional): float copies, rows dc32.px apart (dc32 defaults
// to dc)
int launch_buildP(const Dims &df, const Dims &dc, int kind,
                  const Op14<double> &A, const P27W<double> &P,
                  cudaStream_t s, const P27W<float> &P32 = P27W<float>{},
                  const Dims *dc32 = nullptr);
int launch_buildG(const Dims &df, const Dims &dc, int kind,
                  const P27<double> &P, const Op14<double> &A,
                  const Op14W<double> &out, cudaStream_t s,
                  const Op14W<float> &out32 = Op14W<float>{},
                  const Dims *dc32 = nullptr);

} // namespace pmg
