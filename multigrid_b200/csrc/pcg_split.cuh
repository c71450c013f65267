// MG-preconditioned CG kernels for the refinement paths (mixed, fp64-fast),
// whose preconditioner works on the colour-split finest level
// (split_layout.cuh): the update of x and r writes the preconditioner's
// split right-hand side as it goes, the preconditioned residual z is read
// back from the split correction inside the r.z product, and the operator
// of the finest level is read as code bytes when it is coded. The same
// values and sums as pcg_kernels.cuh's kernels followed by the layout
// conversions (to_split / from_split), with two passes over the level and
// 31 of the matvec's 48 bytes per point fewer.
#pragma once

#include "pcg_kernels.cuh"
#include "split_layout.cuh"

namespace pmg {

// pcg_update_xr_kernel, also writing rs (split) = (R) r
template <typename R>
__global__ void __launch_bounds__(kReduceThreads)
    pcg_update_xr_split_kernel(Dims d, const double *__restrict__ pv,
                               const double *__restrict__ ap,
                               double *__restrict__ x, double *__restrict__ r,
                               R *__restrict__ rs, const PcgState *st,
                               ReduceSlot s) {
  __shared__ double sh[32];
  const double alpha = st->alpha;
  const Split sp = Split::of(d);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      x[p] += alpha * pv[p];
      const double rv = r[p] - alpha * ap[p];
      r[p] = rv;
      rs[sp.at(i, j, k)] = (R)rv;
      acc += rv * rv;
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// z = (double) e (split) on the interior, and the sum of r . z
// (from_split_kernel followed by pcg_dot_kernel, the same bits)
template <typename E>
__global__ void __launch_bounds__(kReduceThreads)
    pcg_dot_split_kernel(Dims d, const double *__restrict__ r,
                         const E *__restrict__ e, double *__restrict__ z,
                         ReduceSlot s) {
  __shared__ double sh[32];
  const Split sp = Split::of(d);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      const double zv = (double)e[sp.at(i, j, k)];
      z[p] = zv;
      acc += r[p] * zv;
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// pcg_matvec_dot_kernel with the couplings and oC from the code bytes and
// the double tables when the level is coded (a uniform branch on the
// device flags; apply7's order either way, so the same bits)
__global__ void __launch_bounds__(kReduceThreads)
    pcg_matvec_dot_code_kernel(Dims d, Op14<double> A,
                               const unsigned char *__restrict__ code,
                               const double *__restrict__ lut64,
                               const double *__restrict__ octab,
                               const int *__restrict__ info,
                               const double *__restrict__ pv,
                               double *__restrict__ ap, ReduceSlot s) {
  __shared__ double sh[32];
  const Split sp = Split::of(d);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  const int sy = d.sy(), sz = d.sz();
  const bool coded = info[6] == 0 && info[7] == 0 && info[8] == 0;
  const double el = coded ? lut64[0] : 0.0, eh = coded ? lut64[1] : 0.0;
  const double nl = coded ? lut64[2] : 0.0, nh = coded ? lut64[3] : 0.0;
  const double ul = coded ? lut64[4] : 0.0, uh = coded ? lut64[5] : 0.0;
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      double y;
      if (coded) {
        const double xn = pv[p + sy], xs = pv[p - sy], xe = pv[p + 1];
        const double xw = pv[p - 1], xd = pv[p - sz], xu = pv[p + sz];
        const double xc = pv[p];
        const unsigned b = code[sp.at(i, j, k)];
        const double cn = (b & 4u) ? nh : nl, cs = (b & 8u) ? nh : nl;
        const double ce = (b & 1u) ? eh : el, cw = (b & 2u) ? eh : el;
        const double cd = (b & 32u) ? uh : ul, cu = (b & 16u) ? uh : ul;
        y = -cn * xn - cs * xs - ce * xe - cw * xw - cd * xd - cu * xu +
            (octab[b & 127u] + 0.0) * xc;
      } else {
        y = apply_op<7>(A, (const double *)nullptr, pv, p, sy, sz);
      }
      ap[p] = y;
      acc += y * pv[p];
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

} // namespace pmg
