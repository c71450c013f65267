// Kernels of the MG-preconditioned CG on the finest level (the reference
// app's CG_solver with the class as preconditioner: CG_Solver.h:45-242,
// PBE_pmgc_class.h:1116-1133, PBE_pmgc_class_with_non_zero_IS.cc:118-131).
//
// Vector kernels take one interior column per thread and kReducePlanes
// planes per block (reduce_grid); the sums are deterministic (block partials
// added in block order). The scalar recurrences run in one-thread kernels on
// a device-resident state, and the stop test sets the condition of the
// graph's while node, so the whole iteration runs without the host.
#pragma once

#include "reduce_kernels.cuh"

namespace pmg {

struct PcgState {
  double tol;
  int max_iters;
  int iters;
  int status; // 0 ok / stopped, 1 diverged, 2 initial residual not finite
  int pad;
  double rs, alpha, beta, r0, rn;
  double hist[1025];
};

// sum over the interior of a * b
__global__ void __launch_bounds__(kReduceThreads)
    pcg_dot_kernel(Dims d, const double *__restrict__ a,
                   const double *__restrict__ b, ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      acc += a[p] * b[p];
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// ap = A p on the interior (the class's finest map); sum of ap * p
__global__ void __launch_bounds__(kReduceThreads)
    pcg_matvec_dot_kernel(Dims d, Op14<double> A,
                          const double *__restrict__ pv,
                          double *__restrict__ ap, ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      const double y =
          apply_op<7>(A, (const double *)nullptr, pv, p, d.sy(), d.sz());
      ap[p] = y;
      acc += y * pv[p];
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// x += alpha p; r -= alpha ap on the interior; sum of r^2
__global__ void __launch_bounds__(kReduceThreads)
    pcg_update_xr_kernel(Dims d, const double *__restrict__ pv,
                         const double *__restrict__ ap, double *__restrict__ x,
                         double *__restrict__ r, const PcgState *st,
                         ReduceSlot s) {
  __shared__ double sh[32];
  const double alpha = st->alpha;
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
      acc += rv * rv;
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// p = z + beta p on the interior
__global__ void __launch_bounds__(kReduceThreads)
    pcg_update_p_kernel(Dims d, const double *__restrict__ z,
                        double *__restrict__ pv, const PcgState *st) {
  const double beta = st->beta;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      pv[p] = z[p] + beta * pv[p];
    }
}

__global__ void pcg_params_kernel(PcgState *st, double tol, int max_iters) {
  st->tol = tol;
  st->max_iters = max_iters;
  st->iters = 0;
  st->status = 0;
}

// rs = r.z, alpha = rs / pAp; no iteration when pAp == 0 (CG_Solver.h:
// 110-116) or the initial residual is zero or not finite
__global__ void pcg_init_kernel(PcgState *st, const double *rr,
                                const double *rz, const double *pap,
                                double n3, cudaGraphConditionalHandle h) {
  const double r0 = sqrt(rr[0] / n3);
  st->r0 = r0;
  st->rn = r0;
  st->hist[0] = r0;
  st->rs = rz[0];
  const bool finite = isfinite(r0);
  st->status = finite ? 0 : 2;
  const bool go = finite && r0 > 0.0 && pap[0] != 0.0 && st->max_iters > 0;
  st->alpha = pap[0] != 0.0 ? st->rs / pap[0] : 0.0;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// beta = r'.z' / r.z (0 when r.z == 0); rs = r'.z' (CG_Solver.h:186-197)
__global__ void pcg_beta_kernel(PcgState *st, const double *rz) {
  st->beta = st->rs == 0.0 ? 0.0 : rz[0] / st->rs;
  st->rs = rz[0];
}

// alpha = rs / pAp (0 when pAp == 0), then the stop test on the updated
// residual's norm sqrt(sum r^2 / n^3) relative to the initial one
__global__ void pcg_check_kernel(PcgState *st, const double *pap,
                                 const double *rr, double n3,
                                 cudaGraphConditionalHandle h) {
  st->alpha = pap[0] == 0.0 ? 0.0 : st->rs / pap[0];
  const int c = ++st->iters;
  const double rn = sqrt(rr[0] / n3);
  st->rn = rn;
  if (c <= 1024)
    st->hist[c] = rn;
  const bool diverged = !isfinite(rn) || rn > 1e6 * st->r0;
  if (diverged)
    st->status = 1;
  const bool converged = st->tol > 0.0 && rn / st->r0 < st->tol;
  cudaGraphSetConditional(
      h, (!diverged && !converged && c < st->max_iters) ? 1u : 0u);
}

} // namespace pmg
