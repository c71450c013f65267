// Coarsest-level CG on a cluster of CTAs with the operator held in shared
// memory.
//
// The one-CTA CG (cg_level_kernel) streams the level's fourteen coefficient
// arrays (17^3 doubles: 550 KB) from L2 through a single SM on every
// iteration. Here a cluster of kCgCtas CTAs splits the level by planes: each
// CTA keeps the coefficients of its planes (and of the plane below, for the
// lower couplings) in its shared memory for the whole solve, holds its
// points' x, r, A p in registers and its planes of p in shared memory, and
// reads the neighbouring planes of p from the neighbouring CTAs' shared
// memory (distributed shared memory). Dot products are block sums summed
// over the cluster in rank order, so every CTA gets the same bits and takes
// the same branch. The iteration is the class's CG (CG_solver,
// CG_Solver.h:45-242, via solve_by_cg<1>): see launch_cg_level.
#pragma once

#include <cooperative_groups.h>

#include "cluster_planes.cuh"
#include "reduce_kernels.cuh"

namespace pmg {

// bytes of dynamic shared memory for an nx x ny level
inline size_t cg_cluster_smem(int nx, int ny) {
  const size_t nxy = (size_t)nx * ny;
  return sizeof(double) * ((kCgMaxPlanes + 1) * 14 * nxy +
                           kCgMaxPlanes * nxy + 2 * kCgCtas + nxy);
}

inline bool cg_cluster_fits(const Dims &d) {
  return d.nx <= kCgMaxN && d.ny <= kCgMaxN && d.nz <= kCgMaxN &&
         (d.nx - 2) * (d.ny - 2) * kCgMaxPlanes <= kCgThreads &&
         d.nz - 2 <= kCgCtas * kCgMaxPlanes;
}

// (A v)(i, j, k) in apply27's order (sums27, then -tO - tU - tD + oC v); a(s,
// di, dj, dk) the coupling slot s at the offset point, v(di, dj, dk) the
// vector there.
template <class CoefFn, class VecFn>
__device__ __forceinline__ double apply27_at(CoefFn a, VecFn v) {
  const double tO = a(kON, 0, 0, 0) * v(0, 1, 0) +
                    a(kON, 0, -1, 0) * v(0, -1, 0) +
                    a(kOE, 0, 0, 0) * v(1, 0, 0) +
                    a(kOE, -1, 0, 0) * v(-1, 0, 0) +
                    a(kONE, 0, 0, 0) * v(1, 1, 0) +
                    a(kONW, 0, 0, 0) * v(-1, 1, 0) +
                    a(kONW, 1, -1, 0) * v(1, -1, 0) +
                    a(kONE, -1, -1, 0) * v(-1, -1, 0);
  const double tU = a(kUC, 0, 0, 0) * v(0, 0, 1) +
                    a(kUN, 0, 0, 0) * v(0, 1, 1) +
                    a(kUS, 0, 0, 0) * v(0, -1, 1) +
                    a(kUE, 0, 0, 0) * v(1, 0, 1) +
                    a(kUW, 0, 0, 0) * v(-1, 0, 1) +
                    a(kUNE, 0, 0, 0) * v(1, 1, 1) +
                    a(kUNW, 0, 0, 0) * v(-1, 1, 1) +
                    a(kUSE, 0, 0, 0) * v(1, -1, 1) +
                    a(kUSW, 0, 0, 0) * v(-1, -1, 1);
  const double tD = a(kUC, 0, 0, -1) * v(0, 0, -1) +
                    a(kUS, 0, 1, -1) * v(0, 1, -1) +
                    a(kUN, 0, -1, -1) * v(0, -1, -1) +
                    a(kUW, 1, 0, -1) * v(1, 0, -1) +
                    a(kUE, -1, 0, -1) * v(-1, 0, -1) +
                    a(kUSW, 1, 1, -1) * v(1, 1, -1) +
                    a(kUSE, -1, 1, -1) * v(-1, 1, -1) +
                    a(kUNW, 1, -1, -1) * v(1, -1, -1) +
                    a(kUNE, -1, -1, -1) * v(-1, -1, -1);
  return (-tO) + (-tU) + (-tD) + (a(kOC, 0, 0, 0) + 0.0) * v(0, 0, 0);
}

__global__ void __cluster_dims__(kCgCtas, 1, 1) __launch_bounds__(kCgThreads)
    cg_cluster_kernel(Dims d, Op14<double> A, const double *__restrict__ rhs,
                      double *__restrict__ x, double thresh, double rel_tol,
                      int class_first_check, int max_iters,
                      int *__restrict__ status) {
  namespace cgs = cooperative_groups;
  cgs::cluster_group cluster = cgs::this_cluster();
  extern __shared__ __align__(16) double cg_smem[];
  const int nx = d.nx, ny = d.ny, nxy = nx * ny;
  // [plane klo-1 .. khi][slot][j][i] coefficients, then p of klo .. khi,
  // then two sets of reduction slots (one per CTA rank), then a zero plane
  double *sA = cg_smem;
  double *sP = sA + (kCgMaxPlanes + 1) * 14 * nxy;
  double *sRed = sP + kCgMaxPlanes * nxy;
  double *zp = sRed + 2 * kCgCtas;
  __shared__ double sh[2 * 32];

  const int rank = (int)cluster.block_rank();
  const int klo = cg_plane_lo(rank, d.nz);
  const int khi = cg_plane_lo(rank + 1, d.nz) - 1; // may be < klo
  const int nplanes = khi - klo + 1;
  const int mi = nx - 2, mj = ny - 2;

  // the coefficients of planes klo-1 .. khi, whole planes (shell included)
  for (int q = threadIdx.x; q < (nplanes + 1) * 14 * nxy; q += blockDim.x) {
    const int lk = q / (14 * nxy), rem = q - lk * 14 * nxy;
    const int slot = rem / nxy, o = rem - slot * nxy;
    const int k = klo - 1 + lk;
    sA[q] = A.a[slot][(long)(k - 1) * nxy + o];
  }
  for (int q = threadIdx.x; q < kCgMaxPlanes * nxy; q += blockDim.x)
    sP[q] = 0.0; // shells of p stay zero
  for (int q = threadIdx.x; q < nxy; q += blockDim.x)
    zp[q] = 0.0;

  // this thread's point
  const int t = threadIdx.x;
  const bool own = t < nplanes * mi * mj;
  int i = 2, j = 2, k = klo;
  if (own) {
    const int lp = t / (mi * mj), r2 = t - lp * mi * mj;
    j = 2 + r2 / mi;
    i = 2 + r2 % mi;
    k = klo + lp;
  }
  const int gi = d.at(i, j, k);
  const int sl = (k - klo) * nxy + (j - 1) * nx + (i - 1); // in sP
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;

  auto coef = [&](int slot, int di, int dj, int dk) -> double {
    const int lk = k + dk - (klo - 1);
    return sA[(lk * 14 + slot) * nxy + (j - 1 + dj) * nx + (i - 1 + di)];
  };
  // plane kk of p: this CTA's planes, the planes next to them from the CTA
  // holding them (distributed shared memory), shell planes zero
  auto p_plane = [&](int kk) -> const double * {
    if (kk < 2 || kk > d.nz - 1)
      return zp;
    if (kk >= klo && kk <= khi)
      return sP + (kk - klo) * nxy;
    const int r = cg_plane_owner(kk, d.nz);
    return cluster.map_shared_rank(sP, r) + (kk - cg_plane_lo(r, d.nz)) * nxy;
  };
  const double *p_c = sP + (k - klo) * nxy;
  const double *p_dn = p_plane(k - 1), *p_up = p_plane(k + 1);
  const int po = (j - 1) * nx + (i - 1);
  auto pval = [&](int di, int dj, int dk) -> double {
    const double *pl = dk == 0 ? p_c : dk < 0 ? p_dn : p_up;
    return pl[po + dj * nx + di];
  };
  auto xval = [&](int di, int dj, int dk) -> double {
    return x[gi + di + dj * nx + dk * nxy];
  };
  // Cluster-wide sum in rank order, the same bits in every CTA: warp sums,
  // the CTA's warp sums added by warp 0 (fixed shuffle tree) and pushed
  // into slot `rank` of every CTA; after the barrier each thread adds its
  // own CTA's kCgCtas slots in rank order. The two slot sets (and the two
  // halves of sh) alternate; a set is written again only after two more
  // cluster barriers, which every reader of its previous contents passed.
  auto cluster_sum = [&](double v, int slot) -> double {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
      sh[slot * 32 + warp] = v;
    __syncthreads();
    if (warp == 0) {
      double b = lane < nw ? sh[slot * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        b += __shfl_down_sync(0xffffffffu, b, o);
      b = __shfl_sync(0xffffffffu, b, 0);
      // every lane stores (lanes 8 apart write the same value)
      cluster.map_shared_rank(sRed, lane % kCgCtas)[slot * kCgCtas + rank] =
          b;
    }
    cluster.sync();
    double s = 0.0;
#pragma unroll
    for (int r = 0; r < kCgCtas; ++r)
      s += sRed[slot * kCgCtas + r];
    return s;
  };

  // r = rhs - A x; p = r; rs = r.r
  double xv = 0.0, rv = 0.0, apv = 0.0;
  __syncthreads(); // coefficients staged
  if (own) {
    xv = x[gi];
    rv = rhs[gi] - apply27_at(coef, xval);
    sP[sl] = rv;
  }
  double rs = cluster_sum(own ? rv * rv : 0.0, 0);
  // Ap and p.Ap (p is visible to the neighbours after the sum's sync)
  if (own)
    apv = apply27_at(coef, pval);
  double pap = cluster_sum(own ? apv * sP[sl] : 0.0, 1);
  int it = 0;
  double res = 0.0;
  if (pap != 0.0) {
    double alpha = rs / pap;
    res = class_first_check ? sqrt(sqrt(rs)) : sqrt(rs);
    const double stop = fmax(thresh, rel_tol * sqrt(rs));
    while (res > stop && it < max_iters) {
      ++it;
      if (own) {
        xv += alpha * sP[sl];
        rv = rv - alpha * apv;
      }
      const double rsn = cluster_sum(own ? rv * rv : 0.0, 0);
      const double beta = rs == 0.0 ? 0.0 : rsn / rs;
      rs = rsn;
      if (own)
        sP[sl] = rv + beta * sP[sl];
      cluster.sync(); // every CTA's new p before anyone reads it
      if (own)
        apv = apply27_at(coef, pval);
      pap = cluster_sum(own ? apv * sP[sl] : 0.0, 1);
      alpha = pap == 0.0 ? 0.0 : rs / pap;
      res = sqrt(rs);
    }
    if (rank == 0 && threadIdx.x == 0) {
      status[0] = it;
      status[1] = (it >= max_iters && res > stop) ? 1 : 0;
    }
  } else if (rank == 0 && threadIdx.x == 0) {
    status[0] = 0;
    status[1] = 0;
  }
  if (own)
    x[gi] = xv;
  cluster.sync(); // no CTA leaves while another may still read its p
}

} // namespace pmg
