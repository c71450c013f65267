// The lowest levels of the mixed-precision V-cycle on a cluster of CTAs with
// every array in shared memory.
//
// bottom_cycle_kernel runs levels 1 .. top in one CTA out of global memory:
// each of its ~80 barrier-separated steps waits for an L2 round trip. Here a
// cluster of kCgCtas CTAs splits the top level (n <= 17) by planes like the
// coarsest-level CG (cg_cluster.cuh): each CTA keeps the coefficients of its
// planes and of the plane below, and its planes of x, f and r, in shared
// memory; the planes next to its own are read from the CTAs holding them
// (distributed shared memory). In a colour sweep only the switch between
// even and odd planes needs a cluster barrier: the four sub-colours of one
// plane parity touch the CTA's own planes only. Rank 0 holds the levels
// below the top (n <= 9) and level 1 whole, runs their part of the cycle
// alone, reads the top level's defect from the other CTAs for the
// restriction and writes the interpolated correction into their r planes.
// The arrays are staged with cp.async; each thread keeps one point per level
// (colour-major, so a colour step is a run of threads), and one warp runs the
// level-1 CG with shuffle sums.
//
// The steps and their per-point arithmetic are bottom_cycle_kernel's (the
// float V-cycle with every level zero-started, v_cycle, PBE_pmgc_class.h:
// 1070-1114); sums over the cluster are taken in rank order, so results are
// deterministic.
#pragma once

#include <cooperative_groups.h>

#include "bottom_cycle.cuh"
#include "cluster_planes.cuh"

namespace pmg {

constexpr int kBcThreads = 512;
constexpr size_t kBcMaxSmem = 200 * 1024; // dynamic, leaves room for static

// byte offsets of the dynamic shared memory (same on host and device)
struct BcLayout {
  size_t tA, tx, tf, tr, zero; // top level, per CTA; tA slot-major
  size_t lA[kBottomMaxLevels], lx[kBottomMaxLevels], // rank 0: levels
      lf[kBottomMaxLevels], lr[kBottomMaxLevels];    // 2 .. top-1
  size_t A1, x1, f1, cr, cp, cap, xf1, ff1;          // rank 0: level 1
  size_t red;                                        // cluster sums
  size_t total;
};

__host__ __device__ inline size_t bc_take(size_t &o, size_t bytes) {
  const size_t r = o;
  o += (bytes + 15) & ~(size_t)15;
  return r;
}

__host__ __device__ inline BcLayout bc_layout(const BottomArgs &a) {
  BcLayout l{};
  size_t o = 0;
  const int T = a.top;
  if (T >= 2) {
    const size_t nxy = (size_t)a.lv[T].d.nx * a.lv[T].d.ny;
    l.tA = bc_take(o, sizeof(float) * (kCgMaxPlanes + 1) * 14 * nxy);
    l.tx = bc_take(o, sizeof(float) * kCgMaxPlanes * nxy);
    l.tf = bc_take(o, sizeof(float) * kCgMaxPlanes * nxy);
    l.tr = bc_take(o, sizeof(float) * kCgMaxPlanes * nxy);
    l.zero = bc_take(o, sizeof(float) * nxy);
  }
  for (int L = 2; L < T; ++L) {
    const size_t n3 = (size_t)a.lv[L].d.count();
    l.lA[L] = bc_take(o, sizeof(float) * 14 * n3);
    l.lx[L] = bc_take(o, sizeof(float) * n3);
    l.lf[L] = bc_take(o, sizeof(float) * n3);
    l.lr[L] = bc_take(o, sizeof(float) * n3);
  }
  const size_t n1 = (size_t)a.lv[1].d.count();
  l.A1 = bc_take(o, sizeof(double) * 14 * n1);
  l.x1 = bc_take(o, sizeof(double) * n1);
  l.f1 = bc_take(o, sizeof(double) * n1);
  l.cr = bc_take(o, sizeof(double) * n1);
  l.cp = bc_take(o, sizeof(double) * n1);
  l.cap = bc_take(o, sizeof(double) * n1);
  l.xf1 = bc_take(o, sizeof(float) * n1);
  l.ff1 = bc_take(o, sizeof(float) * n1);
  l.red = bc_take(o, sizeof(double) * 4);
  l.total = o;
  return l;
}

// The cluster kernel takes levels whose top fits the plane split and whose
// arrays fit one CTA's shared memory.
inline bool bc_fits(const BottomArgs &a) {
  if (a.top < 1 || a.top > kBottomMaxLevels)
    return false;
  if (a.top >= 2) {
    const Dims &d = a.lv[a.top].d;
    if (d.nx > kCgMaxN || d.ny > kCgMaxN || d.nz - 2 > kCgCtas * kCgMaxPlanes)
      return false;
    if ((d.nx - 2) * (d.ny - 2) * kCgMaxPlanes > kBcThreads)
      return false;
  }
  for (int L = 1; L < a.top; ++L)
    if (a.lv[L].d.count() > 9 * 9 * 9)
      return false;
  return bc_layout(a).total <= kBcMaxSmem;
}

// sums27 on arrays given by plane: ak / ad point at slot 0 of the
// coefficients of planes k / k-1 (slot stride ss), xc / xd / xu at planes k,
// k-1, k+1 of x; o is the in-plane offset, w the row length.
template <typename T>
__device__ __forceinline__ void bc_sums27(const T *ak, const T *ad, int ss,
                                          int o, int w, const T *xc,
                                          const T *xd, const T *xu, T &tO,
                                          T &tU, T &tD) {
#define BC_A(s, q) ak[(s) * ss + (q)]
#define BC_D(s, q) ad[(s) * ss + (q)]
  tO = BC_A(kON, o) * xc[o + w] + BC_A(kON, o - w) * xc[o - w] +
       BC_A(kOE, o) * xc[o + 1] + BC_A(kOE, o - 1) * xc[o - 1] +
       BC_A(kONE, o) * xc[o + 1 + w] + BC_A(kONW, o) * xc[o - 1 + w] +
       BC_A(kONW, o + 1 - w) * xc[o + 1 - w] +
       BC_A(kONE, o - 1 - w) * xc[o - 1 - w];
  tU = BC_A(kUC, o) * xu[o] + BC_A(kUN, o) * xu[o + w] +
       BC_A(kUS, o) * xu[o - w] + BC_A(kUE, o) * xu[o + 1] +
       BC_A(kUW, o) * xu[o - 1] + BC_A(kUNE, o) * xu[o + 1 + w] +
       BC_A(kUNW, o) * xu[o - 1 + w] + BC_A(kUSE, o) * xu[o + 1 - w] +
       BC_A(kUSW, o) * xu[o - 1 - w];
  tD = BC_D(kUC, o) * xd[o] + BC_D(kUS, o + w) * xd[o + w] +
       BC_D(kUN, o - w) * xd[o - w] + BC_D(kUW, o + 1) * xd[o + 1] +
       BC_D(kUE, o - 1) * xd[o - 1] + BC_D(kUSW, o + 1 + w) * xd[o + 1 + w] +
       BC_D(kUSE, o - 1 + w) * xd[o - 1 + w] +
       BC_D(kUNW, o + 1 - w) * xd[o + 1 - w] +
       BC_D(kUNE, o - 1 - w) * xd[o - 1 - w];
#undef BC_A
#undef BC_D
}

// (A x) at the point: apply27's order
template <typename T>
__device__ __forceinline__ T bc_apply27(const T *ak, const T *ad, int ss,
                                        int o, int w, const T *xc,
                                        const T *xd, const T *xu) {
  T tO, tU, tD;
  bc_sums27(ak, ad, ss, o, w, xc, xd, xu, tO, tU, tD);
  return (-tO) + (-tU) + (-tD) + (ak[kOC * ss + o] + T(0)) * xc[o];
}

// The t-th interior point, in colour-major order, of planes k0 .. k0+nk-1
// of an nx x ny level (colour (i&1) + 2(j&1) + 4(k&1)); false past the end.
__device__ inline bool bc_point(int t, int nx, int ny, int k0, int nk, int &i,
                                int &j, int &k, int &colour) {
  int start = 0;
  for (int c = 0; c < 8; ++c) {
    const int pi = c & 1, pj = (c >> 1) & 1, pk = c >> 2;
    const int hx = (nx - 1 - pi) / 2, hy = (ny - 1 - pj) / 2;
    const int kf = k0 + ((pk - k0) & 1); // first plane of parity pk
    const int hz = kf > k0 + nk - 1 ? 0 : (k0 + nk - 1 - kf) / 2 + 1;
    const int cnt = hx * hy * hz;
    if (t < start + cnt) {
      const int q = t - start, r = q / hx;
      i = 2 + pi + 2 * (q - r * hx);
      const int kk = r / hy;
      j = 2 + pj + 2 * (r - kk * hy);
      k = kf + 2 * kk;
      colour = c;
      return true;
    }
    start += cnt;
  }
  return false;
}

// One level held whole in this CTA's shared memory (rank 0).
struct BcLevel {
  Dims d;
  float *A, *x, *f, *r; // A: 14 slots of d.count()
};

// eight-colour sweeps on a whole level in this CTA, one point per thread
__device__ void bc_local_gs27(const BcLevel &v, int sweeps) {
  const Dims &d = v.d;
  const int nxy = d.nx * d.ny, n3 = (int)d.count();
  int i, j, k, col;
  const bool ok = bc_point(threadIdx.x, d.nx, d.ny, 2, d.nz - 2, i, j, k, col);
  const int o = (j - 1) * d.nx + (i - 1), pl = (k - 1) * nxy;
  for (int s = 0; s < sweeps; ++s)
    for (int c = 0; c < 8; ++c) {
      if (ok && col == c) {
        float tO, tU, tD;
        bc_sums27(v.A + pl, v.A + pl - nxy, n3, o, d.nx, v.x + pl,
                  v.x + pl - nxy, v.x + pl + nxy, tO, tU, tD);
        v.x[pl + o] = (v.f[pl + o] + (tO + tU + tD)) / v.A[kOC * n3 + pl + o];
      }
      __syncthreads();
    }
}

__device__ void bc_local_defect(const BcLevel &v) {
  const Dims &d = v.d;
  const int nxy = d.nx * d.ny, n3 = (int)d.count();
  int i, j, k, col;
  if (bc_point(threadIdx.x, d.nx, d.ny, 2, d.nz - 2, i, j, k, col)) {
    const int o = (j - 1) * d.nx + (i - 1), pl = (k - 1) * nxy;
    v.r[pl + o] = v.f[pl + o] - bc_apply27(v.A + pl, v.A + pl - nxy, n3, o,
                                           d.nx, v.x + pl, v.x + pl - nxy,
                                           v.x + pl + nxy);
  }
  __syncthreads();
}

// coarse f = restriction of fine r; rfine(K) gives plane K of the fine r
// (restrict_kernel's order: planes 2k-1, 2k, 2k-2, nine terms each)
template <class PlaneFn>
__device__ void bc_restrict(const Dims &fd, const Dims &cd,
                            const P27<float> &P, PlaneFn rfine, float *fc) {
  const int fy = fd.nx;
  for_interior(cd, [&](int i, int j, int k) {
    const int pc = cd.at(i, j, k);
    const int o = (2 * j - 2) * fd.nx + (2 * i - 2);
    float pl[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int b = q * 9;
      const float *r = rfine(q == 0 ? 2 * k - 1 : q == 1 ? 2 * k : 2 * k - 2);
      const float *const *p = P.p;
      pl[q] = p[b + 0][pc] * r[o] + p[b + 1][pc] * r[o + fy] +
              p[b + 2][pc] * r[o - fy] + p[b + 3][pc] * r[o + 1] +
              p[b + 4][pc] * r[o - 1] + p[b + 5][pc] * r[o + 1 + fy] +
              p[b + 6][pc] * r[o - 1 + fy] + p[b + 7][pc] * r[o + 1 - fy] +
              p[b + 8][pc] * r[o - 1 - fy];
    }
    fc[pc] = pl[0] + pl[1] + pl[2];
  });
  __syncthreads();
}

// fine e = interpolation of coarse x (bottom_cycle_kernel's order, one
// coarse cell per thread); rout(K) gives plane K of the fine output, or null
// for a plane this call does not write
template <class PlaneFn>
__device__ void bc_interp(const Dims &cd, const Dims &fd, const P27<float> &P,
                          const float *xin, PlaneFn rout) {
  const int cy = cd.sy(), cz = cd.sz(), fy = fd.nx;
  const int mx = cd.nx - 1, my = cd.ny - 1, m = mx * my * (cd.nz - 1);
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    const int r = q / mx;
    const int ii = q - r * mx + 1;
    const int kk = r / my + 1;
    const int jj = r - (kk - 1) * my + 1;
    const int cc = cd.at(ii, jj, kk);
    const int o = (2 * jj - 2) * fd.nx + (2 * ii - 2);
    const float *const *p = P.p;
    const float x000 = xin[cc], x100 = xin[cc + 1], x010 = xin[cc + cy],
                x001 = xin[cc + cz], x110 = xin[cc + 1 + cy],
                x101 = xin[cc + 1 + cz], x011 = xin[cc + cy + cz],
                x111 = xin[cc + 1 + cy + cz];
    float *lo = rout(2 * kk - 1), *hi = rout(2 * kk);
    if (lo) {
      lo[o] = x000;
      lo[o + 1] = p[3][cc] * x000 + p[4][cc + 1] * x100;
      lo[o + fy] = p[1][cc] * x000 + p[2][cc + cy] * x010;
      lo[o + 1 + fy] = p[5][cc] * x000 + p[6][cc + 1] * x100 +
                       p[7][cc + cy] * x010 + p[8][cc + 1 + cy] * x110;
    }
    if (hi) {
      hi[o] = p[9][cc] * x000 + p[18][cc + cz] * x001;
      hi[o + 1] = p[12][cc] * x000 + p[13][cc + 1] * x100 +
                  p[21][cc + cz] * x001 + p[22][cc + 1 + cz] * x101;
      hi[o + fy] = p[10][cc] * x000 + p[11][cc + cy] * x010 +
                   p[19][cc + cz] * x001 + p[20][cc + cy + cz] * x011;
      hi[o + 1 + fy] =
          p[14][cc] * x000 + p[15][cc + 1] * x100 + p[16][cc + cy] * x010 +
          p[17][cc + 1 + cy] * x110 + p[23][cc + cz] * x001 +
          p[24][cc + 1 + cz] * x101 + p[25][cc + cy + cz] * x011 +
          p[26][cc + 1 + cy + cz] * x111;
    }
  }
  __syncthreads();
}

// omega = (f . x) / (x . A x) over the interior of a whole local level
__device__ double bc_local_damping(const BcLevel &v, double *sh) {
  const Dims &d = v.d;
  const int nxy = d.nx * d.ny, n3 = (int)d.count();
  double up = 0.0, lo = 0.0;
  int i, j, k, col;
  if (bc_point(threadIdx.x, d.nx, d.ny, 2, d.nz - 2, i, j, k, col)) {
    const int o = (j - 1) * d.nx + (i - 1), pl = (k - 1) * nxy;
    up = (double)v.f[pl + o] * (double)v.x[pl + o];
    lo = (double)v.x[pl + o] *
         (double)bc_apply27(v.A + pl, v.A + pl - nxy, n3, o, d.nx, v.x + pl,
                            v.x + pl - nxy, v.x + pl + nxy);
  }
  up = bottom_allsum(up, sh);
  lo = bottom_allsum(lo, sh);
  return up / lo;
}

// sum over warp 0's lanes in lane order of partial sums, in every lane
__device__ __forceinline__ double bc_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}

// Level 1 in double by warp 0: zero-started CG to a relative reduction of
// rtol (bottom_cycle_kernel's level-1 step), then the damping; leaves the
// float copy of x in xf. Returns omega (in every lane).
__device__ double bc_level1(const BottomArgs &a, const double *A1, double *x1,
                            double *f1, double *cr, double *cp, double *cap,
                            const float *ff, float *xf) {
  const Dims d1 = a.lv[1].d;
  const int n1 = (int)d1.count(), nxy1 = d1.nx * d1.ny;
  const int mx = d1.nx - 2, my = d1.ny - 2, m = mx * my * (d1.nz - 2);
  const int lane = threadIdx.x;
  auto at = [&](int q) -> int { // q-th interior point (natural order)
    const int r = q / mx, i = q - r * mx + 2, k = r / my;
    return d1.at(i, r - k * my + 2, k + 2);
  };
  auto ap_at = [&](const double *v, int p) -> double {
    const int pl = (p / nxy1) * nxy1, o = p - pl;
    return bc_apply27(A1 + pl, A1 + pl - nxy1, n1, o, d1.nx, v + pl,
                      v + pl - nxy1, v + pl + nxy1);
  };
  for (int q = lane; q < n1; q += 32)
    f1[q] = (double)ff[q];
  __syncwarp();
  double acc = 0.0;
  for (int q = lane; q < m; q += 32) {
    const int p = at(q);
    const double r = f1[p] - ap_at(x1, p);
    cr[p] = r;
    cp[p] = r;
    acc += r * r;
  }
  double rs = bc_warp_sum(acc);
  __syncwarp();
  acc = 0.0;
  for (int q = lane; q < m; q += 32) {
    const int p = at(q);
    const double ap = ap_at(cp, p);
    cap[p] = ap;
    acc += ap * cp[p];
  }
  double pap = bc_warp_sum(acc);
  int it = 0;
  if (pap != 0.0) {
    double alpha = rs / pap;
    double res = sqrt(rs);
    const double stop = a.rtol * res;
    while (res > stop && it < a.max_iters) {
      ++it;
      acc = 0.0;
      for (int q = lane; q < m; q += 32) {
        const int p = at(q);
        x1[p] += alpha * cp[p];
        const double r = cr[p] - alpha * cap[p];
        cr[p] = r;
        acc += r * r;
      }
      const double rsn = bc_warp_sum(acc);
      const double beta = rs == 0.0 ? 0.0 : rsn / rs;
      rs = rsn;
      for (int q = lane; q < m; q += 32) {
        const int p = at(q);
        cp[p] = cr[p] + beta * cp[p];
      }
      __syncwarp();
      acc = 0.0;
      for (int q = lane; q < m; q += 32) {
        const int p = at(q);
        const double ap = ap_at(cp, p);
        cap[p] = ap;
        acc += ap * cp[p];
      }
      pap = bc_warp_sum(acc);
      alpha = pap == 0.0 ? 0.0 : rs / pap;
      res = sqrt(rs);
    }
  }
  if (lane == 0) {
    a.status[0] = it;
    a.status[1] = it >= a.max_iters ? 1 : 0;
  }
  __syncwarp();
  double up = 0.0, lo = 0.0;
  for (int q = lane; q < m; q += 32) {
    const int p = at(q);
    up += f1[p] * x1[p];
    lo += x1[p] * ap_at(x1, p);
  }
  up = bc_warp_sum(up);
  lo = bc_warp_sum(lo);
  for (int q = lane; q < n1; q += 32)
    xf[q] = (float)x1[q];
  __syncwarp();
  return up / lo;
}

__global__ void __cluster_dims__(kCgCtas, 1, 1) __launch_bounds__(kBcThreads)
    bottom_cluster_kernel(BottomArgs a) {
  namespace cgs = cooperative_groups;
  cgs::cluster_group cluster = cgs::this_cluster();
  extern __shared__ __align__(16) unsigned char bc_smem[];
  __shared__ double sh[32];
  const BcLayout lay = bc_layout(a);
  const int rank = (int)cluster.block_rank();
  const int T = a.top;
  const int tid = threadIdx.x, nt = blockDim.x;
  double *red = (double *)(bc_smem + lay.red);

  // ---- top level: this CTA's planes ----
  const Dims td = a.lv[T].d;
  const int nx = td.nx, nz = td.nz, nxy = td.nx * td.ny;
  const int klo = cg_plane_lo(rank, nz);
  const int khi = cg_plane_lo(rank + 1, nz) - 1;
  const int npl = T >= 2 ? khi - klo + 1 : 0;
  const int TS = (kCgMaxPlanes + 1) * nxy; // slot stride of tA
  float *tA = (float *)(bc_smem + lay.tA); // [slot][plane klo-1 .. khi]
  float *tx = (float *)(bc_smem + lay.tx);
  float *tf = (float *)(bc_smem + lay.tf);
  float *tr = (float *)(bc_smem + lay.tr);
  float *zp = (float *)(bc_smem + lay.zero);
  // plane kk of a distributed top-level array (base: this CTA's copy)
  auto plane = [&](float *base, int kk) -> float * {
    if (kk < 2 || kk > nz - 1)
      return zp;
    if (kk >= klo && kk <= khi)
      return base + (kk - klo) * nxy;
    const int r = cg_plane_owner(kk, nz);
    return cluster.map_shared_rank(base, r) + (kk - cg_plane_lo(r, nz)) * nxy;
  };

  // ---- stage: asynchronous copies, zeroed iterates ----
  if (T >= 2) {
    const BottomLevel &v = a.lv[T];
    const int m = (npl + 1) * nxy;
    for (int s = 0; s < 14; ++s) {
      const float *src = v.A.a[s] + (klo - 2) * nxy;
      for (int q = tid; q < m; q += nt)
        cp_async_zfill<4>(tA + s * TS + q, src + q, true);
    }
    for (int q = tid; q < npl * nxy; q += nt)
      cp_async_zfill<4>(tf + q, v.f + (klo - 1) * nxy + q, true);
    for (int q = tid; q < kCgMaxPlanes * nxy; q += nt) {
      tx[q] = 0.f;
      tr[q] = 0.f;
    }
    for (int q = tid; q < nxy; q += nt)
      zp[q] = 0.f;
  }
  const Dims d1 = a.lv[1].d;
  const int n1 = (int)d1.count();
  double *A1 = (double *)(bc_smem + lay.A1);
  double *x1 = (double *)(bc_smem + lay.x1);
  double *f1 = (double *)(bc_smem + lay.f1);
  double *cr = (double *)(bc_smem + lay.cr);
  double *cp = (double *)(bc_smem + lay.cp);
  double *cap = (double *)(bc_smem + lay.cap);
  float *xf1 = (float *)(bc_smem + lay.xf1);
  float *ff1 = (float *)(bc_smem + lay.ff1);
  auto level = [&](int L) -> BcLevel {
    return BcLevel{a.lv[L].d, (float *)(bc_smem + lay.lA[L]),
                   (float *)(bc_smem + lay.lx[L]),
                   (float *)(bc_smem + lay.lf[L]),
                   (float *)(bc_smem + lay.lr[L])};
  };
  if (rank == 0) {
    for (int L = 2; L < T; ++L) {
      const BcLevel v = level(L);
      const int n3 = (int)v.d.count();
      for (int s = 0; s < 14; ++s)
        for (int q = tid; q < n3; q += nt)
          cp_async_zfill<4>(v.A + s * n3 + q, a.lv[L].A.a[s] + q, true);
      for (int q = tid; q < n3; q += nt) {
        v.x[q] = 0.f;
        v.f[q] = 0.f;
        v.r[q] = 0.f;
      }
    }
    for (int s = 0; s < 14; ++s)
      for (int q = tid; q < n1; q += nt)
        cp_async_zfill<8>(A1 + s * n1 + q, a.A1.a[s] + q, true);
    for (int q = tid; q < n1; q += nt) {
      x1[q] = 0.0;
      cr[q] = 0.0;
      cp[q] = 0.0;
      cap[q] = 0.0;
      xf1[q] = 0.f;
      if (T == 1)
        cp_async_zfill<4>(ff1 + q, a.lv[1].f + q, true);
      else
        ff1[q] = 0.f;
    }
  }
  cp_async_wait_all();
  __syncthreads();
  cluster.sync(); // every CTA's planes staged before anyone reads them

  // this thread's point of the top level, colour-major over the CTA's planes
  int ti = 2, tj = 2, tk = klo, tcol = -1;
  const bool own =
      T >= 2 && bc_point(tid, nx, td.ny, klo, npl, ti, tj, tk, tcol);
  const int to = (tj - 1) * nx + (ti - 1), tlp = tk - klo;
  const float *tak = tA + (tlp + 1) * nxy, *tad = tak - nxy;
  float *txc = tx + tlp * nxy;
  const float *txd = own ? plane(tx, tk - 1) : zp;
  const float *txu = own ? plane(tx, tk + 1) : zp;
  const float *tfc = tf + tlp * nxy;
  // eight-colour sweeps on the top level: the colours of one plane parity
  // touch only this CTA's planes; the parity switch is a cluster barrier
  auto top_gs = [&](int sweeps) {
    for (int s = 0; s < sweeps; ++s)
      for (int c = 0; c < 8; ++c) {
        if (own && tcol == c) {
          float tO, tU, tD;
          bc_sums27(tak, tad, TS, to, nx, txc, txd, txu, tO, tU, tD);
          txc[to] = (tfc[to] + (tO + tU + tD)) / tak[kOC * TS + to];
        }
        if (c == 3 || c == 7)
          cluster.sync();
        else
          __syncthreads();
      }
  };

  // ---- descend ----
  if (T >= 2) {
    top_gs(2);
    if (own)
      tr[tlp * nxy + to] =
          tfc[to] - bc_apply27(tak, tad, TS, to, nx, txc, txd, txu);
    cluster.sync(); // top-level defect visible to rank 0
  }
  if (rank == 0) {
    double omega = 0.0; // damping of the level below the current one
    if (T >= 2)
      bc_restrict(td, a.lv[T - 1].d, a.lv[T - 1].P,
                  [&](int K) -> const float * { return plane(tr, K); },
                  T - 1 >= 2 ? level(T - 1).f : ff1);
    for (int L = T - 1; L >= 2; --L) {
      const BcLevel v = level(L);
      bc_local_gs27(v, 2);
      bc_local_defect(v);
      const int vnxy = v.d.nx * v.d.ny;
      bc_restrict(v.d, a.lv[L - 1].d, a.lv[L - 1].P,
                  [&](int K) -> const float * { return v.r + (K - 1) * vnxy; },
                  L - 1 >= 2 ? level(L - 1).f : ff1);
    }
    if (tid < 32)
      omega = bc_level1(a, A1, x1, f1, cr, cp, cap, ff1, xf1);
    __syncthreads();
    if (tid < 32 && T == 1) {
      for (int q = tid; q < n1; q += 32)
        a.lv[1].x[q] = xf1[q];
      if (tid == 0)
        *a.lv[1].omega = omega;
    }
    if (tid == 0) // warp 0's omega to every thread
      sh[0] = omega;
    __syncthreads();
    omega = sh[0];
    __syncthreads();
    // ascend the local levels
    for (int L = 2; L < T; ++L) {
      const BcLevel v = level(L);
      const int vnxy = v.d.nx * v.d.ny;
      bc_interp(a.lv[L - 1].d, v.d, a.lv[L - 1].P,
                L - 1 >= 2 ? level(L - 1).x : xf1,
                [&](int K) -> float * { return v.r + (K - 1) * vnxy; });
      const float w = (float)omega;
      for (int q = tid; q < (int)v.d.count(); q += nt)
        v.x[q] = v.x[q] + w * v.r[q];
      __syncthreads();
      bc_local_gs27(v, 2);
      omega = bc_local_damping(v, sh);
    }
    if (T >= 2) {
      // interpolate into the top level's r planes (this CTA's and the
      // other CTAs'); shell planes are not stored
      bc_interp(a.lv[T - 1].d, td, a.lv[T - 1].P,
                T - 1 >= 2 ? level(T - 1).x : xf1, [&](int K) -> float * {
                  return K >= 2 && K <= nz - 1 ? plane(tr, K) : nullptr;
                });
      if (tid == 0)
        red[2] = omega;
    }
  }
  if (T < 2) {
    cluster.sync(); // rank 0 done with level 1
    return;
  }

  // ---- ascend the top level ----
  cluster.sync(); // interpolated correction and damping visible
  {
    const float w = (float)cluster.map_shared_rank(red, 0)[2];
    for (int q = tid; q < npl * nxy; q += nt)
      tx[q] = tx[q] + w * tr[q];
  }
  cluster.sync(); // updated x visible before the sweeps read it
  top_gs(2);
  // damping of the top level, summed over the cluster in rank order
  double up = 0.0, lo = 0.0;
  if (own) {
    up = (double)tfc[to] * (double)txc[to];
    lo = (double)txc[to] *
         (double)bc_apply27(tak, tad, TS, to, nx, txc, txd, txu);
  }
  up = cg_block_sum(up, sh);
  __syncthreads();
  lo = cg_block_sum(lo, sh);
  if (tid == 0) {
    red[0] = up;
    red[1] = lo;
  }
  // the top level's x to global memory (shell planes zero)
  {
    float *gx = a.lv[T].x;
    for (int q = tid; q < npl * nxy; q += nt)
      gx[(klo - 1) * nxy + q] = tx[q];
    if (rank == 0)
      for (int q = tid; q < nxy; q += nt) {
        gx[q] = 0.f;
        gx[(nz - 1) * nxy + q] = 0.f;
      }
  }
  cluster.sync();
  if (rank == 0 && tid == 0) {
    double su = 0.0, sl = 0.0;
    for (int r = 0; r < kCgCtas; ++r) {
      const double *rr = cluster.map_shared_rank(red, r);
      su += rr[0];
      sl += rr[1];
    }
    *a.lv[T].omega = su / sl;
  }
  cluster.sync(); // no CTA leaves while rank 0 may still read its sums
}

} // namespace pmg
