// The lowest levels of the mixed-precision V-cycle in one CTA.
//
// Below 17^3 points a level has too little work for a grid-wide launch: the
// smoother alone would be 16 colour launches per sweep pair. This kernel runs
// the whole V-cycle from level `top` (n <= 17) down to level 1 and back in a
// single CTA of 1024 threads, with block barriers in place of launches:
// zero-started eight-colour smoothing in place (a single CTA needs no
// ping-pong), defect, restriction, the double-precision CG on level 1,
// Hackbusch-Reusken damping, interpolation and x += w e — the steps of the
// float V-cycle above it (v_cycle, PBE_pmgc_class.h:1070-1114, with every
// level zero-started), with the same per-point arithmetic. Reductions sum in
// a fixed order, so results are deterministic.
#pragma once

#include "reduce_kernels.cuh"

namespace pmg {

constexpr int kBottomMaxLevels = 4;
constexpr int kBottomMaxN = 17;

struct BottomLevel {
  Dims d;
  Op14<float> A;     // level operator (float), unused on level 1
  P27<float> P;      // prolongation from this level to the next finer one
  float *x, *f, *r;  // iterate, right-hand side, defect / correction
  double *omega;     // damping computed on this level
};

struct BottomArgs {
  int top;                         // finest level handled here (<= 4)
  BottomLevel lv[kBottomMaxLevels + 1];
  Op14<double> A1;                 // level-1 operator (double)
  double *x1, *f1;                 // level-1 iterate / rhs (double)
  double *cg_r, *cg_p, *cg_ap;     // CG work vectors (zero shells)
  double rtol;                     // CG stop: relative residual reduction
  int max_iters;
  int *status;
};

__device__ __forceinline__ double bottom_allsum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads(); // sh may still be read from the previous sum
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
    t += sh[w];
  return t;
}

// all interior points (i, j, k) of d with the given index parities
// (pi, pj, pk < 0 means any), one per thread in turn
template <typename F>
__device__ __forceinline__ void for_interior(const Dims &d, F fn) {
  const int mx = d.nx - 2, my = d.ny - 2, m = mx * my * (d.nz - 2);
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    const int r = q / mx;
    const int i = q - r * mx + 2;
    const int k = r / my;
    const int j = r - k * my + 2;
    fn(i, j, k + 2);
  }
}

__device__ void bottom_gs27(const BottomLevel &v, int sweeps, bool zero) {
  const Dims &d = v.d;
  if (zero) {
    for (int q = threadIdx.x; q < (int)d.count(); q += blockDim.x)
      v.x[q] = 0.f;
    __syncthreads();
  }
  const int sy = d.sy(), sz = d.sz();
  for (int s = 0; s < sweeps; ++s)
    for (int c = 0; c < 8; ++c) {
      const int pi = c & 1, pj = (c >> 1) & 1, pk = (c >> 2) & 1;
      // points with (i%2, j%2, k%2) == (pi, pj, pk): a grid of half size
      const int hx = (d.nx - 2 - pi + 1) / 2, hy = (d.ny - 2 - pj + 1) / 2,
                hz = (d.nz - 2 - pk + 1) / 2;
      const int m = hx * hy * hz;
      for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const int r = q / hx;
        const int i = 2 + pi + 2 * (q - r * hx);
        const int kk = r / hy;
        const int j = 2 + pj + 2 * (r - kk * hy);
        const int k = 2 + pk + 2 * kk;
        const int p = d.at(i, j, k);
        float tO, tU, tD;
        sums27(v.A, v.x, p, sy, sz, tO, tU, tD);
        v.x[p] = (v.f[p] + (tO + tU + tD)) / v.A.a[kOC][p];
      }
      __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) bottom_cycle_kernel(BottomArgs a) {
  __shared__ double sh[32];
  // descend: smooth, defect, restrict
  for (int L = a.top; L >= 2; --L) {
    const BottomLevel &v = a.lv[L];
    const BottomLevel &c = a.lv[L - 1];
    bottom_gs27(v, 2, true);
    const int sy = v.d.sy(), sz = v.d.sz();
    for_interior(v.d, [&](int i, int j, int k) {
      const int p = v.d.at(i, j, k);
      v.r[p] = v.f[p] - apply27(v.A, (const float *)nullptr, v.x, p, sy, sz);
    });
    __syncthreads();
    const int fy = v.d.sy(), fz = v.d.sz();
    for_interior(c.d, [&](int i, int j, int k) {
      const int pc = c.d.at(i, j, k);
      const int f0 = v.d.at(2 * i - 1, 2 * j - 1, 2 * k - 1);
      float pl[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int b = q * 9;
        const int f = f0 + (q == 0 ? 0 : q == 1 ? fz : -fz);
        const float *const *P = c.P.p;
        pl[q] = P[b + 0][pc] * v.r[f] + P[b + 1][pc] * v.r[f + fy] +
                P[b + 2][pc] * v.r[f - fy] + P[b + 3][pc] * v.r[f + 1] +
                P[b + 4][pc] * v.r[f - 1] + P[b + 5][pc] * v.r[f + 1 + fy] +
                P[b + 6][pc] * v.r[f - 1 + fy] +
                P[b + 7][pc] * v.r[f + 1 - fy] +
                P[b + 8][pc] * v.r[f - 1 - fy];
      }
      c.f[pc] = pl[0] + pl[1] + pl[2];
    });
    __syncthreads();
  }

  // level 1: zero-started double CG to a relative reduction of rtol
  {
    const BottomLevel &v = a.lv[1];
    const Dims &d = v.d;
    const int n3 = (int)d.count();
    for (int q = threadIdx.x; q < n3; q += blockDim.x) {
      a.f1[q] = (double)v.f[q];
      a.x1[q] = 0.0;
    }
    __syncthreads();
    const int sy = d.sy(), sz = d.sz();
    const double *nul = nullptr;
    double acc = 0.0;
    for_interior(d, [&](int i, int j, int k) {
      const int p = d.at(i, j, k);
      const double r = a.f1[p] - apply27(a.A1, nul, a.x1, p, sy, sz);
      a.cg_r[p] = r;
      a.cg_p[p] = r;
      acc += r * r;
    });
    double rs = bottom_allsum(acc, sh);
    acc = 0.0;
    for_interior(d, [&](int i, int j, int k) {
      const int p = d.at(i, j, k);
      const double ap = apply27(a.A1, nul, a.cg_p, p, sy, sz);
      a.cg_ap[p] = ap;
      acc += ap * a.cg_p[p];
    });
    double pap = bottom_allsum(acc, sh);
    int it = 0;
    if (pap != 0.0) {
      double alpha = rs / pap;
      double res = sqrt(rs);
      const double stop = a.rtol * res;
      while (res > stop && it < a.max_iters) {
        ++it;
        acc = 0.0;
        for_interior(d, [&](int i, int j, int k) {
          const int p = d.at(i, j, k);
          a.x1[p] += alpha * a.cg_p[p];
          const double r = a.cg_r[p] - alpha * a.cg_ap[p];
          a.cg_r[p] = r;
          acc += r * r;
        });
        const double rsn = bottom_allsum(acc, sh);
        const double beta = rs == 0.0 ? 0.0 : rsn / rs;
        rs = rsn;
        for_interior(d, [&](int i, int j, int k) {
          const int p = d.at(i, j, k);
          a.cg_p[p] = a.cg_r[p] + beta * a.cg_p[p];
        });
        __syncthreads();
        acc = 0.0;
        for_interior(d, [&](int i, int j, int k) {
          const int p = d.at(i, j, k);
          const double ap = apply27(a.A1, nul, a.cg_p, p, sy, sz);
          a.cg_ap[p] = ap;
          acc += ap * a.cg_p[p];
        });
        pap = bottom_allsum(acc, sh);
        alpha = pap == 0.0 ? 0.0 : rs / pap;
        res = sqrt(rs);
      }
    }
    if (threadIdx.x == 0) {
      a.status[0] = it;
      a.status[1] = it >= a.max_iters ? 1 : 0;
    }
    // damping on level 1 in double, then the float copy of x
    double up = 0.0, lo = 0.0;
    for_interior(d, [&](int i, int j, int k) {
      const int p = d.at(i, j, k);
      up += a.f1[p] * a.x1[p];
      lo += a.x1[p] * apply27(a.A1, nul, a.x1, p, sy, sz);
    });
    up = bottom_allsum(up, sh);
    lo = bottom_allsum(lo, sh);
    if (threadIdx.x == 0)
      *v.omega = up / lo;
    for (int q = threadIdx.x; q < n3; q += blockDim.x)
      v.x[q] = (float)a.x1[q];
    __syncthreads();
  }

  // ascend: interpolate, x += w e, smooth; damping of this level for the
  // next finer one
  for (int L = 2; L <= a.top; ++L) {
    const BottomLevel &v = a.lv[L];
    const BottomLevel &c = a.lv[L - 1];
    const int cy = c.d.sy(), cz = c.d.sz();
    const int fy = v.d.sy(), fz = v.d.sz();
    const int mx = c.d.nx - 1, my = c.d.ny - 1, m = mx * my * (c.d.nz - 1);
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
      const int r = q / mx;
      const int ii = q - r * mx + 1;
      const int kk = r / my + 1;
      const int jj = r - (kk - 1) * my + 1;
      const int cc = c.d.at(ii, jj, kk);
      const int f = v.d.at(2 * ii - 1, 2 * jj - 1, 2 * kk - 1);
      const float *const *p = c.P.p;
      const float *xin = c.x;
      float *xout = v.r;
      const float x000 = xin[cc], x100 = xin[cc + 1], x010 = xin[cc + cy],
                  x001 = xin[cc + cz], x110 = xin[cc + 1 + cy],
                  x101 = xin[cc + 1 + cz], x011 = xin[cc + cy + cz],
                  x111 = xin[cc + 1 + cy + cz];
      xout[f] = x000;
      xout[f + 1] = p[3][cc] * x000 + p[4][cc + 1] * x100;
      xout[f + fy] = p[1][cc] * x000 + p[2][cc + cy] * x010;
      xout[f + fz] = p[9][cc] * x000 + p[18][cc + cz] * x001;
      xout[f + 1 + fy] = p[5][cc] * x000 + p[6][cc + 1] * x100 +
                         p[7][cc + cy] * x010 + p[8][cc + 1 + cy] * x110;
      xout[f + 1 + fz] = p[12][cc] * x000 + p[13][cc + 1] * x100 +
                         p[21][cc + cz] * x001 + p[22][cc + 1 + cz] * x101;
      xout[f + fy + fz] = p[10][cc] * x000 + p[11][cc + cy] * x010 +
                          p[19][cc + cz] * x001 + p[20][cc + cy + cz] * x011;
      xout[f + 1 + fy + fz] =
          p[14][cc] * x000 + p[15][cc + 1] * x100 + p[16][cc + cy] * x010 +
          p[17][cc + 1 + cy] * x110 + p[23][cc + cz] * x001 +
          p[24][cc + 1 + cz] * x101 + p[25][cc + cy + cz] * x011 +
          p[26][cc + 1 + cy + cz] * x111;
    }
    __syncthreads();
    const float w = (float)(*c.omega);
    for (int q = threadIdx.x; q < (int)v.d.count(); q += blockDim.x)
      v.x[q] = v.x[q] + w * v.r[q];
    __syncthreads();
    bottom_gs27(v, 2, false);
    // damping on this level (used by the level above)
    const int sy = v.d.sy(), sz = v.d.sz();
    double up = 0.0, lo = 0.0;
    for_interior(v.d, [&](int i, int j, int k) {
      const int p = v.d.at(i, j, k);
      up += (double)v.f[p] * (double)v.x[p];
      lo += (double)v.x[p] *
            (double)apply27(v.A, (const float *)nullptr, v.x, p, sy, sz);
    });
    up = bottom_allsum(up, sh);
    lo = bottom_allsum(lo, sh);
    if (threadIdx.x == 0)
      *v.omega = up / lo;
    __syncthreads();
  }
}

} // namespace pmg
