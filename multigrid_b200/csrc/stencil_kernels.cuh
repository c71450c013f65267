// Stencil kernels of the PMG V-cycle: Gauss-Seidel smoothers, matvec,
// residual and defect, restriction, interpolation (with the damped update).
//
// Every kernel evaluates the per-point arithmetic in the reference's operation
// order (products and sums rounded separately: the library is built with
// --fmad=false), so a double-precision launch reproduces the reference kernel
// bit for bit on the same inputs. Cited per kernel.
#pragma once

#include "pmg_common.cuh"

namespace pmg {

// ---------------------------------------------------------------------------
// Per-point operators
// ---------------------------------------------------------------------------

// Positive neighbour sums of the 27-point operator in the reference order:
// tmpO (8 in-plane), tmpU (9 above), tmpD (9 below), pmgc/gsd.cc:171-204.
template <typename T>
__device__ __forceinline__ void sums27(const Op14<T> &A, const T *x, int p,
                                       int sy, int sz, T &tO, T &tU, T &tD) {
  const T *const *a = A.a;
  tO = a[kON][p] * x[p + sy] + a[kON][p - sy] * x[p - sy] +
       a[kOE][p] * x[p + 1] + a[kOE][p - 1] * x[p - 1] +
       a[kONE][p] * x[p + 1 + sy] + a[kONW][p] * x[p - 1 + sy] +
       a[kONW][p + 1 - sy] * x[p + 1 - sy] +
       a[kONE][p - 1 - sy] * x[p - 1 - sy];
  tU = a[kUC][p] * x[p + sz] + a[kUN][p] * x[p + sy + sz] +
       a[kUS][p] * x[p - sy + sz] + a[kUE][p] * x[p + 1 + sz] +
       a[kUW][p] * x[p - 1 + sz] + a[kUNE][p] * x[p + 1 + sy + sz] +
       a[kUNW][p] * x[p - 1 + sy + sz] + a[kUSE][p] * x[p + 1 - sy + sz] +
       a[kUSW][p] * x[p - 1 - sy + sz];
  tD = a[kUC][p - sz] * x[p - sz] + a[kUS][p + sy - sz] * x[p + sy - sz] +
       a[kUN][p - sy - sz] * x[p - sy - sz] +
       a[kUW][p + 1 - sz] * x[p + 1 - sz] +
       a[kUE][p - 1 - sz] * x[p - 1 - sz] +
       a[kUSW][p + 1 + sy - sz] * x[p + 1 + sy - sz] +
       a[kUSE][p - 1 + sy - sz] * x[p - 1 + sy - sz] +
       a[kUNW][p + 1 - sy - sz] * x[p + 1 - sy - sz] +
       a[kUNE][p - 1 - sy - sz] * x[p - 1 - sy - sz];
}

// (A x)(p) as matveckernel7 / Vmatvec7_1s compute it
// (pmgc/matvecd.h:131-137, pmgc/matvecd.cc:81-88); cc may be null (= 0).
template <typename T>
__device__ __forceinline__ T apply7(const Op14<T> &A, const T *cc, const T *x,
                                    int p, int sy, int sz) {
  const T *oC = A.a[kOC], *oE = A.a[kOE], *oN = A.a[kON], *uC = A.a[kUC];
  const T c = cc ? cc[p] : T(0);
  return -oN[p] * x[p + sy] - oN[p - sy] * x[p - sy] - oE[p] * x[p + 1] -
         oE[p - 1] * x[p - 1] - uC[p - sz] * x[p - sz] - uC[p] * x[p + sz] +
         (oC[p] + c) * x[p];
}

// (A x)(p) as matveckernel27 / Vmatvec27_1s compute it
// (pmgc/matvecd.h:208-239, pmgc/matvecd.cc:142-174): the reference subtracts
// each product from a negated running sum, which rounds exactly like the
// negated positive sum.
template <typename T>
__device__ __forceinline__ T apply27(const Op14<T> &A, const T *cc,
                                     const T *x, int p, int sy, int sz) {
  T tO, tU, tD;
  sums27(A, x, p, sy, sz, tO, tU, tD);
  const T c = cc ? cc[p] : T(0);
  return (-tO) + (-tU) + (-tD) + (A.a[kOC][p] + c) * x[p];
}

template <int KIND, typename T>
__device__ __forceinline__ T apply_op(const Op14<T> &A, const T *cc,
                                      const T *x, int p, int sy, int sz) {
  if constexpr (KIND == 7)
    return apply7(A, cc, x, p, sy, sz);
  else
    return apply27(A, cc, x, p, sy, sz);
}

// ---------------------------------------------------------------------------
// Gauss-Seidel colour sweeps
// ---------------------------------------------------------------------------

// One colour of the red-black sweep on the 7-point operator (Vgsrb7x,
// pmgc/gsd.cc:85-107): updates the interior points with (i+j+k)%2 == want;
// keep = 0 drops the neighbour sum (zero_initialize). One thread per point of
// the colour; blockIdx.z is the plane.
template <typename T>
__global__ void __launch_bounds__(256)
    gs7_color_kernel(Dims d, const T *__restrict__ oC, const T *__restrict__ cc,
                     const T *__restrict__ fc, const T *__restrict__ oE,
                     const T *__restrict__ oN, const T *__restrict__ uC, T *x,
                     int want, T keep) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (j > d.ny - 1)
    return;
  const int i = 2 + ((2 + j + k + want) & 1) +
                2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i > d.nx - 1)
    return;
  const int sy = d.sy(), sz = d.sz();
  const int p = d.at(i, j, k);
  const T s = oN[p] * x[p + sy] + oN[p - sy] * x[p - sy] + oE[p] * x[p + 1] +
              oE[p - 1] * x[p - 1] + uC[p - sz] * x[p - sz] +
              uC[p] * x[p + sz];
  const T c = cc ? cc[p] : T(0);
  x[p] = (fc[p] + keep * s) / (oC[p] + c);
}

// One colour of the eight-colour sweep on the 27-point operator (Vgsrb27x,
// pmgc/gsd.cc:161-209): updates the interior points whose index parities are
// (want&1, want>>1&1, want>>2&1).
template <typename T>
__global__ void __launch_bounds__(256)
    gs27_color_kernel(Dims d, Op14<T> A, const T *__restrict__ cc,
                      const T *__restrict__ fc, T *x, int want) {
  const int i = 2 + (want & 1) +
                2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 2 + ((want >> 1) & 1) +
                2 * (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int k = 2 + ((want >> 2) & 1) + 2 * (int)blockIdx.z;
  if (i > d.nx - 1 || j > d.ny - 1 || k > d.nz - 1)
    return;
  const int sy = d.sy(), sz = d.sz();
  const int p = d.at(i, j, k);
  T tO, tU, tD;
  sums27(A, x, p, sy, sz, tO, tU, tD);
  const T c = cc ? cc[p] : T(0);
  x[p] = (fc[p] + (tO + tU + tD)) / (A.a[kOC][p] + c);
}

// ---------------------------------------------------------------------------
// matvec / residual / defect
// ---------------------------------------------------------------------------

// Interior launch helper: blockIdx.z is the plane, (x, y) cover the row.
struct Interior {
  int i, j, k;
  bool ok;
};
__device__ __forceinline__ Interior interior_point(const Dims &d) {
  Interior t;
  t.i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  t.j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  t.k = blockIdx.z + 2;
  t.ok = t.i <= d.nx - 1 && t.j <= d.ny - 1;
  return t;
}

// y = A x (Vmatvec7_1s / Vmatvec27_1s).
template <int KIND, typename T>
__global__ void __launch_bounds__(256)
    matvec_kernel(Dims d, Op14<T> A, const T *__restrict__ cc,
                  const T *__restrict__ x, T *__restrict__ y) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  y[p] = apply_op<KIND>(A, cc, x, p, d.sy(), d.sz());
}

// (f - A x)(p) in the order of Vmresid7_1s / Vmresid27_1s
// (pmgc/matvecd.cc:402-409, 491-493); cc may be null (= 0).
template <int KIND, typename T>
__device__ __forceinline__ T resid_at(const Op14<T> &A, const T *cc,
                                      const T *fc, const T *x, int p, int sy,
                                      int sz) {
  const T c = cc ? cc[p] : T(0);
  if constexpr (KIND == 7) {
    const T *oC = A.a[kOC], *oE = A.a[kOE], *oN = A.a[kON], *uC = A.a[kUC];
    return fc[p] + oN[p] * x[p + sy] + oN[p - sy] * x[p - sy] +
           oE[p] * x[p + 1] + oE[p - 1] * x[p - 1] + uC[p - sz] * x[p - sz] +
           uC[p] * x[p + sz] - (oC[p] + c) * x[p];
  } else {
    T tO, tU, tD;
    sums27(A, x, p, sy, sz, tO, tU, tD);
    return fc[p] + tO + tU + tD - (A.a[kOC][p] + c) * x[p];
  }
}

// r = f - A x on the interior (Vmresid7_1s / Vmresid27_1s).
template <int KIND, typename T>
__global__ void __launch_bounds__(256)
    mresid_kernel(Dims d, Op14<T> A, const T *__restrict__ cc,
                  const T *__restrict__ fc, const T *__restrict__ x,
                  T *__restrict__ r) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  r[p] = resid_at<KIND>(A, cc, fc, x, p, d.sy(), d.sz());
}

// ---------------------------------------------------------------------------
// Grid transfers
// ---------------------------------------------------------------------------

// Restriction xout = P^T xin on the coarse interior (Vrestrc2,
// pmgc/matvecd.cc:755-794): plane sums over C N S E W NE NW SE SW at the
// fine planes kk, kk+1, kk-1, then tmpO + tmpU + tmpD.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256)
    restrict_kernel(Dims df, Dims dc, const Tin *__restrict__ xin,
                    Tout *__restrict__ xout, P27<Tin> P) {
  const Interior t = interior_point(dc);
  if (!t.ok)
    return;
  const int pc = dc.at(t.i, t.j, t.k);
  const int sy = df.sy(), sz = df.sz();
  const int f0 = df.at(2 * t.i - 1, 2 * t.j - 1, 2 * t.k - 1);
  Tin pl[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int b = q * 9;
    const int f = f0 + (q == 0 ? 0 : q == 1 ? sz : -sz);
    pl[q] = P.p[b + 0][pc] * xin[f] + P.p[b + 1][pc] * xin[f + sy] +
            P.p[b + 2][pc] * xin[f - sy] + P.p[b + 3][pc] * xin[f + 1] +
            P.p[b + 4][pc] * xin[f - 1] + P.p[b + 5][pc] * xin[f + 1 + sy] +
            P.p[b + 6][pc] * xin[f - 1 + sy] +
            P.p[b + 7][pc] * xin[f + 1 - sy] +
            P.p[b + 8][pc] * xin[f - 1 - sy];
  }
  xout[pc] = (Tout)(pl[0] + pl[1] + pl[2]);
}

// Interpolation xout = P xin (VinterpPMG2, pmgc/matvecd.cc:878-960): one
// thread per coarse cell (ii,jj,kk) in [1, n_c-1]^3 writing its eight fine
// points.
template <typename T>
__global__ void __launch_bounds__(256)
    interp_kernel(Dims dc, Dims df, const T *__restrict__ xin,
                  T *__restrict__ xout, P27<T> P) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int kk = blockIdx.z + 1;
  if (ii > dc.nx - 1 || jj > dc.ny - 1)
    return;
  const int cy = dc.sy(), cz = dc.sz();
  const int fy = df.sy(), fz = df.sz();
  const int c = dc.at(ii, jj, kk);
  const int f = df.at(2 * ii - 1, 2 * jj - 1, 2 * kk - 1);
  const T *const *p = P.p;
  // P slots: oPC 0 oPN 1 oPS 2 oPE 3 oPW 4 oPNE 5 oPNW 6 oPSE 7 oPSW 8,
  // u* +9, d* +18.
  const T x000 = xin[c], x100 = xin[c + 1], x010 = xin[c + cy],
          x001 = xin[c + cz], x110 = xin[c + 1 + cy], x101 = xin[c + 1 + cz],
          x011 = xin[c + cy + cz], x111 = xin[c + 1 + cy + cz];
  xout[f] = x000;
  xout[f + 1] = p[3][c] * x000 + p[4][c + 1] * x100;
  xout[f + fy] = p[1][c] * x000 + p[2][c + cy] * x010;
  xout[f + fz] = p[9][c] * x000 + p[18][c + cz] * x001;
  xout[f + 1 + fy] = p[5][c] * x000 + p[6][c + 1] * x100 +
                     p[7][c + cy] * x010 + p[8][c + 1 + cy] * x110;
  xout[f + 1 + fz] = p[12][c] * x000 + p[13][c + 1] * x100 +
                     p[21][c + cz] * x001 + p[22][c + 1 + cz] * x101;
  xout[f + fy + fz] = p[10][c] * x000 + p[11][c + cy] * x010 +
                      p[19][c + cz] * x001 + p[20][c + cy + cz] * x011;
  xout[f + 1 + fy + fz] =
      p[14][c] * x000 + p[15][c + 1] * x100 + p[16][c + cy] * x010 +
      p[17][c + 1 + cy] * x110 + p[23][c + cz] * x001 +
      p[24][c + 1 + cz] * x101 + p[25][c + cy + cz] * x011 +
      p[26][c + 1 + cy + cz] * x111;
}

// x = x + w * (interpolation of xin), fused: interp_kernel's eight values
// per coarse cell (same order and arithmetic), each added at once to the
// fine iterate as the damped update of the padded array adds it, x + w e
// (add_and_multiply_domains, Domain.h:602-623), so the correction never
// goes through memory. The fine points the interpolation does not write
// (the last plane, row and column of the shell) keep x: there the padded
// update adds w * 0, e being zero there. With SPLIT_X
// the fine iterate is in the colour-split row layout (split_layout.cuh).
template <typename T, bool SPLIT_X>
__global__ void __launch_bounds__(256)
    interp_add_kernel(Dims dc, Dims df, const T *__restrict__ xin,
                      P27<T> P, T *__restrict__ x,
                      const double *__restrict__ w) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int kk = blockIdx.z + 1;
  if (ii > dc.nx - 1 || jj > dc.ny - 1)
    return;
  const T ww = (T)(*w);
  const int cy = dc.sy(), cz = dc.sz();
  const int c = dc.at(ii, jj, kk);
  // fine point (2ii-1 + a, 2jj-1 + b, 2kk-1 + c): reference layout
  // f0 + a + b fy + c fz; colour-split layout (split_layout.cuh: halves of
  // hp entries, a multiple of 16) entry ii - 1 of the half of its colour
  // (1 + a + b + c) & 1 in row f0 + b fy + c fz
  const int hp = SPLIT_X ? ((df.nx + 1) / 2 + 15) & ~15 : 0;
  const int fy = SPLIT_X ? 2 * hp : df.sy();
  const int fz = SPLIT_X ? 2 * hp * df.ny : df.sz();
  const int f0 = SPLIT_X ? ((2 * kk - 2) * df.ny + (2 * jj - 2)) * fy + ii - 1
                         : df.at(2 * ii - 1, 2 * jj - 1, 2 * kk - 1);
  // offsets of the points with a = 0 and a = 1 in the rows with b + c even
  // (in the other rows the two swap halves)
  const int ev0 = SPLIT_X ? hp : 0, ev1 = SPLIT_X ? 0 : 1;
  const int od0 = 0, od1 = SPLIT_X ? hp : 1;
  const int e0 = f0 + ev0, e1 = f0 + ev1;
  const T *const *p = P.p;
  const T x000 = xin[c], x100 = xin[c + 1], x010 = xin[c + cy],
          x001 = xin[c + cz], x110 = xin[c + 1 + cy], x101 = xin[c + 1 + cz],
          x011 = xin[c + cy + cz], x111 = xin[c + 1 + cy + cz];
  const T v000 = x000;
  const T v100 = p[3][c] * x000 + p[4][c + 1] * x100;
  const T v010 = p[1][c] * x000 + p[2][c + cy] * x010;
  const T v001 = p[9][c] * x000 + p[18][c + cz] * x001;
  const T v110 = p[5][c] * x000 + p[6][c + 1] * x100 + p[7][c + cy] * x010 +
                 p[8][c + 1 + cy] * x110;
  const T v101 = p[12][c] * x000 + p[13][c + 1] * x100 +
                 p[21][c + cz] * x001 + p[22][c + 1 + cz] * x101;
  const T v011 = p[10][c] * x000 + p[11][c + cy] * x010 +
                 p[19][c + cz] * x001 + p[20][c + cy + cz] * x011;
  const T v111 = p[14][c] * x000 + p[15][c + 1] * x100 +
                 p[16][c + cy] * x010 + p[17][c + 1 + cy] * x110 +
                 p[23][c + cz] * x001 + p[24][c + 1 + cz] * x101 +
                 p[25][c + cy + cz] * x011 + p[26][c + 1 + cy + cz] * x111;
  const int o0 = f0 + od0, o1 = f0 + od1; // rows with b + c odd
  x[e0] = x[e0] + ww * v000;
  x[e1] = x[e1] + ww * v100;
  x[o0 + fy] = x[o0 + fy] + ww * v010;
  x[o0 + fz] = x[o0 + fz] + ww * v001;
  x[o1 + fy] = x[o1 + fy] + ww * v110;
  x[o1 + fz] = x[o1 + fz] + ww * v101;
  x[e0 + fy + fz] = x[e0 + fy + fz] + ww * v011;
  x[e1 + fy + fz] = x[e1 + fy + fz] + ww * v111;
}

// ---------------------------------------------------------------------------
// Elementwise
// ---------------------------------------------------------------------------

// dst = (Tout)src over n entries.
template <typename Tin, typename Tout>
__global__ void convert_kernel(long n, const Tin *__restrict__ src,
                               Tout *__restrict__ dst) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x)
    dst[q] = (Tout)src[q];
}

// dst (rows dd.px apart) = (Tout) src (rows ds.px apart), every point of
// the grid (shell included); the two Dims differ only in their pitch
template <typename Tin, typename Tout>
__global__ void repitch_kernel(Dims ds, Dims dd, const Tin *__restrict__ src,
                               Tout *__restrict__ dst) {
  const long n = (long)ds.nx * ds.ny * ds.nz;
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n;
       g += (long)gridDim.x * blockDim.x) {
    const int i = (int)(g % ds.nx) + 1;
    const long r = g / ds.nx;
    const int j = (int)(r % ds.ny) + 1, k = (int)(r / ds.ny) + 1;
    dst[dd.at(i, j, k)] = (Tout)src[ds.at(i, j, k)];
  }
}

// x64 += (double)e32 on the interior (mixed-precision refinement update).
__global__ void add_correction_kernel(Dims d, double *__restrict__ x,
                                      const float *__restrict__ e);

} // namespace pmg
