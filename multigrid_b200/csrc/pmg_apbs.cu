// Entry points of the pmgc library's APBS-style layer: operators packed as
// one array of diagonals with the stencil size in ipc, the packed matvec and
// residual (Vmatvec, Vmresid: pmgc/matvecd.cc:244-260, 513-529) and the
// Hestenes-Stiefel conjugate gradient Vcghs (pmgc/cgd.cc:60-125).
//
// Packed operator: ac holds numdia columns of nx*ny*nz doubles, column s at
// ac + s*nx*ny*nz, in the order oC oE oN uC (7-point, 4 columns) or oC oE oN
// uC oNE oNW uE uW uN uS uNE uNW uSE uSW (27-point, 14 columns); ipc[10]
// (the reference's VAT(ipc, 11)) is 7 or 27.
#include "launch.cuh"
#include "reduce_kernels.cuh"
#include "pmg_b200.h"

namespace pmg {
namespace {

// Unpacks ac by ipc[10]; 0 on success.
int unpack(const int *ipc, const double *ac, long n3, int *kind,
           Op14<double> *A) {
  PMG_REQUIRE(ipc && ac, "packed operator: null ipc or ac");
  *kind = ipc[10];
  PMG_REQUIRE(*kind == 7 || *kind == 27,
              "packed operator: ipc[10] must be 7 or 27");
  *A = Op14<double>{};
  const int cols = *kind == 7 ? 4 : 14;
  for (int s = 0; s < cols; ++s)
    A->a[s] = ac + (size_t)s * n3;
  return PMG_OK;
}

// r = f - A x (Vmresid order) on the interior; sum of r^2
template <int KIND>
__global__ void __launch_bounds__(kReduceThreads)
    cghs_resid_kernel(Dims d, Op14<double> A, const double *__restrict__ cc,
                      const double *__restrict__ fc,
                      const double *__restrict__ x, double *__restrict__ r,
                      ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      const double v = resid_at<KIND>(A, cc, fc, x, p, d.sy(), d.sz());
      r[p] = v;
      acc += v * v;
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// New direction on the interior: p = r on the first step, else
// p = (p + (1/beta) r) * beta, the reference's Vxaxpy then Vxscal
// (cgd.cc:95-101).
__global__ void __launch_bounds__(kReduceThreads)
    cghs_direction_kernel(Dims d, const double *__restrict__ r,
                          double *__restrict__ pv, double inv_beta,
                          double beta, int first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  if (i > d.nx - 1 || j > d.ny - 1)
    return;
  for (int k = k0; k <= k1; ++k) {
    const int p = d.at(i, j, k);
    pv[p] = first ? r[p] : (pv[p] + inv_beta * r[p]) * beta;
  }
}

// ap = A p (Vmatvec order, cc included) on the interior; sum of p * ap
template <int KIND>
__global__ void __launch_bounds__(kReduceThreads)
    cghs_matvec_kernel(Dims d, Op14<double> A, const double *__restrict__ cc,
                       const double *__restrict__ pv, double *__restrict__ ap,
                       ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      const double y = apply_op<KIND>(A, cc, pv, p, d.sy(), d.sz());
      ap[p] = y;
      acc += pv[p] * y;
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// alpha = rr / pAp; x += alpha p, r += (-alpha) ap on the interior
// (cgd.cc:105-117); sum of the new r^2. rr and pap are device results of
// earlier reductions, read before this launch's own result is written.
__global__ void __launch_bounds__(kReduceThreads)
    cghs_update_kernel(Dims d, const double *__restrict__ pv,
                       const double *__restrict__ ap, double *__restrict__ x,
                       double *__restrict__ r, const double *rr,
                       const double *pap, ReduceSlot s) {
  __shared__ double sh[32];
  const double alpha = rr[0] / pap[0];
  const double malpha = -alpha;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      x[p] += alpha * pv[p];
      const double v = r[p] + malpha * ap[p];
      r[p] = v;
      acc += v * v;
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// Device scratch of one solve: block partials, a ticket, three results
// (r.r ping-pong, p.Ap), freed on every exit.
struct CghsScratch {
  double *partials = nullptr;
  unsigned *ticket = nullptr;
  double *res = nullptr;
  cudaStream_t s;
  explicit CghsScratch(cudaStream_t st) : s(st) {}
  ~CghsScratch() {
    if (partials)
      scratch_free(partials, s);
    if (ticket)
      scratch_free(ticket, s);
    if (res)
      scratch_free(res, s);
  }
};

template <int KIND>
int cghs(const Dims &d, const Op14<double> &A, const double *cc,
         const double *fc, double *x, double *pv, double *ap, double *r,
         int itmax, int *iters, double errtol, int iresid, cudaStream_t s) {
  *iters = 0;
  if (*iters >= itmax && iresid == 0)
    return PMG_OK;
  const dim3 rg = reduce_grid(d), rb = interior_block();
  const size_t nb = (size_t)rg.x * rg.y * rg.z;
  CghsScratch w(s);
  PMG_CUDA_TRY(scratch_alloc((void **)&w.partials, nb * sizeof(double), s));
  PMG_CUDA_TRY(scratch_alloc((void **)&w.ticket, sizeof(unsigned), s));
  PMG_CUDA_TRY(scratch_alloc((void **)&w.res, 3 * sizeof(double), s));
  PMG_CUDA_TRY(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned), s));
  // p's shell must read as zero in A p; the interior is set before use
  PMG_CUDA_TRY(cudaMemsetAsync(pv, 0, sizeof(double) * d.count(), s));
  double *rr[2] = {w.res, w.res + 1}, *pap = w.res + 2;
  auto slot = [&](double *out) {
    return ReduceSlot{w.partials, w.ticket, out};
  };
  auto fetch = [&](const double *dev, double *host) -> int {
    PMG_CUDA_TRY(cudaMemcpyAsync(host, dev, sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
    PMG_CUDA_TRY(cudaStreamSynchronize(s));
    return PMG_OK;
  };

  // r = f - A x; denom = ||r|| (cgd.cc:74-75)
  cghs_resid_kernel<KIND><<<rg, rb, 0, s>>>(d, A, cc, fc, x, r, slot(rr[0]));
  PMG_LAUNCH_CHECK();
  double rhok2 = 0.0, rhok1 = 0.0;
  int rc = fetch(rr[0], &rhok2);
  if (rc != PMG_OK)
    return rc;
  const double denom = sqrt(rhok2);
  if (denom == 0.0 || *iters >= itmax)
    return PMG_OK;
  int cur = 0;
  for (;;) {
    // the stop test on r.r, the same sum as the norm above (cgd.cc:86-93)
    const double rsnrm = sqrt(rhok2);
    if (rsnrm / denom <= errtol || *iters >= itmax)
      break;
    double beta = 0.0, inv_beta = 0.0;
    if (*iters > 0) {
      beta = rhok2 / rhok1;
      inv_beta = 1.0 / beta;
    }
    cghs_direction_kernel<<<rg, rb, 0, s>>>(d, r, pv, inv_beta, beta,
                                            *iters == 0);
    PMG_LAUNCH_CHECK();
    cghs_matvec_kernel<KIND><<<rg, rb, 0, s>>>(d, A, cc, pv, ap, slot(pap));
    PMG_LAUNCH_CHECK();
    rhok1 = rhok2;
    cghs_update_kernel<<<rg, rb, 0, s>>>(d, pv, ap, x, r, rr[cur], pap,
                                         slot(rr[cur ^ 1]));
    PMG_LAUNCH_CHECK();
    cur ^= 1;
    rc = fetch(rr[cur], &rhok2);
    if (rc != PMG_OK)
      return rc;
    ++*iters;
  }
  return PMG_OK;
}

// ---------------------------------------------------------------------------
// The APBS driver, linear case: Vmgdriv / Vmgdriv2 (pmgc/mgdrvd.cc:60-491),
// Vbuildops with Galerkin coarsening (pmgc/mgsubd.cc:63-265, 349-373) and
// the V-cycle Vmvcs (pmgc/mgcsd.cc:61-531). Levels are numbered as APBS
// numbers them: 1 finest .. nlev coarsest.
// ---------------------------------------------------------------------------

// Two opposite faces of x from a boundary map (VfboundPMG,
// pmgc/mikpckd.cc:266-312) or zero when g is null (VfboundPMG00, :235-264).
// group 0: i = 1 and nx over (j, k); 1: j = 1 and ny over (i, k); 2: k = 1
// and nz over (i, j). Launched in that order, so edges keep the later
// group's value.
__global__ void apbs_face_kernel(Dims d, double *__restrict__ x,
                                 const double *__restrict__ g, int group) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int b = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int na = group == 0 ? d.ny : d.nx;
  const int nb = group == 2 ? d.ny : d.nz;
  if (a > na || b > nb)
    return;
  const long face = (long)na * nb, q = (long)(b - 1) * na + (a - 1);
  const double lo = g ? g[q] : 0.0, hi = g ? g[face + q] : 0.0;
  if (group == 0) {
    x[d.at(1, a, b)] = lo;
    x[d.at(d.nx, a, b)] = hi;
  } else if (group == 1) {
    x[d.at(a, 1, b)] = lo;
    x[d.at(a, d.ny, b)] = hi;
  } else {
    x[d.at(a, b, 1)] = lo;
    x[d.at(a, b, d.nz)] = hi;
  }
}

// Interior sums of the driver's norms: mode 0 sum |a| (Vxnrm1), 1 sum a*b
// (Vxdot as documented), 2 sum |a - b| then a = b (istop 2), 3 sum
// (a - b)^2 (istop 3).
__global__ void __launch_bounds__(kReduceThreads)
    apbs_sum_kernel(Dims d, double *__restrict__ a,
                    const double *__restrict__ b, int mode, ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      if (mode == 0) {
        acc += fabs(a[p]);
      } else if (mode == 1) {
        acc += a[p] * b[p];
      } else {
        const double v = a[p] - b[p];
        acc += mode == 2 ? fabs(v) : v * v;
        if (mode == 2)
          a[p] = b[p];
      }
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// r = f - A x (Vmresid order) and its L1 norm: the stop test of istop 0/1
// (mgcsd.cc:467-481).
template <int KIND>
__global__ void __launch_bounds__(kReduceThreads)
    apbs_resid_l1_kernel(Dims d, Op14<double> A, const double *__restrict__ cc,
                         const double *__restrict__ fc,
                         const double *__restrict__ x, double *__restrict__ r,
                         ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      const double v = resid_at<KIND>(A, cc, fc, x, p, d.sy(), d.sz());
      r[p] = v;
      acc += fabs(v);
    }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// Hackbusch-Reusken damping of the coarse correction (mgcsd.cc:431-439):
// w = (x . w0) / (x . A x), A with cc (Vmatvec), over the coarse interior.
template <int KIND>
__global__ void __launch_bounds__(kReduceThreads)
    apbs_damp_kernel(Dims d, Op14<double> A, const double *__restrict__ cc,
                     const double *__restrict__ x,
                     const double *__restrict__ w0, ReduceSlot s,
                     double *__restrict__ w) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  double up = 0.0, lo = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1)
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      up += x[p] * w0[p];
      lo += x[p] * apply_op<KIND>(A, cc, x, p, d.sy(), d.sz());
    }
  double v[2] = {block_sum_2d(up, sh), block_sum_2d(lo, sh)};
  reduce_finish<2>(v, s, w);
}

// ---------------------------------------------------------------------------
// Banded direct solve of a coarsest level (APBS mgsolv 1): Vbuildband
// (pmgc/buildBd.cc:63-303) stores the interior operator in LINPACK upper
// band storage, abd(kk, jj) = A(ii, jj) with kk = ii - jj + m + 1 (lda = m + 1
// rows per column, unknowns x fastest); Vdpbfa / Vdpbsl
// (pmgc/mlinpckd.cc:168-240) factor it as R^T R and solve. The factorisation
// and the two triangular solves are recurrences along the unknowns; they run
// in one thread in LINPACK's order (dot products unrolled by five, Vddot
// :113-165), bit for bit the reference's arithmetic.
// ---------------------------------------------------------------------------

// One column of the band per interior point; cc is not part of it, as in
// the reference (Vbuildband takes ac only). Only couplings with interior
// neighbours are stored: the reference also writes the offsets of shell
// neighbours, which on grids with one interior point along x alias the
// diagonal or pass the end of the column (buildBd.cc:150-247). For
// 27-point operators the coupling with each earlier neighbour q is read
// where the matvec reads it (at q); the reference reads those ten at the
// point below or south of p, which is not the operator its matvec applies.
template <int KIND>
__global__ void band_kernel(Dims d, Op14<double> A, double *__restrict__ abd,
                            int m, int lda) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int i = t.i, j = t.j, k = t.k;
  const int mx = d.nx - 2, my = d.ny - 2;
  const int jj = (k - 2) * mx * my + (j - 2) * mx + (i - 2) + 1;
  double *col = abd + (size_t)(jj - 1) * lda + m; // col[off] = A(jj+off, jj)
  const double *const *a = A.a;
  // the coupling with the earlier neighbour (di, dj, dk), stored at offset
  // di + dj mx + dk mx my, which lies in [-m, -1] for interior neighbours;
  // shell neighbours are skipped
  auto put = [&](int arr, int di, int dj, int dk) {
    const int ii = i + di, jn = j + dj, kn = k + dk;
    if (ii < 2 || ii > d.nx - 1 || jn < 2 || jn > d.ny - 1 || kn < 2 ||
        kn > d.nz - 1)
      return;
    col[di + dj * mx + dk * mx * my] = -a[arr][d.at(ii, jn, kn)];
  };
  col[0] = a[kOC][d.at(i, j, k)];
  put(kOE, -1, 0, 0);
  put(kON, 0, -1, 0);
  if (KIND == 7) {
    put(kUC, 0, 0, -1);
    return;
  }
  put(kONW, 1, -1, 0);
  put(kONE, -1, -1, 0);
  put(kUC, 0, 0, -1);
  put(kUW, 1, 0, -1);
  put(kUE, -1, 0, -1);
  put(kUS, 0, 1, -1);
  put(kUN, 0, -1, -1);
  put(kUSW, 1, 1, -1);
  put(kUSE, -1, 1, -1);
  put(kUNW, 1, -1, -1);
  put(kUNE, -1, -1, -1);
}

// LINPACK's unit-stride dot product: the first n % 5 terms one by one, then
// five-term groups summed left to right and added (Vddot).
__device__ double ddot5(int n, const double *x, const double *y) {
  double t = 0.0;
  if (n <= 0)
    return 0.0;
  const int r = n % 5;
  for (int q = 0; q < r; ++q)
    t += x[q] * y[q];
  if (n < 5)
    return t;
  for (int q = r; q < n; q += 5)
    t += x[q] * y[q] + x[q + 1] * y[q + 1] + x[q + 2] * y[q + 2] +
         x[q + 3] * y[q + 3] + x[q + 4] * y[q + 4];
  return t;
}

#define ABD(r, c) abd[(size_t)((c) - 1) * lda + ((r) - 1)]

// Vdpbfa in one thread; *info = 0 or the first column with a pivot <= 0
__global__ void dpbfa_kernel(double *abd, int lda, int n, int m, int *info) {
  *info = 0;
  for (int j = 1; j <= n; ++j) {
    double s = 0.0;
    int ik = m + 1;
    int jk = max(j - m, 1);
    const int mu = max(m + 2 - j, 1);
    for (int k = mu; k <= m; ++k) {
      double t = ABD(k, j) - ddot5(k - mu, &ABD(ik, jk), &ABD(mu, j));
      t /= ABD(m + 1, jk);
      ABD(k, j) = t;
      s += t * t;
      --ik;
      ++jk;
    }
    s = ABD(m + 1, j) - s;
    if (s <= 0.0) {
      *info = j;
      return;
    }
    ABD(m + 1, j) = sqrt(s);
  }
}

// Vdpbsl in one thread: R^T y = b, then R x = y, in place
__global__ void dpbsl_kernel(const double *abd, int lda, int n, int m,
                             double *b) {
  for (int k = 1; k <= n; ++k) {
    const int lm = min(k - 1, m), la = m + 1 - lm, lb = k - lm;
    const double t = ddot5(lm, &ABD(la, k), &b[lb - 1]);
    b[k - 1] = (b[k - 1] - t) / ABD(m + 1, k);
  }
  for (int kb = 1; kb <= n; ++kb) {
    const int k = n + 1 - kb;
    const int lm = min(k - 1, m), la = m + 1 - lm, lb = k - lm;
    b[k - 1] /= ABD(m + 1, k);
    const double t = -b[k - 1];
    if (lm > 0 && t != 0.0) // Vdaxpy returns early for a zero factor
      for (int q = 0; q < lm; ++q)
        b[lb - 1 + q] += t * ABD(la + q, k);
  }
}
#undef ABD

// interior of x <-> compact vector of the interior unknowns (Vxcopy_small
// with to_compact, Vxcopy_large without; pmgc/mikpckd.cc:78-113)
__global__ void compact_kernel(Dims d, double *__restrict__ x,
                               double *__restrict__ b, int to_compact) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const long q = ((long)(t.k - 2) * (d.ny - 2) + (t.j - 2)) * (d.nx - 2) +
                 (t.i - 2);
  const int p = d.at(t.i, t.j, t.k);
  if (to_compact)
    b[q] = x[p];
  else
    x[p] = b[q];
}

// band sizes of a grid's interior operator (Vbuildband, buildBd.cc:262-280)
void band_dims(const Dims &d, int kind, int *n, int *m, int *lda) {
  const int mx = d.nx - 2, my = d.ny - 2;
  *n = mx * my * (d.nz - 2);
  *m = kind == 7 ? mx * my : mx * my + mx + 1;
  *lda = *m + 1;
}

// zeroes abd, stores the band and factors it; *info read back (synchronises)
int band_factor(const Dims &d, int kind, const Op14<double> &A, double *abd,
                int *info, cudaStream_t s) {
  int n, m, lda;
  band_dims(d, kind, &n, &m, &lda);
  PMG_CUDA_TRY(cudaMemsetAsync(abd, 0, sizeof(double) * lda * n, s));
  if (kind == 7)
    band_kernel<7><<<interior_grid(d), interior_block(), 0, s>>>(d, A, abd, m,
                                                                lda);
  else
    band_kernel<27><<<interior_grid(d), interior_block(), 0, s>>>(d, A, abd,
                                                                 m, lda);
  int *dinfo = nullptr;
  PMG_CUDA_TRY(scratch_alloc((void **)&dinfo, sizeof(int), s));
  dpbfa_kernel<<<1, 1, 0, s>>>(abd, lda, n, m, dinfo);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, s);
  scratch_free(dinfo, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_last_error(e, "Vbuildband", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  return PMG_OK;
}

// Injection of a coefficient map to the next coarser grid (Vbuildcopy0,
// pmgc/mgsubd.cc:578-697): out(a, b, c) = in(2a-1, 2b-1, 2c-1) over the
// whole coarse array, shell included; with keep_c the third index is a
// layer (the two sides of a boundary map) and is not coarsened. Mesh lines
// are (n, 1, 1) arrays.
__global__ void inject_kernel(const double *__restrict__ in,
                              double *__restrict__ out, int na, int nb,
                              int nc, int naf, int nbf, int keep_c) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.z;
  if (a >= na || b >= nb || c >= nc)
    return;
  const int cf = keep_c ? c : 2 * c;
  out[((long)c * nb + b) * na + a] = in[((long)cf * nbf + 2 * b) * naf + 2 * a];
}

// the eleven inputs of the box-method builder, in BoxMaps order
enum { kMx, kMy, kMz, kGx, kGy, kGz, kA1, kA2, kA3, kCcf, kFcf, kMaps };

struct ApbsLevel {
  Dims d;
  int kind;     // 7 (box method: finest, or every level with mgcoar 0) or 27
  int ipc[12];  // ipc[10] = kind, for the packed-operator entry points
  double *ac;   // 4 or 14 columns of d.count()
  double *cc, *fc, *x, *w0;
  double *P[27]; // prolongation from this level to the next finer one
  const double *m[kMaps]; // coefficient maps (mgcoar 0)
  const double *a(int s) const { return ac + (size_t)s * d.count(); }
  double *aw(int s) { return ac + (size_t)s * d.count(); }
};

#define APBS_P27(P)                                                            \
  P[0], P[1], P[2], P[3], P[4], P[5], P[6], P[7], P[8], P[9], P[10], P[11],    \
      P[12], P[13], P[14], P[15], P[16], P[17], P[18], P[19], P[20], P[21],    \
      P[22], P[23], P[24], P[25], P[26]
#define APBS_A14(L)                                                            \
  (L).a(0), (L).a(1), (L).a(2), (L).a(3), (L).a(4), (L).a(5), (L).a(6),        \
      (L).a(7), (L).a(8), (L).a(9), (L).a(10), (L).a(11), (L).a(12), (L).a(13)

Op14<double> level_op(const ApbsLevel &L) {
  Op14<double> A{};
  for (int s = 0; s < (L.kind == 7 ? 4 : 14); ++s)
    A.a[s] = L.a(s);
  return A;
}

// Largest level count with exact coarsening and more than two points per
// axis on every level (Vmaxlev, mgsubd.cc:456-484).
int apbs_maxlev(int n1, int n2, int n3) {
  int lev = 0;
  for (;;) {
    ++lev;
    const int iden = 1 << (lev - 1);
    const int c[3] = {(n1 - 1) / iden + 1, (n2 - 1) / iden + 1,
                      (n3 - 1) / iden + 1};
    const int n[3] = {n1, n2, n3};
    bool done = false;
    for (int a = 0; a < 3; ++a)
      done |= (c[a] - 1) * iden != n[a] - 1 || c[a] <= 2;
    if (done || lev > 30)
      return lev - 1;
  }
}

struct ApbsDriver {
  cudaStream_t s;
  int nlev, mgsmoo, mgsolv = 0;
  double epsiln = 0.0; // stop of the coarsest CG (mgcsd.cc:362-378)
  double *band = nullptr; // factored band of the coarsest level (mgsolv 1)
  int bn = 0, bm = 0, blda = 0;
  ApbsLevel lv[13];
  double *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
  void *block = nullptr; // every level array and work vector
  double *partials = nullptr, *res = nullptr;
  unsigned *ticket = nullptr;
  dim3 rg0;

  explicit ApbsDriver(cudaStream_t st) : s(st) {}
  ~ApbsDriver() {
    if (block)
      scratch_free(block, s);
  }

  ReduceSlot slot(double *out) const {
    return ReduceSlot{partials, ticket, out};
  }

  int fetch(const double *dev, double *host) {
    PMG_CUDA_TRY(cudaMemcpyAsync(host, dev, sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
    PMG_CUDA_TRY(cudaStreamSynchronize(s));
    return PMG_OK;
  }

  int faces(const ApbsLevel &L, double *x, const double *gx,
            const double *gy, const double *gz) {
    const Dims &d = L.d;
    const dim3 b(32, 8);
    apbs_face_kernel<<<dim3(cdiv(d.ny, 32), cdiv(d.nz, 8)), b, 0, s>>>(
        d, x, gx, 0);
    apbs_face_kernel<<<dim3(cdiv(d.nx, 32), cdiv(d.nz, 8)), b, 0, s>>>(
        d, x, gy, 1);
    apbs_face_kernel<<<dim3(cdiv(d.nx, 32), cdiv(d.ny, 8)), b, 0, s>>>(
        d, x, gz, 2);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  }

  int sum(const ApbsLevel &L, double *a, const double *b, int mode,
          double *host) {
    apbs_sum_kernel<<<reduce_grid(L.d), interior_block(), 0, s>>>(
        L.d, a, b, mode, slot(res));
    PMG_LAUNCH_CHECK();
    return fetch(res, host);
  }

  // Vsmooth (smoothd.cc:58-87): red-black GS (then the residual into w1
  // when iresid) or the CG with errtol 0 (its residual is w1).
  int smooth(ApbsLevel &L, const double *f, double *x, int nu, int iadjoint,
             int iresid) {
    const Dims &d = L.d;
    int rc = PMG_OK;
    if (mgsmoo == 4) {
      int it = 0;
      return pmg_Vcghs_d(d.nx, d.ny, d.nz, L.ipc, L.ac, L.cc, f, x, w2, w3,
                         w1, nu, &it, 0.0, iresid, s);
    }
    if (L.kind == 7)
      rc = pmg_Vgsrb7x_d(d.nx, d.ny, d.nz, L.a(0), L.cc, f, L.a(1), L.a(2),
                         L.a(3), x, nu, iadjoint, 0, s);
    else
      rc = pmg_Vgsrb27x_d(d.nx, d.ny, d.nz, L.a(0), L.cc, f, L.a(1), L.a(2),
                          L.a(3), L.a(4), L.a(5), L.a(6), L.a(7), L.a(8),
                          L.a(9), L.a(10), L.a(11), L.a(12), L.a(13), x, nu,
                          0, iadjoint, s);
    if (rc != PMG_OK || !iresid)
      return rc;
    if (L.kind == 7)
      return pmg_Vmresid7_1s_d(d.nx, d.ny, d.nz, L.a(0), L.cc, f, L.a(1),
                               L.a(2), L.a(3), x, w1, s);
    return pmg_Vmresid27_1s_d(d.nx, d.ny, d.nz, L.a(0), L.cc, f, L.a(1),
                              L.a(2), L.a(3), L.a(4), L.a(5), L.a(6), L.a(7),
                              L.a(8), L.a(9), L.a(10), L.a(11), L.a(12),
                              L.a(13), x, w1, s);
  }

  // the coarsest level's solve: mgsolv 0, 100 CG iterations from zero with
  // errtol epsiln = 0 (mgcsd.cc:362-378); mgsolv 1, the banded direct solve
  // of the interior, boundary zero (:380-405)
  int coarse(ApbsLevel &C, const double *f) {
    if (mgsolv == 1) {
      compact_kernel<<<interior_grid(C.d), interior_block(), 0, s>>>(
          C.d, const_cast<double *>(f), w1, 1);
      dpbsl_kernel<<<1, 1, 0, s>>>(band, blda, bn, bm, w1);
      compact_kernel<<<interior_grid(C.d), interior_block(), 0, s>>>(
          C.d, C.x, w1, 0);
      PMG_LAUNCH_CHECK();
      return faces(C, C.x, nullptr, nullptr, nullptr);
    }
    PMG_CUDA_TRY(cudaMemsetAsync(C.x, 0, sizeof(double) * C.d.count(), s));
    int it = 0;
    return pmg_Vcghs_d(C.d.nx, C.d.ny, C.d.nz, C.ipc, C.ac, C.cc, f, C.x, w1,
                       w2, w3, 100, &it, epsiln, 0, s);
  }

  // the stop test's numerator after a cycle (mgcsd.cc:467-519)
  int stop_norm(int istop, double *tru, double *out) {
    ApbsLevel &F = lv[1];
    if (istop == 0 || istop == 1) {
      apbs_resid_l1_kernel<7><<<reduce_grid(F.d), interior_block(), 0, s>>>(
          F.d, level_op(F), F.cc, F.fc, F.x, w1, slot(res));
      PMG_LAUNCH_CHECK();
      return fetch(res, out);
    }
    const int rc = sum(F, tru, F.x, istop == 2 ? 2 : 3, out);
    if (rc == PMG_OK && istop == 3)
      *out = sqrt(*out);
    return rc;
  }

  // Vmvcs (pmgc/mgcsd.cc:61-531) from the finest iterate lv[1].x: the stop
  // test's denominator, then V-cycles until itmax or the stop ratio is at
  // most errtol (one cycle-free coarse solve when nlev is 1). Returns the
  // cycles run and the final ratio.
  int mvcs(int istop, int itmax, double errtol, int nu1, int nu2,
           double *tcf, int *iters, double *ratio) {
    ApbsLevel &F1 = lv[1];
    const Dims &df = F1.d;
    double rsden = 1.0;
    int rc = PMG_OK;
    if (istop == 1) {
      rc = sum(F1, F1.fc, nullptr, 0, &rsden);
    } else if (istop == 2) {
      rsden = sqrt((double)df.nx * df.ny * df.nz);
    } else if (istop == 3) {
      rc = sum(F1, tcf, tcf, 1, &rsden);
      rsden = sqrt(rsden);
    }
    if (rc != PMG_OK)
      return rc;
    if (rsden == 0.0)
      rsden = 1.0;
    int it = 0;
    double rn = 0.0;
    if (nlev == 1) {
      rc = coarse(F1, F1.fc);
      it = 1;
      if (rc == PMG_OK)
        rc = stop_norm(istop, tcf, &rn);
    } else {
      do {
        rc = smooth(F1, F1.fc, F1.x, nu1, 0, 1);
        // the finest residual is kept in the finest w0 (mgcsd.cc:324)
        if (rc == PMG_OK)
          PMG_CUDA_TRY(cudaMemcpyAsync(F1.w0, w1,
                                       sizeof(double) * df.count(),
                                       cudaMemcpyDeviceToDevice, s));
        for (int L = 2; L <= nlev && rc == PMG_OK; ++L) {
          ApbsLevel &F = lv[L - 1], &C = lv[L];
          rc = pmg_Vrestrc2_d(F.d.nx, F.d.ny, F.d.nz, C.d.nx, C.d.ny, C.d.nz,
                              w1, C.w0, APBS_P27(C.P), s);
          if (rc == PMG_OK && L != nlev) {
            PMG_CUDA_TRY(
                cudaMemsetAsync(C.x, 0, sizeof(double) * C.d.count(), s));
            rc = smooth(C, C.w0, C.x, nu1, 0, 1);
          }
        }
        if (rc == PMG_OK)
          rc = coarse(lv[nlev], lv[nlev].w0);
        for (int L = nlev - 1; L >= 1 && rc == PMG_OK; --L) {
          ApbsLevel &F = lv[L], &C = lv[L + 1];
          if (C.kind == 7)
            apbs_damp_kernel<7><<<reduce_grid(C.d), interior_block(), 0, s>>>(
                C.d, level_op(C), C.cc, C.x, C.w0, slot(res), res + 3);
          else
            apbs_damp_kernel<27>
                <<<reduce_grid(C.d), interior_block(), 0, s>>>(
                    C.d, level_op(C), C.cc, C.x, C.w0, slot(res), res + 3);
          P27<double> P;
          for (int q = 0; q < 27; ++q)
            P.p[q] = C.P[q];
          interp_add_kernel<double, false>
              <<<interp_grid(C.d), interior_block(), 0, s>>>(C.d, F.d, C.x, P,
                                                             F.x, res + 3);
          PMG_LAUNCH_CHECK();
          rc = smooth(F, L == 1 ? F.fc : F.w0, F.x, nu2, 1, 0);
        }
        ++it;
        if (rc == PMG_OK)
          rc = stop_norm(istop, tcf, &rn);
      } while (rc == PMG_OK && it < itmax && rn / rsden > errtol);
    }
    *iters = it;
    *ratio = rn / rsden;
    return rc;
  }
};

} // namespace
} // namespace pmg

using namespace pmg;

extern "C" {

int pmg_Vmatvec_d(int nx, int ny, int nz, const int *ipc, const double *ac,
                  const double *cc, const double *x, double *y,
                  pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmatvec: grid size out of range");
  PMG_REQUIRE(x && y, "Vmatvec: null array");
  const Dims d{nx, ny, nz};
  int kind = 0;
  Op14<double> A;
  const int rc = unpack(ipc, ac, d.count(), &kind, &A);
  if (rc != PMG_OK)
    return rc;
  const cudaStream_t s = (cudaStream_t)stream;
  if (kind == 7)
    matvec_kernel<7, double><<<interior_grid(d), interior_block(), 0, s>>>(
        d, A, cc, x, y);
  else
    matvec_kernel<27, double><<<interior_grid(d), interior_block(), 0, s>>>(
        d, A, cc, x, y);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

int pmg_Vmresid_d(int nx, int ny, int nz, const int *ipc, const double *ac,
                  const double *cc, const double *fc, const double *x,
                  double *r, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmresid: grid size out of range");
  PMG_REQUIRE(fc && x && r, "Vmresid: null array");
  const Dims d{nx, ny, nz};
  int kind = 0;
  Op14<double> A;
  const int rc = unpack(ipc, ac, d.count(), &kind, &A);
  if (rc != PMG_OK)
    return rc;
  const cudaStream_t s = (cudaStream_t)stream;
  if (kind == 7)
    mresid_kernel<7, double><<<interior_grid(d), interior_block(), 0, s>>>(
        d, A, cc, fc, x, r);
  else
    mresid_kernel<27, double><<<interior_grid(d), interior_block(), 0, s>>>(
        d, A, cc, fc, x, r);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

int pmg_Vcghs_d(int nx, int ny, int nz, const int *ipc, const double *ac,
                const double *cc, const double *fc, double *x, double *p,
                double *ap, double *r, int itmax, int *iters, double errtol,
                int iresid, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vcghs: grid size out of range");
  PMG_REQUIRE(fc && x && p && ap && r && iters, "Vcghs: null array");
  const Dims d{nx, ny, nz};
  int kind = 0;
  Op14<double> A;
  const int rc = unpack(ipc, ac, d.count(), &kind, &A);
  if (rc != PMG_OK)
    return rc;
  const cudaStream_t s = (cudaStream_t)stream;
  return kind == 7 ? cghs<7>(d, A, cc, fc, x, p, ap, r, itmax, iters, errtol,
                             iresid, s)
                   : cghs<27>(d, A, cc, fc, x, p, ap, r, itmax, iters, errtol,
                              iresid, s);
}

int pmg_Vbuildband_d(int *key, int nx, int ny, int nz, const int *ipc,
                     const double *ac, int *ipcB, double *acB,
                     pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vbuildband: grid size out of range");
  PMG_REQUIRE(key && ipcB && acB, "Vbuildband: null key, ipcB or acB");
  const Dims d{nx, ny, nz};
  int kind = 0;
  Op14<double> A;
  int rc = unpack(ipc, ac, d.count(), &kind, &A);
  if (rc != PMG_OK)
    return rc;
  int n, m, lda, info = 0;
  band_dims(d, kind, &n, &m, &lda);
  rc = band_factor(d, kind, A, acB, &info, (cudaStream_t)stream);
  if (rc != PMG_OK)
    return rc;
  ipcB[0] = n;
  ipcB[1] = m;
  ipcB[2] = lda;
  ipcB[3] = 1; // factored
  *key = info != 0;
  return PMG_OK;
}

int pmg_Vdpbfa_d(double *abd, int lda, int n, int m, int *info,
                 pmg_stream_t stream) {
  PMG_REQUIRE(abd && info, "Vdpbfa: null abd or info");
  PMG_REQUIRE(n >= 0 && m >= 0 && lda >= m + 1, "Vdpbfa: bad n, m or lda");
  const cudaStream_t s = (cudaStream_t)stream;
  int *dinfo = nullptr;
  PMG_CUDA_TRY(scratch_alloc((void **)&dinfo, sizeof(int), s));
  dpbfa_kernel<<<1, 1, 0, s>>>(abd, lda, n, m, dinfo);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, s);
  scratch_free(dinfo, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_last_error(e, "Vdpbfa", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  return PMG_OK;
}

int pmg_Vdpbsl_d(const double *abd, int lda, int n, int m, double *b,
                 pmg_stream_t stream) {
  PMG_REQUIRE(abd && b, "Vdpbsl: null abd or b");
  PMG_REQUIRE(n >= 0 && m >= 0 && lda >= m + 1, "Vdpbsl: bad n, m or lda");
  dpbsl_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(abd, lda, n, m, b);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

int pmg_Vmgdriv_d(const int *iparm, const double *rparm, double *u,
                  const double *xf, const double *yf, const double *zf,
                  const double *gxcf, const double *gycf, const double *gzcf,
                  const double *a1cf, const double *a2cf, const double *a3cf,
                  const double *ccf, const double *fcf, double *tcf,
                  int *iters, int *ierror, double *rsnrm, pmg_stream_t stream) {
  PMG_REQUIRE(iparm && rparm && u, "Vmgdriv: null iparm, rparm or u");
  const int nx = iparm[2], ny = iparm[3], nz = iparm[4], nlev = iparm[5];
  const int nu1 = iparm[6], nu2 = iparm[7], mgkey = iparm[8];
  const int itmax = iparm[9], istop = iparm[10], ipkey = iparm[13];
  const int mode = iparm[15], mgprol = iparm[16], mgcoar = iparm[17];
  const int mgdisc = iparm[18], mgsmoo = iparm[19], mgsolv = iparm[20];
  const int iperf = iparm[21];
  const double errtol = rparm[0];
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmgdriv: grid size out of range");
  PMG_REQUIRE(nlev >= 1 && nlev <= 12 && nlev <= apbs_maxlev(nx, ny, nz),
              "Vmgdriv: nlev does not coarsen the grid exactly");
  PMG_REQUIRE(mode == 0, "Vmgdriv: only the linear mode (iparm mode 0)");
  PMG_REQUIRE(mgkey == 0 || mgkey == 1, "Vmgdriv: mgkey must be 0 or 1");
  PMG_REQUIRE(mgdisc == 0, "Vmgdriv: only the box method (mgdisc 0)");
  PMG_REQUIRE(mgcoar == 0 || mgcoar == 2,
              "Vmgdriv: mgcoar must be 0 (coefficient injection) or 2 "
              "(Galerkin)");
  PMG_REQUIRE(mgprol == 0 || mgprol == 1, "Vmgdriv: mgprol must be 0 or 1");
  PMG_REQUIRE(mgsmoo == 1 || mgsmoo == 4,
              "Vmgdriv: mgsmoo must be 1 (red-black GS) or 4 (CG)");
  PMG_REQUIRE(mgsolv == 0 || mgsolv == 1,
              "Vmgdriv: mgsolv must be 0 (CG) or 1 (banded direct)");
  PMG_REQUIRE(iperf == 0, "Vmgdriv: no eigenvalue analysis (iperf 0)");
  PMG_REQUIRE(istop >= 0 && istop <= 3, "Vmgdriv: istop must be 0 to 3");
  PMG_REQUIRE(istop < 2 || tcf, "Vmgdriv: istop 2 and 3 need tcf");
  PMG_REQUIRE(nu1 >= 0 && nu2 >= 0, "Vmgdriv: negative nu1 or nu2");
  PMG_REQUIRE(xf && yf && zf && gxcf && gycf && gzcf && a1cf && a2cf &&
                  a3cf && ccf && fcf,
              "Vmgdriv: null input array");

  ApbsDriver D((cudaStream_t)stream);
  const cudaStream_t s = D.s;
  D.nlev = nlev;
  D.mgsmoo = mgsmoo;
  D.mgsolv = mgsolv;
  // sizes and one block for everything
  size_t total = 0;
  for (int L = 1; L <= nlev; ++L) {
    ApbsLevel &v = D.lv[L];
    v.d = L == 1 ? Dims{nx, ny, nz}
                 : Dims{(D.lv[L - 1].d.nx - 1) / 2 + 1,
                        (D.lv[L - 1].d.ny - 1) / 2 + 1,
                        (D.lv[L - 1].d.nz - 1) / 2 + 1};
    v.kind = L == 1 || mgcoar == 0 ? 7 : 27;
    for (int q = 0; q < 12; ++q)
      v.ipc[q] = 0;
    v.ipc[10] = v.kind;
    const size_t n = (size_t)v.d.count();
    total += n * ((v.kind == 7 ? 4 : 14) + 3 + (L > 1 ? 1 + 27 : 0));
    if (mgcoar == 0 && L > 1) // coarse maps: 5 grids, lines, boundary maps
      total += 5 * n + v.d.nx + v.d.ny + v.d.nz +
               2 * ((size_t)v.d.ny * v.d.nz + (size_t)v.d.nx * v.d.nz +
                    (size_t)v.d.nx * v.d.ny);
  }
  const size_t nf = (size_t)D.lv[1].d.count();
  D.rg0 = reduce_grid(D.lv[1].d);
  const size_t nblk = (size_t)D.rg0.x * D.rg0.y * D.rg0.z;
  total += 3 * nf + 2 * nblk + 4;
  if (mgsolv == 1) {
    band_dims(D.lv[nlev].d, D.lv[nlev].kind, &D.bn, &D.bm, &D.blda);
    total += (size_t)D.blda * D.bn;
  }
  PMG_CUDA_TRY(scratch_alloc(&D.block, total * sizeof(double) + 64, s));
  PMG_CUDA_TRY(
      cudaMemsetAsync(D.block, 0, total * sizeof(double) + 64, s));
  double *cur = (double *)D.block;
  auto take = [&](size_t n) {
    double *p = cur;
    cur += n;
    return p;
  };
  for (int L = 1; L <= nlev; ++L) {
    ApbsLevel &v = D.lv[L];
    const size_t n = (size_t)v.d.count();
    v.ac = take(n * (v.kind == 7 ? 4 : 14));
    v.cc = take(n);
    v.fc = take(n);
    v.w0 = take(n);
    v.x = L == 1 ? u : take(n);
    for (int q = 0; q < 27; ++q)
      v.P[q] = L > 1 ? take(n) : nullptr;
    if (L == 1) {
      const double *in[kMaps] = {xf,   yf,   zf,   gxcf, gycf, gzcf,
                                 a1cf, a2cf, a3cf, ccf,  fcf};
      for (int q = 0; q < kMaps; ++q)
        v.m[q] = in[q];
    } else if (mgcoar == 0) {
      const Dims &c = v.d;
      const size_t sz[kMaps] = {(size_t)c.nx, (size_t)c.ny, (size_t)c.nz,
                                2 * (size_t)c.ny * c.nz,
                                2 * (size_t)c.nx * c.nz,
                                2 * (size_t)c.nx * c.ny, n, n, n, n, n};
      for (int q = 0; q < kMaps; ++q)
        v.m[q] = take(sz[q]);
    }
  }
  D.w1 = take(nf);
  D.w2 = take(nf);
  D.w3 = take(nf);
  D.partials = take(2 * nblk);
  D.res = take(4);
  if (mgsolv == 1)
    D.band = take((size_t)D.blda * D.bn);
  D.ticket = (unsigned *)cur; // zeroed with the block

  // Vbuildops: the box-method fine operator, then P and the Galerkin
  // operator per level; the coarse cc and fc are the restricted fine ones
  ApbsLevel &F1 = D.lv[1];
  int rc = pmg_VbuildA_fv_d(nx, ny, nz, ipkey, nullptr, nullptr, F1.aw(0),
                            F1.cc, F1.fc, F1.aw(1), F1.aw(2), F1.aw(3), xf, yf,
                            zf, gxcf, gycf, gzcf, a1cf, a2cf, a3cf, ccf, fcf,
                            stream);
  for (int L = 2; L <= nlev && rc == PMG_OK; ++L) {
    ApbsLevel &F = D.lv[L - 1], &C = D.lv[L];
    const Dims &df = F.d, &dc = C.d;
    if (mgprol == 0)
      rc = pmg_VbuildPb_trilin_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz,
                                 APBS_P27(C.P), stream);
    else if (F.kind == 7)
      rc = pmg_VbuildPb_op7_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz,
                              F.a(0), F.a(1), F.a(2), F.a(3), APBS_P27(C.P),
                              stream);
    else
      rc = pmg_VbuildPb_op27_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz,
                               APBS_A14(F), APBS_P27(C.P), stream);
    if (rc != PMG_OK)
      break;
    const double *pc[27];
    double *out[14];
    for (int q = 0; q < 27; ++q)
      pc[q] = C.P[q];
    for (int q = 0; q < 14; ++q)
      out[q] = C.aw(q);
    if (mgcoar == 0) {
      // Vbuildcopy0: the maps injected, then the box method on this grid
      // (mgsubd.cc:141-166); the restricted cc and fc of Galerkin levels do
      // not apply
      const dim3 b(32, 8);
      auto inject = [&](int q, int na, int nb, int nc, int naf, int nbf,
                        int keep) {
        inject_kernel<<<dim3(cdiv(na, 32), cdiv(nb, 8), nc), b, 0, s>>>(
            F.m[q], const_cast<double *>(C.m[q]), na, nb, nc, naf, nbf,
            keep);
      };
      inject(kMx, dc.nx, 1, 1, df.nx, 1, 1);
      inject(kMy, dc.ny, 1, 1, df.ny, 1, 1);
      inject(kMz, dc.nz, 1, 1, df.nz, 1, 1);
      inject(kGx, dc.ny, dc.nz, 2, df.ny, df.nz, 1);
      inject(kGy, dc.nx, dc.nz, 2, df.nx, df.nz, 1);
      inject(kGz, dc.nx, dc.ny, 2, df.nx, df.ny, 1);
      for (int q = kA1; q <= kFcf; ++q)
        inject(q, dc.nx, dc.ny, dc.nz, df.nx, df.ny, 0);
      PMG_LAUNCH_CHECK();
      rc = pmg_VbuildA_fv_d(dc.nx, dc.ny, dc.nz, ipkey, nullptr, nullptr,
                            C.aw(0), C.cc, C.fc, C.aw(1), C.aw(2), C.aw(3),
                            C.m[kMx], C.m[kMy], C.m[kMz], C.m[kGx], C.m[kGy],
                            C.m[kGz], C.m[kA1], C.m[kA2], C.m[kA3], C.m[kCcf],
                            C.m[kFcf], stream);
      continue;
    }
    if (F.kind == 7) {
      rc = pmg_VbuildG_7_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz, pc,
                           F.a(0), F.a(1), F.a(2), F.a(3), out, stream);
    } else {
      const double *a14[14];
      for (int q = 0; q < 14; ++q)
        a14[q] = F.a(q);
      rc = pmg_VbuildG_27_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz, pc, a14,
                            out, stream);
    }
    if (rc == PMG_OK)
      rc = pmg_Vrestrc2_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz, F.cc,
                          C.cc, APBS_P27(C.P), stream);
    if (rc == PMG_OK)
      rc = pmg_Vrestrc2_d(df.nx, df.ny, df.nz, dc.nx, dc.ny, dc.nz, F.fc,
                          C.fc, APBS_P27(C.P), stream);
  }
  if (rc == PMG_OK && mgsolv == 1) {
    // Vbuildband on the coarsest level, factored (mgsubd.cc:245-262)
    int info = 0;
    ApbsLevel &C = D.lv[nlev];
    rc = band_factor(C.d, C.kind, level_op(C), D.band, &info, s);
    PMG_REQUIRE(rc != PMG_OK || info == 0,
                "Vmgdriv: the coarsest operator is not positive definite");
  }
  if (rc != PMG_OK)
    return rc;

  // u starts from zero (mgdrvd.cc:419), then Vmvcs
  PMG_CUDA_TRY(cudaMemsetAsync(u, 0, sizeof(double) * nf, s));
  rc = D.faces(F1, u, nullptr, nullptr, nullptr);
  if (rc != PMG_OK)
    return rc;
  int it = 0;
  double ratio = 0.0;
  rc = D.mvcs(istop, itmax, errtol, nu1, nu2, tcf, &it, &ratio);
  if (rc != PMG_OK)
    return rc;
  rc = D.faces(F1, u, gxcf, gycf, gzcf);
  if (rc != PMG_OK)
    return rc;
  PMG_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters)
    *iters = it;
  if (ierror)
    *ierror = it < itmax ? 0 : 1;
  if (rsnrm)
    *rsnrm = ratio;
  return PMG_OK;
}

int pmg_Vmvcs_d(int nx, int ny, int nz, double *x, const int *iz, double *w0,
                double *w1, double *w2, double *w3, int istop, int itmax,
                int *iters, int *ierror, int nlev, int ilev, int nlev_real,
                int mgsolv, int iok, int iinfo, double epsiln, double errtol,
                double omega, int nu1, int nu2, int mgsmoo, const int *ipc,
                const double *rpc, const double *pc, const double *ac,
                const double *cc, const double *fc, double *tru,
                pmg_stream_t stream) {
  (void)iok;   // the reference's loop always tests (mgcsd.cc:461)
  (void)iinfo; // i/o only
  (void)omega; // damping of the smoothers not offered (mgsmoo 0/2/3)
  (void)rpc;   // no real parameters for the box-method operators
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmvcs: grid size out of range");
  PMG_REQUIRE(iz && ipc, "Vmvcs: null iz or ipc (host arrays)");
  PMG_REQUIRE(x && w0 && w1 && w2 && w3 && ac && cc && fc,
              "Vmvcs: null device array");
  PMG_REQUIRE(nlev >= 1 && nlev <= 12 && ilev >= 1 &&
                  ilev - 1 + nlev + (mgsolv == 1 ? 1 : 0) <= nlev_real,
              "Vmvcs: levels ilev .. ilev+nlev-1 (and the band level for "
              "mgsolv 1) must lie within nlev_real");
  PMG_REQUIRE(nlev == 1 || pc, "Vmvcs: null pc");
  PMG_REQUIRE(mgsmoo == 1 || mgsmoo == 4,
              "Vmvcs: mgsmoo must be 1 (red-black GS) or 4 (CG)");
  PMG_REQUIRE(mgsolv == 0 || mgsolv == 1,
              "Vmvcs: mgsolv must be 0 (CG) or 1 (banded direct)");
  PMG_REQUIRE(istop >= 0 && istop <= 3, "Vmvcs: istop must be 0 to 3");
  PMG_REQUIRE(istop < 2 || tru, "Vmvcs: istop 2 and 3 need tru");
  PMG_REQUIRE(nu1 >= 0 && nu2 >= 0 && itmax >= 0,
              "Vmvcs: negative nu1, nu2 or itmax");
  // iz(field, lev), 1-based, 50 fields per level (Vbuildstr,
  // mgsubd.cc:266-345), as a 0-based offset
  auto IZ = [&](int field, int lev) {
    return (size_t)(iz[(size_t)(lev - 1) * 50 + (field - 1)] - 1);
  };
  ApbsDriver D((cudaStream_t)stream);
  D.nlev = nlev;
  D.mgsmoo = mgsmoo;
  D.mgsolv = mgsolv;
  D.epsiln = epsiln;
  for (int L = 1; L <= nlev; ++L) {
    const int lev = ilev - 1 + L;
    ApbsLevel &v = D.lv[L];
    v.d = L == 1 ? Dims{nx, ny, nz}
                 : Dims{(D.lv[L - 1].d.nx - 1) / 2 + 1,
                        (D.lv[L - 1].d.ny - 1) / 2 + 1,
                        (D.lv[L - 1].d.nz - 1) / 2 + 1};
    PMG_REQUIRE(!bad_dims(v.d.nx, v.d.ny, v.d.nz),
                "Vmvcs: a coarse grid is too small");
    const int *ip = ipc + IZ(5, lev);
    v.kind = ip[10];
    PMG_REQUIRE(v.kind == 7 || v.kind == 27,
                "Vmvcs: ipc(11) of a level must be 7 or 27");
    for (int q = 0; q < 12; ++q)
      v.ipc[q] = ip[q];
    const size_t n = (size_t)v.d.count();
    v.ac = const_cast<double *>(ac) + IZ(7, lev);
    v.cc = const_cast<double *>(cc) + IZ(1, lev);
    v.fc = const_cast<double *>(fc) + IZ(1, lev);
    v.x = x + IZ(1, lev);
    v.w0 = w0 + IZ(1, lev);
    for (int q = 0; q < 27; ++q)
      v.P[q] = L > 1 ? const_cast<double *>(pc) + IZ(11, lev - 1) + q * n
                     : nullptr;
  }
  if (mgsolv == 1) {
    // the factored band sits one level below the coarsest (lpv,
    // mgcsd.cc:380-392): n, m, lda in its ipc, the band in its ac
    const int lpv = ilev - 1 + nlev + 1;
    const int *ipb = ipc + IZ(5, lpv);
    D.bn = ipb[0];
    D.bm = ipb[1];
    D.blda = ipb[2];
    const Dims &c = D.lv[nlev].d;
    PMG_REQUIRE(D.bn == (c.nx - 2) * (c.ny - 2) * (c.nz - 2) && D.bm >= 0 &&
                    D.blda == D.bm + 1,
                "Vmvcs: band sizes in ipc do not fit the coarsest level");
    D.band = const_cast<double *>(ac) + IZ(7, lpv);
  }
  D.w1 = w1;
  D.w2 = w2;
  D.w3 = w3;
  // the reductions' partial sums, result slots and ticket
  cudaStream_t s = D.s;
  D.rg0 = reduce_grid(D.lv[1].d);
  const size_t nblk = (size_t)D.rg0.x * D.rg0.y * D.rg0.z;
  const size_t bytes = (2 * nblk + 4) * sizeof(double) + 64;
  PMG_CUDA_TRY(scratch_alloc(&D.block, bytes, s));
  PMG_CUDA_TRY(cudaMemsetAsync(D.block, 0, bytes, s));
  D.partials = (double *)D.block;
  D.res = D.partials + 2 * nblk;
  D.ticket = (unsigned *)(D.res + 4);
  int it = 0;
  double ratio = 0.0;
  int rc = D.mvcs(istop, itmax, errtol, nu1, nu2, tru, &it, &ratio);
  if (rc != PMG_OK)
    return rc;
  PMG_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters)
    *iters = it;
  if (ierror)
    *ierror = it < itmax ? 0 : 1;
  return PMG_OK;
}

} // extern "C"
