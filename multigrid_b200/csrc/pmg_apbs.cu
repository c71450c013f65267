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

} // extern "C"
