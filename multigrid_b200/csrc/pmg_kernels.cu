#include <map>
#include <mutex>
// Non-template kernels and the per-kernel C-ABI entry points (pmgc names).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "box_builder.cuh"
#include "build_kernels.cuh"
#include "gs27_tiled.cuh"
#include "launch.cuh"
#include "reduce_kernels.cuh"
#include "split_layout.cuh"
#include "cg_cluster.cuh"

namespace pmg {

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
static thread_local char g_last_error[512] = "no error";

void set_last_error(cudaError_t e, const char *what, const char *file,
                    int line) {
  snprintf(g_last_error, sizeof(g_last_error), "%s failed: %s (%s:%d)", what,
           cudaGetErrorString(e), file, line);
}
void set_last_message(const char *msg) {
  snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

namespace {
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[64] = {};
} // namespace

static cudaError_t scratch_pool(cudaMemPool_t *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return e;
  if (dev < 0 || dev >= 64)
    return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mutex);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess)
      return e;
    unsigned long long keep = ~0ull;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}

cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = nullptr;
  const cudaError_t e = scratch_pool(&pool);
  if (e != cudaSuccess)
    return e;
  return cudaMallocFromPoolAsync(ptr, bytes ? bytes : 1, pool, s);
}

cudaError_t scratch_free(void *ptr, cudaStream_t s) {
  return cudaFreeAsync(ptr, s);
}

// ---- tile edge of the 27-point smoother ------------------------------------
namespace {
std::mutex g_tile_mutex;
std::map<std::pair<long, int>, int> g_tiles; // (nx*ny*nz key, esize) -> edge
// 1: measured edges (default); 0: size rule; 8, 16, 32: that edge
int g_tile_mode = 1; // guarded by g_tile_mutex
long tile_key(const Dims &d) {
  return ((long)d.nx * 2048 + d.ny) * 2048 + d.nz;
}
} // namespace

int gs27_tile_for(const Dims &d, int esize) {
  {
    std::lock_guard<std::mutex> lk(g_tile_mutex);
    if (g_tile_mode != 1)
      return g_tile_mode ? g_tile_mode : gs27_tile_by_size(d);
    auto it = g_tiles.find({tile_key(d), esize});
    if (it != g_tiles.end())
      return it->second;
  }
  return gs27_tile_by_size(d);
}

// untuned: enough CTAs for small levels, fewer halo points for large ones
int gs27_tile_by_size(const Dims &d) {
  const int n = d.nx < d.ny ? d.nx : d.ny;
  return n >= 97 ? 32 : n >= 49 ? 16 : 8;
}

bool gs27_autotune_on() {
  std::lock_guard<std::mutex> lk(g_tile_mutex);
  return g_tile_mode == 1;
}

void gs27_tile_record(const Dims &d, int esize, int tile) {
  std::lock_guard<std::mutex> lk(g_tile_mutex);
  g_tiles[{tile_key(d), esize}] = tile;
}

bool gs27_tile_known(const Dims &d, int esize) {
  std::lock_guard<std::mutex> lk(g_tile_mutex);
  return g_tiles.count({tile_key(d), esize}) != 0;
}

template <typename T>
int gs27_tune(const Dims &d, const Op14<T> &A, const T *fc, T *x, T *alt,
              cudaStream_t s) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  PMG_CUDA_TRY(cudaEventCreate(&e0));
  cudaError_t e = cudaEventCreate(&e1);
  int best = 0;
  float best_ms = 0.f, size_ms = 0.f;
  for (int tile : kGs27Tiles) {
    if (e != cudaSuccess)
      break;
    float ms_min = 0.f;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
      T *res = nullptr;
      e = cudaEventRecord(e0, s);
      if (e == cudaSuccess &&
          launch_gs27_pp<T>(d, A, nullptr, fc, x, alt, 2, 0, 0, s, &res,
                            tile) != PMG_OK)
        e = cudaErrorUnknown;
      if (e == cudaSuccess)
        e = cudaEventRecord(e1, s);
      if (e == cudaSuccess)
        e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess)
        e = cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && (rep == 1 || ms < ms_min)) // first run warms up
        ms_min = ms;
    }
    if (e == cudaSuccess && (best == 0 || ms_min < best_ms)) {
      best = tile;
      best_ms = ms_min;
    }
    if (tile == gs27_tile_by_size(d))
      size_ms = ms_min;
  }
  // the size rule's edge stays unless another is clearly faster (timings
  // taken while other work shares the GPU are noisy)
  if (best != gs27_tile_by_size(d) && !(best_ms < 0.9f * size_ms))
    best = gs27_tile_by_size(d);
  cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
  if (e != cudaSuccess) {
    set_last_error(e, "gs27_tune", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  gs27_tile_record(d, (int)sizeof(T), best);
  return PMG_OK;
}

template int gs27_tune<float>(const Dims &, const Op14<float> &,
                              const float *, float *, float *, cudaStream_t);
template int gs27_tune<double>(const Dims &, const Op14<double> &,
                               const double *, double *, double *,
                               cudaStream_t);

// ---------------------------------------------------------------------------
// non-template kernels
// ---------------------------------------------------------------------------
__global__ void add_correction_kernel(Dims d, double *__restrict__ x,
                                      const float *__restrict__ e) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  x[p] = x[p] + (double)e[p];
}

__global__ void buildP_trilin_kernel(Dims dc, P27W<double> P) {
  const Interior t = interior_point(dc);
  if (!t.ok)
    return;
  const int pc = dc.at(t.i, t.j, t.k);
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const int nnz = (dx != 0) + (dy != 0) + (dz != 0);
        P.p[pslot(dx, dy, dz)][pc] = 1.0 / (double)(1 << nnz);
      }
}

// Block-wide sum visible to every thread: warp shuffles, one partial per
// warp in sh[0..31], one barrier, then every thread adds the 32 partials in
// warp order (deterministic). Callers alternate between two sh buffers so
// that a buffer is only rewritten after a later barrier.
__device__ __forceinline__ double cg_allsum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int w = 0; w < nw; ++w)
    t += sh[w];
  return t;
}

template <int K>
__global__ void __launch_bounds__(1024)
    cg_level_kernel(Dims d, Op14<double> A, const double *__restrict__ rhs,
                    double *__restrict__ x, double *__restrict__ r,
                    double *__restrict__ p, double *__restrict__ ap,
                    double thresh, double rel_tol, int class_first_check,
                    int max_iters, int *__restrict__ status) {
  __shared__ double sh[2][32];
  const int m = (d.nx - 2) * (d.ny - 2) * (d.nz - 2);
  const int sy = d.sy(), sz = d.sz();
  int c[K];
#pragma unroll
  for (int t = 0; t < K; ++t) {
    const int q = threadIdx.x + t * blockDim.x;
    int i = 2, j = 2, k = 2;
    if (q < m)
      interior_coords(d, q, i, j, k);
    c[t] = q < m ? d.at(i, j, k) : -1;
  }
  const double *const nul = nullptr;

  // r = rhs - A x; p = r; rs = r.r
  double acc = 0.0;
#pragma unroll
  for (int t = 0; t < K; ++t)
    if (c[t] >= 0) {
      const double v = rhs[c[t]] - apply27(A, nul, x, c[t], sy, sz);
      r[c[t]] = v;
      p[c[t]] = v;
      acc += v * v;
    }
  double rs = cg_allsum(acc, sh[0]);
  // Ap and p.Ap (A p is kept: the next update needs exactly these values)
  acc = 0.0;
#pragma unroll
  for (int t = 0; t < K; ++t)
    if (c[t] >= 0) {
      const double v = apply27(A, nul, p, c[t], sy, sz);
      ap[c[t]] = v;
      acc += v * p[c[t]];
    }
  double pap = cg_allsum(acc, sh[1]);
  int it = 0;
  double res = 0.0;
  if (pap != 0.0) {
    double alpha = rs / pap;
    res = class_first_check ? sqrt(sqrt(rs)) : sqrt(rs);
    const double stop = fmax(thresh, rel_tol * sqrt(rs));
    while (res > stop && it < max_iters) {
      ++it;
      acc = 0.0;
#pragma unroll
      for (int t = 0; t < K; ++t)
        if (c[t] >= 0) {
          x[c[t]] += alpha * p[c[t]];
          const double v = r[c[t]] - alpha * ap[c[t]];
          r[c[t]] = v;
          acc += v * v;
        }
      const double rsn = cg_allsum(acc, sh[0]);
      const double beta = rs == 0.0 ? 0.0 : rsn / rs;
      rs = rsn;
#pragma unroll
      for (int t = 0; t < K; ++t)
        if (c[t] >= 0)
          p[c[t]] = r[c[t]] + beta * p[c[t]];
      __syncthreads();
      acc = 0.0;
#pragma unroll
      for (int t = 0; t < K; ++t)
        if (c[t] >= 0) {
          const double v = apply27(A, nul, p, c[t], sy, sz);
          ap[c[t]] = v;
          acc += v * p[c[t]];
        }
      pap = cg_allsum(acc, sh[1]);
      alpha = pap == 0.0 ? 0.0 : rs / pap;
      res = sqrt(rs);
    }
    if (threadIdx.x == 0) {
      status[0] = it;
      status[1] = (it >= max_iters && res > stop) ? 1 : 0;
    }
  } else if (threadIdx.x == 0) {
    status[0] = 0;
    status[1] = 0;
  }
}

int launch_cg_level(const Dims &d, const Op14<double> &A, const double *rhs,
                    double *x, double *r, double *p, double *ap,
                    double thresh, double rel_tol, int class_first_check,
                    int max_iters, int *status, cudaStream_t s) {
  if (cg_cluster_fits(d)) {
    // levels up to 17^3: a cluster with the operator in shared memory
    const size_t smem = cg_cluster_smem(d.nx, d.ny);
    PMG_CUDA_TRY(set_smem_limit<cg_cluster_kernel>(
        (int)cg_cluster_smem(kCgMaxN, kCgMaxN)));
    cg_cluster_kernel<<<kCgCtas, kCgThreads, smem, s>>>(
        d, A, rhs, x, thresh, rel_tol, class_first_check, max_iters, status);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  }
  const long m = (long)(d.nx - 2) * (d.ny - 2) * (d.nz - 2);
  const int k = (int)((m + 1023) / 1024);
#define PMG_CG(K)                                                              \
  cg_level_kernel<K><<<1, 1024, 0, s>>>(d, A, rhs, x, r, p, ap, thresh,       \
                                        rel_tol, class_first_check,           \
                                        max_iters, status)
  if (k <= 1)
    PMG_CG(1);
  else if (k <= 2)
    PMG_CG(2);
  else if (k <= 4)
    PMG_CG(4);
  else if (k <= 8)
    PMG_CG(8);
  else if (k <= 16)
    PMG_CG(16);
  else if (k <= 32)
    PMG_CG(32);
  else {
    set_last_message("cg_level: level too large for one CTA");
    return PMG_ERR_ARG;
  }
#undef PMG_CG
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

} // namespace pmg

using namespace pmg;

// ---------------------------------------------------------------------------
// argument checks
// ---------------------------------------------------------------------------
static bool bad_pair(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc) {
  return bad_dims(nxf, nyf, nzf) || bad_dims(nxc, nyc, nzc) ||
         nxf != 2 * nxc - 1 || nyf != 2 * nyc - 1 || nzf != 2 * nzc - 1;
}

template <typename T>
static Op14<T> op7(const T *oC, const T *oE, const T *oN, const T *uC) {
  Op14<T> A{};
  A.a[kOC] = oC;
  A.a[kOE] = oE;
  A.a[kON] = oN;
  A.a[kUC] = uC;
  return A;
}
template <typename T>
static Op14<T> op27(const T *oC, const T *oE, const T *oN, const T *uC,
                    const T *oNE, const T *oNW, const T *uE, const T *uW,
                    const T *uN, const T *uS, const T *uNE, const T *uNW,
                    const T *uSE, const T *uSW) {
  return Op14<T>{{oC, oE, oN, uC, oNE, oNW, uE, uW, uN, uS, uNE, uNW, uSE,
                  uSW}};
}
template <typename T> static bool any_null(const Op14<T> &A, int n) {
  for (int s = 0; s < n; ++s)
    if (!A.a[s])
      return true;
  return false;
}

// Runs itmax eight-colour sweeps in place on x with the two-launch tiled
// kernel; the ping-pong partner is a stream-ordered copy of x (same shell).
template <typename T>
static int gs27_inplace(const Dims &d, const Op14<T> &A, const T *cc,
                        const T *fc, T *x, int itmax, int iadjoint,
                        int zero_init, cudaStream_t s) {
  if (itmax == 0) {
    if (zero_init)
      PMG_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(T) * d.count(), s));
    return PMG_OK;
  }
  T *alt = nullptr;
  const size_t bytes = sizeof(T) * d.count();
  PMG_CUDA_TRY(scratch_alloc((void **)&alt, bytes, s));
  int rc = PMG_OK;
  cudaError_t e = cudaSuccess;
  if (zero_init)
    e = cudaMemsetAsync(x, 0, bytes, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(alt, x, bytes, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) {
    T *res = nullptr;
    rc = launch_gs27_pp<T>(d, A, cc, fc, x, alt, itmax, iadjoint, 0, s, &res);
    if (rc == PMG_OK && res != x)
      e = cudaMemcpyAsync(x, res, bytes, cudaMemcpyDeviceToDevice, s);
  }
  scratch_free(alt, s);
  if (e != cudaSuccess) {
    set_last_error(e, "Vgsrb27x", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  return rc;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
// Kernel entry points, for double (_d) and float (_f) arrays.
#define P27_ARGS                                                               \
  oPC, oPN, oPS, oPE, oPW, oPNE, oPNW, oPSE, oPSW, uPC, uPN, uPS, uPE, uPW,    \
      uPNE, uPNW, uPSE, uPSW, dPC, dPN, dPS, dPE, dPW, dPNE, dPNW, dPSE, dPSW

template <typename T>
static int entry_Vmatvec7_1s(int nx, int ny, int nz, const T *oC,
                      const T *cc, const T *oE, const T *oN,
                      const T *uC, const T *x, T *y,
                      pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmatvec7_1s: grid size out of range");
  PMG_REQUIRE(oC && oE && oN && uC && x && y, "Vmatvec7_1s: null array");
  const Dims d{nx, ny, nz};
  matvec_kernel<7, T><<<interior_grid(d), interior_block(),
                             0, (cudaStream_t)stream>>>(
      d, op7(oC, oE, oN, uC), cc, x, y);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

template <typename T>
static int entry_Vmatvec27_1s(int nx, int ny, int nz, const T *oC,
                       const T *cc, const T *oE, const T *oN,
                       const T *uC, const T *oNE, const T *oNW,
                       const T *uE, const T *uW, const T *uN,
                       const T *uS, const T *uNE, const T *uNW,
                       const T *uSE, const T *uSW, const T *x,
                       T *y, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmatvec27_1s: grid size out of range");
  const Op14<T> A =
      op27(oC, oE, oN, uC, oNE, oNW, uE, uW, uN, uS, uNE, uNW, uSE, uSW);
  PMG_REQUIRE(!any_null(A, 14) && x && y, "Vmatvec27_1s: null array");
  const Dims d{nx, ny, nz};
  matvec_kernel<27, T><<<interior_grid(d), interior_block(), 0,
                              (cudaStream_t)stream>>>(d, A, cc, x, y);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

template <typename T>
static int entry_Vmresid7_1s(int nx, int ny, int nz, const T *oC,
                      const T *cc, const T *fc, const T *oE,
                      const T *oN, const T *uC, const T *x,
                      T *r, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmresid7_1s: grid size out of range");
  PMG_REQUIRE(oC && fc && oE && oN && uC && x && r,
              "Vmresid7_1s: null array");
  const Dims d{nx, ny, nz};
  mresid_kernel<7, T><<<interior_grid(d), interior_block(), 0,
                             (cudaStream_t)stream>>>(
      d, op7(oC, oE, oN, uC), cc, fc, x, r);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

template <typename T>
static int entry_Vmresid27_1s(int nx, int ny, int nz, const T *oC,
                       const T *cc, const T *fc, const T *oE,
                       const T *oN, const T *uC, const T *oNE,
                       const T *oNW, const T *uE, const T *uW,
                       const T *uN, const T *uS, const T *uNE,
                       const T *uNW, const T *uSE, const T *uSW,
                       const T *x, T *r, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vmresid27_1s: grid size out of range");
  const Op14<T> A =
      op27(oC, oE, oN, uC, oNE, oNW, uE, uW, uN, uS, uNE, uNW, uSE, uSW);
  PMG_REQUIRE(!any_null(A, 14) && fc && x && r, "Vmresid27_1s: null array");
  const Dims d{nx, ny, nz};
  mresid_kernel<27, T><<<interior_grid(d), interior_block(), 0,
                              (cudaStream_t)stream>>>(d, A, cc, fc, x, r);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

template <typename T>
static int entry_Vrestrc2(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                   const T *xin, T *xout, const T *oPC,
                   const T *oPN, const T *oPS, const T *oPE,
                   const T *oPW, const T *oPNE, const T *oPNW,
                   const T *oPSE, const T *oPSW, const T *uPC,
                   const T *uPN, const T *uPS, const T *uPE,
                   const T *uPW, const T *uPNE, const T *uPNW,
                   const T *uPSE, const T *uPSW, const T *dPC,
                   const T *dPN, const T *dPS, const T *dPE,
                   const T *dPW, const T *dPNE, const T *dPNW,
                   const T *dPSE, const T *dPSW,
                   pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "Vrestrc2: sizes must satisfy n_f = 2 n_c - 1");
  const P27<T> P{{P27_ARGS}};
  for (int s = 0; s < 27; ++s)
    PMG_REQUIRE(P.p[s], "Vrestrc2: null prolongation array");
  PMG_REQUIRE(xin && xout, "Vrestrc2: null array");
  const Dims dc{nxc, nyc, nzc};
  restrict_kernel<T, T><<<interior_grid(dc), interior_block(), 0,
                                    (cudaStream_t)stream>>>(
      Dims{nxf, nyf, nzf}, dc, xin, xout, P);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

template <typename T>
static int entry_VinterpPMG2(int nxc, int nyc, int nzc, int nxf, int nyf,
                      int nzf, const T *xin, T *xout, const T *oPC,
                      const T *oPN, const T *oPS, const T *oPE,
                      const T *oPW, const T *oPNE, const T *oPNW,
                      const T *oPSE, const T *oPSW, const T *uPC,
                      const T *uPN, const T *uPS, const T *uPE,
                      const T *uPW, const T *uPNE, const T *uPNW,
                      const T *uPSE, const T *uPSW, const T *dPC,
                      const T *dPN, const T *dPS, const T *dPE,
                      const T *dPW, const T *dPNE, const T *dPNW,
                      const T *dPSE, const T *dPSW,
                      pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "VinterpPMG2: sizes must satisfy n_f = 2 n_c - 1");
  const P27<T> P{{P27_ARGS}};
  for (int s = 0; s < 27; ++s)
    PMG_REQUIRE(P.p[s], "VinterpPMG2: null prolongation array");
  PMG_REQUIRE(xin && xout, "VinterpPMG2: null array");
  const Dims dc{nxc, nyc, nzc};
  interp_kernel<T><<<interp_grid(dc), interior_block(), 0,
                          (cudaStream_t)stream>>>(dc, Dims{nxf, nyf, nzf},
                                                  xin, xout, P);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

extern "C" {

int pmg_set_autotune(int mode) {
  if (mode != 0 && mode != 1 && mode != 8 && mode != 16 && mode != 32) {
    set_last_message("pmg_set_autotune: mode must be 0, 1, 8, 16 or 32");
    return PMG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_tile_mutex);
  g_tile_mode = mode;
  return PMG_OK;
}

const char *pmg_last_error(void) { return g_last_error; }
const char *pmg_version(void) { return "pmg_b200 0.1 (sm_100a)"; }

#define GS7_BODY(T)                                                            \
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vgsrb7x: grid size out of range");       \
  PMG_REQUIRE(oC && fc && oE && oN && uC && x, "Vgsrb7x: null array");         \
  PMG_REQUIRE(itmax >= 0, "Vgsrb7x: itmax < 0");                               \
  return launch_gs7<T>(Dims{nx, ny, nz}, oC, cc, fc, oE, oN, uC, x, itmax,    \
                       iadjoint, zero_init, (cudaStream_t)stream);

int pmg_Vgsrb7x_d(int nx, int ny, int nz, const double *oC, const double *cc,
                  const double *fc, const double *oE, const double *oN,
                  const double *uC, double *x, int itmax, int iadjoint,
                  int zero_init, pmg_stream_t stream) {
  GS7_BODY(double)
}
int pmg_Vgsrb7x_f(int nx, int ny, int nz, const float *oC, const float *cc,
                  const float *fc, const float *oE, const float *oN,
                  const float *uC, float *x, int itmax, int iadjoint,
                  int zero_init, pmg_stream_t stream) {
  GS7_BODY(float)
}

#define GS27_BODY(T)                                                           \
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "Vgsrb27x: grid size out of range");      \
  const Op14<T> A =                                                            \
      op27<T>(oC, oE, oN, uC, oNE, oNW, uE, uW, uN, uS, uNE, uNW, uSE, uSW);  \
  PMG_REQUIRE(!any_null(A, 14) && fc && x, "Vgsrb27x: null array");            \
  PMG_REQUIRE(itmax >= 0, "Vgsrb27x: itmax < 0");                              \
  return gs27_inplace<T>(Dims{nx, ny, nz}, A, cc, fc, x, itmax, iadjoint,     \
                         zero_init, (cudaStream_t)stream);

int pmg_Vgsrb27x_d(int nx, int ny, int nz, const double *oC, const double *cc,
                   const double *fc, const double *oE, const double *oN,
                   const double *uC, const double *oNE, const double *oNW,
                   const double *uE, const double *uW, const double *uN,
                   const double *uS, const double *uNE, const double *uNW,
                   const double *uSE, const double *uSW, double *x, int itmax,
                   int zero_init, int iadjoint, pmg_stream_t stream) {
  GS27_BODY(double)
}
int pmg_Vgsrb27x_f(int nx, int ny, int nz, const float *oC, const float *cc,
                   const float *fc, const float *oE, const float *oN,
                   const float *uC, const float *oNE, const float *oNW,
                   const float *uE, const float *uW, const float *uN,
                   const float *uS, const float *uNE, const float *uNW,
                   const float *uSE, const float *uSW, float *x, int itmax,
                   int zero_init, int iadjoint, pmg_stream_t stream) {
  GS27_BODY(float)
}

int pmg_Vmatvec7_1s_d(int nx, int ny, int nz, const double *oC,
                      const double *cc, const double *oE, const double *oN,
                      const double *uC, const double *x, double *y,
                      pmg_stream_t stream) {
  return entry_Vmatvec7_1s<double>(nx, ny, nz, oC, cc, oE, oN, uC, x, y,
      stream);
}

int pmg_Vmatvec7_1s_f(int nx, int ny, int nz, const float *oC,
                      const float *cc, const float *oE, const float *oN,
                      const float *uC, const float *x, float *y,
                      pmg_stream_t stream) {
  return entry_Vmatvec7_1s<float>(nx, ny, nz, oC, cc, oE, oN, uC, x, y, stream);
}

int pmg_Vmatvec27_1s_d(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *oE, const double *oN,
                       const double *uC, const double *oNE, const double *oNW,
                       const double *uE, const double *uW, const double *uN,
                       const double *uS, const double *uNE, const double *uNW,
                       const double *uSE, const double *uSW, const double *x,
                       double *y, pmg_stream_t stream) {
  return entry_Vmatvec27_1s<double>(nx, ny, nz, oC, cc, oE, oN, uC, oNE, oNW,
      uE, uW, uN, uS, uNE, uNW, uSE, uSW, x, y, stream);
}

int pmg_Vmatvec27_1s_f(int nx, int ny, int nz, const float *oC,
                       const float *cc, const float *oE, const float *oN,
                       const float *uC, const float *oNE, const float *oNW,
                       const float *uE, const float *uW, const float *uN,
                       const float *uS, const float *uNE, const float *uNW,
                       const float *uSE, const float *uSW, const float *x,
                       float *y, pmg_stream_t stream) {
  return entry_Vmatvec27_1s<float>(nx, ny, nz, oC, cc, oE, oN, uC, oNE, oNW, uE,
      uW, uN, uS, uNE, uNW, uSE, uSW, x, y, stream);
}

int pmg_Vmresid7_1s_d(int nx, int ny, int nz, const double *oC,
                      const double *cc, const double *fc, const double *oE,
                      const double *oN, const double *uC, const double *x,
                      double *r, pmg_stream_t stream) {
  return entry_Vmresid7_1s<double>(nx, ny, nz, oC, cc, fc, oE, oN, uC, x, r,
      stream);
}

int pmg_Vmresid7_1s_f(int nx, int ny, int nz, const float *oC,
                      const float *cc, const float *fc, const float *oE,
                      const float *oN, const float *uC, const float *x,
                      float *r, pmg_stream_t stream) {
  return entry_Vmresid7_1s<float>(nx, ny, nz, oC, cc, fc, oE, oN, uC, x, r,
      stream);
}

int pmg_Vmresid27_1s_d(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *fc, const double *oE,
                       const double *oN, const double *uC, const double *oNE,
                       const double *oNW, const double *uE, const double *uW,
                       const double *uN, const double *uS, const double *uNE,
                       const double *uNW, const double *uSE, const double *uSW,
                       const double *x, double *r, pmg_stream_t stream) {
  return entry_Vmresid27_1s<double>(nx, ny, nz, oC, cc, fc, oE, oN, uC, oNE,
      oNW, uE, uW, uN, uS, uNE, uNW, uSE, uSW, x, r, stream);
}

int pmg_Vmresid27_1s_f(int nx, int ny, int nz, const float *oC,
                       const float *cc, const float *fc, const float *oE,
                       const float *oN, const float *uC, const float *oNE,
                       const float *oNW, const float *uE, const float *uW,
                       const float *uN, const float *uS, const float *uNE,
                       const float *uNW, const float *uSE, const float *uSW,
                       const float *x, float *r, pmg_stream_t stream) {
  return entry_Vmresid27_1s<float>(nx, ny, nz, oC, cc, fc, oE, oN, uC, oNE, oNW,
      uE, uW, uN, uS, uNE, uNW, uSE, uSW, x, r, stream);
}

int pmg_Vrestrc2_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                   const double *xin, double *xout, const double *oPC,
                   const double *oPN, const double *oPS, const double *oPE,
                   const double *oPW, const double *oPNE, const double *oPNW,
                   const double *oPSE, const double *oPSW, const double *uPC,
                   const double *uPN, const double *uPS, const double *uPE,
                   const double *uPW, const double *uPNE, const double *uPNW,
                   const double *uPSE, const double *uPSW, const double *dPC,
                   const double *dPN, const double *dPS, const double *dPE,
                   const double *dPW, const double *dPNE, const double *dPNW,
                   const double *dPSE, const double *dPSW,
                   pmg_stream_t stream) {
  return entry_Vrestrc2<double>(nxf, nyf, nzf, nxc, nyc, nzc, xin, xout, oPC,
      oPN, oPS, oPE, oPW, oPNE, oPNW, oPSE, oPSW, uPC, uPN, uPS, uPE, uPW, uPNE,
      uPNW, uPSE, uPSW, dPC, dPN, dPS, dPE, dPW, dPNE, dPNW, dPSE, dPSW,
      stream);
}

int pmg_Vrestrc2_f(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                   const float *xin, float *xout, const float *oPC,
                   const float *oPN, const float *oPS, const float *oPE,
                   const float *oPW, const float *oPNE, const float *oPNW,
                   const float *oPSE, const float *oPSW, const float *uPC,
                   const float *uPN, const float *uPS, const float *uPE,
                   const float *uPW, const float *uPNE, const float *uPNW,
                   const float *uPSE, const float *uPSW, const float *dPC,
                   const float *dPN, const float *dPS, const float *dPE,
                   const float *dPW, const float *dPNE, const float *dPNW,
                   const float *dPSE, const float *dPSW,
                   pmg_stream_t stream) {
  return entry_Vrestrc2<float>(nxf, nyf, nzf, nxc, nyc, nzc, xin, xout, oPC,
      oPN, oPS, oPE, oPW, oPNE, oPNW, oPSE, oPSW, uPC, uPN, uPS, uPE, uPW, uPNE,
      uPNW, uPSE, uPSW, dPC, dPN, dPS, dPE, dPW, dPNE, dPNW, dPSE, dPSW,
      stream);
}

int pmg_VinterpPMG2_d(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                      const double *xin, double *xout, const double *oPC,
                      const double *oPN, const double *oPS, const double *oPE,
                      const double *oPW, const double *oPNE, const double *oPNW,
                      const double *oPSE, const double *oPSW, const double *uPC,
                      const double *uPN, const double *uPS, const double *uPE,
                      const double *uPW, const double *uPNE, const double *uPNW,
                      const double *uPSE, const double *uPSW, const double *dPC,
                      const double *dPN, const double *dPS, const double *dPE,
                      const double *dPW, const double *dPNE, const double *dPNW,
                      const double *dPSE, const double *dPSW,
                      pmg_stream_t stream) {
  return entry_VinterpPMG2<double>(nxc, nyc, nzc, nxf, nyf, nzf, xin, xout, oPC,
      oPN, oPS, oPE, oPW, oPNE, oPNW, oPSE, oPSW, uPC, uPN, uPS, uPE, uPW, uPNE,
      uPNW, uPSE, uPSW, dPC, dPN, dPS, dPE, dPW, dPNE, dPNW, dPSE, dPSW,
      stream);
}

int pmg_VinterpPMG2_f(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                      const float *xin, float *xout, const float *oPC,
                      const float *oPN, const float *oPS, const float *oPE,
                      const float *oPW, const float *oPNE, const float *oPNW,
                      const float *oPSE, const float *oPSW, const float *uPC,
                      const float *uPN, const float *uPS, const float *uPE,
                      const float *uPW, const float *uPNE, const float *uPNW,
                      const float *uPSE, const float *uPSW, const float *dPC,
                      const float *dPN, const float *dPS, const float *dPE,
                      const float *dPW, const float *dPNE, const float *dPNW,
                      const float *dPSE, const float *dPSW,
                      pmg_stream_t stream) {
  return entry_VinterpPMG2<float>(nxc, nyc, nzc, nxf, nyf, nzf, xin, xout, oPC,
      oPN, oPS, oPE, oPW, oPNE, oPNW, oPSE, oPSW, uPC, uPN, uPS, uPE, uPW, uPNE,
      uPNW, uPSE, uPSW, dPC, dPN, dPS, dPE, dPW, dPNE, dPNW, dPSE, dPSW,
      stream);
}

int pmg_VbuildPb_op7_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                       const double *oC, const double *oE, const double *oN,
                       const double *uC, double *oPC, double *oPN,
                       double *oPS, double *oPE, double *oPW, double *oPNE,
                       double *oPNW, double *oPSE, double *oPSW, double *uPC,
                       double *uPN, double *uPS, double *uPE, double *uPW,
                       double *uPNE, double *uPNW, double *uPSE, double *uPSW,
                       double *dPC, double *dPN, double *dPS, double *dPE,
                       double *dPW, double *dPNE, double *dPNW, double *dPSE,
                       double *dPSW, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "VbuildPb_op7: sizes must satisfy n_f = 2 n_c - 1");
  PMG_REQUIRE(oC && oE && oN && uC, "VbuildPb_op7: null operator array");
  const P27W<double> P{{P27_ARGS}};
  for (int s = 0; s < 27; ++s)
    PMG_REQUIRE(P.p[s], "VbuildPb_op7: null prolongation array");
  return launch_buildP(Dims{nxf, nyf, nzf}, Dims{nxc, nyc, nzc}, 7,
                       op7(oC, oE, oN, uC), P, (cudaStream_t)stream);
}

int pmg_VbuildPb_op27_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                        const double *oC, const double *oE, const double *oN,
                        const double *uC, const double *oNE,
                        const double *oNW, const double *uE, const double *uW,
                        const double *uN, const double *uS, const double *uNE,
                        const double *uNW, const double *uSE,
                        const double *uSW, double *oPC, double *oPN,
                        double *oPS, double *oPE, double *oPW, double *oPNE,
                        double *oPNW, double *oPSE, double *oPSW, double *uPC,
                        double *uPN, double *uPS, double *uPE, double *uPW,
                        double *uPNE, double *uPNW, double *uPSE, double *uPSW,
                        double *dPC, double *dPN, double *dPS, double *dPE,
                        double *dPW, double *dPNE, double *dPNW, double *dPSE,
                        double *dPSW, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "VbuildPb_op27: sizes must satisfy n_f = 2 n_c - 1");
  const Op14<double> A =
      op27(oC, oE, oN, uC, oNE, oNW, uE, uW, uN, uS, uNE, uNW, uSE, uSW);
  PMG_REQUIRE(!any_null(A, 14), "VbuildPb_op27: null operator array");
  const P27W<double> P{{P27_ARGS}};
  for (int s = 0; s < 27; ++s)
    PMG_REQUIRE(P.p[s], "VbuildPb_op27: null prolongation array");
  return launch_buildP(Dims{nxf, nyf, nzf}, Dims{nxc, nyc, nzc}, 27, A, P,
                       (cudaStream_t)stream);
}

int pmg_VbuildPb_trilin_d(int nxf, int nyf, int nzf, int nxc, int nyc,
                          int nzc, double *oPC, double *oPN, double *oPS,
                          double *oPE, double *oPW, double *oPNE, double *oPNW,
                          double *oPSE, double *oPSW, double *uPC, double *uPN,
                          double *uPS, double *uPE, double *uPW, double *uPNE,
                          double *uPNW, double *uPSE, double *uPSW,
                          double *dPC, double *dPN, double *dPS, double *dPE,
                          double *dPW, double *dPNE, double *dPNW,
                          double *dPSE, double *dPSW, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "VbuildPb_trilin: sizes must satisfy n_f = 2 n_c - 1");
  const P27W<double> P{{P27_ARGS}};
  for (int s = 0; s < 27; ++s)
    PMG_REQUIRE(P.p[s], "VbuildPb_trilin: null prolongation array");
  const Dims dc{nxc, nyc, nzc};
  buildP_trilin_kernel<<<interior_grid(dc), interior_block(), 0,
                         (cudaStream_t)stream>>>(dc, P);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

int pmg_VbuildA_fv_d(int nx, int ny, int nz, int ipkey, int *numdia, int *ipc,
                     double *oC, double *cc, double *fc, double *oE,
                     double *oN, double *uC, const double *xf,
                     const double *yf, const double *zf, const double *gxcf,
                     const double *gycf, const double *gzcf,
                     const double *a1cf, const double *a2cf,
                     const double *a3cf, const double *ccf, const double *fcf,
                     pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz), "VbuildA_fv: grid size out of range");
  const BoxMaps m{xf, yf, zf, gxcf, gycf, gzcf, a1cf, a2cf, a3cf, ccf, fcf};
  const BoxOps o{oC, cc, fc, oE, oN, uC};
  PMG_REQUIRE(m.xf && m.yf && m.zf && m.gx && m.gy && m.gz && m.a1 && m.a2 &&
                  m.a3 && m.cc && m.fc,
              "VbuildA_fv: null input array");
  PMG_REQUIRE(o.oC && o.cc && o.fc && o.oE && o.oN && o.uC,
              "VbuildA_fv: null output array");
  if (ipc) {
    ipc[9] = ipkey;
    ipc[10] = 7; // stencil points
    ipc[11] = 1;
  }
  if (numdia)
    *numdia = 4; // stored diagonals
  const Dims d{nx, ny, nz};
  buildA_fv_kernel<<<interior_grid(d), interior_block(), 0,
                     (cudaStream_t)stream>>>(d, m, o);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

int pmg_VbuildG_7_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                    const double *const *p27, const double *oC,
                    const double *oE, const double *oN, const double *uC,
                    double *const *out14, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "VbuildG_7: sizes must satisfy n_f = 2 n_c - 1");
  PMG_REQUIRE(p27 && out14 && oC && oE && oN && uC, "VbuildG_7: null array");
  P27<double> P;
  Op14W<double> out;
  for (int s = 0; s < 27; ++s) {
    P.p[s] = p27[s];
    PMG_REQUIRE(P.p[s], "VbuildG_7: null prolongation array");
  }
  for (int s = 0; s < 14; ++s) {
    out.a[s] = out14[s];
    PMG_REQUIRE(out.a[s], "VbuildG_7: null output array");
  }
  return launch_buildG(Dims{nxf, nyf, nzf}, Dims{nxc, nyc, nzc}, 7, P,
                       op7(oC, oE, oN, uC), out, (cudaStream_t)stream);
}

int pmg_VbuildG_27_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                     const double *const *p27, const double *const *a14,
                     double *const *out14, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_pair(nxf, nyf, nzf, nxc, nyc, nzc),
              "VbuildG_27: sizes must satisfy n_f = 2 n_c - 1");
  PMG_REQUIRE(p27 && a14 && out14, "VbuildG_27: null array");
  P27<double> P;
  Op14<double> A;
  Op14W<double> out;
  for (int s = 0; s < 27; ++s) {
    P.p[s] = p27[s];
    PMG_REQUIRE(P.p[s], "VbuildG_27: null prolongation array");
  }
  for (int s = 0; s < 14; ++s) {
    A.a[s] = a14[s];
    out.a[s] = out14[s];
    PMG_REQUIRE(A.a[s] && out.a[s], "VbuildG_27: null operator array");
  }
  return launch_buildG(Dims{nxf, nyf, nzf}, Dims{nxc, nyc, nzc}, 27, P, A,
                       out, (cudaStream_t)stream);
}

int pmg_cg_level_d(int nx, int ny, int nz, const double *const *a14,
                   const double *rhs, double *x, double thresh, int max_iters,
                   int *iters, pmg_stream_t stream) {
  PMG_REQUIRE(!bad_dims(nx, ny, nz) && nx <= 33 && ny <= 33 && nz <= 33,
              "cg_level: grid must be at most 33^3");
  PMG_REQUIRE(a14 && rhs && x && max_iters >= 0, "cg_level: bad argument");
  Op14<double> A;
  for (int s = 0; s < 14; ++s) {
    A.a[s] = a14[s];
    PMG_REQUIRE(A.a[s], "cg_level: null operator array");
  }
  cudaStream_t s = (cudaStream_t)stream;
  const Dims d{nx, ny, nz};
  const size_t n3 = (size_t)d.count();
  // r, p, Ap (zero shells) and the two status words, stream-ordered.
  char *ws = nullptr;
  const size_t bytes = 3 * n3 * sizeof(double) + 2 * sizeof(int);
  PMG_CUDA_TRY(scratch_alloc((void **)&ws, bytes, s));
  int rc = PMG_OK;
  int host_status[2] = {0, 0};
  double *r = (double *)ws, *p = r + n3, *ap = p + n3;
  int *status = (int *)(ap + n3);
  cudaError_t e = cudaMemsetAsync(ws, 0, bytes, s);
  if (e == cudaSuccess) {
    rc = launch_cg_level(d, A, rhs, x, r, p, ap, thresh, 0.0, 1, max_iters,
                         status, s);
    e = rc == PMG_OK ? cudaSuccess : cudaErrorLaunchFailure;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host_status, status, sizeof(host_status),
                        cudaMemcpyDeviceToHost, s);
  scratch_free(ws, s);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  if (rc != PMG_OK)
    return rc;
  if (e != cudaSuccess) {
    set_last_error(e, "cg_level", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  if (iters)
    *iters = host_status[0];
  if (host_status[1]) {
    set_last_message("cg_level: iteration cap reached above the threshold");
    rc = PMG_ERR_TIMEOUT;
  }
  return rc;
}

} // extern "C"
