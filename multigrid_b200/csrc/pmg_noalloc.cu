// Coarsest-level CG without any device allocation.
//
// pmg_cg_level_d takes its work vectors (residual, search direction, A times
// the search direction) from the stream-ordered allocator on every call.
// Some callers cannot let a library allocate device memory: a host
// application that owns the whole device memory budget through its own pool
// and forbids foreign allocations, a code that must not hit allocator
// synchronisation or out-of-memory failures in the middle of a time step, or
// an embedding whose memory accounting has to be exact. pmg_cg_level_noalloc_d
// runs the same CG kernel on a work area that lives in this library's static
// device memory instead: a file-scope __device__ array sized for the largest
// grid the entry point accepts (17 x 17 x 17 points), which every GPU that
// loads the library keeps until the process exits.
//
// The array is shared by all calls on a device and keeps the last call's
// contents, so each call clears the part it uses (the kernel expects zero
// shells), and two calls that run on the GPU at the same time (on different
// streams) overwrite each other's work vectors.
#include "reduce_kernels.cuh"

namespace {

// Largest accepted grid, points including the shell.
constexpr int kNoAllocMaxPoints = 17 * 17 * 17;
// r, p and A p of the largest grid, then two status words.
constexpr size_t kNoAllocBytes =
    3 * sizeof(double) * kNoAllocMaxPoints + 2 * sizeof(int);

static __device__ __align__(256) unsigned char noalloc_scratch[kNoAllocBytes];

// Device address of noalloc_scratch in the current device's context. In
// host code the array's name is only a stand-in for the symbol, never an
// address a kernel may use. The address is looked up on every call, with
// the caller's device current: a cached address would go stale when the
// context that loaded the module is torn down (cudaDeviceReset) or when
// another context is current, and the lookup is cheap next to the stream
// synchronisation each call does anyway.
int scratch_address(void **out) {
  void *ptr = nullptr;
  PMG_CUDA_TRY(cudaGetSymbolAddress(&ptr, noalloc_scratch));
  *out = ptr;
  return PMG_OK;
}

} // namespace

extern "C" int pmg_cg_level_noalloc_d(int nx, int ny, int nz,
                                      const double *const *a14,
                                      const double *rhs, double *x,
                                      double thresh, int max_iters,
                                      int *iters, pmg_stream_t stream) {
  using namespace pmg;
  if (nx < 3 || ny < 3 || nz < 3) {
    set_last_message("cg_level_noalloc: grid must be at least 3^3");
    return PMG_ERR_ARG;
  }
  if ((long)nx * ny * nz > kNoAllocMaxPoints) {
    set_last_message("cg_level_noalloc: grid larger than the static work "
                     "area (at most 17*17*17 points including the shell)");
    return PMG_ERR_ARG;
  }
  if (!a14 || !rhs || !x || max_iters < 0) {
    set_last_message("cg_level_noalloc: bad argument");
    return PMG_ERR_ARG;
  }
  Op14<double> A;
  for (int s = 0; s < 14; ++s) {
    A.a[s] = a14[s];
    if (!A.a[s]) {
      set_last_message("cg_level_noalloc: null operator array");
      return PMG_ERR_ARG;
    }
  }
  void *base = nullptr;
  int rc = scratch_address(&base);
  if (rc != PMG_OK)
    return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const Dims d{nx, ny, nz};
  const size_t n3 = (size_t)d.count();
  double *r = (double *)base, *p = r + n3, *ap = p + n3;
  int *status = (int *)(ap + n3);
  // the previous call may have left interior values where this grid has its
  // shell, and the status words must start fresh
  PMG_CUDA_TRY(cudaMemsetAsync(base, 0, 3 * n3 * sizeof(double) +
                                            2 * sizeof(int), s));
  rc = launch_cg_level(d, A, rhs, x, r, p, ap, thresh, 0.0, 1, max_iters,
                       status, s);
  if (rc != PMG_OK)
    return rc;
  int host_status[2] = {0, 0};
  PMG_CUDA_TRY(cudaMemcpyAsync(host_status, status, sizeof(host_status),
                               cudaMemcpyDeviceToHost, s));
  PMG_CUDA_TRY(cudaStreamSynchronize(s));
  if (iters)
    *iters = host_status[0];
  if (host_status[1]) {
    set_last_message(
        "cg_level_noalloc: iteration cap reached above the threshold");
    return PMG_ERR_TIMEOUT;
  }
  return PMG_OK;
}
