// Shared device helpers for the PMG kernels (sm_100a).
//
// Grid layout is the reference's (pmgc/vmatrix.h:79-80): an nx*ny*nz array
// per quantity with a one-point Dirichlet shell, x fastest, 1-based
// (i,j,k) -> ((k-1)*ny + (j-1))*nx + (i-1). Grids are at most 1025 points per
// axis, so every linear index fits in 32 bits.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <stdint.h>

#include "../../include/pmg_b200.h"

namespace pmg {

constexpr int kMaxN = 1025;

// nx, ny, nz points per axis; rows px >= nx entries apart (px > nx pads
// the rows of an array to a 16-byte multiple for tensor-memory-access
// copies; every point's index and every stencil offset follow px, the
// entries past nx in a row are never read as grid points).
struct Dims {
  int nx, ny, nz, px;
  Dims() = default;
  __host__ __device__ Dims(int x, int y, int z, int pitch = 0)
      : nx(x), ny(y), nz(z), px(pitch > x ? pitch : x) {}
  __host__ __device__ int sy() const { return px; }
  __host__ __device__ int sz() const { return px * ny; }
  __host__ __device__ int at(int i, int j, int k) const {
    return ((k - 1) * ny + (j - 1)) * px + (i - 1);
  }
  // entries of an array (the padding included)
  __host__ __device__ long count() const { return (long)px * ny * nz; }
};

// The 14 upper diagonals of a symmetric 27-point operator in the reference's
// order oC oE oN uC oNE oNW uE uW uN uS uNE uNW uSE uSW; a 7-point operator
// uses the first four.
template <typename T> struct Op14 {
  const T *a[14];
};
template <typename T> struct Op14W {
  T *a[14];
};
// The 27 prolongation arrays: oP{C,N,S,E,W,NE,NW,SE,SW}, uP*, dP*.
template <typename T> struct P27 {
  const T *p[27];
};
template <typename T> struct P27W {
  T *p[27];
};

// B-byte cp.async into shared memory; reads nothing and writes zero when
// `in` is false (gmem must still be a valid address)
template <int B>
__device__ __forceinline__ void cp_async_zfill(void *smem, const void *gmem,
                                               bool in) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = in ? B : 0;
  if constexpr (B == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s),
                 "l"(gmem), "r"(n)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s),
                 "l"(gmem), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::
                   : "memory");
}

enum OpSlot {
  kOC = 0, kOE, kON, kUC, kONE, kONW, kUE, kUW, kUN, kUS, kUNE, kUNW, kUSE,
  kUSW
};

// Slot of the stored upper diagonal for a neighbour offset, 0 when the offset
// points to the lower half (read from the neighbour) or is the centre.
__host__ __device__ constexpr int upper_slot(int ex, int ey, int ez) {
  return ez == 1
             ? (ey == -1 ? (ex == -1 ? kUSW : ex == 0 ? kUS : kUSE)
                : ey == 0 ? (ex == -1 ? kUW : ex == 0 ? kUC : kUE)
                          : (ex == -1 ? kUNW : ex == 0 ? kUN : kUNE))
         : (ez == 0 && ey == 1) ? (ex == -1 ? kONW : ex == 0 ? kON : kONE)
         : (ez == 0 && ey == 0 && ex == 1) ? kOE
                                           : 0;
}

// Slot in the 27-array prolongation list of fine offset (dx,dy,dz) from a
// coarse point's fine image: plane (o: dz=0, u: +1, d: -1) * 9 + in-plane
// position C N S E W NE NW SE SW.
__host__ __device__ constexpr int pslot(int dx, int dy, int dz) {
  return (dz == 0 ? 0 : dz == 1 ? 9 : 18) +
         (dy == 0 ? (dx == 0 ? 0 : dx == 1 ? 3 : 4)
          : dy == 1 ? (dx == 0 ? 1 : dx == 1 ? 5 : 6)
                    : (dx == 0 ? 2 : dx == 1 ? 7 : 8));
}

// Positive coupling between point p and p + (ex,ey,ez) of a symmetric
// operator; the lower half is read from the upper diagonal stored at the
// neighbour (pmgc/matvecd.h:208-236). Offsets are compile-time after
// unrolling.
template <typename T>
__device__ __forceinline__ T coupling(const Op14<T> &A, const Dims &d, int p,
                                      int ex, int ey, int ez) {
  const int s = upper_slot(ex, ey, ez);
  if (s) {
    const T *a = A.a[s];
    return a ? a[p] : T(0);
  }
  const int s2 = upper_slot(-ex, -ey, -ez);
  const T *a = A.a[s2];
  return a ? a[p + ex + ey * d.sy() + ez * d.sz()] : T(0);
}

// Block-wide sum of one value per thread into thread 0 (any blockDim that is
// a multiple of 32, at most 1024). `sh` needs 32 entries.
template <typename T> __device__ __forceinline__ T block_sum(T v, T *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
    sh[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// block_sum for 2-D blocks (threads numbered x-fastest); result in the
// first thread.
template <typename T> __device__ __forceinline__ T block_sum_2d(T v, T *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nt = blockDim.x * blockDim.y;
  const int lane = tid & 31, w = tid >> 5;
  __syncthreads();
  if (lane == 0)
    sh[w] = v;
  __syncthreads();
  const int nw = (nt + 31) >> 5;
  v = (tid < nw) ? sh[tid] : T(0);
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

} // namespace pmg

// Host-side error plumbing: every entry point returns a pmg_status.
#define PMG_CUDA_TRY(expr)                                                     \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      pmg::set_last_error(_e, #expr, __FILE__, __LINE__);                      \
      return PMG_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

// Argument check of an entry point: the message, then PMG_ERR_ARG.
#define PMG_REQUIRE(cond, msg)                                                 \
  do {                                                                         \
    if (!(cond)) {                                                             \
      pmg::set_last_message(msg);                                              \
      return PMG_ERR_ARG;                                                      \
    }                                                                          \
  } while (0)

namespace pmg {
// Grid sizes an entry point accepts: 3 to kMaxN points per axis.
inline bool bad_dims(int nx, int ny, int nz) {
  return nx < 3 || ny < 3 || nz < 3 || nx > kMaxN || ny > kMaxN ||
         nz > kMaxN;
}
} // namespace pmg

// Raises Kernel's dynamic shared-memory limit to `bytes` on the current
// device, once per device (the attribute belongs to the device's context).
template <auto Kernel> cudaError_t set_smem_limit(int bytes) {
  static std::atomic<int> done[64]; // per device: the limit set so far
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return e;
  if (dev >= 0 && dev < 64 && done[dev].load() >= bytes)
    return cudaSuccess;
  e = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes);
  if (e == cudaSuccess && dev >= 0 && dev < 64)
    done[dev].store(bytes);
  return e;
}

#define PMG_LAUNCH_CHECK()                                                     \
  do {                                                                         \
    cudaError_t _e = cudaGetLastError();                                       \
    if (_e != cudaSuccess) {                                                   \
      pmg::set_last_error(_e, "kernel launch", __FILE__, __LINE__);            \
      return PMG_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

namespace pmg {
void set_last_error(cudaError_t e, const char *what, const char *file,
                    int line);
void set_last_message(const char *msg);
// Stream-ordered scratch of the library: a memory pool of its own per
// device that keeps freed memory (release threshold: unlimited), so
// allocations after the first never map memory again and synchronising a
// stream never trims it (trimming can wait on work of other streams).
cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t s);
cudaError_t scratch_free(void *ptr, cudaStream_t s);
} // namespace pmg
