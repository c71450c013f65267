// Reductions of the PMG path (defect norm, Hackbusch-Reusken damping) and
// the single-CTA coarsest-level CG.
//
// Reductions are deterministic: a fixed grid of blocks accumulates per-thread
// partials over a fixed grid-stride partition, each block writes its partial,
// and the last block to finish (atomic ticket) sums the partials in block
// order. The result therefore depends only on the problem, never on timing or
// on other work sharing the GPU.
#pragma once

#include "stencil_kernels.cuh"

namespace pmg {

constexpr int kReduceThreads = 256;
// Interior reductions launch one thread per point (interior_grid, blocks of
// 32 x 8) and keep one partial sum per block and reduced quantity.

// Device scratch of one reduction site: partials[blocks * NV], ticket
// counter (zero between uses), result[NV].
struct ReduceSlot {
  double *partials;
  unsigned int *ticket;
  double *result;
};

__device__ __forceinline__ void interior_coords(const Dims &d, int q, int &i,
                                                int &j, int &k) {
  const int mx = d.nx - 2, my = d.ny - 2;
  const int r = q / mx;
  i = q - r * mx + 2;
  k = r / my;
  j = r - k * my + 2;
  k += 2;
}

// Finishes a reduction of NV values: called by every block after it has
// computed its block sums v[] (valid in thread 0). The last block sums all
// partials in block order and writes result[]; when ratio != nullptr it also
// stores result[0] / result[1] there (NV == 2).
template <int NV>
__device__ void reduce_finish(const double (&v)[NV], ReduceSlot s,
                              double *ratio) {
  __shared__ bool last;
  __shared__ double sh[32];
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y *
                                                            blockIdx.z);
  const unsigned tid = threadIdx.x + blockDim.x * threadIdx.y;
  const unsigned nt = blockDim.x * blockDim.y;
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q)
      s.partials[(size_t)b * NV + q] = v[q];
    __threadfence();
    const unsigned t = atomicAdd(s.ticket, 1u);
    last = (t == nb - 1);
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  const volatile double *pv = s.partials;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    // each thread adds partials tid, tid + nt, ... in that order; eight
    // loads are issued before their adds, so the tail waits on one load
    // latency per eight partials instead of one per partial
    double acc = 0.0;
    unsigned k = tid;
    for (; k + 7 * nt < nb; k += 8 * nt) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        v[u] = pv[(size_t)(k + u * nt) * NV + q];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        acc += v[u];
    }
    for (; k < nb; k += nt)
      acc += pv[(size_t)k * NV + q];
    acc = block_sum_2d(acc, sh);
    if (tid == 0)
      s.result[q] = acc;
  }
  if (tid == 0) {
    if (ratio)
      *ratio = s.result[0] / s.result[1];
    *s.ticket = 0u;
  }
}

// Reductions take one interior column (i, j) per thread and a run of
// kReducePlanes planes per block (grid: reduce_grid), so each block's partial
// covers enough points to amortise the final step.
constexpr int kReducePlanes = 8;

// sum over the interior of (f - A x)^2 with the defect of the class
// (f - map(x), Convolution.h:137-139 and 170-175); optionally stores the
// defect (cast to Tout) into r. Accumulates in double.
template <int KIND, typename T, typename Tout, bool SPLIT_OUT = false>
__global__ void __launch_bounds__(kReduceThreads)
    defect_norm_kernel(Dims d, Op14<T> A, const T *__restrict__ f,
                       const T *__restrict__ x, Tout *__restrict__ r,
                       ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  const int sy = d.sy(), sz = d.sz();
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1) {
    for (int k = k0; k <= k1; ++k) {
      const int p = d.at(i, j, k);
      const T dv =
          f[p] - apply_op<KIND>(A, (const T *)nullptr, x, p, sy, sz);
      if (r) {
        if constexpr (SPLIT_OUT) {
          // colour-split rows (split_layout.cuh): halves of hp entries (a
          // multiple of 16), point i at entry (i - 1) >> 1 of its colour's
          const int hp = ((d.nx + 1) / 2 + 15) & ~15;
          r[((k - 1) * d.ny + (j - 1)) * 2 * hp + ((i + j + k) & 1) * hp +
            ((i - 1) >> 1)] = (Tout)dv;
        } else {
          r[p] = (Tout)dv;
        }
      }
      acc += (double)dv * (double)dv;
    }
  }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

// Defect only (no reduction): r = f - map(x) on the interior
// (Subtract_Convolve_map, Convolution.h:123-146).
template <int KIND, typename T>
__global__ void __launch_bounds__(256)
    defect_kernel(Dims d, Op14<T> A, const T *__restrict__ f,
                  const T *__restrict__ x, T *__restrict__ r) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  r[p] = f[p] - apply_op<KIND>(A, (const T *)nullptr, x, p, d.sy(), d.sz());
}

// Hackbusch-Reusken damping w = (r . x) / (x . A x) over the interior of a
// 27-point level (get_ideal_lambda, MultigridDomain.h:327-352), accumulated
// in double; the last block stores w. Grid: lambda_grid with PL =
// lambda_planes planes per block. The plane loop has a compile-time length,
// so the loads of a thread's planes can be in flight together; each
// thread's sums still run over its planes in order.
template <typename T, int PL>
__device__ __forceinline__ void ideal_lambda_body(const Dims &d,
                                                  const Op14<T> &A,
                                                  const T *__restrict__ x,
                                                  const T *__restrict__ r,
                                                  const ReduceSlot &s,
                                                  double *__restrict__ w) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * PL;
  const int sy = d.sy(), sz = d.sz();
  double up = 0.0, lo = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1) {
#pragma unroll
    for (int q = 0; q < PL; ++q) {
      const int k = k0 + q;
      if (k <= d.nz - 1) {
        const int p = d.at(i, j, k);
        up += (double)r[p] * (double)x[p];
        lo += (double)x[p] *
              (double)apply27(A, (const T *)nullptr, x, p, sy, sz);
      }
    }
  }
  double v[2];
  v[0] = block_sum_2d(up, sh);
  v[1] = block_sum_2d(lo, sh);
  reduce_finish<2>(v, s, w);
}
template <typename T, int PL>
__global__ void __launch_bounds__(kReduceThreads)
    ideal_lambda_kernel(Dims d, Op14<T> A, const T *__restrict__ x,
                        const T *__restrict__ r, ReduceSlot s,
                        double *__restrict__ w) {
  ideal_lambda_body<T, PL>(d, A, x, r, s, w);
}
// The float four-plane case (levels from 97 points per axis) held to 32
// registers, eight blocks per SM: 63 -> 55 us at 129^3.
template <int PL>
__global__ void __launch_bounds__(kReduceThreads, 8)
    ideal_lambda_r32_kernel(Dims d, Op14<float> A,
                            const float *__restrict__ x,
                            const float *__restrict__ r, ReduceSlot s,
                            double *__restrict__ w) {
  ideal_lambda_body<float, PL>(d, A, x, r, s, w);
}

// Coarsest-level CG of the class, one CTA (CG_solver, CG_Solver.h:45-242 via
// solve_by_cg<1>, PBE_pmgc_class.h:856-860):
//   r = rhs - A x; p = r; rs = r.r; Ap = A p; pAp = Ap.p; stop if pAp == 0;
//   alpha = rs/pAp; res = sqrt(sqrt(rs)) (class_first_check) or sqrt(rs);
//   while res > max(thresh, rel_tol sqrt(rs_0)):
//     x += alpha p; r -= alpha Ap; rs' = r.r; beta = rs'/rs (0 if rs == 0);
//     p = r + beta p; Ap = A p; pAp = Ap.p; alpha = rs/pAp (0 if pAp == 0);
//     res = sqrt(rs)
// bounded by max_iters (the reference loops without a cap). The reference
// applies A to the same p twice per iteration; keeping Ap gives the same
// values with one matvec. The class runs thresh = 1e-8, rel_tol = 0,
// class_first_check = 1. r, p, Ap are scratch arrays whose shells are zero.
// status[0] = iterations, status[1] = 1 when the cap stopped the loop above
// the threshold. Grids up to 33^3 (at most 32 interior points per thread).
int launch_cg_level(const Dims &d, const Op14<double> &A, const double *rhs,
                    double *x, double *r, double *p, double *ap,
                    double thresh, double rel_tol, int class_first_check,
                    int max_iters, int *status, cudaStream_t s);

} // namespace pmg
