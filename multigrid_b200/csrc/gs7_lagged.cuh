// One red-black sweep of the 7-point operator per launch with the second
// colour trailing the first by a few planes, so its reads hit L2.
//
// The reference runs one launch per colour (Vgsrb7x, pmgc/gsd.cc:81-110): the
// second launch streams every coefficient array from DRAM again. Here one
// persistent launch walks a queue of work items in plane order -- the first
// colour of plane k, then the second colour of plane k - kLag -- taken from an
// atomic ticket, so the first and second colour fronts move up the grid a few
// planes apart and the second colour re-reads data the first one has just
// brought into L2. The second colour of plane k depends on the first colour
// of planes k-1, k, k+1 (its neighbours, and the readers of its old values);
// every item of the first colour bumps its plane's counter when its writes
// are visible, and a second-colour item waits for the three counters. Items
// are taken in queue order by running CTAs, so every item waited for is
// already held by a running CTA: the waits end. They are bounded all the
// same; a wait that runs out sets *err and carries on.
//
// Updates are in place with the reference's per-point arithmetic
// (gs7_color_kernel), so a sweep is bit-identical to the two colour launches.
// x is read around L1 (ld.global.cg): the same CTA may have cached a line of
// x before another CTA updated it.
#pragma once

#include <algorithm>

#include "stencil_kernels.cuh"

namespace pmg {

constexpr int kLag = 4;         // planes between the two colour fronts
constexpr int kLagRows = 32;    // rows of a plane per work item
constexpr int kLagThreadsX = 32, kLagThreadsY = 8;

template <typename T>
__global__ void __launch_bounds__(kLagThreadsX *kLagThreadsY)
    gs7_lagged_kernel(Dims d, const T *__restrict__ oC,
                      const T *__restrict__ cc, const T *__restrict__ fc,
                      const T *__restrict__ oE, const T *__restrict__ oN,
                      const T *__restrict__ uC, T *x, int want_first,
                      T keep_first, int *ticket, int *done, int *err) {
  __shared__ int s_item;
  const int planes = d.nz - 2;
  const int bands = (d.ny - 2 + kLagRows - 1) / kLagRows;
  const int steps = planes + kLag;
  const int total = 2 * bands * steps; // includes empty slots at the ends
  const int sy = d.sy(), sz = d.sz();
  const int tid = threadIdx.x + kLagThreadsX * threadIdx.y;
  for (;;) {
    __syncthreads();
    if (tid == 0)
      s_item = atomicAdd(ticket, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= total)
      break;
    // item -> (step, colour, band): at step s the first colour of plane
    // 2 + s and the second colour of plane 2 + s - kLag
    const int step = item / (2 * bands);
    const int rem = item - step * 2 * bands;
    const int second = rem >= bands;
    const int band = second ? rem - bands : rem;
    const int k = 2 + step - (second ? kLag : 0);
    if (k < 2 || k > d.nz - 1)
      continue;
    if (second) {
      if (tid == 0) {
        // first colour of planes k-1, k, k+1 (interior ones) complete
        bool ok = true;
        for (int kk = k - 1; kk <= k + 1; ++kk) {
          if (kk < 2 || kk > d.nz - 1)
            continue;
          const volatile int *c = done + kk;
          int spins = 0;
          while (*c < bands) {
            if (++spins > (1 << 22)) {
              ok = false;
              break;
            }
            __nanosleep(64);
          }
        }
        if (!ok)
          atomicExch(err, 1);
        __threadfence();
      }
      __syncthreads();
    }
    const int want = second ? 1 - want_first : want_first;
    const T keep = second ? T(1) : keep_first;
    const int j_lo = 2 + band * kLagRows;
    const int j_hi = min(j_lo + kLagRows - 1, d.ny - 1);
    for (int j = j_lo + threadIdx.y; j <= j_hi; j += kLagThreadsY) {
      const int i0 = 2 + ((2 + j + k + want) & 1);
      for (int i = i0 + 2 * threadIdx.x; i <= d.nx - 1;
           i += 2 * kLagThreadsX) {
        const int p = d.at(i, j, k);
        const T s = oN[p] * __ldcg(x + p + sy) + oN[p - sy] * __ldcg(x + p - sy) +
                    oE[p] * __ldcg(x + p + 1) + oE[p - 1] * __ldcg(x + p - 1) +
                    uC[p - sz] * __ldcg(x + p - sz) +
                    uC[p] * __ldcg(x + p + sz);
        const T c = cc ? cc[p] : T(0);
        x[p] = (fc[p] + keep * s) / (oC[p] + c);
      }
    }
    if (!second) {
      __threadfence(); // this thread's updates before the plane's counter
      __syncthreads();
      if (tid == 0)
        atomicAdd(done + k, 1);
    }
  }
}

// Device scratch of a lagged launch: ticket, error flag, nz plane counters.
inline size_t gs7_lagged_scratch_ints(const Dims &d) { return 2 + d.nz; }

// nsweeps sweeps in place (Vgsrb7x semantics); sync holds
// gs7_lagged_scratch_ints(d) ints (zeroed here before every sweep); err
// (may be null) collects the wait-timeout flag.
template <typename T>
int launch_gs7_lagged(const Dims &d, const T *oC, const T *cc, const T *fc,
                      const T *oE, const T *oN, const T *uC, T *x, int itmax,
                      int iadjoint, int zero_init, int *sync,
                      cudaStream_t s) {
  int per_sm = 0;
  PMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, gs7_lagged_kernel<T>, kLagThreadsX * kLagThreadsY, 0));
  const int bands = (d.ny - 2 + kLagRows - 1) / kLagRows;
  const int items = 2 * bands * (d.nz - 2 + kLag);
  int dev = 0, sms = 148;
  PMG_CUDA_TRY(cudaGetDevice(&dev));
  PMG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount,
                                      dev));
  const int grid = std::min(items, std::max(1, per_sm) * sms);
  const size_t bytes = sizeof(int) * gs7_lagged_scratch_ints(d);
  for (int it = 0; it < itmax; ++it) {
    // ticket and counters restart; the error flag (sync[1]) accumulates
    PMG_CUDA_TRY(cudaMemsetAsync(sync, 0, sizeof(int), s));
    PMG_CUDA_TRY(cudaMemsetAsync(sync + 2, 0, bytes - 2 * sizeof(int), s));
    const T keep = (it == 0 && zero_init) ? T(0) : T(1);
    gs7_lagged_kernel<T>
        <<<grid, dim3(kLagThreadsX, kLagThreadsY), 0, s>>>(
            d, oC, cc, fc, oE, oN, uC, x, iadjoint, keep, sync, sync + 2,
            sync + 1);
  }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

} // namespace pmg
