// Host launchers of the hierarchy builders (one translation unit: the
// Galerkin kernel is a large unrolled template).
#include "build_kernels.cuh"
#include "launch.cuh"

namespace pmg {

int launch_buildP(const Dims &df, const Dims &dc, int kind,
                  const Op14<double> &A, const P27W<double> &P,
                  cudaStream_t s, const P27W<float> &P32, const Dims *dc32) {
  const Dims d32 = dc32 ? *dc32 : dc;
  const dim3 block(32, 4, 1);
  const dim3 grid(cdiv(dc.nx - 2, 32), cdiv(dc.ny - 2, 4),
                  (unsigned)(dc.nz - 2));
  if (kind == 7)
    buildP_op_kernel<7><<<grid, block, 0, s>>>(df, dc, A, P, P32, d32);
  else
    buildP_op_kernel<27><<<grid, block, 0, s>>>(df, dc, A, P, P32, d32);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

int launch_buildG(const Dims &df, const Dims &dc, int kind,
                  const P27<double> &P, const Op14<double> &A,
                  const Op14W<double> &out, cudaStream_t s,
                  const Op14W<float> &out32, const Dims *dc32) {
  const Dims d32 = dc32 ? *dc32 : dc;
  const dim3 block(32, 4, 1);
  const dim3 grid(cdiv(dc.nx - 2, 32), cdiv(dc.ny - 2, 4),
                  (unsigned)(dc.nz - 2));
  if (kind == 7) {
    buildG_kernel<7><<<grid, block, 0, s>>>(df, dc, P, A, out, out32, d32);
  } else {
    const long m = (long)(dc.nx - 2) * (dc.ny - 2) * (dc.nz - 2);
    buildG_entry_kernel<27><<<dim3(14, (unsigned)((m + 127) / 128)), 128, 0,
                              s>>>(df, dc, P, A, out, out32, d32);
  }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

} // namespace pmg
