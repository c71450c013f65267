// Hierarchy builders: operator-based prolongation and the Galerkin coarse
// operator, double precision, one thread per coarse interior point.
//
// Both follow the definitions rather than the reference's expanded formulas
// (pmgc/buildPd.cc, pmgc/buildGd.cc); the loop structure and summation order
// are identical to the CPU restatement in oracle/pmg_oracle.c, so GPU and
// restatement agree bit for bit, and both agree with the reference to
// rounding.
#pragma once

#include <utility>

#include "pmg_common.cuh"

namespace pmg {

// Operator-based prolongation for every fine neighbour f = c + d of a coarse
// point's fine image c (VbuildPb_op7 pmgc/buildPd.cc:173-555, VbuildPb_op27
// :579-1091):
//   P_d = [sum_{e toward c} a(f,f+e) w(proj(d+e))] / [oC(f) - sum_{e lumped}
//   a(f,f+e)]
// where "toward c" moves only toward c on the axes where d != 0 (and freely
// on the others), "lumped" stays on f's own line/plane, proj keeps d+e on
// the axes where d != 0, w(0) = 1. Faces, then edges, then corners.
// Reference quirk reproduced: in uPE of the 27-point builder the coupling of
// f to (i,j,k) is read as uS(i+1,j+1,k).
template <int KIND>
__global__ void __launch_bounds__(128)
    buildP_op_kernel(Dims df, Dims dc, Op14<double> A, P27W<double> P,
                     P27W<float> P32, Dims dc32) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int kk = blockIdx.z + 2;
  if (ii > dc.nx - 1 || jj > dc.ny - 1)
    return;
  const int pc = dc.at(ii, jj, kk);
  const int sy = df.sy(), sz = df.sz();
  const int c0 = df.at(2 * ii - 1, 2 * jj - 1, 2 * kk - 1);
  double w[27];
#pragma unroll
  for (int s = 0; s < 27; ++s)
    w[s] = 0.0;
  w[pslot(0, 0, 0)] = 1.0;
#pragma unroll
  for (int order = 1; order <= 3; ++order)
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          if ((dx != 0) + (dy != 0) + (dz != 0) != order)
            continue;
          const int fp = c0 + dx + dy * sy + dz * sz;
          double num = 0.0, lump = 0.0;
#pragma unroll
          for (int ez = -1; ez <= 1; ++ez)
#pragma unroll
            for (int ey = -1; ey <= 1; ++ey)
#pragma unroll
              for (int ex = -1; ex <= 1; ++ex) {
                if (!ex && !ey && !ez)
                  continue;
                // 7-point operators only couple along the axes
                if (KIND == 7 && (ex != 0) + (ey != 0) + (ez != 0) != 1)
                  continue;
                const bool on_s = (dx && ex) || (dy && ey) || (dz && ez);
                const bool toward = !(dx && ex && ex != -dx) &&
                                    !(dy && ey && ey != -dy) &&
                                    !(dz && ez && ez != -dz);
                if (on_s && !toward)
                  continue;
                double cpl;
                if (KIND == 27 && dx == 1 && dy == 0 && dz == 1 && ex == -1 &&
                    ey == 0 && ez == -1)
                  cpl = coupling(A, df, fp, 0, 1, -1);
                else
                  cpl = coupling(A, df, fp, ex, ey, ez);
                if (!on_s) {
                  lump += cpl;
                } else {
                  const int vx = dx ? dx + ex : 0, vy = dy ? dy + ey : 0,
                            vz = dz ? dz + ez : 0;
                  num += cpl * w[pslot(vx, vy, vz)];
                }
              }
          w[pslot(dx, dy, dz)] = num / (A.a[kOC][fp] - lump);
        }
#pragma unroll
  for (int s = 0; s < 27; ++s)
    P.p[s][pc] = w[s];
  if (P32.p[0]) { // the mixed path's float copy (rows dc32.px apart)
    const int pc32 = dc32.at(ii, jj, kk);
#pragma unroll
    for (int s = 0; s < 27; ++s)
      P32.p[s][pc32] = (float)w[s];
  }
}

// Constant weights 1, 1/2, 1/4, 1/8 (VbuildPb_trilin, pmgc/buildPd.cc:
// 63-153).
__global__ void buildP_trilin_kernel(Dims dc, P27W<double> P);

// Upper direction D of output slot S (oC oE oN uC oNE oNW uE uW uN uS uNE uNW
// uSE uSW).
__host__ __device__ constexpr int upper_dx(int s) {
  return (s == 1 || s == 4 || s == 6 || s == 10 || s == 12) ? 1
         : (s == 5 || s == 7 || s == 11 || s == 13)         ? -1
                                                             : 0;
}
__host__ __device__ constexpr int upper_dy(int s) {
  return (s == 2 || s == 4 || s == 5 || s == 8 || s == 10 || s == 11) ? 1
         : (s == 9 || s == 12 || s == 13)                             ? -1
                                                                      : 0;
}
__host__ __device__ constexpr int upper_dz(int s) {
  return (s == 3 || s >= 6) ? 1 : 0;
}

// The terms of Galerkin entry S that the fine neighbour f = c + (dx,dy,dz)
// contributes: sum_e P_d(C) A_f(f, f+e) P_{d+e-2D}(C+D), added to acc in e
// order, with A_f(f,f) = oC(f) and A_f(f,g) = -a(f,g) (VbuildG_7
// pmgc/buildGd.cc:438-1361, VbuildG_27 :1364-3274).
template <int KIND, int S>
__device__ __forceinline__ void galerkin_terms(double &acc, const Dims &df,
                                               const Dims &dc,
                                               const P27<double> &P,
                                               const Op14<double> &A, int pc,
                                               int fp, double pw, int dx,
                                               int dy, int dz) {
  constexpr int Dx = upper_dx(S), Dy = upper_dy(S), Dz = upper_dz(S);
  const int pn = pc + Dx + Dy * dc.sy() + Dz * dc.sz();
#pragma unroll
  for (int ez = -1; ez <= 1; ++ez)
#pragma unroll
    for (int ey = -1; ey <= 1; ++ey)
#pragma unroll
      for (int ex = -1; ex <= 1; ++ex) {
        const int tx = dx + ex - 2 * Dx, ty = dy + ey - 2 * Dy,
                  tz = dz + ez - 2 * Dz;
        if (tx < -1 || tx > 1 || ty < -1 || ty > 1 || tz < -1 || tz > 1)
          continue;
        const int nnz = (ex != 0) + (ey != 0) + (ez != 0);
        if (KIND == 7 && nnz > 1)
          continue;
        const double af = nnz == 0 ? A.a[kOC][fp]
                                   : -coupling(A, df, fp, ex, ey, ez);
        if (af == 0.0)
          continue;
        acc += pw * af * P.p[pslot(tx, ty, tz)][pn];
      }
}

// One Galerkin entry: A_c(C, C+D) = sum_{d,e} P_d(C) A_f(c+d, c+d+e)
// P_{d+e-2D}(C+D), the fine neighbours d in (z, y, x) order. Returns the
// stored value: A_c(C,C) for S = 0, -A_c(C,C+D) otherwise.
template <int KIND, int S>
__device__ __forceinline__ double galerkin_entry(const Dims &df,
                                                 const Dims &dc,
                                                 const P27<double> &P,
                                                 const Op14<double> &A,
                                                 int pc, int c0) {
  const int sy = df.sy(), sz = df.sz();
  double acc = 0.0;
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const int fp = c0 + dx + dy * sy + dz * sz;
        galerkin_terms<KIND, S>(acc, df, dc, P, A, pc, fp,
                                P.p[pslot(dx, dy, dz)][pc], dx, dy, dz);
      }
  return S == 0 ? acc : -acc;
}

template <int KIND, int... S>
__device__ __forceinline__ void
galerkin_terms_all(double *acc, const Dims &df, const Dims &dc,
                   const P27<double> &P, const Op14<double> &A, int pc,
                   int fp, double pw, int dx, int dy, int dz,
                   std::integer_sequence<int, S...>) {
  (galerkin_terms<KIND, S>(acc[S], df, dc, P, A, pc, fp, pw, dx, dy, dz),
   ...);
}

// All fourteen entries of one coarse point, the fine neighbour d outermost:
// each entry still adds its terms in galerkin_entry's (d, e) order, so the
// values are the same bits, while P_d(C) and the fine operator around c + d
// are loaded once for the fourteen instead of once per entry, and the
// stores come after all loads. out32 (all null: none) receives the float
// copy of each entry (rows dc32.px apart).
template <int KIND>
__global__ void __launch_bounds__(128)
    buildG_kernel(Dims df, Dims dc, P27<double> P, Op14<double> A,
                  Op14W<double> out, Op14W<float> out32, Dims dc32) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int kk = blockIdx.z + 2;
  if (ii > dc.nx - 1 || jj > dc.ny - 1)
    return;
  const int pc = dc.at(ii, jj, kk);
  const int c0 = df.at(2 * ii - 1, 2 * jj - 1, 2 * kk - 1);
  const int sy = df.sy(), sz = df.sz();
  double acc[14];
#pragma unroll
  for (int s = 0; s < 14; ++s)
    acc[s] = 0.0;
#pragma unroll
  for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const int fp = c0 + dx + dy * sy + dz * sz;
        galerkin_terms_all<KIND>(acc, df, dc, P, A, pc, fp,
                                 P.p[pslot(dx, dy, dz)][pc], dx, dy, dz,
                                 std::make_integer_sequence<int, 14>{});
      }
  const bool f32 = out32.a[0] != nullptr; // the mixed path's float copy
  const int pc32 = dc32.at(ii, jj, kk);
#pragma unroll
  for (int s = 0; s < 14; ++s) {
    const double v = s == 0 ? acc[s] : -acc[s];
    out.a[s][pc] = v;
    if (f32)
      out32.a[s][pc32] = (float)v;
  }
}

// One Galerkin entry per thread (blockIdx.x: the output slot, so the
// fourteen blocks of the same 128 coarse points run back to back and share
// the fine operator in L2), for the 27-point input: a block evaluates one
// entry's unrolled sum for 128 coarse points. With 27 couplings per fine
// point, buildG_kernel's fourteen accumulators need 216 registers (two CTAs
// per SM) and two entries per thread 168; both measured slower than this.
template <int KIND>
__global__ void __launch_bounds__(128)
    buildG_entry_kernel(Dims df, Dims dc, P27<double> P, Op14<double> A,
                        Op14W<double> out, Op14W<float> out32, Dims dc32) {
  const int mx = dc.nx - 2, my = dc.ny - 2;
  const int q = blockIdx.y * blockDim.x + threadIdx.x;
  if (q >= mx * my * (dc.nz - 2))
    return;
  const int r = q / mx, kq = r / my;
  const int ii = q - r * mx + 2, jj = r - kq * my + 2, kk = kq + 2;
  const int pc = dc.at(ii, jj, kk);
  const int c0 = df.at(2 * ii - 1, 2 * jj - 1, 2 * kk - 1);
  const int S = blockIdx.x;
  double v;
  switch (S) {
  case 0: v = galerkin_entry<KIND, 0>(df, dc, P, A, pc, c0); break;
  case 1: v = galerkin_entry<KIND, 1>(df, dc, P, A, pc, c0); break;
  case 2: v = galerkin_entry<KIND, 2>(df, dc, P, A, pc, c0); break;
  case 3: v = galerkin_entry<KIND, 3>(df, dc, P, A, pc, c0); break;
  case 4: v = galerkin_entry<KIND, 4>(df, dc, P, A, pc, c0); break;
  case 5: v = galerkin_entry<KIND, 5>(df, dc, P, A, pc, c0); break;
  case 6: v = galerkin_entry<KIND, 6>(df, dc, P, A, pc, c0); break;
  case 7: v = galerkin_entry<KIND, 7>(df, dc, P, A, pc, c0); break;
  case 8: v = galerkin_entry<KIND, 8>(df, dc, P, A, pc, c0); break;
  case 9: v = galerkin_entry<KIND, 9>(df, dc, P, A, pc, c0); break;
  case 10: v = galerkin_entry<KIND, 10>(df, dc, P, A, pc, c0); break;
  case 11: v = galerkin_entry<KIND, 11>(df, dc, P, A, pc, c0); break;
  case 12: v = galerkin_entry<KIND, 12>(df, dc, P, A, pc, c0); break;
  default: v = galerkin_entry<KIND, 13>(df, dc, P, A, pc, c0); break;
  }
  out.a[S][pc] = v;
  if (out32.a[0])
    out32.a[S][dc32.at(ii, jj, kk)] = (float)v;
}

} // namespace pmg
