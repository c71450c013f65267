// The refinement residual of the mixed and fp64-fast paths, streamed: r =
// f - A x64 on the finest level in double (the class's defect,
// Convolution.h:137-139, with the couplings and oC from the code bytes),
// written rounded to the correction equation's colour-split right-hand side
// (float or double), and its sum of squares (compute_residual_map,
// Convolution.h:156-185). With r null only the sum: the FP64 cycle's stop
// test.
//
// The per-thread kernel (defect_norm_code_kernel) moves the coded format's
// 21 bytes per point and no more but is bound by load latency (ncu: long-
// scoreboard stalls 21 per issue, 38% issue, 2.6 TB/s). Here each CTA owns J
// rows of a chunk of planes and marches along k. Per plane a producer warp
// issues three bulk copies onto the "full" mbarrier of a ring slot: the
// J + 2 rows of x64 around the block (contiguous in the reference layout:
// one copy of ~12 KB), its J rows of f (one copy), and both colour halves of
// its J rows of code bytes (contiguous in the split layout). Consumer warps
// (two per row) compute plane k from the slots of k - 1, k and k + 1 and
// release the slot of k - 1 on its "empty" mbarrier; the producer refills a
// slot once it is released. The per-point arithmetic is
// defect_norm_code_kernel's (apply7's order), so r is the same bits; the
// sum of squares adds the same terms in a different order (per thread over
// its points and planes, then warps, then CTAs in CTA order: deterministic).
//
// Copies run from the 16-byte boundary at or below their first entry; the
// planes past the chunk (halo planes) bring only the block's rows, so no
// copy reads outside the arrays. Every wait is bounded: a warp whose plane
// does not arrive sets *err and stops computing, the producer whose slot is
// not released sets *err and waits (bounded) for its copies in flight, and
// every thread still takes part in the block's reduction, so the kernel
// always ends; the solve's stop test reports PMG_ERR_TIMEOUT.
#pragma once

#include "gs7_stream.cuh"

namespace pmg {

struct ResidCfg {
  static constexpr int J = 4;   // rows per CTA
  static constexpr int WPR = 2; // consumer warps per row
  static constexpr int NC = J * WPR;
  static constexpr int S = 5; // ring stages
  static constexpr int THREADS = 32 * (NC + 1);
};

struct ResidShape {
  int nj, kchunk;
  int xoff, foff, coff, slot; // byte offsets inside a stage, stage bytes
};

inline ResidShape resid_shape(const Dims &d, int resident_ctas) {
  constexpr int J = ResidCfg::J;
  ResidShape sh{};
  sh.nj = (int)cdiv(d.ny - 2, J);
  const int planes = d.nz - 2;
  int nkc = resident_ctas / sh.nj;
  nkc = nkc < 1 ? 1 : nkc > planes ? planes : nkc;
  sh.kchunk = (int)cdiv(planes, nkc);
  auto up128 = [](long b) { return (int)((b + 127) & ~127L); };
  const Split sp = Split::of(d);
  sh.xoff = 0;
  sh.foff = up128(((long)(J + 2) * d.nx + 2) * 8);
  sh.coff = sh.foff + up128(((long)J * d.nx + 2) * 8);
  sh.slot = sh.coff + up128((long)J * sp.pitch());
  return sh;
}
inline size_t resid_smem_bytes(const ResidShape &sh) {
  return (size_t)ResidCfg::S * sh.slot + 2 * ResidCfg::S * sizeof(uint64_t);
}
// dynamic shared memory a CTA may hold next to the kernel's static tables
constexpr size_t kResidMaxSmem = 220 * 1024;
inline bool resid_fits(const Dims &d) {
  return resid_smem_bytes(resid_shape(d, 1)) <= kResidMaxSmem;
}
// CTAs of a streamed residual launch on level d, at most (the partials of
// its reduction slot must hold one entry per CTA)
inline long resid_max_ctas(const Dims &d) {
  return (long)cdiv(d.ny - 2, ResidCfg::J) * (d.nz - 2);
}

// a bulk copy of elements [g0, g1) of an array of esz-byte entries, from the
// 16-byte boundary at or below g0 to the one at or above g1, into the image
// of the array whose element gb (16-byte aligned) is at dst
__device__ __forceinline__ void image_copy(unsigned char *dst,
                                           const void *arr, long gb, long g0,
                                           long g1, int esz, uint64_t *bar) {
  const long a0 = (g0 * esz) & ~15L, a1 = (g1 * esz + 15) & ~15L;
  bulk_load(dst + (a0 - gb * esz), static_cast<const char *>(arr) + a0,
            (unsigned)(a1 - a0), bar);
}
// bytes image_copy moves
__device__ __forceinline__ unsigned image_bytes(long g0, long g1, int esz) {
  return (unsigned)(((g1 * esz + 15) & ~15L) - ((g0 * esz) & ~15L));
}

template <typename R>
__global__ void __launch_bounds__(ResidCfg::THREADS, 2)
    defect_norm_stream_kernel(Dims d, ResidShape sh, Op14<double> A,
                              const double *__restrict__ f,
                              const double *__restrict__ x,
                              const unsigned char *__restrict__ code,
                              const double *__restrict__ lut64,
                              const double *__restrict__ octab,
                              const int *__restrict__ info,
                              R *__restrict__ r, ReduceSlot red, int *err,
                              unsigned extra_tx) {
  constexpr int J = ResidCfg::J, WPR = ResidCfg::WPR, NC = ResidCfg::NC;
  constexpr int S = ResidCfg::S;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ double octab_s[128];
  __shared__ double shred[32];
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + S * sh.slot);
  uint64_t *empty = full + S;
  const Split sp = Split::of(d);
  const int nx = d.nx;
  const int jb = blockIdx.x % sh.nj, kc = blockIdx.x / sh.nj;
  const int j0 = 2 + jb * J;
  const int jn = min(J, d.ny - j0); // own rows j0 .. j0 + jn - 1 <= ny - 1
  const int ka = 2 + kc * sh.kchunk;
  const int kb = min(ka + sh.kchunk - 1, d.nz - 1);
  const int kfirst = ka - 1, klast = kb + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NC);
    }
    fence_mbar_init();
  }
  const bool coded = info[6] == 0 && info[7] == 0;
  const bool oc_coded = coded && info[8] == 0;
  // low / high double value per direction, in registers (selected below,
  // never indexed at run time)
  const double el = coded ? lut64[0] : 0.0, eh = coded ? lut64[1] : 0.0;
  const double nl = coded ? lut64[2] : 0.0, nh = coded ? lut64[3] : 0.0;
  const double ul = coded ? lut64[4] : 0.0, uh = coded ? lut64[5] : 0.0;
  if (oc_coded && threadIdx.x < 128)
    octab_s[threadIdx.x] = octab[threadIdx.x];
  __syncthreads();
  auto slot_of = [&](int kk) { return (kk - kfirst) % S; };
  auto use_of = [&](int kk) { return (kk - kfirst) / S; };
  // image bases (even entries, so 16-byte aligned) of a plane's x rows
  // (from row j0 - 1) and f rows (from row j0)
  auto xbase = [&](int kk) { return (long)d.at(1, j0 - 1, kk) & ~1L; };
  auto fbase = [&](int kk) { return (long)d.at(1, j0, kk) & ~1L; };

  double acc = 0.0;
  if (warp == NC) {
    // producer
    if (lane == 0) {
      // every copy still in flight lands before the producer moves on;
      // one poll budget for all of them
      auto drain = [&](int last) {
        long polls = 0;
        for (int kk = max(kfirst, last - S + 1); kk <= last; ++kk)
          while (!mbar_try_wait(&full[slot_of(kk)], use_of(kk) & 1u)) {
            if (++polls > kTmaMaxPolls)
              return;
            if (polls > 64)
              __nanosleep(64);
          }
      };
      int kk = kfirst;
      for (; kk <= klast; ++kk) {
        const int s = slot_of(kk), u = use_of(kk);
        if (u > 0 && !mbar_wait(&empty[s], (u - 1) & 1u)) {
          atomicOr(err, 1);
          break;
        }
        unsigned char *slot = sm + s * sh.slot;
        const bool own = kk >= ka && kk <= kb;
        // x rows: the block's and, on the planes it computes, the rows
        // above and below them
        const int xf = own ? j0 - 1 : j0, xl = own ? j0 + jn : j0 + jn - 1;
        const long gx0 = d.at(1, xf, kk), gx1 = (long)d.at(1, xl, kk) + nx;
        unsigned tx = image_bytes(gx0, gx1, 8);
        long gf0 = 0, gf1 = 0, gc0 = 0, gc1 = 0;
        if (own) {
          gf0 = d.at(1, j0, kk);
          gf1 = (long)d.at(1, j0 + jn - 1, kk) + nx;
          gc0 = sp.row(j0, kk);
          gc1 = (long)sp.row(j0 + jn - 1, kk) + sp.pitch();
          tx += image_bytes(gf0, gf1, 8) + image_bytes(gc0, gc1, 1);
        }
        mbar_expect_tx(&full[s], tx + extra_tx);
        image_copy(slot + sh.xoff, x, xbase(kk), gx0, gx1, 8, &full[s]);
        if (own) {
          image_copy(slot + sh.foff, f, fbase(kk), gf0, gf1, 8, &full[s]);
          image_copy(slot + sh.coff, code, gc0, gc0, gc1, 1, &full[s]);
        }
      }
      drain(kk - 1);
    }
  } else {
    // consumers: warp w takes row j0 + w / WPR, its (w % WPR)-th run of
    // 128 points of each 128 WPR
    const int rr = warp / WPR, hw = warp % WPR;
    const int jj = j0 + rr;
    int ready = kfirst - 1;
    bool ok = true;
    for (int k = ka; k <= kb && ok; ++k) {
      for (int kk = ready + 1; kk <= k + 1 && ok; ++kk)
        ok = mbar_wait(&full[slot_of(kk)], use_of(kk) & 1u);
      if (!ok) {
        if (lane == 0)
          atomicOr(err, 1);
        break;
      }
      ready = k + 1;
      if (rr < jn) {
        const double *X =
            reinterpret_cast<const double *>(sm + slot_of(k) * sh.slot);
        const double *Xd =
            reinterpret_cast<const double *>(sm + slot_of(k - 1) * sh.slot);
        const double *Xu =
            reinterpret_cast<const double *>(sm + slot_of(k + 1) * sh.slot);
        const double *F = reinterpret_cast<const double *>(
            sm + slot_of(k) * sh.slot + sh.foff);
        const unsigned char *C = sm + slot_of(k) * sh.slot + sh.coff +
                                 (jj - j0) * sp.pitch();
        // entry q = i - 1 of row jj on planes k, k - 1, k + 1, and of f
        const double *xc = X + (d.at(1, jj, k) - xbase(k));
        const double *xd = Xd + (d.at(1, jj, k - 1) - xbase(k - 1));
        const double *xu = Xu + (d.at(1, jj, k + 1) - xbase(k + 1));
        const double *fr = F + (d.at(1, jj, k) - fbase(k));
        // lanes over 32 consecutive points (conflict-free 8-byte shared
        // loads, contiguous stores into each colour half), four rounds
        for (int i0 = 2 + 128 * hw; i0 <= nx - 1; i0 += 128 * WPR) {
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const int i = i0 + 32 * m + lane, q = i - 1;
            if (i > nx - 1)
              break;
            const double xn = xc[q + nx], xs = xc[q - nx], xe = xc[q + 1];
            const double xw = xc[q - 1], xdn = xd[q], xup = xu[q];
            const double xcc = xc[q], fv = fr[q];
            const int p = d.at(i, jj, k);
            double c[6];
            double oc;
            if (coded) {
              const unsigned b = C[((i + jj + k) & 1) * sp.hp + (q >> 1)];
              oc = oc_coded ? octab_s[b & 127u] : A.a[kOC][p];
              c[0] = (b & 1u) ? eh : el;
              c[1] = (b & 2u) ? eh : el;
              c[2] = (b & 4u) ? nh : nl;
              c[3] = (b & 8u) ? nh : nl;
              c[4] = (b & 16u) ? uh : ul;
              c[5] = (b & 32u) ? uh : ul;
            } else {
              couplings64_of(d, A.a[kOE], A.a[kON], A.a[kUC], p, c);
              oc = A.a[kOC][p];
            }
            // apply7's order: -oN x_n - oN_s x_s - oE x_e - oE_w x_w
            // - uC_d x_d - uC x_u + (oC + 0) x
            const double ax = -c[2] * xn - c[3] * xs - c[0] * xe -
                              c[1] * xw - c[5] * xdn - c[4] * xup +
                              (oc + 0.0) * xcc;
            const double dv = fv - ax;
            if (r)
              r[sp.at(i, jj, k)] = (R)dv;
            acc += dv * dv;
          }
        }
      }
      __syncwarp();
      if (lane == 0)
        mbar_arrive(&empty[slot_of(k - 1)]);
    }
  }
  // every thread: the block's sum, then the grid's in block order
  double v[1] = {block_sum_2d(acc, shred)};
  reduce_finish<1>(v, red, nullptr);
}

// The streamed refinement residual on level d (resid_fits(d)); the
// partials of red hold resid_max_ctas(d) entries.
template <typename R>
int launch_resid_stream(const Dims &d, const Op14<double> &A, const double *f,
                        const double *x, const unsigned char *code,
                        const double *lut64, const double *octab,
                        const int *info, R *r, ReduceSlot red, int *err,
                        unsigned extra_tx, cudaStream_t s) {
  auto kern = defect_norm_stream_kernel<R>;
  int dev = 0, sms = 0, per_sm = 0;
  PMG_CUDA_TRY(cudaGetDevice(&dev));
  ResidShape sh = resid_shape(d, 1);
  const size_t smem = resid_smem_bytes(sh);
  {
    const cudaError_t e =
        set_smem_limit<defect_norm_stream_kernel<R>>((int)smem);
    PMG_CUDA_TRY(e);
  }
  PMG_CUDA_TRY(
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PMG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, kern, ResidCfg::THREADS, smem));
  sh = resid_shape(d, sms * (per_sm < 1 ? 1 : per_sm));
  const unsigned g = (unsigned)sh.nj * cdiv(d.nz - 2, sh.kchunk);
  if ((long)g > resid_max_ctas(d)) {
    set_last_message("launch_resid_stream: more CTAs than reduction slots");
    return PMG_ERR_STATE;
  }
  kern<<<g, ResidCfg::THREADS, smem, s>>>(d, sh, A, f, x, code, lut64, octab,
                                           info, r, red, err, extra_tx);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

} // namespace pmg
