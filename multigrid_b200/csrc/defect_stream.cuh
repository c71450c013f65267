// The finest-level defect of the refinement paths' V-cycle, streamed: r =
// f - A x on the colour-split coded level (Subtract_Convolve_map,
// Convolution.h:123-146, in apply7's order; defect7_code_kernel's
// arithmetic), written in the reference layout for the restriction.
//
// The per-thread kernel (defect7_code_kernel) moves the coded format's 13
// bytes per point at ~2.5 TB/s, bound by load latency. Here, as in the
// streamed colour pass (gs7_stream.cuh), each CTA owns J rows of a chunk of
// planes and marches along k: per plane a producer warp issues three bulk
// copies (cp.async.bulk) that take both colour halves, x over the J + 2 rows
// around the block, f and the code bytes over its J rows: in the
// colour-split layout a row's two halves are adjacent and rows follow one
// another, so each is one contiguous run (a tensor box would move it half
// row by half row, ~20 ns each). They land in a ring slot with full / empty
// mbarriers, and consumer warps (two per row, lanes over
// 32 consecutive points, so the reference-layout stores coalesce) compute
// plane k from the slots of k - 1, k and k + 1. A point's seven
// coefficients come from the 128-entry table indexed by its code byte.
// The arithmetic is defect7_code_kernel's, term for term: the same bits.
//
// Every wait is bounded, as in the colour pass: a consumer warp whose
// plane did not arrive sets *err and returns; the producer, whose slot is
// then never released, sets *err, waits (bounded) for its copies in
// flight, and returns.
#pragma once

#include "gs7_stream.cuh"

namespace pmg {

template <typename T> struct DefectCfg {
  static constexpr int J = 4;   // rows per CTA
  static constexpr int WPR = 2; // consumer warps per row
  static constexpr int NC = J * WPR;
  // stages: three float CTAs per SM at 257^3 (a stage holds rows of 2 hp
  // entries, the global layout)
  static constexpr int S = sizeof(T) == 4 ? 5 : 4;
  static constexpr int THREADS = 32 * (NC + 1);
  static constexpr int MIN_CTAS = sizeof(T) == 4 ? 3 : 2;
};

// Geometry of a streamed defect launch: a stage row is a row of the
// colour-split array, two halves of hp entries (bw = bwc = hp).
template <typename T> StreamShape defect_shape(const Dims &d, int resident) {
  constexpr int J = DefectCfg<T>::J;
  StreamShape sh{};
  sh.bw = Split::of(d).hp;
  sh.bwc = sh.bw;
  sh.nj = (int)cdiv(d.ny - 2, J);
  const int planes = d.nz - 2;
  int nkc = resident / sh.nj;
  nkc = nkc < 1 ? 1 : nkc > planes ? planes : nkc;
  sh.kchunk = (int)cdiv(planes, nkc);
  auto up128 = [](int b) { return (b + 127) & ~127; };
  sh.xbytes = (unsigned)((J + 2) * 2 * sh.bw * sizeof(T));
  const unsigned fb = (unsigned)(J * 2 * sh.bw * sizeof(T));
  const unsigned cb = (unsigned)(J * 2 * sh.bwc);
  sh.fcbytes = fb + cb;
  sh.xoff = 0;
  sh.foff = up128((int)sh.xbytes);
  sh.coff = sh.foff + up128((int)fb);
  sh.slot = sh.coff + up128((int)cb);
  return sh;
}
template <typename T> size_t defect_smem_bytes(const StreamShape &sh) {
  return (size_t)DefectCfg<T>::S * sh.slot +
         2 * DefectCfg<T>::S * sizeof(uint64_t);
}
template <typename T> bool defect_fits(const Dims &d) {
  const StreamShape sh = defect_shape<T>(d, 1);
  return sh.bw <= 256 && sh.bwc <= 256 &&
         defect_smem_bytes<T>(sh) <= kStreamMaxSmem;
}

template <typename T>
__global__ void __launch_bounds__(DefectCfg<T>::THREADS,
                                  DefectCfg<T>::MIN_CTAS)
    defect7_stream_kernel(Dims d, StreamShape sh, const T *__restrict__ xg,
                          const T *__restrict__ fg,
                          const unsigned char *__restrict__ codeg,
                          const T *__restrict__ oC,
                          const T *__restrict__ oE, const T *__restrict__ oN,
                          const T *__restrict__ uC,
                          const int *__restrict__ info,
                          const T *__restrict__ lut,
                          const T *__restrict__ octab, T *__restrict__ r,
                          int *err, unsigned extra_tx) {
  constexpr int J = DefectCfg<T>::J, WPR = DefectCfg<T>::WPR;
  constexpr int NC = DefectCfg<T>::NC, S = DefectCfg<T>::S;
  extern __shared__ __align__(128) unsigned char sm[];
  // per code byte (its low seven bits): n, s, e, w, down, up, oC, spare
  __shared__ __align__(16) T ctab[128][8];
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + S * sh.slot);
  uint64_t *empty = full + S;
  const Split sp = Split::of(d);
  const int nx = d.nx;
  const int jb = blockIdx.x % sh.nj, kc = blockIdx.x / sh.nj;
  const int j0 = 2 + jb * J;
  const int jn = min(J, d.ny - j0);
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
  typename LutOf<T>::type L;
  const bool coded = load_lut(info, lut, L);
  const bool oc_coded = coded && info[8] == 0;
  if (oc_coded && threadIdx.x < 128) {
    const unsigned b = threadIdx.x;
    T *t = ctab[b];
    t[0] = (b & 4u) ? L.nh : L.nl;
    t[1] = (b & 8u) ? L.nh : L.nl;
    t[2] = (b & 1u) ? L.eh : L.el;
    t[3] = (b & 2u) ? L.eh : L.el;
    t[4] = (b & 32u) ? L.uh : L.ul;
    t[5] = (b & 16u) ? L.uh : L.ul;
    t[6] = octab[b];
    t[7] = T(0);
  }
  __syncthreads();
  auto slot_of = [&](int kk) { return (kk - kfirst) % S; };
  auto use_of = [&](int kk) { return (kk - kfirst) / S; };

  if (warp == NC) {
    // producer: both halves of x over rows j0 - 1 .. min(j0 + J, ny), of f
    // and the code bytes over rows j0 .. j0 + jn - 1 (planes the block
    // computes); the stage rows past them are never read
    if (lane != 0)
      return;
    const int nrx = min(J + 2, d.ny - j0 + 2);
    const unsigned xb = (unsigned)(nrx * sp.pitch() * sizeof(T));
    const unsigned fb = (unsigned)(jn * sp.pitch() * sizeof(T));
    const unsigned cb = (unsigned)(jn * sp.pitch());
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
    for (int kk = kfirst; kk <= klast; ++kk) {
      const int s = slot_of(kk), u = use_of(kk);
      if (u > 0 && !mbar_wait(&empty[s], (u - 1) & 1u)) {
        atomicOr(err, 1);
        drain(kk - 1);
        return;
      }
      unsigned char *slot = sm + s * sh.slot;
      const bool own = kk >= ka && kk <= kb;
      mbar_expect_tx(&full[s], xb + (own ? fb + cb : 0u) + extra_tx);
      bulk_load(slot + sh.xoff, xg + sp.row(j0 - 1, kk), xb, &full[s]);
      if (own) {
        bulk_load(slot + sh.foff, fg + sp.row(j0, kk), fb, &full[s]);
        bulk_load(slot + sh.coff, codeg + sp.row(j0, kk), cb, &full[s]);
      }
    }
    drain(klast);
    return;
  }

  // consumers: warp w takes row j0 + w / WPR, its (w % WPR)-th run of 128
  // points of each 128 WPR; lanes over 32 consecutive points
  const int rr = warp / WPR, hw = warp % WPR;
  const int jj = j0 + rr;
  const int bw = sh.bw, bwc = sh.bwc;
  int ready = kfirst - 1;
  for (int k = ka; k <= kb; ++k) {
    for (int kk = ready + 1; kk <= k + 1; ++kk)
      if (!mbar_wait(&full[slot_of(kk)], use_of(kk) & 1u)) {
        if (lane == 0)
          atomicOr(err, 1);
        return;
      }
    ready = k + 1;
    if (rr < jn) {
      // stage row t of x holds row j0 - 1 + t, halves of bw entries
      const T *X = reinterpret_cast<const T *>(sm + slot_of(k) * sh.slot +
                                               sh.xoff) +
                   (rr + 1) * 2 * bw;
      const T *Xd = reinterpret_cast<const T *>(
                        sm + slot_of(k - 1) * sh.slot + sh.xoff) +
                    (rr + 1) * 2 * bw;
      const T *Xu = reinterpret_cast<const T *>(
                        sm + slot_of(k + 1) * sh.slot + sh.xoff) +
                    (rr + 1) * 2 * bw;
      const T *F = reinterpret_cast<const T *>(sm + slot_of(k) * sh.slot +
                                               sh.foff) +
                   rr * 2 * bw;
      const unsigned char *C =
          sm + slot_of(k) * sh.slot + sh.coff + rr * 2 * bwc;
      for (int i0 = 2 + 128 * hw; i0 <= nx - 1; i0 += 128 * WPR) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int i = i0 + 32 * m + lane;
          if (i > nx - 1)
            break;
          // own colour c at entry e of half c; every neighbour is in the
          // other half o: west entry (i - 2) >> 1, east i >> 1, the others
          // entry e of rows jj +- 1 and planes k +- 1
          const int c = (i + jj + k) & 1, e = (i - 1) >> 1;
          const int o = (1 - c) * bw, own = c * bw;
          const T xc = X[own + e];
          const T xw = X[o + ((i - 2) >> 1)], xe = X[o + (i >> 1)];
          const T xn = X[2 * bw + o + e], xs = X[-2 * bw + o + e];
          const T xu = Xu[o + e], xd = Xd[o + e];
          const T fv = F[own + e];
          const unsigned b = C[c * bwc + e];
          T ax;
          if (oc_coded) {
            const T *t = ctab[b & 127u];
            ax = -t[0] * xn - t[1] * xs - t[2] * xe - t[3] * xw -
                 t[4] * xd - t[5] * xu + (t[6] + T(0)) * xc;
          } else {
            const int p = sp.at(i, jj, k);
            Couplings<T> cp;
            if (coded) {
              cp.e = (b & 1u) ? L.eh : L.el;
              cp.w = (b & 2u) ? L.eh : L.el;
              cp.n = (b & 4u) ? L.nh : L.nl;
              cp.s = (b & 8u) ? L.nh : L.nl;
              cp.u = (b & 16u) ? L.uh : L.ul;
              cp.dn = (b & 32u) ? L.uh : L.ul;
            } else {
              cp = array_couplings<T>(oE, oN, uC, p, split_nb(sp, p, i, c));
            }
            ax = -cp.n * xn - cp.s * xs - cp.e * xe - cp.w * xw -
                 cp.dn * xd - cp.u * xu + (oC[p] + T(0)) * xc;
          }
          r[d.at(i, jj, k)] = fv - ax;
        }
      }
    }
    __syncwarp();
    if (lane == 0)
      mbar_arrive(&empty[slot_of(k - 1)]);
  }
}

template <typename T> constexpr auto defect_kernel_of() {
  return defect7_stream_kernel<T>;
}

// r (reference layout) = f - A x on the coded split level d (defect_fits);
// x, f, code: the level's colour-split arrays (16-byte aligned).
template <typename T>
int launch_defect7_stream(const T *x, const T *f, const unsigned char *code,
                          const Dims &d, const T *oC,
                          const T *oE, const T *oN, const T *uC,
                          const int *info, const T *lut, const T *octab,
                          T *r, int *err, unsigned extra_tx,
                          cudaStream_t s) {
  constexpr int NT = DefectCfg<T>::THREADS;
  auto kern = defect7_stream_kernel<T>;
  int dev = 0, sms = 0, per_sm = 0;
  PMG_CUDA_TRY(cudaGetDevice(&dev));
  StreamShape sh = defect_shape<T>(d, 1);
  const size_t smem = defect_smem_bytes<T>(sh);
  {
    const cudaError_t e = set_smem_limit<defect_kernel_of<T>()>((int)smem);
    PMG_CUDA_TRY(e);
  }
  PMG_CUDA_TRY(
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PMG_CUDA_TRY(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  sh = defect_shape<T>(d, sms * (per_sm < 1 ? 1 : per_sm));
  const unsigned g = (unsigned)sh.nj * cdiv(d.nz - 2, sh.kchunk);
  kern<<<g, NT, smem, s>>>(d, sh, x, f, code, oC, oE, oN, uC, info, lut,
                           octab, r, err, extra_tx);
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

} // namespace pmg
