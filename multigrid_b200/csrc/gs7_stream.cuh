// Red-black colour pass of the refinement paths' finest level (Vgsrb7x,
// pmgc/gsd.cc:61-111, on the colour-split coded arrays of split_layout.cuh)
// with the level's rows streamed through shared memory by the tensor
// memory accelerator.
//
// The per-point-load pass (gs7_code_color_kernel) moves the coded format's
// bytes and no more, but it executes ~144 instructions per point (address
// arithmetic for nine scalar loads, index and neighbour maths) and keeps
// only what its registers hold in flight, so it runs issue- and
// latency-bound at ~2.6 TB/s (ncu: 77% issue, 38 M warp instructions per
// 257^3 pass). Here each CTA owns J rows of a chunk of planes and marches
// along k. Per plane a producer warp issues three tensor-map boxes onto
// the "full" mbarrier of a slot of a ring of S stages, once every consumer
// warp has released the slot's previous plane on its "empty" mbarrier (no
// block-wide barrier per plane; each consumer warp waits only for the
// planes it reads): the other colour's half of x over J + 2
// rows (the rows above and below the block for the north and south
// neighbours), and the own colour's half of f over the block's J rows. In
// the colour-split layout the other colour is the same half of every row,
// so each is one box; but a box moves row by row, and half-row copies cost
// the copy engine ~20 ns each whatever their size below ~1 KB (measured).
// The own colour's code bytes of the J rows therefore come from a copy of
// the code array blocked by (plane, row block, colour) (code_block_kernel),
// where they are one contiguous run: one bulk copy instead of J rows
// (measured at 257^3: 131 -> 129 us per four float passes, 263 -> 262 us
// double; the pass is bound more by instruction issue than by the copies). Plane k is computed
// from the stages of k - 1, k and k + 1 while the next S - 3 planes are in
// flight, so the bytes in flight are set by the ring, not by registers.
// A warp computes a row: each lane four consecutive points from 16-byte
// shared-memory loads, the one west or east neighbour outside its four by a
// shuffle, and stores the four results with one 16-byte store. A point's
// seven coefficients come from a 128-entry table in shared memory indexed
// by its code byte (two 16-byte loads instead of six bit tests and
// selects and a table lookup). The arithmetic is gs7_code_color_kernel's,
// term for term, so the bits are the same.
//
// A pass reads only the other colour of x and writes only its own, so the
// stages never hold values the pass changes. Rows and planes outside the
// grid (past the last row block, past the last plane) read as zeros from
// the box and are never used. The tensor maps cover this GPU's own arrays
// (no multicast).
//
// Every wait is bounded (gs27_tma.cuh's poll limit): a consumer warp whose
// plane did not arrive sets *err and returns; the producer, whose slot is
// then never released, sets *err, waits (also bounded) for the copies it
// has in flight, and returns; the solve's stop test reports
// PMG_ERR_TIMEOUT.
#pragma once

#include <atomic>
#include <type_traits>

#include "gs27_tma.cuh"
#include "split_layout.cuh"

namespace pmg {

// Rows per CTA, ring stages and threads of the streamed pass by element
// type: one consumer warp per row and one producer warp.
template <typename T> struct StreamCfg {
  static constexpr int J = 8;
  static constexpr int S = sizeof(T) == 4 ? 6 : 4;
  static constexpr int THREADS = 32 * (J + 1);
  // CTAs per SM the ring's shared memory allows at 257^3 (registers capped
  // to match)
  static constexpr int MIN_CTAS = sizeof(T) == 4 ? 3 : 2;
};

// Tensor maps of the colour-split x, f (element type T) and code bytes of a
// level: 4-D, {entry, half, row, plane}; boxes of bw (bwc) entries of one
// half over J + 2 rows (x) or J rows (f, code) of one plane.
struct alignas(64) StreamMaps {
  CUtensorMap x, f, code;
};

// The code bytes blocked for the streamed pass: per plane k, row block jb
// (rows 2 + J jb ..) and colour half h, the J rows' entries 0 .. bwc - 1 of
// half h in a run of J bwc bytes at ((k - 1) nj + jb) 2 + h runs; rows past
// the grid read as zero, as in a box.
static_assert(StreamCfg<float>::J == StreamCfg<double>::J,
              "one blocking serves both element types");
struct CodeBlocks {
  int nj, bwc;
  static CodeBlocks of(const Dims &d) {
    constexpr int J = StreamCfg<float>::J;
    return CodeBlocks{(int)cdiv(d.ny - 2, J),
                      (((d.nx + 1) / 2) + 15) & ~15};
  }
  __host__ __device__ long run() const {
    return (long)StreamCfg<float>::J * bwc;
  }
  __host__ __device__ long bytes(const Dims &d) const {
    return (long)d.nz * nj * 2 * run();
  }
};

__global__ void code_block_kernel(Dims d, CodeBlocks cb,
                                  const unsigned char *__restrict__ code,
                                  unsigned char *__restrict__ out) {
  constexpr int J = StreamCfg<float>::J;
  const Split sp = Split::of(d);
  const long n = cb.bytes(d);
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int e = (int)(t % cb.bwc);
    long q = t / cb.bwc;
    const int r = (int)(q % J);
    q /= J;
    const int h = (int)(q % 2);
    q /= 2;
    const int jb = (int)(q % cb.nj), k = (int)(q / cb.nj) + 1;
    const int j = 2 + jb * J + r;
    out[t] = (j <= d.ny && e < sp.hp) ? code[sp.row(j, k) + h * sp.hp + e]
                                      : (unsigned char)0;
  }
}

// Geometry of one streamed launch (host-computed).
struct StreamShape {
  int nj;     // row blocks
  int kchunk; // planes per CTA
  int bw;     // entries of an x / f box row (a multiple of 16 bytes)
  int bwc;    // entries of a code box row (a multiple of 16)
  int xoff, foff, coff;     // byte offsets of x, f, code inside a stage
  int slot;                 // bytes of a stage (a multiple of 128)
  unsigned xbytes, fcbytes; // transaction bytes: x box; f and code boxes
};

// one box of a 4-D tensor map into shared memory, completing on bar
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map,
                                            int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx"
      "::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

// a plain arrival on an mbarrier (no transaction bytes)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(
                   smem_addr(bar))
               : "memory");
}

// num / (c + 0), rounded to T, with c the divisor of table entry b.
// Double: IEEE division. Float: num times the double reciprocal of the
// divisor, rounded to float. That product is within 2^-51 (relative) of
// num / c (two double roundings), while a quotient of two 24-bit floats
// that is not itself a float lies at least 2^-49 (relative) from every
// rounding midpoint between floats ((a - c m) is a nonzero multiple of the
// smallest exponent's unit), so both round to the same float: the bits of
// the division, without its special-case branch. Quotients that are
// floats, zeros, infinities and NaNs come out the same too.
__device__ __forceinline__ double div_by_table(double num, double c,
                                               const double *, unsigned) {
  return num / (c + 0.0);
}
__device__ __forceinline__ float div_by_table(float num, float,
                                              const double *rtab,
                                              unsigned b) {
  return (float)((double)num * rtab[b]);
}

// a row parity given at compile time (std::true_type / std::false_type) or
// at run time (bool)
__device__ __forceinline__ bool row_parity(bool b) { return b; }
template <bool B>
__device__ __forceinline__ bool row_parity(std::integral_constant<bool, B>) {
  return B;
}

// four consecutive entries
template <typename T> struct alignas(16) Quad {
  T x, y, z, w;
};

// KEEP false: the first pass from a zero iterate (zero_initialize), whose
// neighbour sum is multiplied by 0 as in the per-point pass; true: the sum
// is added as it is (1 * sum is sum, so the multiply is left out).
template <typename T, int J, int S, bool KEEP>
__global__ void __launch_bounds__(StreamCfg<T>::THREADS,
                                  StreamCfg<T>::MIN_CTAS)
    gs7_stream_kernel(const __grid_constant__ StreamMaps maps, Dims d,
                      StreamShape sh, const T *__restrict__ oC,
                      const T *__restrict__ oE, const T *__restrict__ oN,
                      const T *__restrict__ uC, const int *__restrict__ info,
                      const T *__restrict__ lut,
                      const T *__restrict__ octab,
                      const unsigned char *__restrict__ codeb, T *x,
                      int want, int *err, unsigned extra_tx) {
  using V = Quad<T>;
  extern __shared__ __align__(128) unsigned char sm[];
  // per code byte (its low seven bits) the point's seven coefficients in
  // the order the update uses them: n, s, e, w, down, up, oC (one spare)
  __shared__ __align__(16) T ctab[128][8];
  // float: the double reciprocal of each code's divisor oC + 0 (see
  // div_by_table)
  __shared__ double rtab[sizeof(T) == 4 ? 128 : 1];
  // full[s]: the slot's boxes landed (the producer's arrival and their
  // bytes); empty[s]: every consumer warp is done with it
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + S * sh.slot);
  uint64_t *empty = full + S;
  const Split sp = Split::of(d);
  const int jb = blockIdx.x % sh.nj, kc = blockIdx.x / sh.nj;
  const int j0 = 2 + jb * J;
  const int jn = min(J, d.ny - j0); // own rows j0 .. j0 + jn - 1 <= ny - 1
  const int ka = 2 + kc * sh.kchunk;
  const int kb = min(ka + sh.kchunk - 1, d.nz - 1);
  const int kfirst = ka - 1, klast = kb + 1; // staged planes
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], J);
    }
    fence_mbar_init();
  }
  // the coding (uniform): couplings from the code byte, oC from the table
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
    if constexpr (sizeof(T) == 4)
      rtab[b] = 1.0 / (double)(t[6] + T(0));
  }
  __syncthreads();
  auto slot_of = [&](int kk) { return (kk - kfirst) % S; };
  auto use_of = [&](int kk) { return (kk - kfirst) / S; };

  if (warp == J) {
    // producer: the boxes of plane kk into its slot once the slot's
    // previous plane is released (0-based coordinates: entry 0, the half,
    // row j - 1, plane k - 1); the planes the block computes also bring
    // their f and code rows
    if (lane != 0)
      return;
    // every copy still in flight (planes last - S + 1 .. last) lands
    // before the producer leaves; one poll budget for all of them
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
      mbar_expect_tx(&full[s],
                     sh.xbytes + (own ? sh.fcbytes : 0u) + extra_tx);
      tma_load_4d(slot + sh.xoff, &maps.x, 0, 1 - want, j0 - 2, kk - 1,
                  &full[s]);
      if (own) {
        tma_load_4d(slot + sh.foff, &maps.f, 0, want, j0 - 1, kk - 1,
                    &full[s]);
        bulk_load(slot + sh.coff,
                  codeb + ((long)((kk - 1) * sh.nj + jb) * 2 + want) *
                              (J * sh.bwc),
                  (unsigned)(J * sh.bwc), &full[s]);
      }
    }
    drain(klast);
    return;
  }

  // consumers: warp r computes row j0 + r of each plane (a warp past the
  // last row keeps the pace and releases its slots)
  int ready = kfirst - 1; // last plane waited for
  const int bw = sh.bw, bwc = sh.bwc;
  for (int k = ka; k <= kb; ++k) {
    // planes k - 1, k, k + 1 complete
    for (int kk = ready + 1; kk <= k + 1; ++kk)
      if (!mbar_wait(&full[slot_of(kk)], use_of(kk) & 1u)) {
        if (lane == 0)
          atomicOr(err, 1);
        return;
      }
    ready = k + 1;
    const unsigned char *sd = sm + slot_of(k - 1) * sh.slot;
    const unsigned char *sc = sm + slot_of(k) * sh.slot;
    const unsigned char *su = sm + slot_of(k + 1) * sh.slot;
    if (warp < jn) { // warp-uniform
      const int r = warp, j = j0 + r;
      // x stage row rr holds row j0 - 1 + rr: row j is rr = r + 1
      const T *xo = reinterpret_cast<const T *>(sc + sh.xoff) + (r + 1) * bw;
      const T *xn = xo + bw, *xs = xo - bw;
      const T *xu = reinterpret_cast<const T *>(su + sh.xoff) + (r + 1) * bw;
      const T *xd = reinterpret_cast<const T *>(sd + sh.xoff) + (r + 1) * bw;
      const T *fr = reinterpret_cast<const T *>(sc + sh.foff) + r * bw;
      const unsigned char *cr = sc + sh.coff + r * bwc;
      // own points: i = 1 + 2e (odd i, when point 1 of the row has the
      // pass's colour) or 2 + 2e; interior e in [elo, ehi]. West and east
      // are entries e - 1, e (odd i) or e, e + 1 (even i) of the other half.
      const long row = (long)sp.row(j, k) + want * sp.hp;
      // the row's parity is the same for the whole warp. Float: each case
      // compiled on its own, so the per-point selects between them fold away
      // (1-2% per pass at 257^3); double keeps one body, whose two copies
      // would spill (258 against 254 us per four passes)
      auto row_pass = [&](auto odd_c) {
        const bool odd = row_parity(odd_c);
        const int elo = odd ? 1 : 0;
        const int ehi = odd ? (d.nx - 2) / 2 : (d.nx - 3) / 2;
        // every lane takes part in each round (the shuffles); lane g of the
        // round takes entries 4g .. 4g + 3
        for (int g0 = 0; 4 * g0 <= ehi; g0 += 32) {
          const int g = g0 + lane, e4 = 4 * g;
          const bool act = e4 <= ehi;
          V vn{}, vs{}, vu{}, vd{}, vo{}, vf{};
          unsigned cb = 0;
          if (act) {
            vn = *reinterpret_cast<const V *>(xn + e4);
            vs = *reinterpret_cast<const V *>(xs + e4);
            vu = *reinterpret_cast<const V *>(xu + e4);
            vd = *reinterpret_cast<const V *>(xd + e4);
            vo = *reinterpret_cast<const V *>(xo + e4);
            vf = *reinterpret_cast<const V *>(fr + e4);
            cb = *reinterpret_cast<const unsigned *>(cr + e4);
          }
          // the other-half entry just outside the four: e4 - 1 (odd i, the
          // previous lane's last) or e4 + 4 (even i, the next lane's first);
          // read directly where that lane is in another round or idle
          const T up = __shfl_up_sync(0xffffffffu, vo.w, 1);
          const T down = __shfl_down_sync(0xffffffffu, vo.x, 1);
          T edge = odd ? up : down;
          if (act && odd && lane == 0 && e4 > 0)
            edge = xo[e4 - 1];
          if (act && !odd && (lane == 31 || e4 + 4 > ehi))
            edge = xo[e4 + 4];
          const T xw[4] = {odd ? edge : vo.x, odd ? vo.x : vo.y,
                           odd ? vo.y : vo.z, odd ? vo.z : vo.w};
          const T xe[4] = {odd ? vo.x : vo.y, odd ? vo.y : vo.z,
                           odd ? vo.z : vo.w, odd ? vo.w : edge};
          const T an[4] = {vn.x, vn.y, vn.z, vn.w};
          const T as[4] = {vs.x, vs.y, vs.z, vs.w};
          const T au[4] = {vu.x, vu.y, vu.z, vu.w};
          const T ad[4] = {vd.x, vd.y, vd.z, vd.w};
          const T af[4] = {vf.x, vf.y, vf.z, vf.w};
          T out[4];
          if (oc_coded) {
            // every coefficient from the code byte's table entry (the same
            // values gs7_code_color_kernel selects); points outside the row's
            // interior compute from table entries too and are not stored
  #pragma unroll
            for (int m = 0; m < 4; ++m) {
              const T *t = ctab[(cb >> (8 * m)) & 127u];
              const Quad<T> c0 = *reinterpret_cast<const Quad<T> *>(t);
              const Quad<T> c1 = *reinterpret_cast<const Quad<T> *>(t + 4);
              const T sum = c0.x * an[m] + c0.y * as[m] + c0.z * xe[m] +
                            c0.w * xw[m] + c1.x * ad[m] + c1.y * au[m];
              out[m] = div_by_table(KEEP ? af[m] + sum : af[m] + T(0) * sum,
                                    c1.z, rtab,
                                    (cb >> (8 * m)) & 127u);
            }
          } else {
  #pragma unroll
            for (int m = 0; m < 4; ++m) {
              const int e = e4 + m;
              const bool in = act && e >= elo && e <= ehi;
              const unsigned b = (cb >> (8 * m)) & 0xffu;
              const int p = (int)(row + e);
              Couplings<T> cp{};
              if (coded) {
                cp.e = (b & 1u) ? L.eh : L.el;
                cp.w = (b & 2u) ? L.eh : L.el;
                cp.n = (b & 4u) ? L.nh : L.nl;
                cp.s = (b & 8u) ? L.nh : L.nl;
                cp.u = (b & 16u) ? L.uh : L.ul;
                cp.dn = (b & 32u) ? L.uh : L.ul;
              } else if (in) {
                cp = array_couplings<T>(oE, oN, uC, p,
                                        split_nb(sp, p, odd ? 1 : 2, want));
              }
              const T sum = cp.n * an[m] + cp.s * as[m] + cp.e * xe[m] +
                            cp.w * xw[m] + cp.dn * ad[m] + cp.u * au[m];
              const T c = in ? oC[p] : T(1);
              out[m] = (KEEP ? af[m] + sum : af[m] + T(0) * sum) / (c + T(0));
            }
          }
          if (act) {
            T *dst = x + row + e4;
            if (e4 >= elo && e4 + 3 <= ehi) {
              V v;
              v.x = out[0];
              v.y = out[1];
              v.z = out[2];
              v.w = out[3];
              *reinterpret_cast<V *>(dst) = v;
            } else {
  #pragma unroll
              for (int m = 0; m < 4; ++m)
                if (e4 + m >= elo && e4 + m <= ehi)
                  dst[m] = out[m];
            }
          }
        }
      };
      const bool row_odd = ((1 + j + k) & 1) == want;
      if constexpr (sizeof(T) == 4) {
        if (row_odd)
          row_pass(std::true_type{});
        else
          row_pass(std::false_type{});
      } else {
        row_pass(row_odd);
      }
    }
    // plane k - 1 is no longer needed by this warp
    __syncwarp();
    if (lane == 0)
      mbar_arrive(&empty[slot_of(k - 1)]);
  }
}

// Shape of the streamed pass on level d for T: row blocks of J, and planes
// in chunks so that the grid fills the GPU's resident CTAs once.
template <typename T>
StreamShape stream_shape(const Dims &d, int resident_ctas) {
  constexpr int J = StreamCfg<T>::J;
  StreamShape sh{};
  // entries of the longer half, rounded to the four a lane reads at once
  // (16 bytes of float, 32 of double)
  const int hx = (d.nx + 1) / 2;
  sh.bw = (hx + 3) & ~3;
  sh.bwc = (hx + 15) & ~15;
  sh.nj = (int)cdiv(d.ny - 2, J);
  const int planes = d.nz - 2;
  int nkc = resident_ctas / sh.nj;
  nkc = nkc < 1 ? 1 : nkc > planes ? planes : nkc;
  sh.kchunk = (int)cdiv(planes, nkc);
  auto up128 = [](int b) { return (b + 127) & ~127; };
  sh.xbytes = (unsigned)((J + 2) * sh.bw * sizeof(T));
  const unsigned fb = (unsigned)(J * sh.bw * sizeof(T));
  const unsigned cb = (unsigned)(J * sh.bwc);
  sh.fcbytes = fb + cb;
  sh.xoff = 0;
  sh.foff = up128((int)sh.xbytes);
  sh.coff = sh.foff + up128((int)fb);
  sh.slot = sh.coff + up128((int)cb);
  return sh;
}
template <typename T> size_t stream_smem_bytes(const StreamShape &sh) {
  return (size_t)StreamCfg<T>::S * sh.slot +
         2 * StreamCfg<T>::S * sizeof(uint64_t);
}
inline unsigned stream_grid(const Dims &d, const StreamShape &sh) {
  return (unsigned)sh.nj * cdiv(d.nz - 2, sh.kchunk);
}

// Dynamic shared memory a CTA may hold (227 KB less the kernel's static
// coefficient table; the ring must fit) and the widest box row a tensor
// map allows (256 entries): larger levels use the per-point pass.
constexpr size_t kStreamMaxSmem = 227 * 1024 - 128 * 8 * sizeof(double);
template <typename T> bool stream_fits(const Dims &d) {
  const StreamShape sh = stream_shape<T>(d, 1);
  return sh.bw <= 256 && sh.bwc <= 256 &&
         stream_smem_bytes<T>(sh) <= kStreamMaxSmem;
}

template <typename T, bool KEEP = true> constexpr auto stream_kernel_of() {
  return gs7_stream_kernel<T, StreamCfg<T>::J, StreamCfg<T>::S, KEEP>;
}

// itmax red-black sweeps on the coded split arrays (launch_gs7_code's
// semantics) with the streamed pass; maps: the level's x and f maps (boxes
// of stream_shape's widths); codeb: the level's code bytes blocked by
// code_block_kernel; err as in gs7_stream_kernel.
template <typename T>
int launch_gs7_stream(const StreamMaps &maps, const Dims &d, const T *oC,
                      const T *oE, const T *oN, const T *uC, const int *info,
                      const T *lut, const T *octab,
                      const unsigned char *codeb, T *x, int itmax,
                      int iadjoint, int zero_init, int *err,
                      unsigned extra_tx, cudaStream_t s) {
  constexpr int NT = StreamCfg<T>::THREADS;
  auto kern = stream_kernel_of<T>();
  int dev = 0;
  PMG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64)
    dev = 0;
  StreamShape sh = stream_shape<T>(d, 1);
  const size_t smem = stream_smem_bytes<T>(sh);
  {
    cudaError_t e = set_smem_limit<stream_kernel_of<T, true>()>((int)smem);
    PMG_CUDA_TRY(e);
    e = set_smem_limit<stream_kernel_of<T, false>()>((int)smem);
    PMG_CUDA_TRY(e);
  }
  int per_sm = 0, sms = 0;
  PMG_CUDA_TRY(
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PMG_CUDA_TRY(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  sh = stream_shape<T>(d, sms * (per_sm < 1 ? 1 : per_sm));
  const unsigned g = stream_grid(d, sh);
  for (int it = 0; it < itmax; ++it)
    for (int c = 0; c <= 1; ++c) {
      const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
      auto k = zero_init ? stream_kernel_of<T, false>() : kern;
      k<<<g, NT, smem, s>>>(maps, d, sh, oC, oE, oN, uC, info, lut, octab,
                            codeb, x, want, err, extra_tx);
      zero_init = 0;
    }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

} // namespace pmg
