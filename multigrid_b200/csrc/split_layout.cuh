// Colour-split layout of the refinement paths' finest-level arrays.
//
// In the reference layout a red-black colour pass touches every other point
// of a row, so it streams whole cache sectors of every array it reads: one
// sweep moves about twice the bytes it needs. The mixed and fp64-fast paths
// own their copies of the finest operator, right-hand side and correction,
// so they keep every row split by colour: the points with (i + j + k) even
// in the first half of the row, the odd ones in the second, each half
// padded to a multiple of 16 entries (`hp`) so that every half row starts
// on a 16-byte boundary. Entry (i - 1) >> 1 of its colour's half holds
// point i. A colour pass then reads one contiguous half of every row of f
// and the code bytes, and the other colour's half of x, which is the same
// half in every row, so the J rows a block needs of a plane form one
// tensor-map box (gs7_stream.cuh). Its neighbours: i - 1 and i + 1 are
// entries e - (i odd), e + (i even) of the other half of the row; j +- 1
// and k +- 1 are entry e of the other half of the next or previous row or
// plane.
//
// Only the arrays of the finest level use this layout; the kernels here
// read and write them, converting at the boundaries (the double residual,
// the prolongation's correction, the refinement update). The per-point
// arithmetic is the reference-layout kernels', so results are
// bit-identical. The padding entries are zero (the problem's arena is
// cleared at creation) and no update reads them.
#pragma once

#include <climits>
#include <cstring>

#include "launch.cuh"
#include "reduce_kernels.cuh"

namespace pmg {

struct Split {
  int nx, ny, nz, hp; // hp: entries per colour half (a multiple of 16)
  __host__ __device__ static Split of(const Dims &d) {
    return Split{d.nx, d.ny, d.nz, ((d.nx + 1) / 2 + 15) & ~15};
  }
  // entries of a row and of a plane
  __host__ __device__ int pitch() const { return 2 * hp; }
  __host__ __device__ int plane() const { return 2 * hp * ny; }
  __host__ __device__ long count() const { return (long)plane() * nz; }
  // first entry of row (j, k) (its colour-0 half)
  __host__ __device__ int row(int j, int k) const {
    return ((k - 1) * ny + (j - 1)) * pitch();
  }
  // split index of (i, j, k)
  __host__ __device__ int at(int i, int j, int k) const {
    return row(j, k) + ((i + j + k) & 1) * hp + ((i - 1) >> 1);
  }
  // split index of the reference-layout linear index g
  __host__ __device__ int of_linear(long g) const {
    const int i = (int)(g % nx) + 1;
    const long r = g / nx;
    return at(i, (int)(r % ny) + 1, (int)(r / ny) + 1);
  }
};

// dst (split) = (Tout) src (reference layout), every entry
template <typename Tin, typename Tout>
__global__ void to_split_kernel(Dims d, const Tin *__restrict__ src,
                                Tout *__restrict__ dst) {
  const Split sp = Split::of(d);
  const long n = d.count();
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n;
       g += (long)gridDim.x * blockDim.x)
    dst[sp.of_linear(g)] = (Tout)src[g];
}

// dst (reference layout) = (Tout) src (split), every entry
template <typename Tin, typename Tout>
__global__ void from_split_kernel(Dims d, const Tin *__restrict__ src,
                                  Tout *__restrict__ dst) {
  const Split sp = Split::of(d);
  const long n = d.count();
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n;
       g += (long)gridDim.x * blockDim.x)
    dst[g] = (Tout)src[sp.of_linear(g)];
}

// x64 (reference layout) += (double) e (split) on the interior: the
// refinement update of the split correction (float or double)
template <typename E>
__global__ void add_correction_split_kernel(Dims d, double *__restrict__ x,
                                            const E *__restrict__ e) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  x[p] = x[p] + (double)e[Split::of(d).at(t.i, t.j, t.k)];
}

// Neighbour offsets of point i of colour c at split index s: every
// neighbour has the other colour, so it lies in the other half; west and
// east in the same row (entries e - 1, e for odd i; e, e + 1 for even i),
// north / south one row on, up / down one plane on, at entry e.
struct SplitNb {
  int w, e, n, s, u, dn;
};
__device__ __forceinline__ SplitNb split_nb(const Split &sp, int s, int i,
                                            int c) {
  const int o = s + (1 - 2 * c) * sp.hp; // entry e of the other half
  const int odd = i & 1;
  SplitNb nb;
  nb.w = o - odd;
  nb.e = o + 1 - odd;
  nb.n = o + sp.pitch();
  nb.s = o - sp.pitch();
  nb.u = o + sp.plane();
  nb.dn = o - sp.plane();
  return nb;
}

// One colour of the red-black sweep (gs7_color_kernel) on split arrays: the
// points of a row with (i + j + k) % 2 == want are one half of it. One
// thread per point; blockIdx.z is the plane.
template <typename T>
__global__ void __launch_bounds__(256)
    gs7_split_color_kernel(Dims d, const T *__restrict__ oC,
                           const T *__restrict__ fc, const T *__restrict__ oE,
                           const T *__restrict__ oN, const T *__restrict__ uC,
                           T *x, int want, T keep) {
  const Split sp = Split::of(d);
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (j > d.ny - 1)
    return;
  const int i = 2 + ((2 + j + k + want) & 1) +
                2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i > d.nx - 1)
    return;
  const int p = sp.at(i, j, k);
  const SplitNb nb = split_nb(sp, p, i, want);
  const T s = oN[p] * x[nb.n] + oN[nb.s] * x[nb.s] + oE[p] * x[nb.e] +
              oE[nb.w] * x[nb.w] + uC[nb.dn] * x[nb.dn] + uC[p] * x[nb.u];
  x[p] = (fc[p] + keep * s) / (oC[p] + T(0));
}

// itmax red-black sweeps on split arrays (Vgsrb7x semantics, cc = 0)
template <typename T>
int launch_gs7_split(const Dims &d, const T *oC, const T *fc, const T *oE,
                     const T *oN, const T *uC, T *x, int itmax, int iadjoint,
                     int zero_init, cudaStream_t s) {
  for (int it = 0; it < itmax; ++it)
    for (int c = 0; c <= 1; ++c) {
      const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
      const T keep = zero_init ? T(0) : T(1);
      gs7_split_color_kernel<T><<<gs7_grid(d), interior_block(), 0, s>>>(
          d, oC, fc, oE, oN, uC, x, want, keep);
      zero_init = 0;
    }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// r (reference layout) = f - A x with f, x and the 7-point operator split
// (defect_kernel<7>, the class's map order)
template <typename T>
__global__ void __launch_bounds__(256)
    defect7_split_kernel(Dims d, const T *__restrict__ oC,
                         const T *__restrict__ oE, const T *__restrict__ oN,
                         const T *__restrict__ uC, const T *__restrict__ f,
                         const T *__restrict__ x, T *__restrict__ r) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const Split sp = Split::of(d);
  const int p = sp.at(t.i, t.j, t.k);
  const SplitNb nb = split_nb(sp, p, t.i, (t.i + t.j + t.k) & 1);
  const T ax = -oN[p] * x[nb.n] - oN[nb.s] * x[nb.s] - oE[p] * x[nb.e] -
               oE[nb.w] * x[nb.w] - uC[nb.dn] * x[nb.dn] - uC[p] * x[nb.u] +
               (oC[p] + T(0)) * x[p];
  r[d.at(t.i, t.j, t.k)] = f[p] - ax;
}

// ---------------------------------------------------------------------------
// Coded couplings. The class's fine operator has two-valued couplings per
// direction (each face's dielectric is the inside or the outside value, so
// oE, oN and uC each hold two values). A colour pass then needs, per point,
// only which of the two each of its six couplings is: one byte
// (bit 0 oE(p), 1 oE(west), 2 oN(p), 3 oN(south), 4 uC(p), 5 uC(down); a set
// bit selects the larger value), stored in the split layout next to oC. The
// pass reads the byte instead of three float arrays (per sweep 17 bytes per
// point instead of 28) and takes the very same float values from a table,
// so results are bit-identical to the uncoded kernels. The encoding checks
// every coupling a pass reads bit for bit against the two table values;
// for any other operator the kernels read the coupling arrays as before.
// ---------------------------------------------------------------------------
struct CodeLut {
  float el, eh, nl, nh, ul, uh; // low / high value of oE, oN, uC
};

// order-preserving int image of a float (for atomicMin / atomicMax)
__device__ __forceinline__ int float_order(float v) {
  const int i = __float_as_int(v);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ inline float order_float(int i) {
  const int b = i >= 0 ? i : i ^ 0x7fffffff;
  float f;
  memcpy(&f, &b, sizeof f);
  return f;
}

// info[0..5] = min, max of oE, oN, uC over the couplings the interior
// points read (ordered ints; info[0,2,4] start at INT_MAX, [1,3,5] at
// INT_MIN). A grid-stride loop, then warp and block reductions, so only
// one thread per block touches the six global words.
template <typename T>
__global__ void __launch_bounds__(256)
    coupling_range_kernel(Dims d, const T *__restrict__ oE,
                          const T *__restrict__ oN,
                          const T *__restrict__ uC, int *info) {
  __shared__ int sh[6][8];
  int v[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN};
  const Split sp = Split::of(d);
  const int total = (d.nx - 2) * (d.ny - 2) * (d.nz - 2);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += gridDim.x * blockDim.x) {
    int i, j, k;
    interior_coords(d, q, i, j, k);
    const int p = sp.at(i, j, k);
    const SplitNb nb = split_nb(sp, p, i, (i + j + k) & 1);
    // classified by their float values (the double path checks its
    // couplings against the table separately, lut64_check_kernel)
    const int c[6] = {float_order((float)oE[p]), float_order((float)oE[nb.w]),
                      float_order((float)oN[p]), float_order((float)oN[nb.s]),
                      float_order((float)uC[p]), float_order((float)uC[nb.dn])};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      v[2 * a] = min(v[2 * a], min(c[2 * a], c[2 * a + 1]));
      v[2 * a + 1] = max(v[2 * a + 1], max(c[2 * a], c[2 * a + 1]));
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int w = __shfl_xor_sync(0xffffffffu, v[q], o);
      v[q] = (q & 1) ? max(v[q], w) : min(v[q], w);
    }
    if (lane == 0)
      sh[q][warp] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int q = 0; q < 6; ++q) {
      int r = sh[q][0];
      for (int w = 1; w < nw; ++w)
        r = (q & 1) ? max(r, sh[q][w]) : min(r, sh[q][w]);
      if (q & 1)
        atomicMax(&info[q], r);
      else
        atomicMin(&info[q], r);
    }
  }
}

// blocks of coupling_range_kernel: enough to fill the GPU a few times over
inline unsigned coupling_range_blocks(const Dims &d) {
  const long total = (long)(d.nx - 2) * (d.ny - 2) * (d.nz - 2);
  const long want = (total + 255) / 256;
  return (unsigned)(want < 148 * 8 ? want : 148 * 8);
}

// code bytes of the interior points; info[6] |= 1 when a coupling is
// neither table value bit for bit
template <typename T>
__global__ void __launch_bounds__(256)
    coupling_code_kernel(Dims d, const T *__restrict__ oE,
                         const T *__restrict__ oN,
                         const T *__restrict__ uC, int *info,
                         unsigned char *__restrict__ code) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const Split sp = Split::of(d);
  const int p = sp.at(t.i, t.j, t.k);
  const SplitNb nb = split_nb(sp, p, t.i, (t.i + t.j + t.k) & 1);
  const T c[6] = {oE[p], oE[nb.w], oN[p], oN[nb.s], uC[p], uC[nb.dn]};
  unsigned bits = 0;
  bool bad = false;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int v = __float_as_int((float)c[q]);
    const int lo = __float_as_int(order_float(info[(q >> 1) * 2]));
    const int hi = __float_as_int(order_float(info[(q >> 1) * 2 + 1]));
    if (v == hi)
      bits |= 1u << q;
    else if (v != lo)
      bad = true;
  }
  code[p] = (unsigned char)bits;
  if (bad)
    atomicOr(&info[6], 1);
}

// The table of a coded level, read on the device (info written by
// coupling_range_kernel / coupling_code_kernel); false when the level's
// couplings did not all match it, and the uncoded arrays must be used.
__device__ __forceinline__ bool load_lut(const int *info, CodeLut &L) {
  if (info[6] != 0)
    return false;
  L.el = order_float(info[0]);
  L.eh = order_float(info[1]);
  L.nl = order_float(info[2]);
  L.nh = order_float(info[3]);
  L.ul = order_float(info[4]);
  L.uh = order_float(info[5]);
  return true;
}

// The table of a coded double level: lut64 (lut64_store_kernel) holds the
// double value of each direction and bit; usable when the float
// classification held (info[6]) and every double coupling matched its
// entry (info[7]).
struct CodeLut64 {
  double el, eh, nl, nh, ul, uh;
};
__device__ __forceinline__ bool load_lut(const int *info, const float *,
                                         CodeLut &L) {
  return load_lut(info, L);
}
__device__ __forceinline__ bool load_lut(const int *info, const double *lut64,
                                         CodeLut64 &L) {
  const int2 f = *reinterpret_cast<const int2 *>(info + 6);
  if (f.x != 0 || f.y != 0) // info[6], info[7]
    return false;
  const double2 e = *reinterpret_cast<const double2 *>(lut64);
  const double2 n = *reinterpret_cast<const double2 *>(lut64 + 2);
  const double2 u = *reinterpret_cast<const double2 *>(lut64 + 4);
  L.el = e.x;
  L.eh = e.y;
  L.nl = n.x;
  L.nh = n.y;
  L.ul = u.x;
  L.uh = u.y;
  return true;
}
template <typename T> struct LutOf {
  using type = CodeLut;
};
template <> struct LutOf<double> {
  using type = CodeLut64;
};

// ---- the centre coefficient of a coded level ----------------------------
// The class's oC is the sum of a point's six couplings plus kappa^2 eps_out
// outside the ion-exclusion spheres (PBE_pmgc_class.h:67-100, 283-313), so
// for each six-bit coupling code it takes at most two values. Bit 6 of the
// code byte says which; the passes then read oC from a 128-entry table
// (index = the code's low seven bits) instead of an n^3 array. The table is
// found on the device (per code: the least and the largest value), every
// point's oC is checked against it bit for bit (info[8] |= 1 on a third
// value), and the double table is rounded to float for the float passes,
// whose oC is the double one rounded.
__device__ __forceinline__ long long double_order(double v) {
  const long long i = __double_as_longlong(v);
  return i >= 0 ? i : i ^ 0x7fffffffffffffffLL;
}
__device__ __forceinline__ double order_double(long long i) {
  return __longlong_as_double(i >= 0 ? i : i ^ 0x7fffffffffffffffLL);
}

// range[2c], range[2c + 1]: least and largest oC (ordered) of code c
static __global__ void oc_range_init_kernel(long long *range) {
  const int t = threadIdx.x;
  if (t < 128)
    range[t] = (t & 1) ? LLONG_MIN : LLONG_MAX;
}

// Each thread takes runs of kOcRun consecutive interior points of a row
// and folds equal codes in registers (codes change only at the dielectric
// and ion boundaries), then the block's table in shared memory, then one
// global update per code and block.
constexpr int kOcRun = 16;
static __global__ void __launch_bounds__(256)
    oc_range_kernel(Dims d, const double *__restrict__ oC,
                    const unsigned char *__restrict__ code,
                    long long *range) {
  __shared__ long long sh[128];
  for (int t = threadIdx.x; t < 128; t += blockDim.x)
    sh[t] = (t & 1) ? LLONG_MIN : LLONG_MAX;
  __syncthreads();
  const Split sp = Split::of(d);
  const int mx = d.nx - 2;
  const int runs_per_row = (mx + kOcRun - 1) / kOcRun;
  const long runs = (long)runs_per_row * (d.ny - 2) * (d.nz - 2);
  for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < runs;
       r += (long)gridDim.x * blockDim.x) {
    const long row = r / runs_per_row;
    const int i0 = 2 + (int)(r - row * runs_per_row) * kOcRun;
    const int j = 2 + (int)(row % (d.ny - 2)), k = 2 + (int)(row / (d.ny - 2));
    const int i1 = min(i0 + kOcRun - 1, d.nx - 1);
    int cur = -1;
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (int i = i0; i <= i1; ++i) {
      const int c = code[sp.at(i, j, k)] & 63;
      const long long v = double_order(oC[d.at(i, j, k)]);
      if (c != cur) {
        if (cur >= 0) {
          atomicMin(&sh[2 * cur], lo);
          atomicMax(&sh[2 * cur + 1], hi);
        }
        cur = c;
        lo = hi = v;
      } else {
        lo = min(lo, v);
        hi = max(hi, v);
      }
    }
    if (cur >= 0) {
      atomicMin(&sh[2 * cur], lo);
      atomicMax(&sh[2 * cur + 1], hi);
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < 64; c += blockDim.x)
    if (sh[2 * c] != LLONG_MAX) {
      atomicMin(&range[2 * c], sh[2 * c]);
      atomicMax(&range[2 * c + 1], sh[2 * c + 1]);
    }
}

inline unsigned oc_range_blocks(const Dims &d) {
  const long runs = (long)((d.nx - 2 + kOcRun - 1) / kOcRun) * (d.ny - 2) *
                    (d.nz - 2);
  const long want = (runs + 255) / 256;
  return (unsigned)(want < 148 * 4 ? want : 148 * 4);
}

// bit 6 of every interior code byte (oC is the code's larger value), and
// info[8] |= 1 where oC is neither of the code's two values
static __global__ void __launch_bounds__(256)
    oc_code_kernel(Dims d, const double *__restrict__ oC,
                   const long long *__restrict__ range, int *info,
                   unsigned char *__restrict__ code) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int sidx = Split::of(d).at(t.i, t.j, t.k);
  const unsigned b = code[sidx] & 63u;
  const long long v = __double_as_longlong(oC[d.at(t.i, t.j, t.k)]);
  const long long lo = __double_as_longlong(order_double(range[2 * b]));
  const long long hi = __double_as_longlong(order_double(range[2 * b + 1]));
  code[sidx] = (unsigned char)(b | (v == hi ? 64u : 0u));
  if (v != lo && v != hi)
    atomicOr(&info[8], 1);
}

// the tables: tab64[c + 64 bit] = the code's low (bit 0) or high (bit 1)
// value, tab32 the same rounded to float; codes no point has read 0
static __global__ void oc_table_kernel(const long long *__restrict__ range,
                                double *tab64, float *tab32) {
  const int t = threadIdx.x; // 128 threads: t = c + 64 bit
  if (t >= 128)
    return;
  const int c = t & 63, bit = t >> 6;
  const bool used = range[2 * c] != LLONG_MAX;
  const double v = used ? order_double(range[2 * c + bit]) : 0.0;
  tab64[t] = v;
  if (tab32)
    tab32[t] = (float)v;
}

// oC of a coded point: the table entry of the code's low seven bits
template <typename T>
__device__ __forceinline__ T oc_of(const T *tab, unsigned b) {
  return tab[b & 127u];
}

// the six couplings of point p from the arrays (split layout)
template <typename T> struct Couplings {
  T e, w, n, s, u, dn;
};
template <typename T>
__device__ __forceinline__ Couplings<T>
array_couplings(const T *oE, const T *oN, const T *uC, int p,
                const SplitNb &nb) {
  Couplings<T> c;
  c.e = oE[p];
  c.w = oE[nb.w];
  c.n = oN[p];
  c.s = oN[nb.s];
  c.u = uC[p];
  c.dn = uC[nb.dn];
  return c;
}

// gs7_split_color_kernel taking the couplings from the code byte when the
// level is coded (a uniform branch on the device flag, so the choice needs
// no host round trip and a captured graph serves either case). With the
// couplings coded a point moves about 17 bytes, so each thread takes PTS
// points of its half row (32 apart: a warp stays contiguous) and issues
// all their loads before computing, to keep enough bytes in flight.
// (Issuing the x loads before the coding flag is read raised the float
// kernel to 40 registers and 6 blocks per SM: 173 -> 186 us per four passes
// at 257^3; with one point per thread, 32 registers, 178 us.)
template <typename T, int PTS>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4)
    gs7_code_color_kernel(Dims d, const T *__restrict__ oC,
                          const T *__restrict__ fc, const T *__restrict__ oE,
                          const T *__restrict__ oN, const T *__restrict__ uC,
                          const unsigned char *__restrict__ code,
                          const int *__restrict__ info,
                          const T *__restrict__ lut,
                          const T *__restrict__ octab, T *x, int want,
                          T keep) {
  const Split sp = Split::of(d);
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (j > d.ny - 1)
    return;
  const int i0 = 2 + ((2 + j + k + want) & 1) +
                 2 * (int)(blockIdx.x * blockDim.x * PTS + threadIdx.x);
  if (i0 > d.nx - 1)
    return;
  int p[PTS];
  bool ok[PTS];
  unsigned b[PTS];
#pragma unroll
  for (int r = 0; r < PTS; ++r) {
    const int i = i0 + 64 * r;
    ok[r] = i <= d.nx - 1;
    p[r] = sp.at(ok[r] ? i : i0, j, k);
    b[r] = code[p[r]]; // every interior point has a byte
  }
  typename LutOf<T>::type L;
  const bool coded = load_lut(info, lut, L);
  const bool oc_coded = coded && info[8] == 0;
  T s[PTS], f[PTS], c[PTS];
#pragma unroll
  for (int r = 0; r < PTS; ++r) {
    // every point of the thread has colour want and the parity of i0
    const SplitNb nb = split_nb(sp, p[r], i0, want);
    Couplings<T> cp;
    if (coded) {
      cp.e = (b[r] & 1u) ? L.eh : L.el;
      cp.w = (b[r] & 2u) ? L.eh : L.el;
      cp.n = (b[r] & 4u) ? L.nh : L.nl;
      cp.s = (b[r] & 8u) ? L.nh : L.nl;
      cp.u = (b[r] & 16u) ? L.uh : L.ul;
      cp.dn = (b[r] & 32u) ? L.uh : L.ul;
    } else {
      cp = array_couplings<T>(oE, oN, uC, p[r], nb);
    }
    s[r] = cp.n * x[nb.n] + cp.s * x[nb.s] + cp.e * x[nb.e] +
           cp.w * x[nb.w] + cp.dn * x[nb.dn] + cp.u * x[nb.u];
    f[r] = fc[p[r]];
    c[r] = oc_coded ? oc_of(octab, b[r]) : oC[p[r]];
  }
#pragma unroll
  for (int r = 0; r < PTS; ++r)
    if (ok[r])
      x[p[r]] = (f[r] + keep * s[r]) / (c[r] + T(0));
}

// points per thread of the coded colour pass
constexpr int kCodePts = 2;

template <typename T>
int launch_gs7_code(const Dims &d, const T *oC, const T *fc, const T *oE,
                    const T *oN, const T *uC, const unsigned char *code,
                    const int *info, const T *lut, const T *octab, T *x,
                    int itmax, int iadjoint, int zero_init, cudaStream_t s) {
  const dim3 g(cdiv(cdiv(d.nx - 2, 2), 32 * kCodePts), cdiv(d.ny - 2, 8),
               (unsigned)(d.nz - 2));
  for (int it = 0; it < itmax; ++it)
    for (int c = 0; c <= 1; ++c) {
      const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
      const T keep = zero_init ? T(0) : T(1);
      gs7_code_color_kernel<T, kCodePts><<<g, interior_block(), 0, s>>>(
          d, oC, fc, oE, oN, uC, code, info, lut, octab, x, want, keep);
      zero_init = 0;
    }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// defect7_split_kernel with the couplings from the code byte when coded;
// two points per thread (32 apart in the row) for the same reason as the
// colour pass
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4)
    defect7_code_kernel(Dims d, const T *__restrict__ oC,
                        const T *__restrict__ oE, const T *__restrict__ oN,
                        const T *__restrict__ uC,
                        const unsigned char *__restrict__ code,
                        const int *__restrict__ info,
                        const T *__restrict__ lut,
                        const T *__restrict__ octab, const T *__restrict__ f,
                        const T *__restrict__ x, T *__restrict__ r) {
  const int i0 = blockIdx.x * blockDim.x * 2 + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k = blockIdx.z + 2;
  if (i0 > d.nx - 1 || j > d.ny - 1)
    return;
  const Split sp = Split::of(d);
  int ii[2], p[2];
  bool ok[2];
  unsigned b[2];
  // loads independent of the coding first (see gs7_code_color_kernel)
  T xv[2][7], fv[2], cv[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    ii[q] = i0 + 32 * q;
    ok[q] = ii[q] <= d.nx - 1;
    if (!ok[q])
      ii[q] = i0;
    p[q] = sp.at(ii[q], j, k);
    b[q] = code[p[q]];
    const SplitNb nb =
        split_nb(sp, p[q], ii[q], (ii[q] + j + k) & 1);
    xv[q][0] = x[nb.n];
    xv[q][1] = x[nb.s];
    xv[q][2] = x[nb.e];
    xv[q][3] = x[nb.w];
    xv[q][4] = x[nb.dn];
    xv[q][5] = x[nb.u];
    xv[q][6] = x[p[q]];
    fv[q] = f[p[q]];
  }
  typename LutOf<T>::type L;
  const bool coded = load_lut(info, lut, L);
  const bool oc_coded = coded && info[8] == 0;
  T out[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    cv[q] = oc_coded ? oc_of(octab, b[q]) : oC[p[q]];
    Couplings<T> c;
    if (coded) {
      c.e = (b[q] & 1u) ? L.eh : L.el;
      c.w = (b[q] & 2u) ? L.eh : L.el;
      c.n = (b[q] & 4u) ? L.nh : L.nl;
      c.s = (b[q] & 8u) ? L.nh : L.nl;
      c.u = (b[q] & 16u) ? L.uh : L.ul;
      c.dn = (b[q] & 32u) ? L.uh : L.ul;
    } else {
      c = array_couplings<T>(oE, oN, uC, p[q],
                             split_nb(sp, p[q], ii[q], (ii[q] + j + k) & 1));
    }
    const T ax = -c.n * xv[q][0] - c.s * xv[q][1] - c.e * xv[q][2] -
                 c.w * xv[q][3] - c.dn * xv[q][4] - c.u * xv[q][5] +
                 (cv[q] + T(0)) * xv[q][6];
    out[q] = fv[q] - ax;
  }
#pragma unroll
  for (int q = 0; q < 2; ++q)
    if (ok[q])
      r[d.at(ii[q], j, k)] = out[q];
}

// ---- the double operator of the same level (the refinement residual) ----
// The double couplings take the code bytes of the float ones when each
// direction's double values are two as well: lut64[2q + bit] holds the
// double value of direction q (E, N, U) for a bit, and info[7] is set when
// any double coupling differs from its entry bit for bit.
template <typename T>
__device__ __forceinline__ void couplings64_of(const Dims &d, const T *oE,
                                               const T *oN, const T *uC,
                                               int p, T (&c)[6]) {
  c[0] = oE[p];
  c[1] = oE[p - 1];
  c[2] = oN[p];
  c[3] = oN[p - d.sy()];
  c[4] = uC[p];
  c[5] = uC[p - d.sz()];
}

// pass 1: every point stores its double couplings under their bits (equal
// values when the level is two-valued; pass 2 finds out)
template <typename T>
__global__ void __launch_bounds__(256)
    lut64_store_kernel(Dims d, const T *__restrict__ oE,
                       const T *__restrict__ oN, const T *__restrict__ uC,
                       const unsigned char *__restrict__ code, T *lut64) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  const unsigned b = code[Split::of(d).at(t.i, t.j, t.k)];
  T c[6];
  couplings64_of(d, oE, oN, uC, p, c);
#pragma unroll
  for (int q = 0; q < 6; ++q)
    lut64[2 * (q >> 1) + ((b >> q) & 1u)] = c[q];
}

// pass 2: info[7] |= 1 on any double coupling that is not its entry
template <typename T>
__global__ void __launch_bounds__(256)
    lut64_check_kernel(Dims d, const T *__restrict__ oE,
                       const T *__restrict__ oN, const T *__restrict__ uC,
                       const unsigned char *__restrict__ code,
                       const T *__restrict__ lut64, int *info) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int p = d.at(t.i, t.j, t.k);
  const unsigned b = code[Split::of(d).at(t.i, t.j, t.k)];
  T c[6];
  couplings64_of(d, oE, oN, uC, p, c);
  bool bad = false;
#pragma unroll
  for (int q = 0; q < 6; ++q)
    bad |= __double_as_longlong(c[q]) !=
           __double_as_longlong(lut64[2 * (q >> 1) + ((b >> q) & 1u)]);
  if (bad)
    atomicOr(&info[7], 1);
}

// defect_norm_kernel<7, double, float, true> (the refinement residual r =
// f - A x64, written to the split float right-hand side, and its sum of
// squares) with the double couplings from the code bytes when both codings
// hold: the same values, the same order, the same bits.
template <typename T, typename R>
__global__ void __launch_bounds__(kReduceThreads, 6)
    defect_norm_code_kernel(Dims d, Op14<T> A, const T *__restrict__ f,
                            const T *__restrict__ x,
                            const unsigned char *__restrict__ code,
                            const T *__restrict__ lut64,
                            const T *__restrict__ octab,
                            const int *__restrict__ info,
                            R *__restrict__ r, ReduceSlot s) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int k0 = 2 + blockIdx.z * kReducePlanes;
  const int k1 = min(k0 + kReducePlanes - 1, d.nz - 1);
  const int sy = d.sy(), sz = d.sz();
  const bool coded = info[6] == 0 && info[7] == 0;
  const bool oc_coded = coded && info[8] == 0;
  // low / high double value per direction, in registers (selected below,
  // never indexed at run time)
  const T el = coded ? lut64[0] : T(0), eh = coded ? lut64[1] : T(0);
  const T nl = coded ? lut64[2] : T(0), nh = coded ? lut64[3] : T(0);
  const T ul = coded ? lut64[4] : T(0), uh = coded ? lut64[5] : T(0);
  const Split sp = Split::of(d);
  double acc = 0.0;
  if (i <= d.nx - 1 && j <= d.ny - 1) {
    // unrolled over the block's planes so the loads of several planes are
    // in flight together; acc still adds the planes in order
#pragma unroll
    for (int q = 0; q < kReducePlanes; ++q) {
      const int k = k0 + q;
      if (k > k1)
        break;
      const int p = d.at(i, j, k);
      const int sidx = sp.at(i, j, k);
      // the loads that do not depend on the code byte first, so a plane
      // costs one memory round trip
      const T xn = x[p + sy], xs = x[p - sy], xe = x[p + 1], xw = x[p - 1];
      const T xd = x[p - sz], xu = x[p + sz], xc = x[p], fv = f[p];
      T c[6];
      T oc;
      if (coded) {
        const unsigned b = code[sidx];
        oc = oc_coded ? oc_of(octab, b) : A.a[kOC][p];
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
      // apply7's order: -oN x_n - oN_s x_s - oE x_e - oE_w x_w - uC_d x_d
      // - uC x_u + (oC + 0) x
      const T ax = -c[2] * xn - c[3] * xs - c[0] * xe - c[1] * xw -
                   c[5] * xd - c[4] * xu + (oc + T(0)) * xc;
      const T dv = fv - ax;
      r[sidx] = (R)dv;
      acc += (double)dv * (double)dv;
    }
  }
  double v[1] = {block_sum_2d(acc, sh)};
  reduce_finish<1>(v, s, nullptr);
}

inline dim3 defect7_code_grid(const Dims &d) {
  return dim3(cdiv(d.nx - 2, 64), cdiv(d.ny - 2, 8), (unsigned)(d.nz - 2));
}

} // namespace pmg
