// Problem handle: the PBE_linear_problem class (PBE_pmgc_class.h:112-1174)
// with runtime sizes, its Galerkin hierarchy resident in one device arena,
// the V-cycle, and the FP64 / mixed-precision solves.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <new>

#include "build_kernels.cuh"
#include "bottom_cluster.cuh"
#include "bottom_cycle.cuh"
#include "gs27_tiled.cuh"
#include "gs27_tma.cuh"
#include "gs7_stream.cuh"
#include "resid_stream.cuh"
#include "defect_stream.cuh"

#include <cudaTypedefs.h>
#include "launch.cuh"
#include "pcg_kernels.cuh"
#include "pcg_split.cuh"
#include "split_layout.cuh"
#include "reduce_kernels.cuh"

namespace pmg {

constexpr int kMaxLevels = 12;
constexpr int kCgMaxIters = 20000;
constexpr int kProfSlots = 8 * (kMaxLevels + 1);

struct LevelBuf {
  int n = 0;
  Dims d{};
  long n3 = 0;
  // the float arrays of the level (mixed path): rows padded to a 16-byte
  // multiple on the levels the 27-point smoother stages by tensor-memory
  // access (between the one-launch bottom levels and the finest level),
  // else d
  Dims d32{};
  long n3_32 = 0;
  // tensor maps of the padded float iterate and its ping-pong partner (the
  // 27-point smoother's x staging)
  struct TmaMaps {
    CUtensorMap x, xalt;
  } tma;
  bool tma_ok = false;
  int tma_tile = 0; // the tile edge the maps' boxes are made for
  // the padded float levels of the 32 tile class: the fourteen couplings
  // again, split by the parity of i (gs27_tma_kernel's copies)
  CoefSplit cs{};
  float *opc[14] = {};
  // the refinement paths' finest level: tensor maps of the colour-split
  // correction and right-hand side (the streamed colour pass; its code
  // bytes come from codeb)
  StreamMaps smaps;
  // the streamed defect (defect_stream.cuh, bulk copies of the same
  // arrays) fits the level
  bool defect_ok = false;
  double *op[14] = {};
  double *P[27] = {}; // prolongation from this level to level+1
  double *x = nullptr, *f = nullptr, *r = nullptr;
  double *xalt = nullptr; // ping-pong partner of x for the 27-point smoother
  float *op32[14] = {};
  float *P32[27] = {};
  float *x32 = nullptr, *f32 = nullptr, *r32 = nullptr;
  float *xalt32 = nullptr;
  double *omega = nullptr; // damping computed on this level (device)
  // mixed / fp64-fast finest level: coded couplings (split_layout.cuh) and
  // their table
  unsigned char *code = nullptr;
  // the code bytes blocked for the streamed colour pass (CodeBlocks)
  unsigned char *codeb = nullptr;
  int *code_info = nullptr; // device: ranges and the mismatch flags
  double *lut64 = nullptr;  // device: the double couplings of the codes
  // device: the centre coefficient by code (bit 6 of the code byte) and the
  // per-code ranges it is found from
  double *octab64 = nullptr;
  float *octab32 = nullptr;
  long long *oc_range = nullptr;
  // fp64-fast finest level: the correction, its right-hand side and the
  // operator (oC oE oN uC) in the colour-split layout, double
  double *xs = nullptr, *fs = nullptr;
  double *ops[4] = {};

  Op14<double> A64(int nops) const {
    Op14<double> A{};
    for (int s = 0; s < nops; ++s)
      A.a[s] = op[s];
    return A;
  }
  Op14<float> A32(int nops) const {
    Op14<float> A{};
    for (int s = 0; s < nops; ++s)
      A.a[s] = op32[s];
    return A;
  }
  P27<double> Pc() const {
    P27<double> p;
    for (int s = 0; s < 27; ++s)
      p.p[s] = P[s];
    return p;
  }
  P27<float> Pc32() const {
    P27<float> p;
    for (int s = 0; s < 27; ++s)
      p.p[s] = P32[s];
    return p;
  }
};

// Two-pass arena planner: the first pass (base == nullptr) only counts.
struct Arena {
  char *base = nullptr;
  size_t off = 0;
  template <typename T> T *take(long count) {
    off = (off + 255) & ~size_t(255);
    T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
    off += sizeof(T) * (size_t)count;
    return p;
  }
};

// The arrays a refinement-step V-cycle (vcycle_ref) works on, by its
// arithmetic type: float copies on every level (mixed), or the double
// arrays, with the colour-split copies on the finest level (fp64-fast).
template <typename T> struct LevelArrays;
template <> struct LevelArrays<float> {
  static float *x(LevelBuf &v) { return v.x32; }
  static float *f(LevelBuf &v) { return v.f32; }
  static float *r(LevelBuf &v) { return v.r32; }
  static float *alt(LevelBuf &v) { return v.xalt32; }
  static float *fine_op(LevelBuf &v, int s) { return v.op32[s]; }
  static const float *lut(LevelBuf &) { return nullptr; }
  static const float *octab(LevelBuf &v) { return v.octab32; }
  static const Dims &dims(const LevelBuf &v) { return v.d32; }
  static Op14<float> A(const LevelBuf &v) { return v.A32(14); }
  static P27<float> P(const LevelBuf &v) { return v.Pc32(); }
};
template <> struct LevelArrays<double> {
  static double *x(LevelBuf &v) { return v.xs ? v.xs : v.x; }
  static double *f(LevelBuf &v) { return v.fs ? v.fs : v.f; }
  static double *r(LevelBuf &v) { return v.r; }
  static double *alt(LevelBuf &v) { return v.xalt; }
  static double *fine_op(LevelBuf &v, int s) { return v.ops[s]; }
  static const double *lut(LevelBuf &v) { return v.lut64; }
  static const double *octab(LevelBuf &v) { return v.octab64; }
  static const Dims &dims(const LevelBuf &v) { return v.d; }
  static Op14<double> A(const LevelBuf &v) { return v.A64(14); }
  static P27<double> P(const LevelBuf &v) { return v.Pc(); }
};

// Fine-level set-up from atoms on the GPU (pmg_setup_gpu.cu).
int setup_fine_device(int n, double h, const double *atoms_host, int natoms,
                      const pmg_physics *ph, double *oC, double *oE,
                      double *oN, double *uC, double *f, double *x0,
                      cudaStream_t st);

// Device-resident state of one solve (pmg_solve_start): parameters, the
// residual history and the outcome, written by the solve graph's control
// kernels and copied to pinned host memory at its end.
constexpr int kMaxHist = 1024;
struct SolveState {
  double tol;
  int max_cycles;
  int cycles;
  // 0 running / converged / capped, 1 diverged, 2 r0 not finite, 3 a
  // staged copy (27-point smoother, streamed finest pass or residual) did
  // not arrive
  int status;
  int pad;
  double r0, r;
  double hist[kMaxHist + 1];
};

} // namespace pmg

using namespace pmg;

struct pmg_problem {
  int base = 0, nlev = 0, precision = 0;
  double box = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t created_stream = nullptr; // destroyed with the problem
  char *arena = nullptr;
  size_t arena_bytes = 0;
  LevelBuf lv[kMaxLevels + 1];
  double *cg_r = nullptr, *cg_p = nullptr, *cg_ap = nullptr;
  int *cg_status = nullptr;
  // device: set by the staged kernels (gs27_tma_kernel, gs7_stream_kernel,
  // defect_norm_stream_kernel) on a lost stage
  int *kernel_err = nullptr;
  int num_sms = 0;
  // Relative stopping threshold of the coarsest CG on the mixed path's
  // correction equation (the FP64 path keeps the class's absolute 1e-8).
  double coarse_rtol = 1e-4;
  // Mixed path: levels 1 .. bottom_top (n <= 17) run in one CTA
  // (bottom_cycle_kernel); 0 when level 1 is too large.
  int bottom_top = 0;
  // pmg_set_tma_staging when the problem was created (read once, so that
  // both passes of plan() lay out the same arrays)
  bool tma_on = true;
  ReduceSlot red_norm{}, red_lambda{};
  double *h_pinned = nullptr; // [0] residual sum, [1..] spare
  int *h_status = nullptr;
  bool fine_set = false, built = false;
  // One V-cycle (plus the residual norm) captured as a CUDA graph.
  cudaGraphExec_t cycle_exec = nullptr;
  // A whole solve as one graph: initial residual, then a device-side while
  // loop over cycles (conditional node), then the state copy to the host.
  cudaGraphExec_t solve_exec = nullptr;
  long long solve_pre_kernels = 0, solve_body_kernels = 0;
  SolveState *d_state = nullptr; // arena
  SolveState *h_state = nullptr; // pinned
  cudaEvent_t done_ev = nullptr;
  bool solve_pending = false;
  bool host_loop = false; // pmg_problem_set_host_loop
  bool throughput = false; // pmg_problem_set_throughput_mode
  bool use_codes = true;   // pmg_problem_set_coded_couplings
  // the finest colour passes stream their rows through shared memory
  // (gs7_stream.cuh); fixed at creation by pmg_set_finest_streaming
  bool stream_fine = false;
  // MG-preconditioned CG on the finest level (allocated on first use):
  // right-hand side, iterate, residual, preconditioned residual, search
  // direction, A times it; three reduction slots; the iteration state.
  struct {
    char *mem = nullptr;
    size_t bytes = 0;
    double *b = nullptr, *xs = nullptr, *r = nullptr, *z = nullptr,
           *pv = nullptr, *ap = nullptr;
    ReduceSlot rr{}, rz{}, pap{};
    PcgState *d_st = nullptr, *h_st = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long head_kernels = 0, body_kernels = 0;
  } pcg;
  // kernel launches issued by this problem (build, solve, graph replays)
  long long launches = 0;
  long long cycle_kernels = 0; // kernel nodes in the captured cycle graph
  // phase timing (pmg_problem_set_profiling)
  bool prof_on = false;
  cudaEvent_t prof_ev[2][kProfSlots] = {};
  bool prof_used[kProfSlots] = {};
  double prof_ms[kProfSlots] = {};
  long prof_count[kProfSlots] = {};
};

namespace {

// pmg_set_tma_staging: problems created while it is off use gs27_tiled.cuh
// on every level (the same bits)
std::atomic<int> g_tma_on{1};
bool tma_disabled() { return g_tma_on.load() == 0; }
// pmg_set_finest_streaming: problems created while it is off use the
// per-point-load colour pass (gs7_code_color_kernel) on the finest level
std::atomic<int> g_stream_on{1};
// pmg_test_tma_short_delivery: extra bytes every stage waits for
std::atomic<unsigned> g_tma_extra_tx{0};

int level_n(int base, int L) { return base * (1 << L) + 1; }

// The damping reduction of a coarse level (ideal_lambda_kernel with the
// level's planes per block)
template <typename T>
void launch_ideal_lambda(const Dims &d, const Op14<T> &A, const T *x,
                         const T *r, ReduceSlot red, double *w,
                         cudaStream_t s) {
  const dim3 g = lambda_grid(d), b = interior_block();
  const int pl = lambda_planes(d);
  if (pl == 4) {
    if constexpr (sizeof(T) == sizeof(float))
      ideal_lambda_r32_kernel<4><<<g, b, 0, s>>>(d, A, x, r, red, w);
    else
      ideal_lambda_kernel<T, 4><<<g, b, 0, s>>>(d, A, x, r, red, w);
  } else if (pl == 2) {
    ideal_lambda_kernel<T, 2><<<g, b, 0, s>>>(d, A, x, r, red, w);
  } else {
    ideal_lambda_kernel<T, 1><<<g, b, 0, s>>>(d, A, x, r, red, w);
  }
}

// Mixed path: the top level of the one-launch bottom cycle (the levels up
// to 17 points per axis); 0 on the other paths.
int bottom_top_of(int base, int nlev, int precision) {
  int top = 0;
  if (precision == PMG_PREC_MIXED)
    for (int L = 1; L < nlev && L <= kBottomMaxLevels; ++L)
      if (level_n(base, L) <= kBottomMaxN)
        top = L;
  return top;
}

// Lays out every device array of a problem; with a.base == nullptr only
// counts bytes.
void plan(pmg_problem *p, Arena &a) {
  const bool mixed = p->precision == PMG_PREC_MIXED;
  // the finest level's colour-split double copies and code bytes: fp64-fast
  // (its correction equation) and FP64 (the class's cycle on split copies
  // of x and f, converted at the level's V-cycle)
  const bool fast = p->precision == PMG_PREC_FP64_FAST ||
                    p->precision == PMG_PREC_FP64;
  const int bottom_top = bottom_top_of(p->base, p->nlev, p->precision);
  for (int L = 1; L <= p->nlev; ++L) {
    LevelBuf &v = p->lv[L];
    v.n = level_n(p->base, L);
    v.d = Dims{v.n, v.n, v.n};
    v.n3 = v.d.count();
    const bool fine = L == p->nlev;
    const bool pitched = mixed && !fine && L > bottom_top;
    v.d32 = pitched ? Dims{v.n, v.n, v.n, (v.n + 3) & ~3} : v.d;
    v.n3_32 = v.d32.count();
    const int nops = fine ? 4 : 14;
    for (int s = 0; s < 14; ++s)
      v.op[s] = s < nops ? a.take<double>(v.n3) : nullptr;
    for (int s = 0; s < 27; ++s)
      v.P[s] = fine ? nullptr : a.take<double>(v.n3);
    // The mixed path keeps double iterates only on the finest level (x64,
    // f) and on level 1 (the double CG).
    const bool need64 = !mixed || fine || L == 1;
    v.x = need64 ? a.take<double>(v.n3) : nullptr;
    v.f = need64 ? a.take<double>(v.n3) : nullptr;
    v.r = (mixed && L > 1) ? nullptr : a.take<double>(v.n3);
    // ping-pong partners of the eight-colour smoother (levels 2 .. nlev-1)
    const bool smoothed = L > 1 && !fine;
    v.xalt = (smoothed && !mixed) ? a.take<double>(v.n3) : nullptr;
    v.omega = a.take<double>(1);
    // the refinement paths' finest operator, correction, its right-hand
    // side and the code bytes are colour-split (split_layout.cuh)
    const long ns = fine ? Split::of(v.d).count() : 0;
    if (mixed) {
      const long m = v.n3_32;
      const long mf = fine ? ns : m;
      for (int s = 0; s < 14; ++s)
        v.op32[s] = (L > 1 && s < nops) ? a.take<float>(mf) : nullptr;
      for (int s = 0; s < 27; ++s)
        v.P32[s] = fine ? nullptr : a.take<float>(m);
      v.x32 = a.take<float>(mf);
      v.f32 = a.take<float>(mf);
      v.r32 = L > 1 ? a.take<float>(m) : nullptr; // reference layout
      v.xalt32 = smoothed ? a.take<float>(m) : nullptr;
      v.cs = CoefSplit::of(v.d32);
      const bool wide =
          pitched && gs27_tile_by_size(v.d32) == 32 && p->tma_on;
      for (int s = 0; s < 14; ++s)
        v.opc[s] = wide ? a.take<float>(v.cs.count(v.d32.nz)) : nullptr;
      v.code = fine ? a.take<unsigned char>(ns) : nullptr;
      v.codeb = fine ? a.take<unsigned char>(CodeBlocks::of(v.d).bytes(v.d))
                     : nullptr;
      v.code_info = fine ? a.take<int>(12) : nullptr;
      v.lut64 = fine ? a.take<double>(6) : nullptr;
      v.octab64 = fine ? a.take<double>(128) : nullptr;
      v.octab32 = fine ? a.take<float>(128) : nullptr;
      v.oc_range = fine ? a.take<long long>(128) : nullptr;
    }
    if (fast && fine) {
      for (int s = 0; s < 4; ++s)
        v.ops[s] = a.take<double>(ns);
      v.xs = a.take<double>(ns);
      v.fs = a.take<double>(ns);
      v.code = a.take<unsigned char>(ns);
      v.codeb = a.take<unsigned char>(CodeBlocks::of(v.d).bytes(v.d));
      v.code_info = a.take<int>(12);
      v.lut64 = a.take<double>(6);
      v.octab64 = a.take<double>(128);
      v.oc_range = a.take<long long>(128);
    }
  }
  const long n1 = p->lv[1].n3;
  p->cg_r = a.take<double>(n1);
  p->cg_p = a.take<double>(n1);
  p->cg_ap = a.take<double>(n1);
  p->cg_status = a.take<int>(2);
  p->kernel_err = a.take<int>(1);
  p->d_state = a.take<SolveState>(1);
  // partials of the largest launch using each slot: the finest level's
  // reductions, and the damping on any coarse level
  const dim3 gf = reduce_grid(p->lv[p->nlev].d);
  long blocks = (long)gf.x * gf.y * gf.z;
  // the streamed refinement residual's CTAs (resid_stream.cuh)
  blocks = std::max(blocks, resid_max_ctas(p->lv[p->nlev].d));
  for (int L = 1; L < p->nlev; ++L) {
    const dim3 g = lambda_grid(p->lv[L].d);
    blocks = std::max(blocks, (long)g.x * g.y * g.z);
  }
  for (ReduceSlot *s : {&p->red_norm, &p->red_lambda}) {
    s->partials = a.take<double>(2L * blocks);
    s->ticket = a.take<unsigned int>(1);
    s->result = a.take<double>(2);
  }
}

int check_shape(int base, int nlev) {
  if (base < 1 || nlev < 2 || nlev > kMaxLevels)
    return PMG_ERR_ARG;
  if ((long)base * (1L << nlev) + 1 > kMaxN)
    return PMG_ERR_ARG;
  return PMG_OK;
}

// ---- phase timing ------------------------------------------------------------
// Optional CUDA-event timing of every V-cycle phase, recorded inside the
// captured cycle graph. Slot = level * 8 + phase; level 0 holds the
// finest-level residual (0), the refinement update (1) and conversions (2).
enum Phase {
  kPhPre = 0, kPhDefect, kPhRestrict, kPhCoarse, kPhLambda, kPhInterp,
  kPhAxpy, kPhPost
};
enum GlobalPhase { kPhResidual = 0, kPhCorrect = 1, kPhConvert = 2 };

// Inside stream capture a plain cudaEventRecord only orders work; the
// external flag (valid only while capturing) makes the captured node record
// the event for timing.
void prof_record(pmg_problem *p, cudaEvent_t ev) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(p->stream, &st);
  if (st == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(ev, p->stream, cudaEventRecordExternal);
  else
    cudaEventRecord(ev, p->stream);
}
void prof_begin(pmg_problem *p, int slot) {
  if (p->prof_on)
    prof_record(p, p->prof_ev[0][slot]);
}
void prof_end(pmg_problem *p, int slot) {
  if (p->prof_on) {
    prof_record(p, p->prof_ev[1][slot]);
    p->prof_used[slot] = true;
  }
}
void prof_collect(pmg_problem *p) {
  if (!p->prof_on)
    return;
  for (int q = 0; q < kProfSlots; ++q)
    if (p->prof_used[q]) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p->prof_ev[0][q], p->prof_ev[1][q]) ==
          cudaSuccess) {
        p->prof_ms[q] += ms;
        p->prof_count[q] += 1;
      }
    }
  // a failed query must not surface as the next launch's error
  (void)cudaGetLastError();
}

// ---- V-cycle pieces (FP64) ------------------------------------------------

// nsweeps smoothing sweeps on level L (smooth_domain_sol,
// PBE_pmgc_class.h:868-927): red-black in place on the finest level,
// two-launch eight-colour (ping-pong between x and xalt) below. *cur is the
// buffer holding the iterate on entry and on return.
int smooth64(pmg_problem *p, int L, int nsweeps, int zero_init,
             double **cur) {
  LevelBuf &v = p->lv[L];
  if (L == p->nlev && *cur == v.xs) { // the split coded copies
    if (p->stream_fine)
      return launch_gs7_stream<double>(
          v.smaps, v.d, v.ops[kOC], v.ops[kOE], v.ops[kON], v.ops[kUC],
          v.code_info, v.lut64, v.octab64, v.codeb, v.xs, nsweeps, 0,
          zero_init, p->kernel_err, g_tma_extra_tx.load(), p->stream);
    return launch_gs7_code<double>(v.d, v.ops[kOC], v.fs, v.ops[kOE],
                                   v.ops[kON], v.ops[kUC], v.code,
                                   v.code_info, v.lut64, v.octab64, v.xs,
                                   nsweeps, 0, zero_init, p->stream);
  }
  if (L == p->nlev)
    return launch_gs7<double>(v.d, v.op[kOC], nullptr, v.f, v.op[kOE],
                              v.op[kON], v.op[kUC], *cur, nsweeps, 0,
                              zero_init, p->stream);
  double *alt = *cur == v.x ? v.xalt : v.x;
  return launch_gs27_pp<double>(v.d, v.A64(14), nullptr, v.f, *cur, alt,
                                nsweeps, 0, zero_init, p->stream, cur);
}

// Coarsest level: the class's CG (absolute 1e-8, first test on
// sqrt(sqrt(r.r))) on the FP64 path; on the refinement paths (mixed,
// fp64-fast) a zero-started CG to coarse_rtol relative to its initial
// residual.
int cg_level1(pmg_problem *p, const double *rhs, double *x) {
  LevelBuf &v = p->lv[1];
  if (p->precision != PMG_PREC_FP64)
    return launch_cg_level(v.d, v.A64(14), rhs, x, p->cg_r, p->cg_p,
                           p->cg_ap, 0.0, p->coarse_rtol, 0, kCgMaxIters,
                           p->cg_status, p->stream);
  return launch_cg_level(v.d, v.A64(14), rhs, x, p->cg_r, p->cg_p, p->cg_ap,
                         1e-8, 0.0, 1, kCgMaxIters, p->cg_status, p->stream);
}

// v_cycle of the class (PBE_pmgc_class.h:1070-1114) on level L.
int vcycle64(pmg_problem *p, int L, int as_preconditioner) {
  cudaStream_t s = p->stream;
  LevelBuf &v = p->lv[L];
  const int sl = L * 8;
  if (L == 1) {
    prof_begin(p, sl + kPhCoarse);
    int rc = cg_level1(p, v.f, v.x);
    prof_end(p, sl + kPhCoarse);
    return rc;
  }
  LevelBuf &c = p->lv[L - 1];
  const int kind = L == p->nlev ? 7 : 27;
  int rc;
  // the finest level runs on its colour-split coded copies (the kernels of
  // the refinement paths, the class's per-point arithmetic: the same bits);
  // x and f are converted at the level's V-cycle (f each time: the
  // preconditioner's right-hand side changes per call)
  const bool split = kind == 7 && p->use_codes && v.xs != nullptr;
  double *x = split ? v.xs : v.x;
  const int zero_init = (L != p->nlev) || as_preconditioner;
  if (split) {
    to_split_kernel<double, double><<<flat_grid(v.n3), 256, 0, s>>>(v.d, v.f,
                                                                    v.fs);
    to_split_kernel<double, double><<<flat_grid(v.n3), 256, 0, s>>>(v.d, v.x,
                                                                    v.xs);
    PMG_LAUNCH_CHECK();
  }
  prof_begin(p, sl + kPhPre);
  if ((rc = smooth64(p, L, 2, zero_init, &x)))
    return rc;
  prof_end(p, sl + kPhPre);
  prof_begin(p, sl + kPhDefect);
  if (split)
    defect7_code_kernel<double>
        <<<defect7_code_grid(v.d), interior_block(), 0, s>>>(
            v.d, v.ops[kOC], v.ops[kOE], v.ops[kON], v.ops[kUC], v.code,
            v.code_info, v.lut64, v.octab64, v.fs, x, v.r);
  else if (kind == 7)
    defect_kernel<7, double><<<interior_grid(v.d), interior_block(), 0, s>>>(
        v.d, v.A64(4), v.f, x, v.r);
  else
    defect_kernel<27, double><<<interior_grid(v.d), interior_block(), 0, s>>>(
        v.d, v.A64(14), v.f, x, v.r);
  prof_end(p, sl + kPhDefect);
  prof_begin(p, sl + kPhRestrict);
  restrict_kernel<double, double>
      <<<interior_grid(c.d), interior_block(), 0, s>>>(v.d, c.d, v.r, c.f,
                                                       c.Pc());
  prof_end(p, sl + kPhRestrict);
  PMG_LAUNCH_CHECK();
  if ((rc = vcycle64(p, L - 1, 0)))
    return rc;
  prof_begin(p, sl + kPhLambda);
  launch_ideal_lambda<double>(c.d, c.A64(14), c.x, c.f, p->red_lambda,
                              c.omega, s);
  prof_end(p, sl + kPhLambda);
  // x += w * (interpolated correction), one pass
  prof_begin(p, sl + kPhInterp);
  if (split)
    interp_add_kernel<double, true>
        <<<interp_grid(c.d), interior_block(), 0, s>>>(c.d, v.d, c.x, c.Pc(),
                                                       x, c.omega);
  else
    interp_add_kernel<double, false>
        <<<interp_grid(c.d), interior_block(), 0, s>>>(c.d, v.d, c.x, c.Pc(),
                                                       x, c.omega);
  prof_end(p, sl + kPhInterp);
  PMG_LAUNCH_CHECK();
  prof_begin(p, sl + kPhPost);
  if ((rc = smooth64(p, L, 2, 0, &x)))
    return rc;
  prof_end(p, sl + kPhPost);
  if (x != (split ? v.xs : v.x)) {
    set_last_message("vcycle64: iterate left the level's buffer");
    return PMG_ERR_STATE;
  }
  if (split) {
    from_split_kernel<double, double><<<flat_grid(v.n3), 256, 0, s>>>(
        v.d, v.xs, v.x);
    PMG_LAUNCH_CHECK();
  }
  return PMG_OK;
}

// Residual sum of squares of the finest level into red_norm.result[0] and
// then into pinned host memory (not synchronised here).
int residual_norm_async(pmg_problem *p, bool to_host = true) {
  LevelBuf &v = p->lv[p->nlev];
  prof_begin(p, kPhResidual);
  if (p->use_codes && p->stream_fine && resid_fits(v.d)) {
    // the streamed coded residual, its sum only (resid_stream.cuh)
    int rc = launch_resid_stream<double>(
        v.d, v.A64(4), v.f, v.x, v.code, v.lut64, v.octab64, v.code_info,
        (double *)nullptr, p->red_norm, p->kernel_err, g_tma_extra_tx.load(),
        p->stream);
    if (rc)
      return rc;
  } else {
    defect_norm_kernel<7, double, double>
        <<<reduce_grid(v.d), interior_block(), 0, p->stream>>>(
            v.d, v.A64(4), v.f, v.x, (double *)nullptr, p->red_norm);
  }
  prof_end(p, kPhResidual);
  PMG_LAUNCH_CHECK();
  if (to_host)
    PMG_CUDA_TRY(cudaMemcpyAsync(p->h_pinned, p->red_norm.result,
                                 sizeof(double), cudaMemcpyDeviceToHost,
                                 p->stream));
  return PMG_OK;
}

double norm_from_sum(const pmg_problem *p, double s) {
  const double n3 = (double)p->lv[p->nlev].n3;
  return sqrt(s / n3);
}

// ---- the 27-point smoother by tensor-memory access (gs27_tma.cuh) -----------


PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f,
                                cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    (void)cudaGetLastError();
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// A 3-D map of one padded float array of the level: extent nx x ny x nz
// (the padding reads as outside), rows px apart, boxes of a tile of size
// class tt (TmaBox, 2 tt + 12 by tt / 2 + 8, for tt = 32; TmaSqBox,
// tt + 12 by tt + 8, below).
bool encode_level_map(CUtensorMap *m, const float *base, const Dims &d,
                      int tt) {
  auto enc = tensor_map_encoder();
  if (!enc || !base || (d.px * sizeof(float)) % 16 != 0)
    return false;
  const cuuint64_t dims[3] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny,
                              (cuuint64_t)d.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)d.px * sizeof(float),
                                 (cuuint64_t)d.px * d.ny * sizeof(float)};
  const cuuint32_t box[3] = {
      (cuuint32_t)(tt == 32 ? 2 * tt + 12 : tt + 12),
      (cuuint32_t)(tt == 32 ? tt / 2 + 8 : tt + 8), 1};
  const cuuint32_t elem[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims,
             strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of every padded level (their arrays are fixed for the life
// of the problem); a level whose maps cannot be made uses gs27_tiled.cuh.
void encode_tma_maps(pmg_problem *p) {
  for (int L = 2; L < p->nlev; ++L) {
    LevelBuf &v = p->lv[L];
    v.tma_ok = false;
    if (v.d32.px == v.d.px || !v.xalt32 || v.d32.nx - 2 < 1)
      continue;
    // the size rule's tile edge (gs27_tiled.cuh)
    v.tma_tile = gs27_tile_by_size(v.d32);
    if (v.tma_tile == 32 && !v.opc[0])
      continue;
    bool ok = encode_level_map(&v.tma.x, v.x32, v.d32, v.tma_tile);
    ok = ok && encode_level_map(&v.tma.xalt, v.xalt32, v.d32, v.tma_tile);
    v.tma_ok = ok;
  }
}

// A 4-D map {entry, half, row, plane} of one colour-split array of the
// level (split_layout.cuh): boxes of bw entries of one half (or of both)
// over `rows` rows of one plane.
bool encode_split_map(CUtensorMap *m, const void *base, CUtensorMapDataType t,
                      int esz, const Dims &d, int bw, int rows,
                      int halves = 1) {
  auto enc = tensor_map_encoder();
  if (!enc || !base || ((uintptr_t)base & 15) != 0)
    return false;
  const Split sp = Split::of(d);
  const cuuint64_t dims[4] = {(cuuint64_t)sp.hp, 2, (cuuint64_t)d.ny,
                              (cuuint64_t)d.nz};
  const cuuint64_t strides[3] = {(cuuint64_t)sp.hp * esz,
                                 (cuuint64_t)sp.pitch() * esz,
                                 (cuuint64_t)sp.plane() * esz};
  const cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)halves,
                             (cuuint32_t)rows, 1};
  const cuuint32_t elem[4] = {1, 1, 1, 1};
  return enc(m, t, 4, const_cast<void *>(base), dims, strides, box, elem,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The finest colour passes of a refinement path can be streamed
// (gs7_stream.cuh): the level fits the stage ring and the box width, and
// the tensor maps of its correction, right-hand side and code bytes could
// be made (their arrays are fixed for the life of the problem).
template <typename T>
bool encode_stream_maps(LevelBuf &v, const T *x, const T *f) {
  if (!stream_fits<T>(v.d))
    return false;
  const StreamShape sh = stream_shape<T>(v.d, 1);
  constexpr int J = StreamCfg<T>::J;
  const CUtensorMapDataType t = sizeof(T) == 4
                                    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  v.defect_ok = defect_fits<T>(v.d);
  // (the streamed pass reads its code bytes by bulk copies of the blocked
  // copy, not by a map)
  return encode_split_map(&v.smaps.x, x, t, sizeof(T), v.d, sh.bw, J + 2) &&
         encode_split_map(&v.smaps.f, f, t, sizeof(T), v.d, sh.bw, J);
}
bool stream_fine_ok(pmg_problem *p) {
  LevelBuf &v = p->lv[p->nlev];
  if (p->precision == PMG_PREC_MIXED)
    return encode_stream_maps<float>(v, v.x32, v.f32);
  return encode_stream_maps<double>(v, v.xs, v.fs);
}

// nsweeps eight-colour sweeps of a padded float level (launch_gs27_pp's
// order and ping-pong, the colours forward), *cur in and out.
int launch_gs27_tma(pmg_problem *p, LevelBuf &v, int nsweeps, int zero_init,
                    float **cur) {
  cudaStream_t s = p->stream;
  const Dims &d = v.d32;
  if (zero_init)
    PMG_CUDA_TRY(cudaMemsetAsync(*cur, 0, sizeof(float) * v.n3_32, s));
  const int tt = v.tma_tile;
  // tiles of 2 tt x tt / 2 points (TmaBox) for tt = 32, else tt x tt
  const unsigned tx = tt == 32 ? cdiv(d.nx - 2, 2 * tt) : cdiv(d.nx - 2, tt);
  const unsigned ty = tt == 32 ? cdiv(d.ny - 2, tt / 2) : cdiv(d.ny - 2, tt);
  const int order = 0 | 1 << 2 | 2 << 4 | 3 << 6;
  Op14<float> Ac{};
  for (int q = 0; q < 14; ++q)
    Ac.a[q] = v.opc[q];
  const Op14<float> A = v.A32(14);
  float *c = *cur;
  float *a = c == v.x32 ? v.xalt32 : v.x32;
  for (int sw = 0; sw < nsweeps; ++sw) {
    const CUtensorMap &mc = c == v.x32 ? v.tma.x : v.tma.xalt;
    const CUtensorMap &ma = c == v.x32 ? v.tma.xalt : v.tma.x;
    for (int ph = 0; ph < 2; ++ph) {
      const int kfirst = ph == 0 ? 2 : 3;
      const int planes = kfirst > d.nz - 1 ? 0 : (d.nz - 1 - kfirst) / 2 + 1;
      if (planes == 0)
        continue;
      Gs27TmaMaps m;
      m.own = mc;
      m.nb = ph == 0 ? mc : ma;
      const dim3 g(tx, ty, (unsigned)planes);
      const unsigned xt = g_tma_extra_tx.load();
      if (tt == 32)
        gs27_tma_kernel<32><<<g, Gs27Tile<32>::THREADS, 0, s>>>(
            m, d, v.cs, Ac, v.f32, a, kfirst, p->kernel_err, xt);
      else if (tt == 16)
        gs27_tma_square_kernel<16><<<g, Gs27Tile<16>::THREADS, 0, s>>>(
            m, d, A, v.f32, a, kfirst, order, p->kernel_err, xt);
      else
        gs27_tma_square_kernel<8><<<g, Gs27Tile<8>::THREADS, 0, s>>>(
            m, d, A, v.f32, a, kfirst, order, p->kernel_err, xt);
    }
    std::swap(c, a);
  }
  PMG_LAUNCH_CHECK();
  *cur = c;
  return PMG_OK;
}

// ---- refinement paths (mixed, fp64-fast) -----------------------------------

// Smoothing sweeps of a refinement-step V-cycle on level L in type T: on the
// finest level the colour-split red-black pass, with the couplings from the
// code bytes when they are coded; below, the eight-colour smoother with
// ping-pong buffers. *cur holds the iterate on entry and on return.
template <typename T>
int smooth_ref(pmg_problem *p, int L, int nsweeps, int zero_init, T **cur) {
  using A = LevelArrays<T>;
  LevelBuf &v = p->lv[L];
  // (the streamed pass's tensor maps cover the level's own correction and
  // right-hand side)
  if (L == p->nlev && p->use_codes && p->stream_fine && *cur == A::x(v))
    return launch_gs7_stream<T>(v.smaps, v.d, A::fine_op(v, kOC),
                                A::fine_op(v, kOE), A::fine_op(v, kON),
                                A::fine_op(v, kUC), v.code_info, A::lut(v),
                                A::octab(v), v.codeb, *cur, nsweeps, 0,
                                zero_init, p->kernel_err,
                                g_tma_extra_tx.load(), p->stream);
  if (L == p->nlev && p->use_codes)
    return launch_gs7_code<T>(v.d, A::fine_op(v, kOC), A::f(v),
                              A::fine_op(v, kOE), A::fine_op(v, kON),
                              A::fine_op(v, kUC), v.code, v.code_info,
                              A::lut(v), A::octab(v), *cur, nsweeps, 0,
                              zero_init, p->stream);
  if (L == p->nlev) // colour-split layout (split_layout.cuh)
    return launch_gs7_split<T>(v.d, A::fine_op(v, kOC), A::f(v),
                               A::fine_op(v, kOE), A::fine_op(v, kON),
                               A::fine_op(v, kUC), *cur, nsweeps, 0,
                               zero_init, p->stream);
  if constexpr (sizeof(T) == sizeof(float))
    if (v.tma_ok)
      return launch_gs27_tma(p, v, nsweeps, zero_init, cur);
  T *alt = *cur == A::x(v) ? A::alt(v) : A::x(v);
  return launch_gs27_pp<T>(A::dims(v), A::A(v), nullptr, A::f(v), *cur, alt,
                           nsweeps, 0, zero_init, p->stream, cur);
}

// Arguments of the one-CTA cycle over levels 1 .. top.
BottomArgs bottom_args(pmg_problem *p, int top) {
  BottomArgs a{};
  a.top = top;
  for (int L = 1; L <= top; ++L) {
    LevelBuf &v = p->lv[L];
    BottomLevel &b = a.lv[L];
    b.d = v.d;
    b.A = v.A32(L > 1 ? 14 : 0);
    b.P = v.Pc32();
    b.x = v.x32;
    b.f = v.f32;
    b.r = v.r32;
    b.omega = v.omega;
  }
  a.A1 = p->lv[1].A64(14);
  a.x1 = p->lv[1].x;
  a.f1 = p->lv[1].f;
  a.cg_r = p->cg_r;
  a.cg_p = p->cg_p;
  a.cg_ap = p->cg_ap;
  a.rtol = p->coarse_rtol;
  a.max_iters = kCgMaxIters;
  a.status = p->cg_status;
  return a;
}

// Levels 1 .. top of the mixed V-cycle in one launch: on a cluster with
// every array in shared memory when they fit (bottom_cluster.cuh), else, or
// in throughput mode, in one CTA out of global memory (bottom_cycle.cuh).
// The cluster is faster for a solve alone, but it can start only when eight
// SMs of one GPC are idle at once, which many concurrent solves rarely
// leave (measured: serving saturation 111 against 133 solves/s).
int launch_bottom(pmg_problem *p, int top) {
  const BottomArgs a = bottom_args(p, top);
  cudaStream_t s = p->stream;
  if (!p->throughput && bc_fits(a)) {
    PMG_CUDA_TRY(set_smem_limit<bottom_cluster_kernel>((int)kBcMaxSmem));
    bottom_cluster_kernel<<<kCgCtas, kBcThreads, bc_layout(a).total, s>>>(a);
  } else {
    bottom_cycle_kernel<<<1, 1024, 0, s>>>(a);
  }
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// V-cycle in type T on the correction equation, every level zero-started
// (v_cycle with as_preconditioner, PBE_pmgc_class.h:1070-1114); level 1 in
// double. T = float is the mixed path, T = double fp64-fast.
template <typename T> int vcycle_ref(pmg_problem *p, int L) {
  using A = LevelArrays<T>;
  constexpr bool kFloat = sizeof(T) == sizeof(float);
  cudaStream_t s = p->stream;
  LevelBuf &v = p->lv[L];
  const int sl = L * 8;
  if (L == 1) {
    prof_begin(p, sl + kPhCoarse);
    if (kFloat)
      convert_kernel<float, double><<<flat_grid(v.n3), 256, 0, s>>>(
          v.n3, v.f32, v.f);
    PMG_CUDA_TRY(cudaMemsetAsync(v.x, 0, sizeof(double) * v.n3, s));
    int rc = cg_level1(p, v.f, v.x);
    prof_end(p, sl + kPhCoarse);
    return rc;
  }
  LevelBuf &c = p->lv[L - 1];
  const int kind = L == p->nlev ? 7 : 27;
  int rc;
  T *x = A::x(v);
  const bool bottom_below = kFloat && L - 1 <= p->bottom_top;
  prof_begin(p, sl + kPhPre);
  if ((rc = smooth_ref<T>(p, L, 2, 1, &x)))
    return rc;
  prof_end(p, sl + kPhPre);
  prof_begin(p, sl + kPhDefect);
  if (kFloat && kind == 7 && p->use_codes && p->stream_fine && v.defect_ok &&
      x == A::x(v)) {
    // streamed (defect_stream.cuh); float only (the double version, two
    // CTAs per SM, was slower than the per-thread kernel: 114 against
    // 110 us at 257^3)
    if ((rc = launch_defect7_stream<T>(
             x, A::f(v), v.code, v.d, A::fine_op(v, kOC), A::fine_op(v, kOE),
             A::fine_op(v, kON), A::fine_op(v, kUC), v.code_info, A::lut(v),
             A::octab(v), A::r(v), p->kernel_err, g_tma_extra_tx.load(), s)))
      return rc;
  } else if (kind == 7 && p->use_codes)
    defect7_code_kernel<T>
        <<<defect7_code_grid(v.d), interior_block(), 0, s>>>(
            v.d, A::fine_op(v, kOC), A::fine_op(v, kOE), A::fine_op(v, kON),
            A::fine_op(v, kUC), v.code, v.code_info, A::lut(v), A::octab(v),
            A::f(v), x, A::r(v));
  else if (kind == 7) // split arrays in, reference-layout defect out
    defect7_split_kernel<T><<<interior_grid(v.d), interior_block(), 0, s>>>(
        v.d, A::fine_op(v, kOC), A::fine_op(v, kOE), A::fine_op(v, kON),
        A::fine_op(v, kUC), A::f(v), x, A::r(v));
  else
    defect_kernel<27, T><<<interior_grid(v.d), interior_block(), 0, s>>>(
        A::dims(v), A::A(v), A::f(v), x, A::r(v));
  prof_end(p, sl + kPhDefect);
  prof_begin(p, sl + kPhRestrict);
  restrict_kernel<T, T><<<interior_grid(c.d), interior_block(), 0, s>>>(
      A::dims(v), A::dims(c), A::r(v), A::f(c), A::P(c));
  prof_end(p, sl + kPhRestrict);
  PMG_LAUNCH_CHECK();
  if (bottom_below) {
    // levels 1 .. L-1 in one CTA; it also leaves the damping of level L-1
    prof_begin(p, sl + kPhCoarse);
    if ((rc = launch_bottom(p, L - 1)))
      return rc;
    prof_end(p, sl + kPhCoarse);
    PMG_LAUNCH_CHECK();
  } else if ((rc = vcycle_ref<T>(p, L - 1))) {
    return rc;
  }
  prof_begin(p, sl + kPhLambda);
  if (bottom_below) {
    // damping computed by the bottom kernel
  } else if (L - 1 == 1) {
    launch_ideal_lambda<double>(c.d, c.A64(14), c.x, c.f, p->red_lambda,
                                c.omega, s);
    if (kFloat)
      convert_kernel<double, float><<<flat_grid(c.n3), 256, 0, s>>>(
          c.n3, c.x, c.x32);
  } else {
    launch_ideal_lambda<T>(A::dims(c), A::A(c), A::x(c), A::f(c),
                           p->red_lambda, c.omega, s);
  }
  prof_end(p, sl + kPhLambda);
  // x += w * (interpolated correction), one pass
  prof_begin(p, sl + kPhInterp);
  if (kind == 7) // the finest iterate is split
    interp_add_kernel<T, true><<<interp_grid(c.d), interior_block(), 0, s>>>(
        A::dims(c), v.d, A::x(c), A::P(c), x, c.omega);
  else
    interp_add_kernel<T, false>
        <<<interp_grid(c.d), interior_block(), 0, s>>>(
            A::dims(c), A::dims(v), A::x(c), A::P(c), x, c.omega);
  prof_end(p, sl + kPhInterp);
  PMG_LAUNCH_CHECK();
  prof_begin(p, sl + kPhPost);
  if ((rc = smooth_ref<T>(p, L, 2, 0, &x)))
    return rc;
  prof_end(p, sl + kPhPost);
  if (x != A::x(v)) {
    set_last_message("vcycle_ref: iterate left the level's buffer");
    return PMG_ERR_STATE;
  }
  return PMG_OK;
}

// r64 = f - A x64 on the finest level, written into the correction
// equation's split right-hand side (float for mixed, double for fp64-fast),
// its sum of squares into red_norm and pinned host memory.
int refine_residual_async(pmg_problem *p, bool to_host = true) {
  LevelBuf &v = p->lv[p->nlev];
  const dim3 g = reduce_grid(v.d), b = interior_block();
  cudaStream_t s = p->stream;
  prof_begin(p, kPhResidual);
  // the streamed residual (resid_stream.cuh) on the problems whose colour
  // passes stream; the same r, the sum of squares in another fixed order
  const bool streamed = p->use_codes && p->stream_fine && resid_fits(v.d);
  if (streamed && p->precision == PMG_PREC_MIXED) {
    int rc = launch_resid_stream<float>(
        v.d, v.A64(4), v.f, v.x, v.code, v.lut64, v.octab64, v.code_info,
        v.f32, p->red_norm, p->kernel_err, g_tma_extra_tx.load(), s);
    if (rc)
      return rc;
  } else if (streamed) {
    int rc = launch_resid_stream<double>(
        v.d, v.A64(4), v.f, v.x, v.code, v.lut64, v.octab64, v.code_info,
        v.fs, p->red_norm, p->kernel_err, g_tma_extra_tx.load(), s);
    if (rc)
      return rc;
  } else if (p->precision == PMG_PREC_MIXED) {
    if (p->use_codes)
      defect_norm_code_kernel<double, float><<<g, b, 0, s>>>(
          v.d, v.A64(4), v.f, v.x, v.code, v.lut64, v.octab64, v.code_info,
          v.f32, p->red_norm);
    else
      defect_norm_kernel<7, double, float, true><<<g, b, 0, s>>>(
          v.d, v.A64(4), v.f, v.x, v.f32, p->red_norm);
  } else {
    if (p->use_codes)
      defect_norm_code_kernel<double, double><<<g, b, 0, s>>>(
          v.d, v.A64(4), v.f, v.x, v.code, v.lut64, v.octab64, v.code_info,
          v.fs, p->red_norm);
    else
      defect_norm_kernel<7, double, double, true><<<g, b, 0, s>>>(
          v.d, v.A64(4), v.f, v.x, v.fs, p->red_norm);
  }
  prof_end(p, kPhResidual);
  PMG_LAUNCH_CHECK();
  if (to_host)
    PMG_CUDA_TRY(cudaMemcpyAsync(p->h_pinned, p->red_norm.result,
                                 sizeof(double), cudaMemcpyDeviceToHost,
                                 p->stream));
  return PMG_OK;
}

// One refinement step: V-cycle on the correction (float or double), x64 +=
// e, new residual.
int refine_step(pmg_problem *p, bool to_host = true) {
  LevelBuf &v = p->lv[p->nlev];
  const bool mixed = p->precision == PMG_PREC_MIXED;
  int rc = mixed ? vcycle_ref<float>(p, p->nlev)
                 : vcycle_ref<double>(p, p->nlev);
  if (rc)
    return rc;
  prof_begin(p, kPhCorrect);
  if (mixed)
    add_correction_split_kernel<float>
        <<<interior_grid(v.d), interior_block(), 0, p->stream>>>(v.d, v.x,
                                                                 v.x32);
  else
    add_correction_split_kernel<double>
        <<<interior_grid(v.d), interior_block(), 0, p->stream>>>(v.d, v.x,
                                                                 v.xs);
  prof_end(p, kPhCorrect);
  PMG_LAUNCH_CHECK();
  return refine_residual_async(p, to_host);
}

// Kernel nodes of a graph (conditional bodies are counted by their own
// graph). The type query fails on conditional nodes; that failure is
// expected and cleared, so call this with no other error pending.
long long count_kernel_nodes(cudaGraph_t g) {
  size_t nn = 0;
  long long k = 0;
  if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn) {
    cudaGraphNode_t *nodes = new cudaGraphNode_t[nn];
    if (cudaGraphGetNodes(g, nodes, &nn) == cudaSuccess)
      for (size_t q = 0; q < nn; ++q) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess &&
            t == cudaGraphNodeTypeKernel)
          ++k;
      }
    delete[] nodes;
  }
  (void)cudaGetLastError();
  return k;
}

// One cycle with its residual: FP64 V-cycle + residual norm, or the mixed
// refinement step. to_host adds the copy of the residual sum to pinned
// memory (the host-driven loop); the device-driven loop keeps it on the GPU.
int cycle_with_residual(pmg_problem *p, bool to_host) {
  if (p->precision != PMG_PREC_FP64)
    return refine_step(p, to_host);
  int rc = vcycle64(p, p->nlev, 0);
  return rc ? rc : residual_norm_async(p, to_host);
}

// Captures one cycle (FP64: V-cycle + residual; mixed: refinement step) as a
// CUDA graph on first use.
int ensure_graph(pmg_problem *p) {
  if (p->cycle_exec)
    return PMG_OK;
  cudaGraph_t g = nullptr;
  PMG_CUDA_TRY(
      cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
  int rc = cycle_with_residual(p, true);
  cudaError_t e = cudaStreamEndCapture(p->stream, &g);
  if (rc) {
    if (g)
      cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) {
    set_last_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  p->cycle_kernels = count_kernel_nodes(g);
  e = cudaGraphInstantiate(&p->cycle_exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    p->cycle_exec = nullptr;
    set_last_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  return PMG_OK;
}

// ---- device-driven solve loop ----------------------------------------------
// The class's solve loop (PBE_pmgc_class.h:1139-1152: r0, then V-cycles until
// r / r0 < tol) with the decisions taken on the GPU: the stop test sets the
// condition of a while node, so a whole solve is one graph launch with no
// host round trip per cycle. The arithmetic of the test (sqrt of the sum over
// n^3, the ratio, the divergence guard) is the host loop's.

__global__ void solve_params_kernel(SolveState *st, double tol,
                                    int max_cycles) {
  st->tol = tol;
  st->max_cycles = max_cycles;
  st->cycles = 0;
  st->status = 0;
}

__global__ void solve_init_kernel(SolveState *st, const double *sum,
                                  double n3, const int *kernel_err,
                                  cudaGraphConditionalHandle h) {
  const double r0 = sqrt(sum[0] / n3);
  st->r0 = r0;
  st->r = r0;
  st->hist[0] = r0;
  const bool finite = isfinite(r0);
  // a staged copy of the initial residual that did not arrive leaves its
  // sum incomplete: no cycle runs, the solve reports the lost stage
  const bool lost = *kernel_err != 0;
  st->status = lost ? 3 : finite ? 0 : 2;
  cudaGraphSetConditional(
      h, (!lost && finite && r0 > 0.0 && st->max_cycles > 0) ? 1u : 0u);
}

__global__ void solve_check_kernel(SolveState *st, const double *sum,
                                   double n3, const int *kernel_err,
                                   cudaGraphConditionalHandle h) {
  const double r = sqrt(sum[0] / n3);
  const int c = ++st->cycles;
  if (c <= kMaxHist)
    st->hist[c] = r;
  st->r = r;
  const double r0 = st->r0;
  const bool diverged = !isfinite(r) || r > 1e6 * r0;
  const bool lost = *kernel_err != 0;
  if (diverged)
    st->status = 1;
  if (lost)
    st->status = 3;
  const bool go =
      !diverged && !lost && !(r / r0 < st->tol) && c < st->max_cycles;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// Takes a pending runtime error left by a graph-building call that reports
// through the last-error slot only, naming the step.
int graph_step_ok(const char *step) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    return PMG_OK;
  set_last_error(e, step, __FILE__, __LINE__);
  return PMG_ERR_CUDA;
}

// Builds [head] -> while (cond) { body } -> [tail] as one executable graph.
// head(h), body(h) and tail() enqueue work on the problem's stream (captured)
// and return a pmg_status; head and body launch the kernels that set the
// while node's condition h. The loop ends only through body's stop test, so
// a body whose capture yields fewer than two kernels is refused.
template <class Head, class Body, class Tail>
int build_loop_graph(pmg_problem *p, Head head, Body body, Tail tail,
                     cudaGraphExec_t *exec, long long *head_kernels,
                     long long *body_kernels) {
  cudaGraph_t g = nullptr, bg = nullptr;
  cudaGraphConditionalHandle h;
  cudaGraphNode_t cond = nullptr;
  int rc = PMG_OK;
  (void)cudaGetLastError();
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e == cudaSuccess)
    e = cudaGraphConditionalHandleCreate(&h, g, 0,
                                         cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    if (g)
      cudaGraphDestroy(g);
    set_last_error(e, "loop graph: conditional handle", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  e = cudaStreamBeginCaptureToGraph(p->stream, g, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = head(h);
    if (!rc)
      rc = graph_step_ok("loop graph: head");
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaStreamCaptureStatus cs;
    if (!rc)
      e = cudaStreamGetCaptureInfo(p->stream, &cs, nullptr, nullptr, &deps,
                                   &ndeps);
    if (!rc && e == cudaSuccess) {
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&cond, g, deps, ndeps, &cp);
      if (e == cudaSuccess) {
        bg = cp.conditional.phGraph_out[0];
        e = cudaStreamUpdateCaptureDependencies(
            p->stream, &cond, 1, cudaStreamSetCaptureDependencies);
      }
    }
    if (!rc && e == cudaSuccess)
      rc = tail();
    cudaGraph_t out = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(p->stream, &out);
    if (e == cudaSuccess)
      e = e2;
  }
  if (!rc && e == cudaSuccess)
    rc = graph_step_ok("loop graph: head capture");
  if (!rc && e == cudaSuccess)
    *head_kernels = count_kernel_nodes(g);
  if (!rc && e == cudaSuccess) {
    e = cudaStreamBeginCaptureToGraph(p->stream, bg, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess)
      rc = graph_step_ok("loop graph: body capture");
    if (e == cudaSuccess && !rc) {
      rc = body(h);
      if (!rc)
        rc = graph_step_ok("loop graph: body");
      cudaGraph_t out = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(p->stream, &out);
      if (e == cudaSuccess)
        e = e2;
    }
  }
  if (!rc && e == cudaSuccess) {
    *body_kernels = count_kernel_nodes(bg);
    if (*body_kernels < 2) {
      set_last_message("loop graph: loop body was not captured");
      rc = PMG_ERR_STATE;
    } else {
      e = cudaGraphInstantiate(exec, g, 0);
    }
  }
  cudaGraphDestroy(g);
  if (rc)
    return rc;
  if (e != cudaSuccess) {
    *exec = nullptr;
    set_last_error(e, "loop graph", __FILE__, __LINE__);
    return PMG_ERR_CUDA;
  }
  return PMG_OK;
}

// The solve graph: [initial residual, init] -> while (cond) {cycle, check}
// -> copy of the state to pinned memory.
int ensure_solve_graph(pmg_problem *p) {
  if (p->solve_exec)
    return PMG_OK;
  const bool refine = p->precision != PMG_PREC_FP64;
  const double n3 = (double)p->lv[p->nlev].n3;
  auto head = [&](cudaGraphConditionalHandle h) -> int {
    int rc = refine ? refine_residual_async(p, false)
                    : residual_norm_async(p, false);
    if (rc)
      return rc;
    solve_init_kernel<<<1, 1, 0, p->stream>>>(
        p->d_state, p->red_norm.result, n3, p->kernel_err, h);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  };
  auto body = [&](cudaGraphConditionalHandle h) -> int {
    int rc = cycle_with_residual(p, false);
    if (rc)
      return rc;
    solve_check_kernel<<<1, 1, 0, p->stream>>>(
        p->d_state, p->red_norm.result, n3, p->kernel_err, h);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  };
  auto tail = [&]() -> int {
    PMG_CUDA_TRY(cudaMemcpyAsync(p->h_state, p->d_state, sizeof(SolveState),
                                 cudaMemcpyDeviceToHost, p->stream));
    return PMG_OK;
  };
  return build_loop_graph(p, head, body, tail, &p->solve_exec,
                          &p->solve_pre_kernels, &p->solve_body_kernels);
}

// Drops the captured graphs (their kernels bake in thresholds and modes).
void drop_graphs(pmg_problem *p) {
  if (p->cycle_exec) {
    cudaGraphExecDestroy(p->cycle_exec);
    p->cycle_exec = nullptr;
  }
  if (p->solve_exec) {
    cudaGraphExecDestroy(p->solve_exec);
    p->solve_exec = nullptr;
  }
  if (p->pcg.exec) {
    cudaGraphExecDestroy(p->pcg.exec);
    p->pcg.exec = nullptr;
  }
}

// ---- MG-preconditioned CG ----------------------------------------------------

int pcg_alloc(pmg_problem *p) {
  if (p->pcg.mem)
    return PMG_OK;
  const LevelBuf &v = p->lv[p->nlev];
  const dim3 g = reduce_grid(v.d);
  const long blocks = (long)g.x * g.y * g.z;
  Arena a;
  for (int pass = 0; pass < 2; ++pass) {
    a.off = 0;
    double **vec[6] = {&p->pcg.b, &p->pcg.xs, &p->pcg.r, &p->pcg.z,
                       &p->pcg.pv, &p->pcg.ap};
    for (double **q : vec)
      *q = a.take<double>(v.n3);
    for (ReduceSlot *sl : {&p->pcg.rr, &p->pcg.rz, &p->pcg.pap}) {
      sl->partials = a.take<double>(blocks);
      sl->ticket = a.take<unsigned int>(1);
      sl->result = a.take<double>(1);
    }
    p->pcg.d_st = a.take<PcgState>(1);
    if (pass == 0) {
      PMG_CUDA_TRY(cudaMalloc((void **)&p->pcg.mem, a.off));
      p->pcg.bytes = a.off;
      a.base = p->pcg.mem;
    }
  }
  PMG_CUDA_TRY(cudaMemsetAsync(p->pcg.mem, 0, p->pcg.bytes, p->stream));
  if (!p->pcg.h_st)
    PMG_CUDA_TRY(cudaMallocHost((void **)&p->pcg.h_st, sizeof(PcgState)));
  return PMG_OK;
}

// z = M r: one zero-started V-cycle on r (the class's operator(),
// PBE_pmgc_class.h:1116-1133) -- FP64 V-cycle, or the float V-cycle of the
// mixed path. The finest iterate (shell zero) and, for FP64, the finest
// right-hand side are borrowed as the V-cycle's work arrays.
int precondition(pmg_problem *p, const double *r, double *z) {
  LevelBuf &v = p->lv[p->nlev];
  cudaStream_t s = p->stream;
  const size_t b = sizeof(double) * v.n3;
  if (p->precision == PMG_PREC_MIXED) {
    to_split_kernel<double, float><<<flat_grid(v.n3), 256, 0, s>>>(v.d, r,
                                                                   v.f32);
    PMG_LAUNCH_CHECK();
    int rc = vcycle_ref<float>(p, p->nlev);
    if (rc)
      return rc;
    from_split_kernel<float, double><<<flat_grid(v.n3), 256, 0, s>>>(
        v.d, v.x32, z);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  }
  if (p->precision == PMG_PREC_FP64_FAST) {
    to_split_kernel<double, double><<<flat_grid(v.n3), 256, 0, s>>>(v.d, r,
                                                                    v.fs);
    PMG_LAUNCH_CHECK();
    int rc = vcycle_ref<double>(p, p->nlev);
    if (rc)
      return rc;
    from_split_kernel<double, double><<<flat_grid(v.n3), 256, 0, s>>>(
        v.d, v.xs, z);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  }
  PMG_CUDA_TRY(cudaMemcpyAsync(v.f, r, b, cudaMemcpyDeviceToDevice, s));
  PMG_CUDA_TRY(cudaMemsetAsync(v.x, 0, b, s));
  int rc = vcycle64(p, p->nlev, 1);
  if (rc)
    return rc;
  PMG_CUDA_TRY(cudaMemcpyAsync(z, v.x, b, cudaMemcpyDeviceToDevice, s));
  return PMG_OK;
}

// The PCG graph (CG_solver, CG_Solver.h:45-242, with the MG
// preconditioner): head r = b - A x, z = M r, p = z, rs = r.z, Ap, pAp,
// alpha; body x += alpha p, r -= alpha Ap, z = M r, beta, p = z + beta p,
// Ap, pAp, alpha, stop test; tail: iterate and right-hand side back into
// the problem, state to pinned memory.
int ensure_pcg_graph(pmg_problem *p) {
  if (p->pcg.exec)
    return PMG_OK;
  LevelBuf &v = p->lv[p->nlev];
  cudaStream_t s = p->stream;
  const double n3 = (double)v.n3;
  const size_t b = sizeof(double) * v.n3;
  auto &c = p->pcg;
  const dim3 rg = reduce_grid(v.d), rb = interior_block();
  const bool mixed = p->precision == PMG_PREC_MIXED;
  const bool split = p->precision != PMG_PREC_FP64;
  // the refinement paths' finest operator as code bytes (pcg_split.cuh);
  // the device flags say whether the coding holds
  const bool coded = split && p->use_codes;
  auto matvec = [&]() {
    if (coded)
      pcg_matvec_dot_code_kernel<<<rg, rb, 0, s>>>(
          v.d, v.A64(4), v.code, v.lut64, v.octab64, v.code_info, c.pv, c.ap,
          c.pap);
    else
      pcg_matvec_dot_kernel<<<rg, rb, 0, s>>>(v.d, v.A64(4), c.pv, c.ap,
                                              c.pap);
  };
  auto head = [&](cudaGraphConditionalHandle h) -> int {
    PMG_CUDA_TRY(cudaMemcpyAsync(c.xs, v.x, b, cudaMemcpyDeviceToDevice, s));
    PMG_CUDA_TRY(cudaMemcpyAsync(c.b, v.f, b, cudaMemcpyDeviceToDevice, s));
    defect_norm_kernel<7, double, double>
        <<<rg, rb, 0, s>>>(v.d, v.A64(4), c.b, c.xs, c.r, c.rr);
    PMG_LAUNCH_CHECK();
    int rc = precondition(p, c.r, c.z);
    if (rc)
      return rc;
    PMG_CUDA_TRY(cudaMemcpyAsync(c.pv, c.z, b, cudaMemcpyDeviceToDevice, s));
    pcg_dot_kernel<<<rg, rb, 0, s>>>(v.d, c.r, c.z, c.rz);
    matvec();
    pcg_init_kernel<<<1, 1, 0, s>>>(c.d_st, c.rr.result, c.rz.result,
                                    c.pap.result, n3, h);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  };
  auto body = [&](cudaGraphConditionalHandle h) -> int {
    int rc;
    if (split) {
      // r and the split right-hand side in one pass, the V-cycle, then z
      // from the split correction inside r.z
      if (mixed)
        pcg_update_xr_split_kernel<float><<<rg, rb, 0, s>>>(
            v.d, c.pv, c.ap, c.xs, c.r, v.f32, c.d_st, c.rr);
      else
        pcg_update_xr_split_kernel<double><<<rg, rb, 0, s>>>(
            v.d, c.pv, c.ap, c.xs, c.r, v.fs, c.d_st, c.rr);
      PMG_LAUNCH_CHECK();
      rc = mixed ? vcycle_ref<float>(p, p->nlev)
                 : vcycle_ref<double>(p, p->nlev);
      if (rc)
        return rc;
      if (mixed)
        pcg_dot_split_kernel<float>
            <<<rg, rb, 0, s>>>(v.d, c.r, v.x32, c.z, c.rz);
      else
        pcg_dot_split_kernel<double>
            <<<rg, rb, 0, s>>>(v.d, c.r, v.xs, c.z, c.rz);
    } else {
      pcg_update_xr_kernel<<<rg, rb, 0, s>>>(v.d, c.pv, c.ap, c.xs, c.r,
                                             c.d_st, c.rr);
      PMG_LAUNCH_CHECK();
      if ((rc = precondition(p, c.r, c.z)))
        return rc;
      pcg_dot_kernel<<<rg, rb, 0, s>>>(v.d, c.r, c.z, c.rz);
    }
    pcg_beta_kernel<<<1, 1, 0, s>>>(c.d_st, c.rz.result);
    pcg_update_p_kernel<<<rg, rb, 0, s>>>(v.d, c.z, c.pv, c.d_st);
    matvec();
    pcg_check_kernel<<<1, 1, 0, s>>>(c.d_st, c.pap.result, c.rr.result, n3,
                                     h);
    PMG_LAUNCH_CHECK();
    return PMG_OK;
  };
  auto tail = [&]() -> int {
    PMG_CUDA_TRY(cudaMemcpyAsync(v.x, c.xs, b, cudaMemcpyDeviceToDevice, s));
    PMG_CUDA_TRY(cudaMemcpyAsync(v.f, c.b, b, cudaMemcpyDeviceToDevice, s));
    PMG_CUDA_TRY(cudaMemcpyAsync(c.h_st, c.d_st, sizeof(PcgState),
                                 cudaMemcpyDeviceToHost, s));
    return PMG_OK;
  };
  return build_loop_graph(p, head, body, tail, &c.exec, &c.head_kernels,
                          &c.body_kernels);
}

// Bit 6 of the finest code bytes and the centre-coefficient tables
// (split_layout.cuh, oc_range_kernel ... oc_table_kernel), after the
// coupling codes.
int build_oc_codes(pmg_problem *p, LevelBuf &v) {
  cudaStream_t s = p->stream;
  oc_range_init_kernel<<<1, 128, 0, s>>>(v.oc_range);
  oc_range_kernel<<<oc_range_blocks(v.d), 256, 0, s>>>(v.d, v.op[kOC],
                                                       v.code, v.oc_range);
  oc_code_kernel<<<interior_grid(v.d), interior_block(), 0, s>>>(
      v.d, v.op[kOC], v.oc_range, v.code_info, v.code);
  oc_table_kernel<<<1, 128, 0, s>>>(v.oc_range, v.octab64, v.octab32);
  p->launches += 4;
  PMG_LAUNCH_CHECK();
  return PMG_OK;
}

// A new problem starts from the state of a freshly constructed class: the
// coarse iterates are zero (the coarsest CG warm-starts from its level's
// iterate, so a previous solve's values would change the result).
int new_problem_loaded(pmg_problem *p) {
  for (int L = 1; L < p->nlev; ++L) {
    LevelBuf &c = p->lv[L];
    if (c.x)
      PMG_CUDA_TRY(
          cudaMemsetAsync(c.x, 0, sizeof(double) * c.n3, p->stream));
    if (c.x32)
      PMG_CUDA_TRY(
          cudaMemsetAsync(c.x32, 0, sizeof(float) * c.n3_32, p->stream));
  }
  p->fine_set = true;
  p->built = false;
  return PMG_OK;
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

long long pmg_problem_bytes(int base, int nlev, int precision) {
  if (check_shape(base, nlev))
    return -1;
  pmg_problem tmp;
  tmp.base = base;
  tmp.nlev = nlev;
  tmp.precision = precision;
  tmp.tma_on = !tma_disabled();
  Arena a;
  plan(&tmp, a);
  return (long long)a.off;
}

int pmg_problem_create(int base, int nlev, double box, int precision,
                       pmg_stream_t stream, pmg_problem **out) {
  if (!out || check_shape(base, nlev) ||
      (precision != PMG_PREC_FP64 && precision != PMG_PREC_MIXED &&
       precision != PMG_PREC_FP64_FAST)) {
    set_last_message("pmg_problem_create: bad argument");
    return PMG_ERR_ARG;
  }
  *out = nullptr;
  pmg_problem *p = new (std::nothrow) pmg_problem();
  if (!p)
    return PMG_ERR_NOMEM;
  p->base = base;
  p->nlev = nlev;
  p->box = box;
  p->precision = precision;
  p->bottom_top = bottom_top_of(base, nlev, precision);
  p->tma_on = !tma_disabled();
  Arena a;
  plan(p, a);
  p->arena_bytes = a.off;
  cudaError_t e = cudaMalloc((void **)&p->arena, p->arena_bytes);
  if (e != cudaSuccess) {
    delete p;
    set_last_error(e, "cudaMalloc(problem arena)", __FILE__, __LINE__);
    return PMG_ERR_NOMEM;
  }
  Arena b;
  b.base = p->arena;
  plan(p, b);
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount,
                             dev);
    (void)cudaGetLastError();
    if (p->tma_on)
      encode_tma_maps(p);
    p->stream_fine = g_stream_on.load() != 0 && stream_fine_ok(p);
  }
  if (stream) {
    p->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    p->own_stream = e == cudaSuccess;
    if (p->own_stream)
      p->created_stream = p->stream;
  }
  if (e == cudaSuccess)
    e = cudaMallocHost((void **)&p->h_pinned, 4 * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMallocHost((void **)&p->h_state, sizeof(SolveState));
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&p->done_ev, cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(p->arena, 0, p->arena_bytes, p->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(p->stream);
  if (e != cudaSuccess) {
    set_last_error(e, "pmg_problem_create", __FILE__, __LINE__);
    pmg_problem_destroy(p);
    return PMG_ERR_CUDA;
  }
  *out = p;
  return PMG_OK;
}

int pmg_problem_destroy(pmg_problem *p) {
  if (!p)
    return PMG_OK;
  if (p->stream)
    cudaStreamSynchronize(p->stream);
  drop_graphs(p);
  if (p->pcg.mem)
    cudaFree(p->pcg.mem);
  if (p->pcg.h_st)
    cudaFreeHost(p->pcg.h_st);
  if (p->done_ev)
    cudaEventDestroy(p->done_ev);
  if (p->h_state)
    cudaFreeHost(p->h_state);
  for (int e = 0; e < 2; ++e)
    for (int q = 0; q < kProfSlots; ++q)
      if (p->prof_ev[e][q])
        cudaEventDestroy(p->prof_ev[e][q]);
  if (p->arena)
    cudaFree(p->arena);
  if (p->h_pinned)
    cudaFreeHost(p->h_pinned);
  if (p->created_stream) {
    cudaStreamSynchronize(p->created_stream);
    cudaStreamDestroy(p->created_stream);
  }
  delete p;
  return PMG_OK;
}

int pmg_problem_set_coarse_rtol(pmg_problem *p, double rtol) {
  if (!p || !(rtol >= 0.0) || rtol >= 1.0) {
    set_last_message("pmg_problem_set_coarse_rtol: need 0 <= rtol < 1");
    return PMG_ERR_ARG;
  }
  p->coarse_rtol = rtol;
  drop_graphs(p); // the captured cycles bake the threshold in
  return PMG_OK;
}

int pmg_set_finest_streaming(int on) {
  g_stream_on.store(on != 0);
  return PMG_OK;
}

int pmg_set_tma_staging(int on) {
  g_tma_on.store(on != 0);
  return PMG_OK;
}

int pmg_test_tma_short_delivery(int bytes) {
  if (bytes < 0 || bytes % 16 != 0 || bytes > (1 << 20)) {
    set_last_message("pmg_test_tma_short_delivery: bytes must be a multiple "
                     "of 16 in [0, 2^20]");
    return PMG_ERR_ARG;
  }
  g_tma_extra_tx.store((unsigned)bytes);
  return PMG_OK;
}

int pmg_problem_set_host_loop(pmg_problem *p, int on) {
  if (!p)
    return PMG_ERR_ARG;
  p->host_loop = on != 0;
  return PMG_OK;
}

int pmg_problem_set_coded_couplings(pmg_problem *p, int on) {
  if (!p)
    return PMG_ERR_ARG;
  if ((bool)on != p->use_codes)
    drop_graphs(p); // the captured cycles bake the kernel choice in
  p->use_codes = on != 0;
  return PMG_OK;
}

int pmg_problem_coded_couplings(pmg_problem *p, int *coded) {
  if (!p || !coded)
    return PMG_ERR_ARG;
  *coded = 0;
  const LevelBuf &v = p->lv[p->nlev];
  if (!p->built || !p->use_codes)
    return PMG_OK;
  int flag[2] = {1, 1};
  PMG_CUDA_TRY(cudaMemcpyAsync(flag, v.code_info + 6, sizeof(flag),
                               cudaMemcpyDeviceToHost, p->stream));
  PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
  // the float coding; the double paths also need the double couplings to
  // match
  *coded = flag[0] == 0 &&
           (p->precision == PMG_PREC_MIXED || flag[1] == 0);
  return PMG_OK;
}

int pmg_problem_finest_streamed(pmg_problem *p, int *streamed) {
  if (!p || !streamed)
    return PMG_ERR_ARG;
  *streamed = p->stream_fine && p->use_codes;
  return PMG_OK;
}

int pmg_problem_set_throughput_mode(pmg_problem *p, int on) {
  if (!p)
    return PMG_ERR_ARG;
  if ((bool)on != p->throughput)
    drop_graphs(p); // the captured cycles bake the kernel choice in
  p->throughput = on != 0;
  return PMG_OK;
}

int pmg_problem_set_profiling(pmg_problem *p, int on) {
  if (!p)
    return PMG_ERR_ARG;
  if (on && !p->prof_ev[0][0]) {
    for (int e = 0; e < 2; ++e)
      for (int q = 0; q < kProfSlots; ++q)
        PMG_CUDA_TRY(cudaEventCreate(&p->prof_ev[e][q]));
  }
  if ((bool)on != p->prof_on)
    drop_graphs(p);
  p->prof_on = on != 0;
  return PMG_OK;
}

int pmg_problem_profile(pmg_problem *p, double *ms, long long *counts,
                        int cap, int reset) {
  if (!p)
    return PMG_ERR_ARG;
  for (int q = 0; q < kProfSlots && q < cap; ++q) {
    if (ms)
      ms[q] = p->prof_ms[q];
    if (counts)
      counts[q] = p->prof_count[q];
  }
  if (reset)
    for (int q = 0; q < kProfSlots; ++q) {
      p->prof_ms[q] = 0.0;
      p->prof_count[q] = 0;
    }
  return kProfSlots;
}

long long pmg_problem_launches(pmg_problem *p) { return p ? p->launches : -1; }

pmg_stream_t pmg_problem_stream(pmg_problem *p) {
  return p ? (pmg_stream_t)p->stream : nullptr;
}

int pmg_problem_set_fine(pmg_problem *p, const double *oC, const double *oE,
                         const double *oN, const double *uC, const double *f,
                         const double *x0) {
  if (!p || !oC || !oE || !oN || !uC || !f || !x0) {
    set_last_message("pmg_problem_set_fine: null argument");
    return PMG_ERR_ARG;
  }
  LevelBuf &v = p->lv[p->nlev];
  const size_t b = sizeof(double) * v.n3;
  const double *src[6] = {oC, oE, oN, uC, f, x0};
  double *dst[6] = {v.op[kOC], v.op[kOE], v.op[kON], v.op[kUC], v.f, v.x};
  for (int q = 0; q < 6; ++q)
    PMG_CUDA_TRY(
        cudaMemcpyAsync(dst[q], src[q], b, cudaMemcpyDefault, p->stream));
  return new_problem_loaded(p);
}

int pmg_problem_set_atoms(pmg_problem *p, const double *atoms, int natoms,
                          const pmg_physics *phys) {
  if (!p || !phys || natoms < 0 || (natoms > 0 && !atoms)) {
    set_last_message("pmg_problem_set_atoms: bad argument");
    return PMG_ERR_ARG;
  }
  LevelBuf &v = p->lv[p->nlev];
  const double h = p->box / (double)(v.n - 1);
  const int rc = setup_fine_device(v.n, h, atoms, natoms, phys, v.op[kOC],
                                   v.op[kOE], v.op[kON], v.op[kUC], v.f, v.x,
                                   p->stream);
  if (rc)
    return rc;
  return new_problem_loaded(p);
}

int pmg_build_hierarchy(pmg_problem *p, int trilinear) {
  if (!p)
    return PMG_ERR_ARG;
  if (!p->fine_set) {
    set_last_message("pmg_build_hierarchy: fine level not set");
    return PMG_ERR_STATE;
  }
  cudaStream_t s = p->stream;
  const bool mixed = p->precision == PMG_PREC_MIXED;
  int rc;
  for (int L = p->nlev; L >= 2; --L) {
    LevelBuf &f = p->lv[L], &c = p->lv[L - 1];
    const int kind = L == p->nlev ? 7 : 27;
    P27W<double> Pw;
    for (int q = 0; q < 27; ++q)
      Pw.p[q] = c.P[q];
    // the mixed path's float copies are written by the builders (interior
    // entries; the shells stay zero from the arena's clearing)
    P27W<float> P32w{};
    Op14W<float> out32{};
    // the builders write the float copies (rows c.d32.px apart)
    if (mixed) {
      for (int q = 0; q < 27; ++q)
        P32w.p[q] = c.P32[q];
      for (int q = 0; q < 14; ++q)
        out32.a[q] = c.op32[q]; // null on level 1
    }
    if (trilinear) {
      buildP_trilin_kernel<<<interior_grid(c.d), interior_block(), 0, s>>>(
          c.d, Pw);
      PMG_LAUNCH_CHECK();
    } else if ((rc = launch_buildP(f.d, c.d, kind, f.A64(kind == 7 ? 4 : 14),
                                   Pw, s, P32w, &c.d32))) {
      return rc;
    }
    p->launches += 2; // prolongation + Galerkin operator
    Op14W<double> out;
    for (int q = 0; q < 14; ++q)
      out.a[q] = c.op[q];
    if ((rc = launch_buildG(f.d, c.d, kind, c.Pc(),
                            f.A64(kind == 7 ? 4 : 14), out, s, out32,
                            &c.d32)))
      return rc;
  }
  if (mixed) {
    LevelBuf &v = p->lv[p->nlev];
    const unsigned g = flat_grid(v.n3);
    for (int q = 0; q < 14; ++q)
      if (v.op32[q]) { // the finest float operator is split
        to_split_kernel<double, float><<<g, 256, 0, s>>>(v.d, v.op[q],
                                                         v.op32[q]);
        ++p->launches;
      }
    // coded couplings of the finest float operator, when it has two values
    // per direction (split_layout.cuh)
    const int init[12] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN,
                          0,       0,       0,       0,       0,       0};
    PMG_CUDA_TRY(cudaMemcpyAsync(v.code_info, init, sizeof(init),
                                 cudaMemcpyHostToDevice, s));
    const dim3 ig = interior_grid(v.d), ib = interior_block();
    coupling_range_kernel<float><<<coupling_range_blocks(v.d), 256, 0, s>>>(
        v.d, v.op32[kOE], v.op32[kON], v.op32[kUC], v.code_info);
    coupling_code_kernel<float><<<ig, ib, 0, s>>>(
        v.d, v.op32[kOE], v.op32[kON], v.op32[kUC], v.code_info, v.code);
    lut64_store_kernel<double><<<ig, ib, 0, s>>>(
        v.d, v.op[kOE], v.op[kON], v.op[kUC], v.code, v.lut64);
    lut64_check_kernel<double><<<ig, ib, 0, s>>>(
        v.d, v.op[kOE], v.op[kON], v.op[kUC], v.code, v.lut64, v.code_info);
    p->launches += 4;
    if ((rc = build_oc_codes(p, v)))
      return rc;
    // the streamed pass's blocked copy of the finished code bytes
    code_block_kernel<<<flat_grid(CodeBlocks::of(v.d).bytes(v.d)), 256, 0,
                        s>>>(v.d, CodeBlocks::of(v.d), v.code, v.codeb);
    ++p->launches;
    // the staged smoother's split copies of the padded levels' couplings
    for (int L = 2; L < p->nlev; ++L) {
      LevelBuf &c = p->lv[L];
      if (!c.tma_ok || !c.opc[0])
        continue;
      Op14W<float> o;
      for (int q = 0; q < 14; ++q)
        o.a[q] = c.opc[q];
      coef_split_kernel<<<flat_grid(c.n3), 256, 0, s>>>(c.d32, c.cs,
                                                        c.A32(14), o);
      ++p->launches;
    }
    if (trilinear) // the trilinear builder writes double only
      for (int L = 1; L < p->nlev; ++L) {
        LevelBuf &c = p->lv[L];
        for (int q = 0; q < 27; ++q) {
          repitch_kernel<double, float><<<flat_grid(c.n3), 256, 0, s>>>(
              c.d, c.d32, c.P[q], c.P32[q]);
          ++p->launches;
        }
      }
    PMG_LAUNCH_CHECK();
  }
  if (p->precision != PMG_PREC_MIXED) {
    // fp64-fast and FP64: the finest double operator split by colour, and
    // its coded couplings
    // (classified by their float values, then checked bit for bit in
    // double: info[7] keeps the arrays in use when they do not match)
    LevelBuf &v = p->lv[p->nlev];
    const unsigned g = flat_grid(v.n3);
    for (int q = 0; q < 4; ++q) {
      to_split_kernel<double, double><<<g, 256, 0, s>>>(v.d, v.op[q],
                                                        v.ops[q]);
      ++p->launches;
    }
    const int init[12] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN,
                          0,       0,       0,       0,       0,       0};
    PMG_CUDA_TRY(cudaMemcpyAsync(v.code_info, init, sizeof(init),
                                 cudaMemcpyHostToDevice, s));
    const dim3 ig = interior_grid(v.d), ib = interior_block();
    coupling_range_kernel<double><<<coupling_range_blocks(v.d), 256, 0, s>>>(
        v.d, v.ops[kOE], v.ops[kON], v.ops[kUC], v.code_info);
    coupling_code_kernel<double><<<ig, ib, 0, s>>>(
        v.d, v.ops[kOE], v.ops[kON], v.ops[kUC], v.code_info, v.code);
    lut64_store_kernel<double><<<ig, ib, 0, s>>>(
        v.d, v.op[kOE], v.op[kON], v.op[kUC], v.code, v.lut64);
    lut64_check_kernel<double><<<ig, ib, 0, s>>>(
        v.d, v.op[kOE], v.op[kON], v.op[kUC], v.code, v.lut64, v.code_info);
    p->launches += 4;
    if ((rc = build_oc_codes(p, v)))
      return rc;
    // the streamed pass's blocked copy of the finished code bytes
    code_block_kernel<<<flat_grid(CodeBlocks::of(v.d).bytes(v.d)), 256, 0,
                        s>>>(v.d, CodeBlocks::of(v.d), v.code, v.codeb);
    ++p->launches;
    PMG_LAUNCH_CHECK();
  }
  // tile edge of the 27-point smoother, measured once per grid size (every
  // edge gives the same bits; the levels' iterates serve as scratch and are
  // cleared afterwards)
  for (int L = 2; L < p->nlev; ++L) {
    LevelBuf &v = p->lv[L];
    const size_t n3 = (size_t)v.n3;
    if (p->precision == PMG_PREC_MIXED) {
      if (L <= p->bottom_top || v.tma_ok || gs27_tile_known(v.d32, 4) ||
          !gs27_autotune_on())
        continue;
      if ((rc = gs27_tune<float>(v.d32, v.A32(14), v.f32, v.x32, v.xalt32,
                                 s)))
        return rc;
      PMG_CUDA_TRY(cudaMemsetAsync(v.x32, 0, sizeof(float) * v.n3_32, s));
      PMG_CUDA_TRY(cudaMemsetAsync(v.xalt32, 0, sizeof(float) * v.n3_32, s));
    } else {
      if (gs27_tile_known(v.d, 8) || !gs27_autotune_on())
        continue;
      if ((rc = gs27_tune<double>(v.d, v.A64(14), v.f, v.x, v.xalt, s)))
        return rc;
      PMG_CUDA_TRY(cudaMemsetAsync(v.x, 0, sizeof(double) * n3, s));
      PMG_CUDA_TRY(cudaMemsetAsync(v.xalt, 0, sizeof(double) * n3, s));
    }
  }
  p->built = true;
  return PMG_OK;
}

int pmg_vcycle(pmg_problem *p, int as_preconditioner) {
  if (!p)
    return PMG_ERR_ARG;
  if (!p->built) {
    set_last_message("pmg_vcycle: hierarchy not built");
    return PMG_ERR_STATE;
  }
  if (p->precision != PMG_PREC_FP64) {
    set_last_message("pmg_vcycle: FP64 problems only");
    return PMG_ERR_ARG;
  }
  return vcycle64(p, p->nlev, as_preconditioner);
}

int pmg_compute_residual_2(pmg_problem *p, double *out) {
  if (!p || !out)
    return PMG_ERR_ARG;
  if (!p->fine_set)
    return PMG_ERR_STATE;
  int rc = residual_norm_async(p);
  if (rc)
    return rc;
  PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
  *out = norm_from_sum(p, p->h_pinned[0]);
  return PMG_OK;
}

// Host-driven loop: one cycle graph per launch and a residual read-back per
// cycle (used with phase timing, whose event records cannot sit in a
// conditional body, and for histories longer than the device state holds).
static int solve_host_loop(pmg_problem *p, double tol, int max_cycles,
                           int *cycles, double *relres, double *hist) {
  const bool refine = p->precision != PMG_PREC_FP64;
  PMG_CUDA_TRY(cudaMemsetAsync(p->kernel_err, 0, sizeof(int), p->stream));
  int rc = refine ? refine_residual_async(p) : residual_norm_async(p);
  if (rc)
    return rc;
  ++p->launches;
  PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
  const double r0 = norm_from_sum(p, p->h_pinned[0]);
  if (hist)
    hist[0] = r0;
  if (!isfinite(r0)) {
    if (cycles)
      *cycles = 0;
    if (relres)
      *relres = r0;
    set_last_message("pmg_solve: initial residual is not finite");
    return PMG_ERR_DIVERGED;
  }
  if ((rc = ensure_graph(p)))
    return rc;
  int c = 0;
  double r = r0;
  rc = PMG_OK;
  while (c < max_cycles && r0 > 0.0) {
    PMG_CUDA_TRY(cudaGraphLaunch(p->cycle_exec, p->stream));
    p->launches += p->cycle_kernels;
    PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
    prof_collect(p);
    ++c;
    r = norm_from_sum(p, p->h_pinned[0]);
    if (hist)
      hist[c] = r;
    if (!isfinite(r) || r > 1e6 * r0) {
      set_last_message("pmg_solve: residual diverged");
      rc = PMG_ERR_DIVERGED;
      break;
    }
    if (r / r0 < tol)
      break;
  }
  if (cycles)
    *cycles = c;
  if (relres)
    *relres = r0 > 0.0 ? r / r0 : 0.0;
  int lost = 0;
  PMG_CUDA_TRY(cudaMemcpy(&lost, p->kernel_err, sizeof(int),
                          cudaMemcpyDeviceToHost));
  if (rc == PMG_OK && lost) {
    set_last_message("pmg_solve: a staged copy (27-point smoother, "
                     "streamed finest pass or residual) did not arrive "
                     "(bounded wait ran out)");
    rc = PMG_ERR_TIMEOUT;
  }
  return rc;
}

int pmg_solve_start(pmg_problem *p, double tol, int max_cycles) {
  if (!p || max_cycles < 0 || max_cycles > kMaxHist || !(tol >= 0.0)) {
    set_last_message("pmg_solve_start: bad argument (0 <= max_cycles <= "
                     "1024, tol >= 0)");
    return PMG_ERR_ARG;
  }
  if (!p->built) {
    set_last_message("pmg_solve_start: hierarchy not built");
    return PMG_ERR_STATE;
  }
  if (p->solve_pending) {
    set_last_message("pmg_solve_start: a solve is already in flight");
    return PMG_ERR_STATE;
  }
  if (p->prof_on) {
    set_last_message("pmg_solve_start: phase timing needs pmg_solve");
    return PMG_ERR_STATE;
  }
  int rc = ensure_solve_graph(p);
  if (rc)
    return rc;
  PMG_CUDA_TRY(cudaMemsetAsync(p->kernel_err, 0, sizeof(int), p->stream));
  solve_params_kernel<<<1, 1, 0, p->stream>>>(p->d_state, tol, max_cycles);
  PMG_LAUNCH_CHECK();
  PMG_CUDA_TRY(cudaGraphLaunch(p->solve_exec, p->stream));
  PMG_CUDA_TRY(cudaEventRecord(p->done_ev, p->stream));
  p->solve_pending = true;
  return PMG_OK;
}

int pmg_solve_poll(pmg_problem *p, int *done) {
  if (!p || !done)
    return PMG_ERR_ARG;
  if (!p->solve_pending) {
    *done = 1;
    return PMG_OK;
  }
  const cudaError_t e = cudaEventQuery(p->done_ev);
  if (e == cudaErrorNotReady) {
    *done = 0;
    return PMG_OK;
  }
  PMG_CUDA_TRY(e);
  *done = 1;
  return PMG_OK;
}

int pmg_solve_finish(pmg_problem *p, int *cycles, double *relres,
                     double *hist) {
  if (!p)
    return PMG_ERR_ARG;
  if (!p->solve_pending) {
    set_last_message("pmg_solve_finish: no solve in flight");
    return PMG_ERR_STATE;
  }
  p->solve_pending = false;
  PMG_CUDA_TRY(cudaEventSynchronize(p->done_ev));
  const SolveState &st = *p->h_state;
  p->launches += 1 + p->solve_pre_kernels +
                 (long long)st.cycles * p->solve_body_kernels;
  if (cycles)
    *cycles = st.cycles;
  if (relres)
    *relres = st.status == 2 ? st.r0 : (st.r0 > 0.0 ? st.r / st.r0 : 0.0);
  if (hist)
    for (int c = 0; c <= st.cycles && c <= kMaxHist; ++c)
      hist[c] = st.hist[c];
  if (st.status == 2) {
    set_last_message("pmg_solve: initial residual is not finite");
    return PMG_ERR_DIVERGED;
  }
  if (st.status == 1) {
    set_last_message("pmg_solve: residual diverged");
    return PMG_ERR_DIVERGED;
  }
  if (st.status == 3) {
    set_last_message("pmg_solve: a staged copy (27-point smoother, "
                     "streamed finest pass or residual) did not arrive "
                     "(bounded wait ran out)");
    return PMG_ERR_TIMEOUT;
  }
  return PMG_OK;
}

int pmg_solve(pmg_problem *p, double tol, int max_cycles, int *cycles,
              double *relres, double *hist) {
  if (!p || max_cycles < 0)
    return PMG_ERR_ARG;
  if (!p->built) {
    set_last_message("pmg_solve: hierarchy not built");
    return PMG_ERR_STATE;
  }
  if (p->solve_pending) {
    set_last_message("pmg_solve: a solve is already in flight");
    return PMG_ERR_STATE;
  }
  if (p->prof_on || p->host_loop || max_cycles > kMaxHist)
    return solve_host_loop(p, tol, max_cycles, cycles, relres, hist);
  int rc = pmg_solve_start(p, tol, max_cycles);
  if (rc)
    return rc;
  return pmg_solve_finish(p, cycles, relres, hist);
}

int pmg_pcg_solve(pmg_problem *p, double tol, int max_iters, int *iters,
                  double *relres, double *hist) {
  if (!p || max_iters < 0 || max_iters > 1024 || !(tol >= 0.0)) {
    set_last_message("pmg_pcg_solve: bad argument (0 <= max_iters <= 1024, "
                     "tol >= 0)");
    return PMG_ERR_ARG;
  }
  if (!p->built) {
    set_last_message("pmg_pcg_solve: hierarchy not built");
    return PMG_ERR_STATE;
  }
  if (p->solve_pending || p->prof_on) {
    set_last_message("pmg_pcg_solve: a solve is in flight or phase timing "
                     "is on");
    return PMG_ERR_STATE;
  }
  int rc = pcg_alloc(p);
  if (!rc)
    rc = ensure_pcg_graph(p);
  if (rc)
    return rc;
  pcg_params_kernel<<<1, 1, 0, p->stream>>>(p->pcg.d_st, tol, max_iters);
  PMG_LAUNCH_CHECK();
  PMG_CUDA_TRY(cudaGraphLaunch(p->pcg.exec, p->stream));
  PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
  const PcgState &st = *p->pcg.h_st;
  p->launches += 1 + p->pcg.head_kernels +
                 (long long)st.iters * p->pcg.body_kernels;
  if (iters)
    *iters = st.iters;
  if (relres)
    *relres = st.status == 2 ? st.r0 : (st.r0 > 0.0 ? st.rn / st.r0 : 0.0);
  if (hist)
    for (int c = 0; c <= st.iters && c <= 1024; ++c)
      hist[c] = st.hist[c];
  if (st.status == 2) {
    set_last_message("pmg_pcg_solve: initial residual is not finite");
    return PMG_ERR_DIVERGED;
  }
  if (st.status == 1) {
    set_last_message("pmg_pcg_solve: residual diverged");
    return PMG_ERR_DIVERGED;
  }
  return PMG_OK;
}

int pmg_get_potential(pmg_problem *p, double *dst) {
  if (!p || !dst)
    return PMG_ERR_ARG;
  LevelBuf &v = p->lv[p->nlev];
  PMG_CUDA_TRY(cudaMemcpyAsync(dst, v.x, sizeof(double) * v.n3,
                               cudaMemcpyDefault, p->stream));
  PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return PMG_OK;
}

int pmg_get_potential_async(pmg_problem *p, double *dst) {
  if (!p || !dst)
    return PMG_ERR_ARG;
  LevelBuf &v = p->lv[p->nlev];
  PMG_CUDA_TRY(cudaMemcpyAsync(dst, v.x, sizeof(double) * v.n3,
                               cudaMemcpyDefault, p->stream));
  return PMG_OK;
}

int pmg_problem_set_stream(pmg_problem *p, pmg_stream_t stream) {
  if (!p || (!stream && !p->created_stream)) {
    set_last_message("pmg_problem_set_stream: null argument");
    return PMG_ERR_ARG;
  }
  if (!stream)
    stream = (pmg_stream_t)p->created_stream;
  if (p->solve_pending) {
    set_last_message("pmg_problem_set_stream: a solve is in flight");
    return PMG_ERR_STATE;
  }
  if ((cudaStream_t)stream == p->stream)
    return PMG_OK;
  // work already queued on the old stream precedes work on the new one
  cudaEvent_t ev = nullptr;
  PMG_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, p->stream);
  if (e == cudaSuccess)
    e = cudaStreamWaitEvent((cudaStream_t)stream, ev, 0);
  cudaEventDestroy(ev);
  PMG_CUDA_TRY(e);
  p->stream = (cudaStream_t)stream;
  return PMG_OK;
}

int pmg_get_level(pmg_problem *p, int level, double *dst) {
  if (!p || !dst || level < 1 || level >= p->nlev)
    return PMG_ERR_ARG;
  LevelBuf &v = p->lv[level];
  const size_t b = sizeof(double) * v.n3;
  for (int q = 0; q < 27; ++q)
    PMG_CUDA_TRY(cudaMemcpyAsync(dst + q * v.n3, v.P[q], b, cudaMemcpyDefault,
                                 p->stream));
  for (int q = 0; q < 14; ++q)
    PMG_CUDA_TRY(cudaMemcpyAsync(dst + (27 + q) * v.n3, v.op[q], b,
                                 cudaMemcpyDefault, p->stream));
  PMG_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return PMG_OK;
}

} // extern "C"
