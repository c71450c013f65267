/* pmg_b200 — C ABI of the B200-native PMG (Galerkin multigrid) solver for
 * the linearized Poisson-Boltzmann equation.
 *
 * Drop-in boundary for the reference's pmgc kernels and its
 * pmgc_solver::PBE_linear_problem class (jabruniessner/multigrid, ported from
 * APBS pmgc). Each entry point below names the reference routine it replaces
 * as file:line in that project.
 *
 * Conventions (all entry points):
 *  - Grid arrays are the reference's: nx*ny*nz values including the
 *    one-point Dirichlet shell, x fastest, 1-based
 *    VAT3(m,i,j,k) = m[(k-1)*ny*nx + (j-1)*nx + (i-1)] (pmgc/vmatrix.h:79-80).
 *  - Kernel entry points take DEVICE pointers and a CUDA stream in place of
 *    the reference's sycl::queue&; they are asynchronous on that stream, like
 *    the reference's in-order queue. Entry points that return a scalar to the
 *    host synchronise the stream, as the reference's reductions do (.wait()).
 *  - The caller owns every array passed in; the library never frees caller
 *    memory. Unused APBS arguments of the reference (ipc, rpc) are dropped.
 *  - Every function returns a pmg_status: 0 on success, negative on error;
 *    pmg_last_error() describes the last failure on the calling thread.
 *  - _d entry points compute in double, _f in float.
 */
#ifndef PMG_B200_H
#define PMG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

struct CUstream_st;
typedef struct CUstream_st *pmg_stream_t; /* == cudaStream_t */

typedef enum {
  PMG_OK = 0,
  PMG_ERR_ARG = -1,      /* invalid size, null pointer, bad option        */
  PMG_ERR_CUDA = -2,     /* a CUDA call failed (see pmg_last_error)      */
  PMG_ERR_NOMEM = -3,    /* device allocation failed                      */
  PMG_ERR_DIVERGED = -4, /* residual became NaN/Inf or stagnated          */
  PMG_ERR_TIMEOUT = -5,  /* a bounded device wait or iteration cap ran out */
  PMG_ERR_BUDGET = -6,   /* admission refused: device-memory budget       */
  PMG_ERR_STATE = -7     /* call out of order (e.g. solve before build)   */
} pmg_status;

/* Human-readable description of the last error on this thread. */
const char *pmg_last_error(void);
/* Library version string. */
const char *pmg_version(void);

/* ======================================================================
 * pmgc kernels (device pointers, stream-ordered)
 * ==================================================================== */

/* Red-black Gauss-Seidel on the 7-point operator, itmax sweeps of two
 * colours; colour c updates (i+j+k)%2 == (1-iadjoint)*c + iadjoint*(1-c);
 * zero_init drops the neighbour sum in the first colour.
 * Replaces pmgc::Vgsrb7x, pmgc/gsd.cc:60-111. cc may be NULL (= 0). */
int pmg_Vgsrb7x_d(int nx, int ny, int nz, const double *oC, const double *cc,
                  const double *fc, const double *oE, const double *oN,
                  const double *uC, double *x, int itmax, int iadjoint,
                  int zero_init, pmg_stream_t stream);
int pmg_Vgsrb7x_f(int nx, int ny, int nz, const float *oC, const float *cc,
                  const float *fc, const float *oE, const float *oN,
                  const float *uC, float *x, int itmax, int iadjoint,
                  int zero_init, pmg_stream_t stream);

/* Eight-colour Gauss-Seidel on the 27-point operator; colour
 * (i%2)+2(j%2)+4(k%2) visited in order c*(1-iadjoint) + iadjoint*(7-c);
 * zero_init clears x first. Argument order follows the reference
 * (x, itmax, zero_initialize, iadjoint).
 * Replaces pmgc::Vgsrb27x, pmgc/gsd.cc:113-212. cc may be NULL. */
int pmg_Vgsrb27x_d(int nx, int ny, int nz, const double *oC, const double *cc,
                   const double *fc, const double *oE, const double *oN,
                   const double *uC, const double *oNE, const double *oNW,
                   const double *uE, const double *uW, const double *uN,
                   const double *uS, const double *uNE, const double *uNW,
                   const double *uSE, const double *uSW, double *x, int itmax,
                   int zero_init, int iadjoint, pmg_stream_t stream);
int pmg_Vgsrb27x_f(int nx, int ny, int nz, const float *oC, const float *cc,
                   const float *fc, const float *oE, const float *oN,
                   const float *uC, const float *oNE, const float *oNW,
                   const float *uE, const float *uW, const float *uN,
                   const float *uS, const float *uNE, const float *uNW,
                   const float *uSE, const float *uSW, float *x, int itmax,
                   int zero_init, int iadjoint, pmg_stream_t stream);

/* y = A x on the interior (7-point). Replaces pmgc::Vmatvec7_1s,
 * pmgc/matvecd.cc:61-90 (and the class map matveckernel7,
 * pmgc/matvecd.h:117-138). */
int pmg_Vmatvec7_1s_d(int nx, int ny, int nz, const double *oC,
                      const double *cc, const double *oE, const double *oN,
                      const double *uC, const double *x, double *y,
                      pmg_stream_t stream);
/* The same on float arrays. */
int pmg_Vmatvec7_1s_f(int nx, int ny, int nz, const float *oC,
                      const float *cc, const float *oE, const float *oN,
                      const float *uC, const float *x, float *y,
                      pmg_stream_t stream);
/* y = A x on the interior (27-point). Replaces pmgc::Vmatvec27_1s,
 * pmgc/matvecd.cc:103-176 (and matveckernel27, pmgc/matvecd.h:179-240). */
int pmg_Vmatvec27_1s_d(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *oE, const double *oN,
                       const double *uC, const double *oNE, const double *oNW,
                       const double *uE, const double *uW, const double *uN,
                       const double *uS, const double *uNE, const double *uNW,
                       const double *uSE, const double *uSW, const double *x,
                       double *y, pmg_stream_t stream);
/* The same on float arrays. */
int pmg_Vmatvec27_1s_f(int nx, int ny, int nz, const float *oC,
                       const float *cc, const float *oE, const float *oN,
                       const float *uC, const float *oNE, const float *oNW,
                       const float *uE, const float *uW, const float *uN,
                       const float *uS, const float *uNE, const float *uNW,
                       const float *uSE, const float *uSW, const float *x,
                       float *y, pmg_stream_t stream);

/* r = f - A x on the interior (7-point). Replaces pmgc::Vmresid7_1s,
 * pmgc/matvecd.cc:381-411. */
int pmg_Vmresid7_1s_d(int nx, int ny, int nz, const double *oC,
                      const double *cc, const double *fc, const double *oE,
                      const double *oN, const double *uC, const double *x,
                      double *r, pmg_stream_t stream);
/* The same on float arrays. */
int pmg_Vmresid7_1s_f(int nx, int ny, int nz, const float *oC,
                      const float *cc, const float *fc, const float *oE,
                      const float *oN, const float *uC, const float *x,
                      float *r, pmg_stream_t stream);
/* r = f - A x on the interior (27-point). Replaces pmgc::Vmresid27_1s,
 * pmgc/matvecd.cc:425-495. */
int pmg_Vmresid27_1s_d(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *fc, const double *oE,
                       const double *oN, const double *uC, const double *oNE,
                       const double *oNW, const double *uE, const double *uW,
                       const double *uN, const double *uS, const double *uNE,
                       const double *uNW, const double *uSE, const double *uSW,
                       const double *x, double *r, pmg_stream_t stream);
/* The same on float arrays. */
int pmg_Vmresid27_1s_f(int nx, int ny, int nz, const float *oC,
                       const float *cc, const float *fc, const float *oE,
                       const float *oN, const float *uC, const float *oNE,
                       const float *oNW, const float *uE, const float *uW,
                       const float *uN, const float *uS, const float *uNE,
                       const float *uNW, const float *uSE, const float *uSW,
                       const float *x, float *r, pmg_stream_t stream);

/* Restriction xout = P^T xin on the coarse interior.
 * Replaces pmgc::Vrestrc2, pmgc/matvecd.cc:695-799. */
int pmg_Vrestrc2_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                   const double *xin, double *xout, const double *oPC,
                   const double *oPN, const double *oPS, const double *oPE,
                   const double *oPW, const double *oPNE, const double *oPNW,
                   const double *oPSE, const double *oPSW, const double *uPC,
                   const double *uPN, const double *uPS, const double *uPE,
                   const double *uPW, const double *uPNE, const double *uPNW,
                   const double *uPSE, const double *uPSW, const double *dPC,
                   const double *dPN, const double *dPS, const double *dPE,
                   const double *dPW, const double *dPNE, const double *dPNW,
                   const double *dPSE, const double *dPSW,
                   pmg_stream_t stream);
/* The same on float arrays. */
int pmg_Vrestrc2_f(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                   const float *xin, float *xout, const float *oPC,
                   const float *oPN, const float *oPS, const float *oPE,
                   const float *oPW, const float *oPNE, const float *oPNW,
                   const float *oPSE, const float *oPSW, const float *uPC,
                   const float *uPN, const float *uPS, const float *uPE,
                   const float *uPW, const float *uPNE, const float *uPNW,
                   const float *uPSE, const float *uPSW, const float *dPC,
                   const float *dPN, const float *dPS, const float *dPE,
                   const float *dPW, const float *dPNE, const float *dPNW,
                   const float *dPSE, const float *dPSW,
                   pmg_stream_t stream);

/* Operator-based interpolation xout = P xin: every coarse (ii,jj,kk) in
 * [1,n_c-1]^3 writes its eight fine points.
 * Replaces pmgc::VinterpPMG2, pmgc/matvecd.cc:819-964. */
int pmg_VinterpPMG2_d(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                      const double *xin, double *xout, const double *oPC,
                      const double *oPN, const double *oPS, const double *oPE,
                      const double *oPW, const double *oPNE, const double *oPNW,
                      const double *oPSE, const double *oPSW, const double *uPC,
                      const double *uPN, const double *uPS, const double *uPE,
                      const double *uPW, const double *uPNE, const double *uPNW,
                      const double *uPSE, const double *uPSW, const double *dPC,
                      const double *dPN, const double *dPS, const double *dPE,
                      const double *dPW, const double *dPNE, const double *dPNW,
                      const double *dPSE, const double *dPSW,
                      pmg_stream_t stream);
/* The same on float arrays. */
int pmg_VinterpPMG2_f(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                      const float *xin, float *xout, const float *oPC,
                      const float *oPN, const float *oPS, const float *oPE,
                      const float *oPW, const float *oPNE, const float *oPNW,
                      const float *oPSE, const float *oPSW, const float *uPC,
                      const float *uPN, const float *uPS, const float *uPE,
                      const float *uPW, const float *uPNE, const float *uPNW,
                      const float *uPSE, const float *uPSW, const float *dPC,
                      const float *dPN, const float *dPS, const float *dPE,
                      const float *dPW, const float *dPNE, const float *dPNW,
                      const float *dPSE, const float *dPSW,
                      pmg_stream_t stream);

/* Operator-based prolongation from a 7-point fine operator (27 outputs on
 * the coarse grid). Replaces pmgc::VbuildPb_op7, pmgc/buildPd.cc:172-555. */
int pmg_VbuildPb_op7_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                       const double *oC, const double *oE, const double *oN,
                       const double *uC, double *oPC, double *oPN,
                       double *oPS, double *oPE, double *oPW, double *oPNE,
                       double *oPNW, double *oPSE, double *oPSW, double *uPC,
                       double *uPN, double *uPS, double *uPE, double *uPW,
                       double *uPNE, double *uPNW, double *uPSE, double *uPSW,
                       double *dPC, double *dPN, double *dPS, double *dPE,
                       double *dPW, double *dPNE, double *dPNW, double *dPSE,
                       double *dPSW, pmg_stream_t stream);
/* Operator-based prolongation from a 27-point fine operator.
 * Replaces pmgc::VbuildPb_op27, pmgc/buildPd.cc:578-1091. */
int pmg_VbuildPb_op27_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                        const double *oC, const double *oE, const double *oN,
                        const double *uC, const double *oNE,
                        const double *oNW, const double *uE, const double *uW,
                        const double *uN, const double *uS, const double *uNE,
                        const double *uNW, const double *uSE,
                        const double *uSW, double *oPC, double *oPN,
                        double *oPS, double *oPE, double *oPW, double *oPNE,
                        double *oPNW, double *oPSE, double *oPSW, double *uPC,
                        double *uPN, double *uPS, double *uPE, double *uPW,
                        double *uPNE, double *uPNW, double *uPSE, double *uPSW,
                        double *dPC, double *dPN, double *dPS, double *dPE,
                        double *dPW, double *dPNE, double *dPNW, double *dPSE,
                        double *dPSW, pmg_stream_t stream);
/* Constant (trilinear) prolongation weights.
 * Replaces pmgc::VbuildPb_trilin, pmgc/buildPd.cc:62-153. */
int pmg_VbuildPb_trilin_d(int nxf, int nyf, int nzf, int nxc, int nyc,
                          int nzc, double *oPC, double *oPN, double *oPS,
                          double *oPE, double *oPW, double *oPNE, double *oPNW,
                          double *oPSE, double *oPSW, double *uPC, double *uPN,
                          double *uPS, double *uPE, double *uPW, double *uPNE,
                          double *uPNW, double *uPSE, double *uPSW,
                          double *dPC, double *dPN, double *dPS, double *dPE,
                          double *dPW, double *dPNE, double *dPNW,
                          double *dPSE, double *dPSW, pmg_stream_t stream);

/* Box-method (finite volume) fine operator of the APBS driver from the
 * coefficient maps on a tensor mesh: oC, cc, fc, oE, oN, uC on the interior
 * (the shell is not written) from the mesh lines xf (nx), yf (ny), zf (nz),
 * the Dirichlet values gxcf (ny*nz*2), gycf (nx*nz*2), gzcf (nx*ny*2; side
 * 1 = low face, 2 = high face), the face maps a1cf, a2cf, a3cf, the kappa
 * map ccf and the source fcf (all device arrays). Host bookkeeping as the
 * reference: ipc[9..11] = ipkey, 7, 1 (ipc may be NULL, else 12 ints) and
 * *numdia = 4 (may be NULL); the unused rpc is dropped. Every interior plane
 * is built (the reference's launch takes its k extent from ny, the same when
 * ny == nz).
 * Replaces pmgc::VbuildA_fv, pmgc/buildAd.cc:63-212. */
int pmg_VbuildA_fv_d(int nx, int ny, int nz, int ipkey, int *numdia, int *ipc,
                     double *oC, double *cc, double *fc, double *oE,
                     double *oN, double *uC, const double *xf,
                     const double *yf, const double *zf, const double *gxcf,
                     const double *gycf, const double *gzcf,
                     const double *a1cf, const double *a2cf,
                     const double *a3cf, const double *ccf, const double *fcf,
                     pmg_stream_t stream);

/* Galerkin coarse operator A_c = P^T A_f P from a 7-point fine operator:
 * 14 coarse diagonals XoC..XuSW. Replaces pmgc::VbuildG_7,
 * pmgc/buildGd.cc:437-1361. p27 = the 27 prolongation arrays in list order,
 * out14 = the 14 outputs (host arrays of device pointers). */
int pmg_VbuildG_7_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                    const double *const *p27, const double *oC,
                    const double *oE, const double *oN, const double *uC,
                    double *const *out14, pmg_stream_t stream);
/* Galerkin coarse operator from a 27-point fine operator (a14 = fine
 * diagonals oC..uSW). Replaces pmgc::VbuildG_27, pmgc/buildGd.cc:1363-3274. */
int pmg_VbuildG_27_d(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                     const double *const *p27, const double *const *a14,
                     double *const *out14, pmg_stream_t stream);

/* ======================================================================
 * APBS-style entry points: packed operators (device pointers)
 *
 * ac holds the operator's diagonals as consecutive columns of nx*ny*nz
 * doubles: oC oE oN uC for a 7-point operator, oC oE oN uC oNE oNW uE uW uN
 * uS uNE uNW uSE uSW for a 27-point one. ipc is a host array of at least 11
 * ints whose ipc[10] (the reference's VAT(ipc, 11)) is 7 or 27, as
 * pmg_VbuildA_fv_d leaves it. The unused rpc is dropped.
 * ==================================================================== */

/* y = A x on the interior, dispatched on ipc[10].
 * Replaces pmgc::Vmatvec, pmgc/matvecd.cc:244-260. */
int pmg_Vmatvec_d(int nx, int ny, int nz, const int *ipc, const double *ac,
                  const double *cc, const double *x, double *y,
                  pmg_stream_t stream);

/* r = f - A x on the interior, dispatched on ipc[10].
 * Replaces pmgc::Vmresid, pmgc/matvecd.cc:513-529. */
int pmg_Vmresid_d(int nx, int ny, int nz, const int *ipc, const double *ac,
                  const double *cc, const double *fc, const double *x,
                  double *r, pmg_stream_t stream);

/* Hestenes-Stiefel conjugate gradient from the initial x: r = f - A x,
 * then iterations until ||r|| / ||r_0|| <= errtol or itmax iterations
 * (*iters, host, gets the count). p, ap, r are work arrays of nx*ny*nz
 * doubles (r ends as the last residual): p is cleared first (its shell
 * must read as zero), ap and r are used on the interior. With itmax <= 0
 * and iresid == 0 nothing runs. Reads one scalar
 * back per iteration (synchronises the stream each time), as the reference
 * does. The reference's dot product returns x.x instead of x.y and its axpy
 * starts its range at index 0 (pmgc/mikpckd.cc:115-129, 192-222); this
 * implements the algorithm they document: p.Ap in the step length and
 * updates on the interior. omega and iadjoint, unused by the reference's
 * CG, are dropped.
 * Replaces pmgc::Vcghs, pmgc/cgd.cc:60-125. */
int pmg_Vcghs_d(int nx, int ny, int nz, const int *ipc, const double *ac,
                const double *cc, const double *fc, double *x, double *p,
                double *ap, double *r, int itmax, int *iters, double errtol,
                int iresid, pmg_stream_t stream);

/* Band storage of a level's interior operator and its R^T R factorisation,
 * for the direct coarse solve: acB (device, lda*n doubles with n the
 * interior unknowns, m = (nx-2)(ny-2) for 7-point and (nx-2)(ny-2)+(nx-2)+1
 * for 27-point operators, lda = m + 1) is zeroed, filled in LINPACK upper
 * band storage (unknowns x fastest) and factored in place. ipcB (host, 4
 * ints) gets n, m, lda, 1; *key (host) 0, or 1 when a pivot was not
 * positive (the operator is not positive definite). The factorisation runs
 * in one GPU thread in LINPACK's order; synchronises the stream. For
 * 27-point operators the couplings are stored where the matvec reads them;
 * the reference reads ten of them at other points (buildBd.cc:170-245).
 * Replaces pmgc::Vbuildband, pmgc/buildBd.cc:252-303. */
int pmg_Vbuildband_d(int *key, int nx, int ny, int nz, const int *ipc,
                     const double *ac, int *ipcB, double *acB,
                     pmg_stream_t stream);

/* In-place R^T R factorisation of a symmetric positive definite band matrix
 * (device abd, LINPACK upper band storage, lda >= m + 1); *info (host) 0 or
 * the first column whose pivot was not positive. One GPU thread;
 * synchronises the stream. Replaces pmgc::Vdpbfa, pmgc/mlinpckd.cc:168-207. */
int pmg_Vdpbfa_d(double *abd, int lda, int n, int m, int *info,
                 pmg_stream_t stream);

/* Solves R^T R x = b in place with a factor from pmg_Vdpbfa_d (device b, n
 * values). One GPU thread. Replaces pmgc::Vdpbsl,
 * pmgc/mlinpckd.cc:209-240. */
int pmg_Vdpbsl_d(const double *abd, int lda, int n, int m, double *b,
                 pmg_stream_t stream);

/* The APBS V-cycle loop on a hierarchy the caller built (Vbuildops or its
 * own), in APBS's packed multilevel storage: for level lev the iterate,
 * w0, cc, fc and tru start at offset iz(1,lev), the operator's ac at
 * iz(7,lev) (4 or 14 columns of n_lev doubles), its ipc at iz(5,lev) (host;
 * ipc(11) = 7 or 27), and the prolongation from lev+1 to lev at iz(11,lev)
 * (27 columns of n_(lev+1)). iz is the host copy of the 50 x nlev_real
 * integer table of Vbuildstr (pmgc/mgsubd.cc:266-345), column-major,
 * 1-based offsets. Runs levels ilev .. ilev+nlev-1 with level ilev of size
 * nx x ny x nz: per cycle nu1 red-black GS sweeps (mgsmoo 1) or CG steps
 * (mgsmoo 4) and the residual going down, the coarsest level by 100 CG
 * iterations to epsiln (mgsolv 0) or by the factored band stored one level
 * further down (mgsolv 1: n, m, lda in that level's ipc, the band in its
 * ac), the Hackbusch-Reusken damped correction and nu2 sweeps with the
 * colours reversed going up; until itmax cycles or the stop ratio of istop
 * 0-3 (tru needed for 2 and 3) is at most errtol. x (level ilev) is the
 * starting iterate and the result. Device arrays: x, w0, pc, ac, cc, fc,
 * tru (packed) and w1, w2, w3 (the finest size). Host outputs (may be
 * NULL): *iters cycles, *ierror 0 or 1 (itmax reached). iok, iinfo, omega
 * and rpc are accepted for the reference's signature and not used. Reads
 * one scalar back per cycle and per CG iteration; synchronises the stream.
 * Replaces pmgc::Vmvcs (pmgc/mgcsd.cc:61-531). */
int pmg_Vmvcs_d(int nx, int ny, int nz, double *x, const int *iz, double *w0,
                double *w1, double *w2, double *w3, int istop, int itmax,
                int *iters, int *ierror, int nlev, int ilev, int nlev_real,
                int mgsolv, int iok, int iinfo, double epsiln, double errtol,
                double omega, int nu1, int nu2, int mgsmoo, const int *ipc,
                const double *rpc, const double *pc, const double *ac,
                const double *cc, const double *fc, double *tru,
                pmg_stream_t stream);

/* The APBS iparm/rparm multigrid driver, linear case: builds the box-method
 * fine operator from the coefficient maps (as pmg_VbuildA_fv_d), the
 * prolongations and Galerkin operators of nlev levels, then runs V-cycles
 * from u = 0 until the stop test passes or itmax cycles ran, and writes the
 * boundary values onto u's shell. iparm and rparm are 0-based copies of the
 * reference's 1-based arrays (Vpackmg order, pmgc/mgsubd.cc:538-576):
 *   iparm[2..5] nx ny nz nlev   iparm[6..7] nu1 nu2   iparm[8] mgkey (0|1)
 *   iparm[9] itmax   iparm[10] istop (0 absolute L1 residual, 1 relative L1
 *   residual, 2 L1 change of the iterate, 3 L2 error against tcf)
 *   iparm[13] ipkey   iparm[15] mode (0)   iparm[16] mgprol (0 trilinear,
 *   1 operator-based)   iparm[17] mgcoar (0 coefficient maps injected and
 *   the box method per level, 2 Galerkin)   iparm[18] mgdisc
 *   (0 box method)   iparm[19] mgsmoo (1 red-black GS, 4 CG)   iparm[20]
 *   mgsolv (0 CG on the coarsest level, 1 banded direct solve as
 *   pmg_Vbuildband_d / pmg_Vdpbsl_d)   iparm[21] iperf (0)
 *   rparm[0] errtol
 * Other values of those parameters return PMG_ERR_ARG (the reference leaves
 * them untranslated or cannot build them). Level 1 is the finest; each
 * level's cycle follows Vmvcs: nu1 GS sweeps (colours forward) and the
 * residual going down, 100 CG iterations (or the band solve) on the
 * coarsest level, the
 * Hackbusch-Reusken damped correction and nu2 sweeps with the colours
 * reversed going up. Device arrays: u (n^3), xf/yf/zf (mesh lines), the
 * boundary maps gxcf/gycf/gzcf, a1cf a2cf a3cf ccf fcf (n^3), tcf (the true
 * solution; needed for istop 2/3, which overwrites it with the iterate,
 * else may be NULL). Host outputs (may be NULL): *iters cycles, *ierror 0
 * or 1 (itmax reached), *rsnrm the final stop ratio. Reads one scalar back
 * per cycle and per CG iteration; synchronises the stream. The reference's
 * helpers compute x.x for x.y, start axpys at index 0 and fill only parts of
 * the boundary faces (pmgc/mikpckd.cc:115-312); this follows what they
 * document.
 * Replaces pmgc::Vmgdriv (pmgc/mgdrvd.cc:60-491) with Vbuildops
 * (pmgc/mgsubd.cc:63-265) and Vmvcs (pmgc/mgcsd.cc:61-531); the work
 * arrays iwork/rwork are the library's own. */
int pmg_Vmgdriv_d(const int *iparm, const double *rparm, double *u,
                  const double *xf, const double *yf, const double *zf,
                  const double *gxcf, const double *gycf, const double *gzcf,
                  const double *a1cf, const double *a2cf, const double *a3cf,
                  const double *ccf, const double *fcf, double *tcf,
                  int *iters, int *ierror, double *rsnrm, pmg_stream_t stream);

/* ======================================================================
 * Class-level helpers of PBE_linear_problem (device pointers)
 * ==================================================================== */

/* Coarsest-level CG exactly as the class runs it: warm start from x,
 * absolute stop sqrt(r.r) <= thresh (the first test on sqrt(sqrt(r.r))),
 * early exit when the first p.Ap is 0, at most max_iters iterations (the
 * reference has no cap). a14 = 14 diagonals (host array of device
 * pointers). *iters (host) gets the iteration count. One CTA; grids up to
 * 33^3. Synchronises the stream. Replaces cg_solver::CG_solver with
 * thresh_criterion, CG_Solver.h:45-242, as called by solve_by_cg,
 * PBE_pmgc_class.h:856-860. */
int pmg_cg_level_d(int nx, int ny, int nz, const double *const *a14,
                   const double *rhs, double *x, double thresh, int max_iters,
                   int *iters, pmg_stream_t stream);

/* Same CG as pmg_cg_level_d, for callers that cannot let a library allocate
 * device memory (an application that hands all device memory to its own
 * pool, or must not meet allocator stalls or out-of-memory errors inside a
 * time step). The work vectors live in a static device array of this
 * library (about 118 KB, held by every GPU that loads the library until the
 * process exits), so grids are limited to 17*17*17 points including the
 * shell; larger grids return PMG_ERR_ARG. Every call looks up the array's
 * device address in the current device's context (so a cudaDeviceReset
 * between calls is harmless). All calls on a device share the array: each
 * call clears the part it uses, and calls that overlap on the GPU (e.g. on
 * two streams) corrupt each other. Grids of at most 17 points per axis run
 * as the cluster kernel, which keeps its vectors on chip (only the array's
 * two status words are used); the other accepted shapes (e.g. 19 x 13 x 19)
 * run the one-CTA kernel on the array's work vectors. Synchronises the
 * stream. No counterpart in the reference. */
int pmg_cg_level_noalloc_d(int nx, int ny, int nz, const double *const *a14,
                           const double *rhs, double *x, double thresh,
                           int max_iters, int *iters, pmg_stream_t stream);

/* ======================================================================
 * Fine-level set-up from atoms (host)
 * ==================================================================== */

/* Physical parameters of a linearized PB problem. */
typedef struct {
  double eps_in;         /* solute dielectric (reference: epsilon_p)        */
  double eps_out;        /* solvent dielectric (reference: epsilon_r)       */
  double ionic_strength; /* 1:1 salt, mol/l                                 */
  double ion_radius;     /* Angstrom, inflates the ion-exclusion spheres    */
  double temperature;    /* K                                               */
  double probe_radius;   /* Angstrom; 0 = van der Waals dielectric boundary */
} pmg_physics;

/* Inverse Debye length (1/Angstrom) and the vacuum permittivity in the
 * reference's reduced units (e^2 / (kT Angstrom)); KappaA and epsilon,
 * scientific_quantities.h:8-55. Either output may be NULL. */
int pmg_kappa(const pmg_physics *phys, double *kappa, double *eps0);

/* Builds the fine level of an n^3 grid with spacing h (host arrays, n^3
 * doubles each) from natoms rows (x, y, z, radius, charge) in the grid's
 * frame (grid point (i0,i1,i2) sits at (i0 h, i1 h, i2 h); coordinate 0 lies
 * on the slowest array axis, as the reference's Position[0]):
 *   oE oN uC  eps/h^2 at the staggered points (x fastest: oE), eps_in inside
 *             the solute, eps_out outside;
 *   oC        sum of the six face coefficients plus kappa^2 eps_out outside
 *             the ion-exclusion spheres (interior only);
 *   f         trilinear charges q / eps0 / h^3;
 *   x0        multiple Debye-Hueckel boundary values on the shell, 0 inside.
 * Replaces initialize_epsilons, set_up_rhs and initialize_boundary of the
 * class, PBE_pmgc_class.h:141-349 (probe_radius 0 reproduces them). */
int pmg_setup_fine(int n, double h, const double *atoms, int natoms,
                   const pmg_physics *phys, double *oC, double *oE,
                   double *oN, double *uC, double *f, double *x0);

/* The same set-up on the GPU into device arrays (n^3 doubles each),
 * stream-ordered on `stream` (scratch from the stream-ordered allocator);
 * atoms are host rows, validated like pmg_setup_fine. oE oN uC oC and f are
 * bit-identical to pmg_setup_fine (same marking bounds and sums, charges
 * summed per grid point in atom order); x0 uses CUDA's exp and agrees to a
 * few ulp. */
int pmg_setup_fine_d(int n, double h, const double *atoms, int natoms,
                     const pmg_physics *phys, double *oC, double *oE,
                     double *oN, double *uC, double *f, double *x0,
                     pmg_stream_t stream);

/* ---- File formats ------------------------------------------------------
 * PQR atoms (read_pqr_file, fileio.cc:10-53): every non-REMARK line of
 * exactly ten fields gives one row (x, y, z, radius, charge) from fields
 * 6-8, 10 and 9. With atoms == NULL only counts; returns PMG_ERR_ARG when
 * the file cannot be read or holds more than cap atoms. */
int pmg_read_pqr(const char *path, double *atoms, int cap, int *count);
/* OpenDX grid file of an nx x ny x nz array in array order (x fastest), the
 * reference's print_dx_to_stream (Domain.h:136-185): counts slowest axis
 * first (nz ny nx), origin (xmin, ymin, zmin), spacing box_length / (nz - 1)
 * on every axis (box_length is the extent of the slowest axis, as in the
 * reference), three values per line. */
int pmg_write_dx(const char *path, const double *values, int nx, int ny,
                 int nz, double xmin, double ymin, double zmin,
                 double box_length);

/* ======================================================================
 * Problem handle: PBE_linear_problem<base, nlev, box> with runtime sizes
 * (PBE_pmgc_class.h:112-1174). Level L has n_L = base*2^L + 1 points per
 * axis; level nlev is the finest, level 1 the coarsest (CG).
 * ==================================================================== */

typedef struct pmg_problem pmg_problem;

typedef enum {
  PMG_PREC_FP64 = 0,  /* V-cycles in double (the reference's arithmetic)  */
  PMG_PREC_MIXED = 1, /* float V-cycles inside double iterative refinement */
  /* double V-cycles with the mixed path's structure: zero-started V-cycles
   * on the correction equation inside the same double refinement loop, the
   * finest level on colour-split arrays with coded couplings; the fastest
   * all-double solve (not the reference's cycle, so its potential agrees
   * with the reference's to the stopping tolerance, not to rounding). */
  PMG_PREC_FP64_FAST = 2
} pmg_precision;

/* The mixed path's 27-point smoother stages each tile's operator, right-hand
 * side and iterate planes in shared memory with tensor-memory-access copies
 * on the levels between its one-launch bottom levels and the finest level
 * (their float rows are padded to a 16-byte multiple for it). on = 0 makes
 * problems created afterwards use the per-point-load kernel instead; both
 * give the same bits. No counterpart in the reference. */
int pmg_set_tma_staging(int on);

/* The refinement paths' finest red-black colour passes stream the level's
 * rows through shared memory: per plane, one bulk copy per row of the other
 * colour's iterate and of the own colour's right-hand side and code bytes,
 * into a ring of stages, so the bytes in flight are set by the ring and not
 * by registers. on = 0 makes problems created afterwards use the
 * per-point-load pass instead; both give the same bits. No counterpart in
 * the reference (Vgsrb7x, pmgc/gsd.cc:61-111, is the arithmetic of both).
 * A lost stage is reported like the staged 27-point smoother's. */
int pmg_set_finest_streaming(int on);

/* For testing the staged smoother's error path: every tensor-memory-access
 * stage of solves launched or captured afterwards waits for `bytes` more
 * than its boxes deliver (a multiple of 16, 0 restores the normal count),
 * so each bounded wait runs out (about 0.1 s), the kernel records the lost
 * stage and returns, and the solve reports PMG_ERR_TIMEOUT with the context
 * still usable. A captured solve graph keeps the value it was captured
 * with: use new problems on both sides of the switch. */
int pmg_test_tma_short_delivery(int bytes);

/* Creates a problem on the current CUDA device; allocates its hierarchy.
 * stream may be NULL (a private stream is created). */
int pmg_problem_create(int base, int nlev, double box, int precision,
                       pmg_stream_t stream, pmg_problem **out);
/* Frees the handle and everything it allocated. */
int pmg_problem_destroy(pmg_problem *p);
/* Device bytes held by a problem of this shape (for admission control). */
long long pmg_problem_bytes(int base, int nlev, int precision);

/* Loads the fine level: oC (kappa^2 folded in), oE, oN, uC, the right-hand
 * side f and the initial iterate x0 whose shell holds the boundary values.
 * Pointers may be host or device memory (copied). Replaces filling the
 * class's maps by initialize_epsilons / set_up_rhs / initialize_boundary,
 * PBE_pmgc_class.h:191-349. */
int pmg_problem_set_fine(pmg_problem *p, const double *oC, const double *oE,
                         const double *oN, const double *uC, const double *f,
                         const double *x0);

/* Loads the finest level from atoms with the GPU set-up (pmg_setup_fine_d
 * at spacing box / (n - 1)) straight into the problem's arrays: only the
 * atoms cross PCIe. Replaces the class's set-up chain (initialize_boundary,
 * initialize_epsilons, set_up_rhs; PBE_pmgc_class.h:141-349). */
int pmg_problem_set_atoms(pmg_problem *p, const double *atoms, int natoms,
                          const pmg_physics *phys);

/* Builds the Galerkin hierarchy (P then A_c per level); trilinear != 0 uses
 * constant weights. Replaces buildmultilevelops, PBE_pmgc_class.h:351-617. */
int pmg_build_hierarchy(pmg_problem *p, int trilinear);

/* One V-cycle of the class (v_cycle, PBE_pmgc_class.h:1070-1114); with
 * as_preconditioner != 0 every level is zero-initialised. FP64 problems
 * only. */
int pmg_vcycle(pmg_problem *p, int as_preconditioner);

/* sqrt(sum_interior (f - A x)^2 / n^3) of the finest level; synchronises.
 * Replaces compute_residual_2, PBE_pmgc_class.h:768-772. */
int pmg_compute_residual_2(pmg_problem *p, double *out);

/* Solves to compute_residual_2()/r0 < tol with at most max_cycles V-cycles
 * (FP64) or refinement steps (mixed): the solve loop of the class's apps
 * (PBE_pmgc_class_test.cc:124-146). *cycles and *relres (host) get the
 * cycles run and the final relative residual; hist (host, may be NULL,
 * max_cycles+1 entries) the residual norm per cycle. Returns
 * PMG_ERR_DIVERGED on NaN/Inf or stagnation. Runs as one graph launch with
 * the stop test on the GPU (pmg_solve_start + pmg_solve_finish) unless phase
 * timing is on or max_cycles > 1024 (then one launch and one read-back per
 * cycle); both take the same decisions. */
int pmg_solve(pmg_problem *p, double tol, int max_cycles, int *cycles,
              double *relres, double *hist);

/* MG-preconditioned CG on the finest level, the reference app's outer
 * solver (PBE_pmgc_class_with_non_zero_IS.cc:118-131: CG_solver,
 * CG_Solver.h:45-242, with the class as preconditioner, operator(),
 * PBE_pmgc_class.h:1116-1133 -- one zero-started V-cycle per application,
 * FP64 or, for mixed problems, the float V-cycle). Starts from the loaded
 * iterate and stops after max_iters (<= 1024) iterations or, with tol > 0,
 * once sqrt(sum r^2 / n^3) of the recursively updated residual is below tol
 * times its initial value (tol = 0: the app's counting criterion). The
 * result replaces the finest iterate (pmg_get_potential); *iters, *relres
 * and hist (max_iters + 1 entries, may be NULL) as for pmg_solve. The whole
 * iteration is one graph launch (stop test on the GPU). Allocates 6 n^3
 * doubles on first use. */
int pmg_pcg_solve(pmg_problem *p, double tol, int max_iters, int *iters,
                  double *relres, double *hist);

/* Asynchronous solve (no reference counterpart; the class's loop is
 * synchronous): enqueues the whole solve on the problem's stream as one
 * graph launch whose while node repeats cycle + stop test on the GPU, and
 * returns at once. 0 <= max_cycles <= 1024. One solve in flight per
 * problem; independent problems on their own streams overlap on the
 * device. */
int pmg_solve_start(pmg_problem *p, double tol, int max_cycles);
/* *done = 1 once the solve started by pmg_solve_start has finished on the
 * GPU (also when none is in flight); never blocks. */
int pmg_solve_poll(pmg_problem *p, int *done);
/* Waits for the solve in flight and reports it like pmg_solve. */
int pmg_solve_finish(pmg_problem *p, int *cycles, double *relres,
                     double *hist);

/* Copies the finest iterate (n^3 doubles incl. shell) to dst (host or
 * device). */
int pmg_get_potential(pmg_problem *p, double *dst);

/* pmg_get_potential without the wait: the copy is queued on the problem's
 * stream (dst must stay valid until the stream reaches it). */
int pmg_get_potential_async(pmg_problem *p, double *dst);

/* Moves the problem to another stream (no solve may be in flight); work
 * already queued on the old stream stays ordered before later work. The
 * captured graphs are launched on whichever stream the problem has. NULL
 * returns a problem created without a stream to the stream it created. */
int pmg_problem_set_stream(pmg_problem *p, pmg_stream_t stream);

/* Copies level L's hierarchy out (host or device dst): 27 prolongation
 * arrays then 14 operator arrays, n_L^3 doubles each; L in [1, nlev-1]. */
int pmg_get_level(pmg_problem *p, int level, double *dst);

/* Mixed precision: relative residual reduction at which the coarsest-level
 * CG stops on each correction (default 1e-4; the FP64 path always runs the
 * class's absolute 1e-8 test). */
int pmg_problem_set_coarse_rtol(pmg_problem *p, double rtol);

/* on != 0: pmg_solve drives its cycles from the host (one cycle-graph
 * launch and one residual read-back per cycle) instead of the single graph
 * with the device-side stop test; same decisions, same results. For tools
 * that cannot look inside graphs with conditional nodes (kernel profilers).
 * No reference counterpart. */
int pmg_problem_set_host_loop(pmg_problem *p, int on);

/* Mixed precision: the finest float smoother and defect read the couplings
 * as one code byte per point with a two-value table per direction whenever
 * the fine operator has two values per coupling direction (the class's
 * dielectric faces do), and the coupling arrays otherwise; results are the
 * same bits either way. on = 0 keeps the arrays (default 1). */
int pmg_problem_set_coded_couplings(pmg_problem *p, int on);
/* *coded = 1 when the built mixed problem's finest couplings are coded and
 * in use. Synchronises the problem's stream. */
int pmg_problem_coded_couplings(pmg_problem *p, int *coded);
/* *streamed = 1 when the problem's finest colour passes and refinement
 * residual stream their rows through shared memory (mixed and fp64-fast
 * problems created with pmg_set_finest_streaming on, levels that fit the
 * stage ring). No reference counterpart. */
int pmg_problem_finest_streamed(pmg_problem *p, int *streamed);

/* on != 0: choose kernels for many solves sharing the GPU rather than for
 * the latency of this one: the mixed path's lowest levels run in one CTA
 * instead of an 8-CTA cluster with its arrays in shared memory (a cluster
 * starts only when eight SMs of one GPC are idle at once). Same arithmetic
 * per point; the mixed results may differ in the last bits (sums in another
 * order). The serving runtime sets it on the problems it creates. Default
 * off. No reference counterpart. */
int pmg_problem_set_throughput_mode(pmg_problem *p, int on);

/* Tile edge of the 27-point smoother, for the whole process. mode 1 (the
 * default): pmg_build_hierarchy times the edges 8, 16 and 32 on each level
 * size the first time it meets it and keeps the fastest (the size rule's
 * edge unless another is more than 10% faster); mode 0: the size rule (32
 * from 97 points per axis, 16 from 49, else 8); mode 8, 16 or 32: that
 * edge everywhere. Every edge gives the same results. Use mode 0 under
 * kernel profilers, which serialise and replay launches so that timings
 * taken there mean nothing. Other modes: PMG_ERR_ARG. No reference
 * counterpart. */
int pmg_set_autotune(int mode);

/* Phase timing: with on != 0, pmg_solve records CUDA events around every
 * phase of every cycle (inside the captured cycle graph) and accumulates the
 * elapsed times. */
int pmg_problem_set_profiling(pmg_problem *p, int on);
/* Accumulated phase times (ms) and counts; slot = level * 8 + phase with
 * phase 0 pre-smoothing, 1 defect, 2 restriction, 3 coarsest solve,
 * 4 damping, 5 interpolation, 6 x += w e, 7 post-smoothing; level 0 holds
 * 0 finest-level residual norm, 1 refinement update. Returns the number of
 * slots; reset != 0 clears the accumulators. */
int pmg_problem_profile(pmg_problem *p, double *ms, long long *counts,
                        int cap, int reset);

/* Kernels this problem has launched so far (hierarchy builds, residuals and
 * every kernel node of each replayed cycle graph). */
long long pmg_problem_launches(pmg_problem *p);

/* The class's stream (for callers that enqueue around a solve). */
pmg_stream_t pmg_problem_stream(pmg_problem *p);

/* ---- Serving: continuous batching of independent solves ------------------
 * No reference counterpart: the reference solves one molecule per process
 * (PBE_pmgc_class_test.cc:84-146). A server owns a worker thread that admits
 * requests in arrival order against a device-memory budget (the bytes of
 * every problem it holds, pmg_problem_bytes), keeps each admitted solve's
 * hierarchy resident in its own problem (reused for later requests of the
 * same grid and precision), runs up to max_inflight solves at once, each as
 * one graph launch on its own stream (pmg_solve_start), so cycles of
 * different grid sizes overlap on the device, and reports completions. A
 * request's arithmetic does not depend on what else is in flight: its result
 * is bit-identical alone and in the mix. */
typedef struct pmg_server pmg_server;

typedef struct pmg_request {
  int base, nlev;          /* grid: n = base * 2^nlev + 1 per axis        */
  double box;              /* domain edge (Angstrom)                      */
  int precision;           /* pmg_precision                               */
  const double *fine[6];   /* oC oE oN uC f x0, n^3 each, host or device; */
                           /* valid until the request's completion        */
  double *potential;       /* n^3 result (host or device), may be NULL    */
  double tol;              /* relative residual target                    */
  int max_cycles;          /* 0 .. 1024                                   */
  long long tag;           /* caller's identifier, echoed back            */
  int hierarchy;           /* 0: levels as given; 1: the deepest levels   */
                           /* of the same grid (pmg_levels_for(n, 12, 5)) */
  const double *atoms;     /* non-NULL: load the fine level from these    */
                           /* host rows (x y z radius charge) with the GPU*/
                           /* set-up (pmg_problem_set_atoms); fine[] is   */
                           /* then ignored                                */
  int natoms;
  pmg_physics physics;     /* set-up parameters when atoms is non-NULL    */
} pmg_request;

typedef struct pmg_completion {
  long long tag;
  int status;              /* pmg_status of the solve                    */
  int cycles;
  double relres;
  double t_submit, t_admit, t_done; /* seconds since server creation      */
  char message[160];       /* error text when status != PMG_OK            */
} pmg_completion;

typedef struct pmg_server_stats {
  int queued, inflight, idle_problems;
  long long held_bytes, peak_bytes, budget_bytes;
  long long completed, created_problems, evicted_problems;
  /* host time of the worker: issuing requests (set-up / load, build,
   * solve launch) and retiring them (results copied out), total and
   * longest single call, seconds */
  double issue_s, issue_max_s, retire_s, retire_max_s;
} pmg_server_stats;

/* (base, nlev) with n = base * 2^nlev + 1, the largest nlev <= max_levels
 * whose coarsest grid 2 * base + 1 has at least min_coarse points (grid-size
 * rule of Vcorsr, pmgc/mgsubd.cc:395-413, applied as far as it goes). */
int pmg_levels_for(int n, int max_levels, int min_coarse, int *base,
                   int *nlev);

/* budget_bytes > 0; 1 <= max_inflight <= 256. Uses the current device. */
int pmg_server_create(long long budget_bytes, int max_inflight,
                      pmg_server **out);
/* Enqueues a copy of *r; never blocks on the GPU. A request larger than the
 * whole budget completes with PMG_ERR_BUDGET. */
int pmg_server_submit(pmg_server *s, const pmg_request *r);
/* Moves up to cap completions into out (*n of them), waiting up to
 * timeout_s seconds for the first one (0: no wait). */
int pmg_server_wait(pmg_server *s, pmg_completion *out, int cap, int *n,
                    double timeout_s);
int pmg_server_get_stats(pmg_server *s, pmg_server_stats *st);
/* Finishes the queued and in-flight work, then frees everything. */
int pmg_server_destroy(pmg_server *s);

/* Batched solves: every request through one server with the given budget,
 * all admitted as memory allows; out[i] belongs to reqs[i]. */
int pmg_batch_solve(const pmg_request *reqs, int count, long long budget_bytes,
                    int max_inflight, pmg_completion *out);

#ifdef __cplusplus
}
#endif

#endif /* PMG_B200_H */
