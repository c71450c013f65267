/* CPU restatement of the reference PMG path (oracle, test infrastructure).
 *
 * Plain C99, double precision, single thread. This is the checker that
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use; the
 * product (multigrid_b200/) never links or calls it.
 *
 * Every function restates one reference routine and cites it. Grid arrays use
 * the reference layout: nx*ny*nz doubles with a one-point shell, x fastest,
 * 1-based (i,j,k) -> ((k-1)*ny + (j-1))*nx + (i-1)  (pmgc/vmatrix.h:79-80).
 *
 * Operators are held as 14 "upper" diagonals (oC oE oN uC oNE oNW uE uW uN uS
 * uNE uNW uSE uSW, pmgc/buildGd.h:281-494); a 7-point operator sets only
 * oC oE oN uC and leaves the other ten NULL. Off-diagonal entries are stored
 * as positive couplings: A(p, p+d) = -coef. Prolongations are 27 arrays on
 * the coarse grid in the order oPC oPN oPS oPE oPW oPNE oPNW oPSE oPSW,
 * uP*, dP* (pmgc/matvecd.cc:696-704).
 */
#ifndef PMG_ORACLE_H
#define PMG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* 14-diagonal operator; kind 7 or 27. */
typedef struct {
  int kind;
  const double *a[14];
} pmgo_op;

/* ---- single kernels ------------------------------------------------- */
void pmgo_gsrb7x(int nx, int ny, int nz, const double *oC, const double *cc,
                 const double *fc, const double *oE, const double *oN,
                 const double *uC, double *x, int itmax, int iadjoint,
                 int zero_init);
void pmgo_gsrb27x(int nx, int ny, int nz, const double *const *a14,
                  const double *cc, const double *fc, double *x, int itmax,
                  int iadjoint, int zero_init);
void pmgo_matvec(int nx, int ny, int nz, const pmgo_op *A, const double *cc,
                 const double *x, double *y);
void pmgo_mresid(int nx, int ny, int nz, const pmgo_op *A, const double *cc,
                 const double *fc, const double *x, double *r);
void pmgo_restrc2(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                  const double *xin, double *xout, const double *const *p27);
void pmgo_interp2(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                  const double *xin, double *xout, const double *const *p27);
void pmgo_buildP_op(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                    const pmgo_op *A, double *const *p27);
void pmgo_buildP_trilin(int nxc, int nyc, int nzc, double *const *p27);
/* Hestenes-Stiefel CG of the APBS layer (Vcghs, documented dot/axpy);
 * returns the iteration count. */
int pmgo_cghs(int nx, int ny, int nz, const pmgo_op *A, const double *cc,
              const double *fc, double *x, double *p, double *ap, double *r,
              int itmax, double errtol, int iresid);
/* APBS iparm/rparm driver, linear case (Vmgdriv, Vbuildops with Galerkin
 * coarsening, Vmvcs). iparm/rparm are 0-based copies of the reference's
 * 1-based arrays. u: n^3 in/out (solution with the boundary values on the
 * shell); tcf: the true solution for istop 2/3 (overwritten by istop 2),
 * else may be NULL. Returns 0, -1 (bad nlev), -2 (out of memory) or -3
 * (mgsolv 1: the coarsest operator is not positive definite). */
int pmgo_mgdriv(const int *iparm, const double *rparm, double *u,
                const double *xf, const double *yf, const double *zf,
                const double *gxcf, const double *gycf, const double *gzcf,
                const double *a1cf, const double *a2cf, const double *a3cf,
                const double *ccf, const double *fcf, double *tcf,
                int *iters_out, int *ierror_out, double *rsnrm_out);
/* Banded direct solver of the APBS layer (Vbuildband, Vdpbfa, Vdpbsl):
 * band storage (abd zeroed by the caller, (m+1)*n doubles), in-place
 * factorisation (returns info), in-place solve. */
void pmgo_buildband(int nx, int ny, int nz, const pmgo_op *A, int *n_out,
                    int *m_out, int *lda_out, double *abd);
int pmgo_dpbfa(double *abd, int lda, int n, int m);
void pmgo_dpbsl(const double *abd, int lda, int n, int m, double *b);
/* Box-method fine operator from coefficient maps (VbuildA_fv). */
void pmgo_buildA_fv(int nx, int ny, int nz, int ipkey, int *numdia, int *ipc,
                    double *oC, double *cc, double *fc, double *oE,
                    double *oN, double *uC, const double *xf,
                    const double *yf, const double *zf, const double *gxcf,
                    const double *gycf, const double *gzcf,
                    const double *a1cf, const double *a2cf,
                    const double *a3cf, const double *ccf,
                    const double *fcf);
void pmgo_buildG(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                 const double *const *p27, const pmgo_op *A,
                 double *const *out14);

/* ---- the class's map-based helpers ---------------------------------- */
void pmgo_defect(int nx, int ny, int nz, const pmgo_op *A, const double *f,
                 const double *x, double *r);
double pmgo_residual2(int nx, int ny, int nz, const pmgo_op *A,
                      const double *f, const double *x);
double pmgo_ideal_lambda(int nx, int ny, int nz, const pmgo_op *A,
                         const double *x, const double *r);
int pmgo_cg(int nx, int ny, int nz, const pmgo_op *A, const double *rhs,
            double *x, double thresh);

/* ---- whole solve ----------------------------------------------------- */
/* Fine inputs as in the reference class: oC has kappa^2 folded in, x0 holds
 * the Dirichlet boundary on its shell. Levels: n_L = base*2^L + 1.
 * trilinear selects constant prolongation weights. Returns V-cycles run or a
 * negative value on allocation failure. hist[0..cycles] gets the residual
 * norms. */
int pmgo_solve(int base, int nlev, const double *oC, const double *oE,
               const double *oN, const double *uC, const double *f,
               const double *x0, double tol, int max_cycles, int trilinear,
               double *x_out, double *hist);

/* Hierarchy in the layout of pmgref_hierarchy: for L = nlev-1 .. 1, the 27
 * prolongation arrays then the 14 operator arrays of level L. Returns the
 * number of doubles written, or -1 if cap is too small. */
/* MG-preconditioned CG on the finest level (CG_Solver.h:45-242 with the
 * class as preconditioner, PBE_pmgc_class.h:1116-1133); see pmg_oracle.c. */
int pmgo_pcg(int base, int nlev, const double *oC, const double *oE,
             const double *oN, const double *uC, const double *f,
             const double *x0, int max_iters, double tol, double *x_out,
             double *hist);

long pmgo_hierarchy(int base, int nlev, const double *oC, const double *oE,
                    const double *oN, const double *uC, int trilinear,
                    double *out, long cap);

/* ---- fine-level set-up from atoms (pmg_oracle_setup.c) ---------------- */
/* kappa (1/Angstrom) and eps0 (e^2 / (kT Angstrom)) of the physics
 * (scientific_quantities.h:7-55). */
void pmgo_physics(double eps_out, double ionic_strength, double temperature,
                  double *kappa, double *eps0);
/* Fine level of an n^3 grid from natoms rows (x, y, z, radius, charge) in
 * the grid frame: face coefficients, oC with kappa^2 eps_out folded in,
 * trilinear charges, multiple Debye-Hueckel boundary on the shell
 * (PBE_pmgc_class.h:141-349). probe_radius 0 is the reference's van der
 * Waals marking; > 0 the molecular surface. Returns 0, -1 on a bad argument
 * or an atom outside the grid, -2 on allocation failure. */
int pmgo_setup_fine(int n, double h, const double *atoms, int natoms,
                    double eps_in, double eps_out, double ionic_strength,
                    double ion_radius, double temperature,
                    double probe_radius, double *oC, double *oE, double *oN,
                    double *uC, double *f, double *x0);

#ifdef __cplusplus
}
#endif

#endif
