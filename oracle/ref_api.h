/* C interface of the reference-built oracle (oracle/_ref/libpmgc_ref*.so).
 *
 * TEST INFRASTRUCTURE ONLY. These entry points wrap the reference's own
 * PBE_pmgc_class.h (class pmgc_solver::PBE_linear_problem) and pmgc kernels,
 * compiled with g++ against the host SYCL shim in oracle/shim. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load them, as the
 * checker or the timed CPU reference — never as part of the product path.
 *
 * Array convention (same as the reference, pmgc/vmatrix.h:79-80): every grid
 * array holds nx*ny*nz doubles including the one-point Dirichlet shell,
 * x fastest: VAT3(m,i,j,k) = m[(k-1)*ny*nx + (j-1)*nx + (i-1)].
 *
 * Coarse-operator order (14 arrays): oC oE oN uC oNE oNW uE uW uN uS uNE uNW
 * uSE uSW (pmgc/buildGd.h:281-494). Prolongation order (27 arrays): oPC oPN
 * oPS oPE oPW oPNE oPNW oPSE oPSW, uP*, dP* (pmgc/matvecd.cc:696-704).
 */
#ifndef PMGC_REF_API_H
#define PMGC_REF_API_H

#ifdef __cplusplus
extern "C" {
#endif

/* Grid configurations compiled into the oracle: fills base/nlev/box of up to
 * cap entries, returns the total count. */
int pmgref_configs(int *base, int *nlev, double *box, int cap);

/* Fine level of the class's PMG problem.
 *   oC     centre coefficient with kappa^2*eps folded in (cc stays 0)
 *   oE oN uC  face coefficients eps/h^2 (upper-neighbour convention)
 *   f      right-hand side
 *   x0     initial iterate; its shell holds the Dirichlet boundary values */
typedef struct {
  const double *oC, *oE, *oN, *uC, *f, *x0;
} pmgref_fine;

/* Builds the Galerkin hierarchy (buildmultilevelops,
 * PBE_pmgc_class.h:351-617) and loops v_cycle (PBE_pmgc_class.h:1070-1114)
 * until compute_residual_2()/r0 < tol or max_cycles cycles ran.
 * x_out: fine potential (nx^3); hist: max_cycles+1 residual norms
 * (compute_residual_2, PBE_pmgc_class.h:768); *cycles: V-cycles run.
 * trilinear != 0 selects VbuildPb_trilin instead of VbuildPb_op7/op27.
 * Returns 0, or -1 for an unknown (base, nlev). */
int pmgref_solve(int base, int nlev, const pmgref_fine *in, double tol,
                 int max_cycles, int trilinear, double *x_out, double *hist,
                 int *cycles);

/* Same set-up, then exactly `ncycles` V-cycles with no residual checks in
 * between (for timing a bounded sample). Returns 0 or -1. */
int pmgref_cycles(int base, int nlev, const pmgref_fine *in, int ncycles,
                  double *x_out);

/* Builds only the hierarchy and copies it out. For each coarse level
 * L = nlev-1 down to 1 the output holds, back to back, the 27 prolongation
 * arrays (level L) then the 14 operator arrays (level L), each n_L^3 doubles
 * with n_L = base*2^L + 1. Returns the number of doubles written or -1. */
long pmgref_hierarchy(int base, int nlev, const pmgref_fine *in,
                      int trilinear, double *out, long cap);

/* One coarsest-level CG solve as v_cycle<1> runs it (solve_by_cg<1>,
 * PBE_pmgc_class.h:856-860; CG_solver, CG_Solver.h:45-242) on level 1 of a
 * (base, nlev) problem: op14 = the 14 level-1 operator arrays, rhs, x in/out
 * (warm start). Returns 0 or -1. */
int pmgref_cg_level1(int base, int nlev, const double *const *op14,
                     const double *rhs, double *x);

/* The class's own set-up from atoms with the reference's compiled-in
 * constants (epsilon_p 4.0, epsilon_r 78.4; scientific_quantities.h:14-15):
 * initialize_boundary, initialize_epsilons, set_up_rhs
 * (PBE_pmgc_class.h:141-349). atoms: n rows of (x, y, z, radius, charge) in
 * the grid's frame (origin at the first shell point). Outputs fine oC, oE, oN,
 * uC, f and x0 (boundary on the shell, zero inside); box comes from the
 * compiled-in configuration. Returns 0 or -1. */
int pmgref_setup(int base, int nlev, const double *atoms, int natoms,
                 double ionic_strength, double ion_radius, double *oC,
                 double *oE, double *oN, double *uC, double *f, double *x0);

/* MG-preconditioned CG of the reference app
 * (PBE_pmgc_class_with_non_zero_IS.cc:123-131): CG_solver
 * (CG_Solver.h:45-242) on the finest level with the class as preconditioner
 * (operator(), PBE_pmgc_class.h:1116-1133: one zero-started V-cycle),
 * counting criterion of `iters` iterations. The class's own finest iterate
 * starts at zero (the app never sets its boundary); x0 (with the Dirichlet
 * shell) is the CG's initial guess. Writes the iterate to x_out. */
int pmgref_pcg(int base, int nlev, const pmgref_fine *in, int iters,
               double *x_out);

/* Single pmgc kernels (pmgc/*.cc), called on host arrays. */
int pmgref_Vgsrb7x(int nx, int ny, int nz, const double *oC, const double *cc,
                   const double *fc, const double *oE, const double *oN,
                   const double *uC, double *x, int itmax, int iadjoint,
                   int zero_init);
int pmgref_Vgsrb27x(int nx, int ny, int nz, const double *const *op14,
                    const double *cc, const double *fc, double *x, int itmax,
                    int iadjoint, int zero_init);
int pmgref_Vmatvec7_1s(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *oE, const double *oN,
                       const double *uC, const double *x, double *y);
int pmgref_Vmatvec27_1s(int nx, int ny, int nz, const double *const *op14,
                        const double *cc, const double *x, double *y);
int pmgref_Vmresid7_1s(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *fc, const double *oE,
                       const double *oN, const double *uC, const double *x,
                       double *r);
int pmgref_Vmresid27_1s(int nx, int ny, int nz, const double *const *op14,
                        const double *cc, const double *fc, const double *x,
                        double *r);
int pmgref_Vrestrc2(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                    const double *xin, double *xout, const double *const *p27);
int pmgref_VinterpPMG2(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                       const double *xin, double *xout,
                       const double *const *p27);
int pmgref_VbuildPb_op7(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                        const double *oC, const double *oE, const double *oN,
                        const double *uC, double *const *p27);
int pmgref_VbuildPb_op27(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                         const double *const *op14, double *const *p27);
int pmgref_VbuildPb_trilin(int nxf, int nyf, int nzf, int nxc, int nyc,
                           int nzc, double *const *p27);
int pmgref_VbuildG_7(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                     const double *const *p27, const double *oC,
                     const double *oE, const double *oN, const double *uC,
                     double *const *out14);
int pmgref_VbuildG_27(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                      const double *const *p27, const double *const *op14,
                      double *const *out14);

/* The reference's box-method fine builder VbuildA_fv
 * (pmgc/buildAd.cc:63-212) as compiled: ipc needs 12 ints (it writes
 * ipc[9..11]), numdia one; rpc is unused by it. */
int pmgref_VbuildA_fv(int nx, int ny, int nz, int ipkey, int *numdia,
                      int *ipc, double *oC, double *cc, double *fc,
                      double *oE, double *oN, double *uC, const double *xf,
                      const double *yf, const double *zf, const double *gxcf,
                      const double *gycf, const double *gzcf,
                      const double *a1cf, const double *a2cf,
                      const double *a3cf, const double *ccf,
                      const double *fcf);

/* The reference's banded coarse solver as compiled: Vbuildband
 * (pmgc/buildBd.cc:252-303: LINPACK band storage of the interior operator,
 * then Vdpbfa, pmgc/mlinpckd.cc:168-207) and Vdpbsl (:209-240). ac: the
 * packed operator (4 or 14 columns for numdia 7 or 27); ipcB gets n, m,
 * lda, 1; acB (zeroed by the caller) lda*n doubles. Returns key (0, or 1
 * when the factorisation met a non-positive pivot). */
int pmgref_Vbuildband(int nx, int ny, int nz, int numdia, double *ac,
                      int *ipcB, double *acB);
int pmgref_Vdpbfa(double *abd, int lda, int n, int m);
int pmgref_Vdpbsl(double *abd, int lda, int n, int m, double *b);

/* The reference's PQR reader (read_pqr_file, fileio.cc:10-53): rows (x, y,
 * z, radius, charge) of up to cap atoms; *count gets the number read.
 * Returns -1 when the file holds more than cap. */
int pmgref_read_pqr(const char *path, double *atoms, int cap, int *count);

/* The reference's OpenDX writer (Grid::print_dx_to_stream,
 * Domain.h:136-185) on a grid of interior lengths (slowest axis first)
 * 4 x 5 x 6 (shape 0) or 7 x 7 x 7 (shape 1) with a one-point padding,
 * values in array order; the text goes to out (cap bytes). Returns its
 * length, or minus the bytes needed. */
long pmgref_write_dx(int shape, const double *values, double xmin,
                     double ymin, double zmin, double box, char *out,
                     long cap);

#ifdef __cplusplus
}
#endif

#endif
