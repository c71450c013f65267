/* CPU restatement of the reference PMG path (oracle, test infrastructure).
 * See pmg_oracle.h for conventions. Each routine cites the reference routine
 * it restates; the per-point arithmetic of the smoothers, matvecs, residuals
 * and transfers keeps the reference's operation order so that single-kernel
 * FP64 results can be compared bit for bit. The prolongation and Galerkin
 * builders are a generic formulation of the same operators (see the comments
 * there) and agree with the reference to rounding.
 */
#include "pmg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IX(nx, ny, i, j, k)                                                    \
  (((size_t)((k)-1) * (size_t)(ny) + (size_t)((j)-1)) * (size_t)(nx) +          \
   (size_t)((i)-1))

/* Index of the stored upper diagonal for a neighbour offset (ex,ey,ez), or 0
 * when the offset is not an upper one. 1..13 = oE oN uC oNE oNW uE uW uN uS
 * uNE uNW uSE uSW. */
static int upper_slot(int ex, int ey, int ez) {
  if (ez == 1) {
    static const int t[3][3] = {/* ey=-1 */ {13, 9, 12},
                                /* ey= 0 */ {7, 3, 6},
                                /* ey=+1 */ {11, 8, 10}};
    return t[ey + 1][ex + 1];
  }
  if (ez == 0 && ey == 1)
    return ex == 1 ? 4 : (ex == 0 ? 2 : 5);
  if (ez == 0 && ey == 0 && ex == 1)
    return 1;
  return 0;
}

/* Positive coupling between fine point (i,j,k) and (i+ex, j+ey, k+ez) of a
 * symmetric 14-diagonal operator: the lower half is read from the upper
 * diagonal stored at the neighbour (pmgc/matvecd.h:208-236). */
static double coupling(const pmgo_op *A, int nx, int ny, int i, int j, int k,
                       int ex, int ey, int ez) {
  int s = upper_slot(ex, ey, ez);
  if (s) {
    const double *a = A->a[s];
    return a ? a[IX(nx, ny, i, j, k)] : 0.0;
  }
  s = upper_slot(-ex, -ey, -ez);
  const double *a = A->a[s];
  return a ? a[IX(nx, ny, i + ex, j + ey, k + ez)] : 0.0;
}

/* ------------------------------------------------------------------------
 * Gauss-Seidel smoothers
 * ---------------------------------------------------------------------- */

/* Red-black GS on the 7-point operator: Vgsrb7x, pmgc/gsd.cc:61-111.
 * Colour c of each sweep updates (i+j+k)%2 == (1-iad)*c + iad*(1-c) on the
 * 1-based interior; zero_init drops the neighbour sum in the very first
 * colour only (the flag is cleared after each colour, gsd.cc:108). */
void pmgo_gsrb7x(int nx, int ny, int nz, const double *oC, const double *cc,
                 const double *fc, const double *oE, const double *oN,
                 const double *uC, double *x, int itmax, int iadjoint,
                 int zero_init) {
  const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
  for (int it = 1; it <= itmax; ++it) {
    for (int c = 0; c <= 1; ++c) {
      const int want = (1 - iadjoint) * c + iadjoint * (1 - c);
      const double keep = zero_init ? 0.0 : 1.0;
      for (int k = 2; k <= nz - 1; ++k)
        for (int j = 2; j <= ny - 1; ++j)
          for (int i = 2; i <= nx - 1; ++i) {
            if ((i + j + k) % 2 != want)
              continue;
            const size_t p = IX(nx, ny, i, j, k);
            const double s = oN[p] * x[p + sy] + oN[p - sy] * x[p - sy] +
                             oE[p] * x[p + 1] + oE[p - 1] * x[p - 1] +
                             uC[p - sz] * x[p - sz] + uC[p] * x[p + sz];
            x[p] = (fc[p] + keep * s) / (oC[p] + cc[p]);
          }
      zero_init = 0;
    }
  }
}

/* The 27-point neighbour sums in the reference's order: tmpO (8 in-plane),
 * tmpU (9 above), tmpD (9 below); pmgc/gsd.cc:171-204,
 * pmgc/matvecd.cc:142-170. */
static void sums27(const double *const *a, const double *x, size_t p,
                   size_t sy, size_t sz, double *tO, double *tU, double *tD) {
  const double *oE = a[1], *oN = a[2], *uC = a[3], *oNE = a[4], *oNW = a[5];
  const double *uE = a[6], *uW = a[7], *uN = a[8], *uS = a[9], *uNE = a[10];
  const double *uNW = a[11], *uSE = a[12], *uSW = a[13];
  *tO = +oN[p] * x[p + sy] + oN[p - sy] * x[p - sy] + oE[p] * x[p + 1] +
        oE[p - 1] * x[p - 1] + oNE[p] * x[p + 1 + sy] +
        oNW[p] * x[p - 1 + sy] + oNW[p + 1 - sy] * x[p + 1 - sy] +
        oNE[p - 1 - sy] * x[p - 1 - sy];
  *tU = +uC[p] * x[p + sz] + uN[p] * x[p + sy + sz] + uS[p] * x[p - sy + sz] +
        uE[p] * x[p + 1 + sz] + uW[p] * x[p - 1 + sz] +
        uNE[p] * x[p + 1 + sy + sz] + uNW[p] * x[p - 1 + sy + sz] +
        uSE[p] * x[p + 1 - sy + sz] + uSW[p] * x[p - 1 - sy + sz];
  *tD = +uC[p - sz] * x[p - sz] + uS[p + sy - sz] * x[p + sy - sz] +
        uN[p - sy - sz] * x[p - sy - sz] + uW[p + 1 - sz] * x[p + 1 - sz] +
        uE[p - 1 - sz] * x[p - 1 - sz] +
        uSW[p + 1 + sy - sz] * x[p + 1 + sy - sz] +
        uSE[p - 1 + sy - sz] * x[p - 1 + sy - sz] +
        uNW[p + 1 - sy - sz] * x[p + 1 - sy - sz] +
        uNE[p - 1 - sy - sz] * x[p - 1 - sy - sz];
}

/* Eight-colour GS on the 27-point operator: Vgsrb27x, pmgc/gsd.cc:114-212.
 * Colour (i%2) + 2(j%2) + 4(k%2) on 1-based indices, visited in the order
 * c*(1-iad) + iad*(7-c); zero_init clears the whole array first
 * (gsd.cc:154-156). */
void pmgo_gsrb27x(int nx, int ny, int nz, const double *const *a,
                  const double *cc, const double *fc, double *x, int itmax,
                  int iadjoint, int zero_init) {
  const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
  if (zero_init)
    memset(x, 0, sizeof(double) * (size_t)nx * ny * nz);
  for (int it = 1; it <= itmax; ++it)
    for (int c = 0; c < 8; ++c) {
      const int want = c * (1 - iadjoint) + iadjoint * (7 - c);
      for (int k = 2; k <= nz - 1; ++k)
        for (int j = 2; j <= ny - 1; ++j)
          for (int i = 2; i <= nx - 1; ++i) {
            if ((i % 2) + 2 * (j % 2) + 4 * (k % 2) != want)
              continue;
            const size_t p = IX(nx, ny, i, j, k);
            double tO, tU, tD;
            sums27(a, x, p, sy, sz, &tO, &tU, &tD);
            x[p] = (fc[p] + (tO + tU + tD)) / (a[0][p] + cc[p]);
          }
    }
}

/* ------------------------------------------------------------------------
 * Matrix-vector products and residuals
 * ---------------------------------------------------------------------- */

/* y = A x on the interior with the reference's rounding order:
 * 7-point Vmatvec7_1s / matveckernel7 (pmgc/matvecd.cc:62-90,
 * pmgc/matvecd.h:118-139); 27-point Vmatvec27_1s / matveckernel27
 * (pmgc/matvecd.cc:104-176, pmgc/matvecd.h:180-240). */
static double apply_at(int nx, int ny, const pmgo_op *A, const double *cc,
                       const double *x, int i, int j, int k) {
  const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
  const size_t p = IX(nx, ny, i, j, k);
  const double *const *a = A->a;
  const double ccp = cc ? cc[p] : 0.0;
  if (A->kind == 7) {
    const double *oC = a[0], *oE = a[1], *oN = a[2], *uC = a[3];
    return -oN[p] * x[p + sy] - oN[p - sy] * x[p - sy] - oE[p] * x[p + 1] -
           oE[p - 1] * x[p - 1] - uC[p - sz] * x[p - sz] - uC[p] * x[p + sz] +
           (oC[p] + ccp) * x[p];
  }
  double tO, tU, tD;
  sums27(a, x, p, sy, sz, &tO, &tU, &tD);
  /* the reference negates every product; -(a*b) is exact, so summing the
   * negated products equals negating the positive sum term by term */
  return (-tO) + (-tU) + (-tD) + (a[0][p] + ccp) * x[p];
}

void pmgo_matvec(int nx, int ny, int nz, const pmgo_op *A, const double *cc,
                 const double *x, double *y) {
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        y[IX(nx, ny, i, j, k)] = apply_at(nx, ny, A, cc, x, i, j, k);
}

/* r = f - A x in the rounding order of Vmresid7_1s / Vmresid27_1s
 * (pmgc/matvecd.cc:382-411, 426-495): f plus the positive neighbour sums,
 * minus the centre term. */
void pmgo_mresid(int nx, int ny, int nz, const pmgo_op *A, const double *cc,
                 const double *fc, const double *x, double *r) {
  const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
  const double *const *a = A->a;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t p = IX(nx, ny, i, j, k);
        const double ccp = cc ? cc[p] : 0.0;
        if (A->kind == 7) {
          const double *oC = a[0], *oE = a[1], *oN = a[2], *uC = a[3];
          r[p] = fc[p] + oN[p] * x[p + sy] + oN[p - sy] * x[p - sy] +
                 oE[p] * x[p + 1] + oE[p - 1] * x[p - 1] +
                 uC[p - sz] * x[p - sz] + uC[p] * x[p + sz] -
                 (oC[p] + ccp) * x[p];
        } else {
          double tO, tU, tD;
          sums27(a, x, p, sy, sz, &tO, &tU, &tD);
          r[p] = fc[p] + tO + tU + tD - (a[0][p] + ccp) * x[p];
        }
      }
}

/* Defect of the class: r = f - map(x) with map = matveckernel7/27 and cc = 0
 * (Subtract_Convolve_map, Convolution.h:123-146; get_map,
 * PBE_pmgc_class.h:619-698). Interior only. */
void pmgo_defect(int nx, int ny, int nz, const pmgo_op *A, const double *f,
                 const double *x, double *r) {
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t p = IX(nx, ny, i, j, k);
        r[p] = f[p] - apply_at(nx, ny, A, NULL, x, i, j, k);
      }
}

/* sqrt(sum over the interior of (f - A x)^2 / (nx*ny*nz)): the class's
 * compute_residual_2 (Convolution.h:156-185; num_values counts the shell). */
double pmgo_residual2(int nx, int ny, int nz, const pmgo_op *A,
                      const double *f, const double *x) {
  double s = 0.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t p = IX(nx, ny, i, j, k);
        const double d = f[p] - apply_at(nx, ny, A, NULL, x, i, j, k);
        s += d * d;
      }
  return sqrt(s / ((double)nx * ny * nz));
}

/* Hackbusch-Reusken damping (r . x) / (x . A x) over the interior:
 * get_ideal_lambda, MultigridDomain.h:327-359 (accumulators start at 0). */
double pmgo_ideal_lambda(int nx, int ny, int nz, const pmgo_op *A,
                         const double *x, const double *r) {
  double up = 0.0, lo = 0.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t p = IX(nx, ny, i, j, k);
        up += r[p] * x[p];
        lo += x[p] * apply_at(nx, ny, A, NULL, x, i, j, k);
      }
  return up / lo;
}

/* ------------------------------------------------------------------------
 * Grid transfers
 * ---------------------------------------------------------------------- */

/* Offsets of the nine in-plane prolongation stencils in list order
 * C N S E W NE NW SE SW, and the plane order o (dz=0), u (+1), d (-1). */
static const int kPlaneDx[9] = {0, 0, 0, 1, -1, 1, -1, 1, -1};
static const int kPlaneDy[9] = {0, 1, -1, 0, 0, 1, 1, -1, -1};
static const int kPlaneDz[3] = {0, 1, -1};

/* Slot in the 27-array list of the prolongation weight for fine offset
 * (dx,dy,dz) from the coarse point's fine image. */
static int pslot(int dx, int dy, int dz) {
  int s = 0;
  for (; s < 9; ++s)
    if (kPlaneDx[s] == dx && kPlaneDy[s] == dy)
      break;
  const int plane = dz == 0 ? 0 : (dz == 1 ? 1 : 2);
  return plane * 9 + s;
}

/* Restriction r_c = P^T r_f: Vrestrc2, pmgc/matvecd.cc:696-799. Coarse
 * interior (i,j,k) reads fine (ii,jj,kk) = 2(i,j,k)-1 and its 26 neighbours;
 * sums tmpO, tmpU, tmpD in list order. */
void pmgo_restrc2(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                  const double *xin, double *xout, const double *const *P) {
  (void)nzf;
  for (int k = 2; k <= nzc - 1; ++k)
    for (int j = 2; j <= nyc - 1; ++j)
      for (int i = 2; i <= nxc - 1; ++i) {
        const size_t pc = IX(nxc, nyc, i, j, k);
        const int ii = 2 * i - 1, jj = 2 * j - 1, kk = 2 * k - 1;
        double t[3];
        for (int pl = 0; pl < 3; ++pl) {
          double s = 0.0;
          for (int q = 0; q < 9; ++q) {
            const double w = P[pl * 9 + q][pc];
            const double v = xin[IX(nxf, nyf, ii + kPlaneDx[q],
                                    jj + kPlaneDy[q], kk + kPlaneDz[pl])];
            s = q == 0 ? w * v : s + w * v;
          }
          t[pl] = s;
        }
        xout[pc] = t[0] + t[1] + t[2];
      }
}

/* Prolongation e_f = P e_c: VinterpPMG2, pmgc/matvecd.cc:820-964. Each
 * coarse (ii,jj,kk) in [1, n_c-1]^3 writes the eight fine points
 * (2ii-1+{0,1}, 2jj-1+{0,1}, 2kk-1+{0,1}); fine index n_f is never written. */
void pmgo_interp2(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                  const double *xin, double *xout, const double *const *P) {
  (void)nzf;
#define PC(name, a, b, c) P[name][IX(nxc, nyc, a, b, c)]
#define XC(a, b, c) xin[IX(nxc, nyc, a, b, c)]
#define XF(a, b, c) xout[IX(nxf, nyf, a, b, c)]
  enum { oPC, oPN, oPS, oPE, oPW, oPNE, oPNW, oPSE, oPSW,
         uPC, uPN, uPS, uPE, uPW, uPNE, uPNW, uPSE, uPSW,
         dPC, dPN, dPS, dPE, dPW, dPNE, dPNW, dPSE, dPSW };
  for (int kk = 1; kk <= nzc - 1; ++kk)
    for (int jj = 1; jj <= nyc - 1; ++jj)
      for (int ii = 1; ii <= nxc - 1; ++ii) {
        const int i = 2 * ii - 1, j = 2 * jj - 1, k = 2 * kk - 1;
        /* a fine point on a coarse point */
        XF(i, j, k) = XC(ii, jj, kk);
        /* fine points between two coarse points along x, y, z */
        XF(i + 1, j, k) = PC(oPE, ii, jj, kk) * XC(ii, jj, kk) +
                          PC(oPW, ii + 1, jj, kk) * XC(ii + 1, jj, kk);
        XF(i, j + 1, k) = PC(oPN, ii, jj, kk) * XC(ii, jj, kk) +
                          PC(oPS, ii, jj + 1, kk) * XC(ii, jj + 1, kk);
        XF(i, j, k + 1) = PC(uPC, ii, jj, kk) * XC(ii, jj, kk) +
                          PC(dPC, ii, jj, kk + 1) * XC(ii, jj, kk + 1);
        /* fine points in the middle of four coarse points (xy, xz, yz) */
        XF(i + 1, j + 1, k) = PC(oPNE, ii, jj, kk) * XC(ii, jj, kk) +
                              PC(oPNW, ii + 1, jj, kk) * XC(ii + 1, jj, kk) +
                              PC(oPSE, ii, jj + 1, kk) * XC(ii, jj + 1, kk) +
                              PC(oPSW, ii + 1, jj + 1, kk) *
                                  XC(ii + 1, jj + 1, kk);
        XF(i + 1, j, k + 1) = PC(uPE, ii, jj, kk) * XC(ii, jj, kk) +
                              PC(uPW, ii + 1, jj, kk) * XC(ii + 1, jj, kk) +
                              PC(dPE, ii, jj, kk + 1) * XC(ii, jj, kk + 1) +
                              PC(dPW, ii + 1, jj, kk + 1) *
                                  XC(ii + 1, jj, kk + 1);
        XF(i, j + 1, k + 1) = PC(uPN, ii, jj, kk) * XC(ii, jj, kk) +
                              PC(uPS, ii, jj + 1, kk) * XC(ii, jj + 1, kk) +
                              PC(dPN, ii, jj, kk + 1) * XC(ii, jj, kk + 1) +
                              PC(dPS, ii, jj + 1, kk + 1) *
                                  XC(ii, jj + 1, kk + 1);
        /* the fine point in the middle of eight coarse points */
        XF(i + 1, j + 1, k + 1) =
            +PC(uPNE, ii, jj, kk) * XC(ii, jj, kk) +
            PC(uPNW, ii + 1, jj, kk) * XC(ii + 1, jj, kk) +
            PC(uPSE, ii, jj + 1, kk) * XC(ii, jj + 1, kk) +
            PC(uPSW, ii + 1, jj + 1, kk) * XC(ii + 1, jj + 1, kk) +
            PC(dPNE, ii, jj, kk + 1) * XC(ii, jj, kk + 1) +
            PC(dPNW, ii + 1, jj, kk + 1) * XC(ii + 1, jj, kk + 1) +
            PC(dPSE, ii, jj + 1, kk + 1) * XC(ii, jj + 1, kk + 1) +
            PC(dPSW, ii + 1, jj + 1, kk + 1) * XC(ii + 1, jj + 1, kk + 1);
      }
#undef PC
#undef XC
#undef XF
}

/* ------------------------------------------------------------------------
 * Operator-based prolongation (VbuildPb_op7 pmgc/buildPd.cc:173-555,
 * VbuildPb_op27 :579-1091), restated as one rule for every fine neighbour
 * f = c + d of a coarse point's fine image c, d in {-1,0,1}^3 \ {0}:
 *
 *   S    = axes with d_a != 0 (the directions being interpolated across),
 *   P_d  = [ sum_{e in N(d)} a(f, f+e) * w(proj(d+e)) ]
 *          / [ oC(f) - sum_{e in L(d)} a(f, f+e) ],
 *   N(d) = { e : e_a in {0, -d_a} for a in S, not all zero on S,
 *                e_b in {-1,0,1} for b not in S }     (couplings toward c),
 *   L(d) = { e != 0 : e_a = 0 for a in S }            (lumped onto the
 *                                                       diagonal),
 *   proj(v) keeps v on S and zeroes it elsewhere, w(0) = 1 and w(v) = P_v.
 *
 * Faces (|S|=1) come first, then edges (|S|=2), then corners (|S|=3), so
 * every w on the right is already known. a(.,.) is the positive coupling of
 * the fine operator (7- or 27-point); the 7-point reference formulas are the
 * same rule with only axis couplings present.
 * ---------------------------------------------------------------------- */
void pmgo_buildP_op(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                    const pmgo_op *A, double *const *P) {
  (void)nzf;
  for (int kk = 2; kk <= nzc - 1; ++kk)
    for (int jj = 2; jj <= nyc - 1; ++jj)
      for (int ii = 2; ii <= nxc - 1; ++ii) {
        const size_t pc = IX(nxc, nyc, ii, jj, kk);
        const int ci = 2 * ii - 1, cj = 2 * jj - 1, ck = 2 * kk - 1;
        double w[27];
        for (int s = 0; s < 27; ++s)
          w[s] = 0.0;
        w[pslot(0, 0, 0)] = 1.0;
        for (int order = 1; order <= 3; ++order)
          for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
              for (int dx = -1; dx <= 1; ++dx) {
                const int d[3] = {dx, dy, dz};
                if ((dx != 0) + (dy != 0) + (dz != 0) != order)
                  continue;
                const int fi = ci + dx, fj = cj + dy, fk = ck + dz;
                double num = 0.0, lump = 0.0;
                for (int ez = -1; ez <= 1; ++ez)
                  for (int ey = -1; ey <= 1; ++ey)
                    for (int ex = -1; ex <= 1; ++ex) {
                      const int e[3] = {ex, ey, ez};
                      if (!ex && !ey && !ez)
                        continue;
                      int toward = 1, on_s = 0;
                      for (int a = 0; a < 3; ++a) {
                        if (d[a] == 0)
                          continue;
                        if (e[a] != 0 && e[a] != -d[a])
                          toward = 0;
                        if (e[a] != 0)
                          on_s = 1;
                      }
                      double cpl = coupling(A, nxf, nyf, fi, fj, fk, ex, ey,
                                            ez);
                      /* Reference quirk kept for parity: for uPE of the
                       * 27-point builder the coupling to (i, j, k) — the
                       * coarse point's own fine image, offset (-1,0,-1) from
                       * f — is read as uS(i+1, j+1, k), the coupling of f
                       * to (i+1, j+1, k) (pmgc/buildPd.cc uPE numerator,
                       * first line). uPNE and uPSE inherit it through uPE. */
                      if (A->kind == 27 && dx == 1 && dy == 0 && dz == 1 &&
                          ex == -1 && ey == 0 && ez == -1)
                        cpl = coupling(A, nxf, nyf, fi, fj, fk, 0, 1, -1);
                      if (!on_s) {
                        lump += cpl;
                      } else if (toward) {
                        int v[3];
                        for (int a = 0; a < 3; ++a)
                          v[a] = d[a] ? d[a] + e[a] : 0;
                        num += cpl * w[pslot(v[0], v[1], v[2])];
                      }
                    }
                const double diag = A->a[0][IX(nxf, nyf, fi, fj, fk)];
                w[pslot(dx, dy, dz)] = num / (diag - lump);
              }
        for (int s = 0; s < 27; ++s)
          P[s][pc] = w[s];
      }
}

/* Constant weights 1, 1/2, 1/4, 1/8 by the number of nonzero offset
 * components: VbuildPb_trilin, pmgc/buildPd.cc:63-153. */
void pmgo_buildP_trilin(int nxc, int nyc, int nzc, double *const *P) {
  for (int kk = 2; kk <= nzc - 1; ++kk)
    for (int jj = 2; jj <= nyc - 1; ++jj)
      for (int ii = 2; ii <= nxc - 1; ++ii) {
        const size_t pc = IX(nxc, nyc, ii, jj, kk);
        for (int pl = 0; pl < 3; ++pl)
          for (int q = 0; q < 9; ++q) {
            const int nnz =
                (kPlaneDx[q] != 0) + (kPlaneDy[q] != 0) + (kPlaneDz[pl] != 0);
            P[pl * 9 + q][pc] = 1.0 / (double)(1 << nnz);
          }
      }
}

/* Box-method (finite volume) fine operator of the APBS driver from the
 * harmonic coefficient maps: VbuildA_fv, pmgc/buildAd.cc:63-212. Mesh
 * coordinates xf/yf/zf are 1-based per axis; the boundary maps are
 * gx(j,k,side) on ny x nz x 2, gy(i,k,side) on nx x nz x 2, gz(i,j,side) on
 * nx x ny x 2 (side 1: low face, 2: high face). Every interior point gets
 * the face weights (product of the two transverse widths over four times
 * the normal width), the control volume (three widths over eight), the
 * scaled source and kappa term, the diagonal as the six weighted coupling
 * sum, the upper couplings zeroed on the high faces, and the Dirichlet
 * values of boundary neighbours moved into fc in the order E, N, U, W, S, D.
 * The expressions keep the reference's operand order. All interior planes
 * are built; the reference's launch takes its k extent from ny
 * (buildAd.cc:116), which is the same for ny == nz. ipc[9..11] get ipkey, 7
 * and 1, *numdia 4 (buildAd.cc:102-107). */
void pmgo_buildA_fv(int nx, int ny, int nz, int ipkey, int *numdia, int *ipc,
                    double *oC, double *cc, double *fc, double *oE,
                    double *oN, double *uC, const double *xf,
                    const double *yf, const double *zf, const double *gxcf,
                    const double *gycf, const double *gzcf,
                    const double *a1cf, const double *a2cf,
                    const double *a3cf, const double *ccf,
                    const double *fcf) {
  if (ipc) {
    ipc[9] = ipkey;
    ipc[10] = 7;
    ipc[11] = 1;
  }
  if (numdia)
    *numdia = 4;
  const double diag = 1.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t p = IX(nx, ny, i, j, k);
        const size_t pw = IX(nx, ny, i - 1, j, k);
        const size_t ps = IX(nx, ny, i, j - 1, k);
        const size_t pd = IX(nx, ny, i, j, k - 1);
        const double hzm1 = zf[k - 1] - zf[k - 2], hz = zf[k] - zf[k - 1];
        const double hym1 = yf[j - 1] - yf[j - 2], hy = yf[j] - yf[j - 1];
        const double hxm1 = xf[i - 1] - xf[i - 2], hx = xf[i] - xf[i - 1];
        const double wE = diag * (hym1 + hy) * (hzm1 + hz) / (4.0 * hx);
        const double wW = diag * (hym1 + hy) * (hzm1 + hz) / (4.0 * hxm1);
        const double wN = diag * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hy);
        const double wS = diag * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hym1);
        const double wU = diag * (hxm1 + hx) * (hym1 + hy) / (4.0 * hz);
        const double wD = diag * (hxm1 + hx) * (hym1 + hy) / (4.0 * hzm1);
        const double vol =
            diag * (hxm1 + hx) * (hym1 + hy) * (hzm1 + hz) / 8.0;
        double f = vol * fcf[p];
        cc[p] = vol * ccf[p];
        oC[p] = wE * a1cf[p] + wW * a1cf[pw] + wN * a2cf[p] + wS * a2cf[ps] +
                wU * a3cf[p] + wD * a3cf[pd];
        const int e = i != nx - 1, n = j != ny - 1, u = k != nz - 1;
        const int w = i != 2, s = j != 2, d = k != 2;
        oE[p] = e * wE * a1cf[p];
        f += (1 - e) * wE * a1cf[p] *
             gxcf[(size_t)ny * nz + (size_t)(k - 1) * ny + (j - 1)];
        oN[p] = n * wN * a2cf[p];
        f += (1 - n) * wN * a2cf[p] *
             gycf[(size_t)nx * nz + (size_t)(k - 1) * nx + (i - 1)];
        uC[p] = u * wU * a3cf[p];
        f += (1 - u) * wU * a3cf[p] *
             gzcf[(size_t)nx * ny + (size_t)(j - 1) * nx + (i - 1)];
        f += (1 - w) * wW * a1cf[pw] * gxcf[(size_t)(k - 1) * ny + (j - 1)];
        f += (1 - s) * wS * a2cf[ps] * gycf[(size_t)(k - 1) * nx + (i - 1)];
        f += (1 - d) * wD * a3cf[pd] * gzcf[(size_t)(j - 1) * nx + (i - 1)];
        fc[p] = f;
      }
}

/* ------------------------------------------------------------------------
 * Galerkin coarse operator A_c = P^T A_f P (VbuildG_7, pmgc/buildGd.cc:
 * 438-1361; VbuildG_27, :1364-3274), computed from its definition: for a
 * coarse point C and an upper direction D (or D = 0),
 *
 *   A_c(C, C+D) = sum_{d, e} P_d(C) * A_f(c+d, c+d+e) * P_{d+e-2D}(C+D)
 *
 * over d in {-1,0,1}^3 (fine support of C) and fine couplings e with
 * d+e-2D in {-1,0,1}^3 (the fine point lies in the support of C+D).
 * A_f(f,f) = oC(f), A_f(f,g) = -a(f,g). The stored coarse entries are
 * XoC = A_c(C,C) and X<dir> = -A_c(C, C+dir), on the coarse interior.
 * ---------------------------------------------------------------------- */
static const int kUpper[14][3] = {
    {0, 0, 0},  {1, 0, 0},  {0, 1, 0},   {0, 0, 1},  {1, 1, 0},
    {-1, 1, 0}, {1, 0, 1},  {-1, 0, 1},  {0, 1, 1},  {0, -1, 1},
    {1, 1, 1},  {-1, 1, 1}, {1, -1, 1},  {-1, -1, 1}};

void pmgo_buildG(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                 const double *const *P, const pmgo_op *A,
                 double *const *out) {
  (void)nzf;
  for (int kk = 2; kk <= nzc - 1; ++kk)
    for (int jj = 2; jj <= nyc - 1; ++jj)
      for (int ii = 2; ii <= nxc - 1; ++ii) {
        const size_t pc = IX(nxc, nyc, ii, jj, kk);
        const int ci = 2 * ii - 1, cj = 2 * jj - 1, ck = 2 * kk - 1;
        for (int s = 0; s < 14; ++s) {
          const int *D = kUpper[s];
          const size_t pn = IX(nxc, nyc, ii + D[0], jj + D[1], kk + D[2]);
          double acc = 0.0;
          for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
              for (int dx = -1; dx <= 1; ++dx) {
                const double pw = P[pslot(dx, dy, dz)][pc];
                const int fi = ci + dx, fj = cj + dy, fk = ck + dz;
                for (int ez = -1; ez <= 1; ++ez)
                  for (int ey = -1; ey <= 1; ++ey)
                    for (int ex = -1; ex <= 1; ++ex) {
                      const int tx = dx + ex - 2 * D[0];
                      const int ty = dy + ey - 2 * D[1];
                      const int tz = dz + ez - 2 * D[2];
                      if (tx < -1 || tx > 1 || ty < -1 || ty > 1 || tz < -1 ||
                          tz > 1)
                        continue;
                      double af;
                      if (!ex && !ey && !ez)
                        af = A->a[0][IX(nxf, nyf, fi, fj, fk)];
                      else
                        af = -coupling(A, nxf, nyf, fi, fj, fk, ex, ey, ez);
                      if (af == 0.0)
                        continue;
                      acc += pw * af * P[pslot(tx, ty, tz)][pn];
                    }
              }
          out[s][pc] = s == 0 ? acc : -acc;
        }
      }
}

/* ------------------------------------------------------------------------
 * Coarsest-level CG of the class (CG_solver, CG_Solver.h:45-242, run by
 * solve_by_cg<1>, PBE_pmgc_class.h:856-860): warm start from x, interior
 * dot products, absolute stop sqrt(r.r) <= thresh, the first test taking
 * the square root twice (CG_Solver.h:135,140), return when the first p.Ap
 * is zero. An iteration cap (absent in the reference, which would loop
 * forever on stagnation) bounds the loop; returns the iterations run.
 * ---------------------------------------------------------------------- */
/* Interior dot product (the documented Vxdot, pmgc/mikpckd.cc:192-222,
 * whose reference body sums x.x instead), serial order. */
static double idot(int nx, int ny, int nz, const double *a, const double *b) {
  double s = 0.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t q = IX(nx, ny, i, j, k);
        s += a[q] * b[q];
      }
  return s;
}

/* Hestenes-Stiefel CG of the APBS layer: Vcghs, pmgc/cgd.cc:60-125, with
 * the dot products and axpys it documents (x.y; interior updates, where the
 * reference's Vxaxpy starts its range at index 0, mikpckd.cc:115-129).
 * r = f - A x (Vmresid order), denom = ||r||; loop: stop when
 * ||r||/denom <= errtol or iters >= itmax; p = r on the first step, else
 * p += (1/beta) r then p *= beta (beta = rho_k / rho_{k-1}); ap = A p
 * (Vmatvec order, cc included); alpha = rho_k / p.ap; x += alpha p;
 * r += (-alpha) ap. p, ap, r are caller work arrays (p is cleared first,
 * so that its shell reads as zero); returns the count. */
int pmgo_cghs(int nx, int ny, int nz, const pmgo_op *A, const double *cc,
              const double *fc, double *x, double *p, double *ap, double *r,
              int itmax, double errtol, int iresid) {
  int iters = 0;
  if (iters >= itmax && iresid == 0)
    return 0;
  /* p's shell must read as zero in A p (the reference leaves whatever the
   * work array held there) */
  memset(p, 0, sizeof(double) * (size_t)nx * ny * nz);
  pmgo_mresid(nx, ny, nz, A, cc, fc, x, r);
  const double denom = sqrt(idot(nx, ny, nz, r, r));
  if (denom == 0.0 || iters >= itmax)
    return 0;
  double rhok1 = 0.0;
  for (;;) {
    const double rhok2 = idot(nx, ny, nz, r, r);
    if (sqrt(rhok2) / denom <= errtol || iters >= itmax)
      break;
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          const size_t q = IX(nx, ny, i, j, k);
          if (iters == 0) {
            p[q] = r[q];
          } else {
            const double beta = rhok2 / rhok1, inv = 1.0 / beta;
            p[q] = (p[q] + inv * r[q]) * beta;
          }
        }
    pmgo_matvec(nx, ny, nz, A, cc, p, ap);
    const double alpha = rhok2 / idot(nx, ny, nz, p, ap);
    rhok1 = rhok2;
    const double malpha = -alpha;
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          const size_t q = IX(nx, ny, i, j, k);
          x[q] += alpha * p[q];
          r[q] = r[q] + malpha * ap[q];
        }
    ++iters;
  }
  return iters;
}

/* ------------------------------------------------------------------------
 * Banded direct solve of a coarsest level (the APBS mgsolv 1 path):
 * Vbuildband (pmgc/buildBd.cc:63-303) stores the interior operator in
 * LINPACK upper band storage, abd(kk, jj) = A(ii, jj) with kk = ii - jj +
 * m + 1 (1-based, lda = m + 1 rows per column), unknowns ordered x fastest;
 * Vdpbfa / Vdpbsl (pmgc/mlinpckd.cc:168-240) factor it as R^T R and solve.
 * The dot products keep LINPACK's unrolled order (Vddot, :113-165).
 * ---------------------------------------------------------------------- */
static double ddot5(int n, const double *x, const double *y) {
  double t = 0.0;
  if (n <= 0)
    return 0.0;
  const int r = n % 5;
  for (int i = 0; i < r; ++i)
    t += x[i] * y[i];
  if (n < 5)
    return t;
  for (int i = r; i < n; i += 5)
    t += x[i] * y[i] + x[i + 1] * y[i + 1] + x[i + 2] * y[i + 2] +
         x[i + 3] * y[i + 3] + x[i + 4] * y[i + 4];
  return t;
}

/* Band storage of the interior operator (the caller zeroes abd, lda*n);
 * cc is not part of it, as in the reference (Vbuildband takes ac only).
 * Only couplings with interior neighbours are stored. The reference also
 * writes the offsets of shell neighbours, which wrap to the previous row or
 * plane (a shell coefficient, zero for operators built on the interior);
 * on grids with one interior point along x (3 points) some of those
 * offsets alias the diagonal or pass the end of the column, i.e. of the
 * array (buildBd.cc:150-247). For 27-point operators the reference reads
 * the ten diagonal couplings at the point below or south of p, which is not
 * the operator its matvec applies; this stores the coupling with each
 * earlier neighbour q where the matvec reads it, at q. */
void pmgo_buildband(int nx, int ny, int nz, const pmgo_op *A, int *n_out,
                    int *m_out, int *lda_out, double *abd) {
  const int mx = nx - 2, my = ny - 2;
  const int n = mx * my * (nz - 2);
  const int m = A->kind == 7 ? mx * my : mx * my + mx + 1, lda = m + 1;
  const double *const *a = A->a;
  *n_out = n;
  *m_out = m;
  *lda_out = lda;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const int jj = (k - 2) * mx * my + (j - 2) * mx + (i - 2) + 1;
        double *col = abd + (size_t)(jj - 1) * lda;
        /* row offset ii - jj, coefficient array, its point (di, dj, dk) */
/* only couplings with interior neighbours (whose offset lies in [-m, -1]) */
#define BAND(off, arr, di, dj, dk, sign)                                       \
  do {                                                                         \
    if (i + (di) >= 2 && i + (di) <= nx - 1 && j + (dj) >= 2 &&              \
        j + (dj) <= ny - 1 && k + (dk) >= 2 && k + (dk) <= nz - 1)             \
      col[(off) + m] =                                                         \
          sign a[arr][IX(nx, ny, i + (di), j + (dj), k + (dk))];               \
  } while (0)
        BAND(0, 0, 0, 0, 0, +);
        BAND(-1, 1, -1, 0, 0, -);
        BAND(-mx, 2, 0, -1, 0, -);
        if (A->kind == 7) {
          BAND(-mx * my, 3, 0, 0, -1, -);
          continue;
        }
        /* the coupling with the earlier neighbour q = p + d is stored at q
         * as the diagonal pointing back to p (the matvec's convention) */
        BAND(-mx + 1, 5, 1, -1, 0, -);      /* oNW(i+1, j-1, k)   */
        BAND(-mx - 1, 4, -1, -1, 0, -);     /* oNE(i-1, j-1, k)   */
        BAND(-mx * my, 3, 0, 0, -1, -);     /* uC(i, j, k-1)      */
        BAND(-mx * my + 1, 7, 1, 0, -1, -); /* uW(i+1, j, k-1)    */
        BAND(-mx * my - 1, 6, -1, 0, -1, -); /* uE(i-1, j, k-1)   */
        BAND(-mx * my + mx, 9, 0, 1, -1, -); /* uS(i, j+1, k-1)   */
        BAND(-mx * my - mx, 8, 0, -1, -1, -); /* uN(i, j-1, k-1)  */
        BAND(-mx * my + mx + 1, 13, 1, 1, -1, -);  /* uSW(i+1, j+1)  */
        BAND(-mx * my + mx - 1, 12, -1, 1, -1, -); /* uSE(i-1, j+1)  */
        BAND(-mx * my - mx + 1, 11, 1, -1, -1, -); /* uNW(i+1, j-1)  */
        BAND(-mx * my - mx - 1, 10, -1, -1, -1, -); /* uNE(i-1, j-1) */
#undef BAND
      }
}

/* R^T R factorisation in place; returns info (0, or the column whose pivot
 * was not positive). */
int pmgo_dpbfa(double *abd, int lda, int n, int m) {
#define ABD(r, c) abd[(size_t)((c) - 1) * lda + ((r) - 1)]
  for (int j = 1; j <= n; ++j) {
    double s = 0.0;
    int ik = m + 1;
    int jk = j - m > 1 ? j - m : 1;
    const int mu = m + 2 - j > 1 ? m + 2 - j : 1;
    for (int k = mu; k <= m; ++k) {
      double t = ABD(k, j) - ddot5(k - mu, &ABD(ik, jk), &ABD(mu, j));
      t /= ABD(m + 1, jk);
      ABD(k, j) = t;
      s += t * t;
      --ik;
      ++jk;
    }
    s = ABD(m + 1, j) - s;
    if (s <= 0.0)
      return j;
    ABD(m + 1, j) = sqrt(s);
  }
  return 0;
}

/* Solves R^T R x = b in place (b: n values). */
void pmgo_dpbsl(const double *abd, int lda, int n, int m, double *b) {
  for (int k = 1; k <= n; ++k) {
    const int lm = k - 1 < m ? k - 1 : m;
    const int la = m + 1 - lm, lb = k - lm;
    const double t = ddot5(lm, &ABD(la, k), &b[lb - 1]);
    b[k - 1] = (b[k - 1] - t) / ABD(m + 1, k);
  }
  for (int kb = 1; kb <= n; ++kb) {
    const int k = n + 1 - kb;
    const int lm = k - 1 < m ? k - 1 : m;
    const int la = m + 1 - lm, lb = k - lm;
    b[k - 1] /= ABD(m + 1, k);
    const double t = -b[k - 1];
    if (lm > 0 && t != 0.0)
      for (int i = 0; i < lm; ++i)
        b[lb - 1 + i] += t * ABD(la + i, k);
  }
#undef ABD
}

/* ------------------------------------------------------------------------
 * APBS iparm/rparm driver, linear case: Vmgdriv / Vmgdriv2
 * (pmgc/mgdrvd.cc:60-491) with Vbuildops (pmgc/mgsubd.cc:63-265, Galerkin
 * coarsening) and the V-cycle Vmvcs (pmgc/mgcsd.cc:61-531), restated with
 * the semantics the code documents where the reference's own helpers are
 * wrong (x.y dot products, interior axpys, all six boundary faces).
 * Levels are numbered as APBS does: 1 finest .. nlev coarsest.
 * ---------------------------------------------------------------------- */
typedef struct {
  int nx, ny, nz, kind;
  double *a[14], *cc, *fc, *x, *w0, *P[27];
  double *m[11]; /* coarse coefficient maps (mgcoar 0), BOX_IN order */
} alevel;

/* Injection to the next coarser grid (Vbuildcopy0, mgsubd.cc:578-697):
 * out(a, b, c) = in(2a-1, 2b-1, 2c-1); keep_c: c is a layer index. */
static void inject(const double *in, double *out, int na, int nb, int nc,
                   int naf, int nbf, int keep_c) {
  for (int c = 0; c < nc; ++c)
    for (int b = 0; b < nb; ++b)
      for (int a = 0; a < na; ++a)
        out[((size_t)c * nb + b) * na + a] =
            in[((size_t)(keep_c ? c : 2 * c) * nbf + 2 * b) * naf + 2 * a];
}

static double inorm1(int nx, int ny, int nz, const double *a) {
  double s = 0.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        s += fabs(a[IX(nx, ny, i, j, k)]);
  return s;
}

static pmgo_op aop(const alevel *L) {
  pmgo_op o;
  o.kind = L->kind;
  for (int s = 0; s < 14; ++s)
    o.a[s] = L->a[s];
  return o;
}

/* Vsmooth (smoothd.cc:58-87): meth 1 red-black GS (nu sweeps, then the
 * residual into r when iresid), meth 4 the CG Vcghs (nu iterations,
 * errtol 0). */
static void asmooth(const alevel *L, const double *f, double *x, int nu,
                    int iadjoint, int iresid, int meth, double *r, double *w2,
                    double *w3) {
  const pmgo_op o = aop(L);
  if (meth == 4) {
    pmgo_cghs(L->nx, L->ny, L->nz, &o, L->cc, f, x, w2, w3, r, nu, 0.0,
              iresid);
    return;
  }
  if (L->kind == 7)
    pmgo_gsrb7x(L->nx, L->ny, L->nz, L->a[0], L->cc, f, L->a[1], L->a[2],
                L->a[3], x, nu, iadjoint, 0);
  else
    pmgo_gsrb27x(L->nx, L->ny, L->nz, (const double *const *)L->a, L->cc, f,
                 x, nu, iadjoint, 0);
  if (iresid)
    pmgo_mresid(L->nx, L->ny, L->nz, &o, L->cc, f, x, r);
}

/* Six faces of x from the boundary maps (VfboundPMG, mikpckd.cc:266-312,
 * ibound != 0), or zero (VfboundPMG00, :235-264) when gx is NULL. */
static void afbound(int nx, int ny, int nz, double *x, const double *gx,
                    const double *gy, const double *gz) {
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      x[IX(nx, ny, 1, j, k)] = gx ? gx[(size_t)(k - 1) * ny + (j - 1)] : 0.0;
      x[IX(nx, ny, nx, j, k)] =
          gx ? gx[(size_t)ny * nz + (size_t)(k - 1) * ny + (j - 1)] : 0.0;
    }
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) {
      x[IX(nx, ny, i, 1, k)] = gy ? gy[(size_t)(k - 1) * nx + (i - 1)] : 0.0;
      x[IX(nx, ny, i, ny, k)] =
          gy ? gy[(size_t)nx * nz + (size_t)(k - 1) * nx + (i - 1)] : 0.0;
    }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      x[IX(nx, ny, i, j, 1)] = gz ? gz[(size_t)(j - 1) * nx + (i - 1)] : 0.0;
      x[IX(nx, ny, i, j, nz)] =
          gz ? gz[(size_t)nx * ny + (size_t)(j - 1) * nx + (i - 1)] : 0.0;
    }
}

/* The coarsest level's solve (mgcsd.cc:362-405): mgsolv 0, 100 CG
 * iterations from zero with errtol epsiln = 0; mgsolv 1, the factored band
 * applied to the interior of f, boundary zero. */
static void acoarse(alevel *C, const double *f, int mgsolv,
                    const double *band, int bn, int bm, int blda, double *w1,
                    double *w2, double *w3) {
  const size_t n = (size_t)C->nx * C->ny * C->nz;
  if (mgsolv == 1) {
    size_t q = 0;
    for (int k = 2; k <= C->nz - 1; ++k)
      for (int j = 2; j <= C->ny - 1; ++j)
        for (int i = 2; i <= C->nx - 1; ++i)
          w1[q++] = f[IX(C->nx, C->ny, i, j, k)];
    pmgo_dpbsl(band, blda, bn, bm, w1);
    q = 0;
    for (int k = 2; k <= C->nz - 1; ++k)
      for (int j = 2; j <= C->ny - 1; ++j)
        for (int i = 2; i <= C->nx - 1; ++i)
          C->x[IX(C->nx, C->ny, i, j, k)] = w1[q++];
    afbound(C->nx, C->ny, C->nz, C->x, NULL, NULL, NULL);
    return;
  }
  const pmgo_op o = aop(C);
  memset(C->x, 0, sizeof(double) * n);
  pmgo_cghs(C->nx, C->ny, C->nz, &o, C->cc, f, C->x, w1, w2, w3, 100, 0.0, 0);
}

/* The stop test's numerator after a cycle (mgcsd.cc:467-519): istop 0/1
 * the L1 norm of f - A u, 2 the L1 norm of tru - u (then tru = u), 3 the
 * L2 norm of tru - u. */
static double astop(const alevel *L, int istop, const double *u, double *tru,
                    double *w1) {
  const int nx = L->nx, ny = L->ny, nz = L->nz;
  if (istop == 0 || istop == 1) {
    const pmgo_op o = aop(L);
    pmgo_mresid(nx, ny, nz, &o, L->cc, L->fc, u, w1);
    return inorm1(nx, ny, nz, w1);
  }
  double s = 0.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t q = IX(nx, ny, i, j, k);
        const double d = tru[q] - u[q];
        s += istop == 2 ? fabs(d) : d * d;
        if (istop == 2)
          tru[q] = u[q];
      }
  return istop == 2 ? s : sqrt(s);
}

int pmgo_mgdriv(const int *iparm, const double *rparm, double *u,
                const double *xf, const double *yf, const double *zf,
                const double *gxcf, const double *gycf, const double *gzcf,
                const double *a1cf, const double *a2cf, const double *a3cf,
                const double *ccf, const double *fcf, double *tcf,
                int *iters_out, int *ierror_out, double *rsnrm_out) {
  const int nx = iparm[2], ny = iparm[3], nz = iparm[4], nlev = iparm[5];
  const int nu1 = iparm[6], nu2 = iparm[7], itmax = iparm[9];
  const int istop = iparm[10], ipkey = iparm[13], mgprol = iparm[16];
  const int mgsmoo = iparm[19], mgsolv = iparm[20], mgcoar = iparm[17];
  const double errtol = rparm[0];
  if (nlev < 1 || nlev > 12)
    return -1;
  alevel lv[13];
  memset(lv, 0, sizeof(lv));
  int ok = 1;
  for (int L = 1; L <= nlev; ++L) {
    alevel *v = &lv[L];
    v->nx = L == 1 ? nx : (lv[L - 1].nx - 1) / 2 + 1;
    v->ny = L == 1 ? ny : (lv[L - 1].ny - 1) / 2 + 1;
    v->nz = L == 1 ? nz : (lv[L - 1].nz - 1) / 2 + 1;
    v->kind = L == 1 || mgcoar == 0 ? 7 : 27;
    const size_t n = (size_t)v->nx * v->ny * v->nz;
    for (int s = 0; s < (v->kind == 7 ? 4 : 14); ++s)
      ok &= (v->a[s] = calloc(n, sizeof(double))) != NULL;
    ok &= (v->cc = calloc(n, sizeof(double))) != NULL;
    ok &= (v->fc = calloc(n, sizeof(double))) != NULL;
    ok &= (v->w0 = calloc(n, sizeof(double))) != NULL;
    v->x = L == 1 ? u : calloc(n, sizeof(double));
    ok &= v->x != NULL;
    if (L > 1)
      for (int s = 0; s < 27; ++s)
        ok &= (v->P[s] = calloc(n, sizeof(double))) != NULL;
    if (L > 1 && mgcoar == 0) {
      const size_t sz[11] = {(size_t)v->nx, (size_t)v->ny, (size_t)v->nz,
                             2 * (size_t)v->ny * v->nz,
                             2 * (size_t)v->nx * v->nz,
                             2 * (size_t)v->nx * v->ny, n, n, n, n, n};
      for (int q = 0; q < 11; ++q)
        ok &= (v->m[q] = calloc(sz[q], sizeof(double))) != NULL;
    }
  }
  const size_t nf = (size_t)nx * ny * nz;
  double *w1 = calloc(nf, sizeof(double)), *w2 = calloc(nf, sizeof(double));
  double *w3 = calloc(nf, sizeof(double));
  double *tru = NULL, *band = NULL;
  int bn = 0, bm = 0, blda = 0;
  ok &= w1 && w2 && w3;
  int iters = 0;
  double rsnrm = 0.0;
  if (!ok)
    goto done;
  /* Vbuildops: fine operator from the maps, then P and Galerkin per level;
   * the coarse cc and fc are the restricted fine ones (Vbuildgaler0,
   * mgsubd.cc:349-373). */
  pmgo_buildA_fv(nx, ny, nz, ipkey, NULL, NULL, lv[1].a[0], lv[1].cc,
                 lv[1].fc, lv[1].a[1], lv[1].a[2], lv[1].a[3], xf, yf, zf,
                 gxcf, gycf, gzcf, a1cf, a2cf, a3cf, ccf, fcf);
  for (int L = 2; L <= nlev; ++L) {
    const alevel *F = &lv[L - 1];
    alevel *C = &lv[L];
    const pmgo_op fo = aop(F);
    if (mgprol == 0)
      pmgo_buildP_trilin(C->nx, C->ny, C->nz, C->P);
    else
      pmgo_buildP_op(F->nx, F->ny, F->nz, C->nx, C->ny, C->nz, &fo, C->P);
    if (mgcoar == 0) { /* maps injected, box method on this grid */
      const double *fm[11] = {xf,   yf,   zf,   gxcf, gycf, gzcf,
                              a1cf, a2cf, a3cf, ccf,  fcf};
      const double *const *src = L == 2 ? fm : (const double *const *)F->m;
      inject(src[0], C->m[0], C->nx, 1, 1, F->nx, 1, 1);
      inject(src[1], C->m[1], C->ny, 1, 1, F->ny, 1, 1);
      inject(src[2], C->m[2], C->nz, 1, 1, F->nz, 1, 1);
      inject(src[3], C->m[3], C->ny, C->nz, 2, F->ny, F->nz, 1);
      inject(src[4], C->m[4], C->nx, C->nz, 2, F->nx, F->nz, 1);
      inject(src[5], C->m[5], C->nx, C->ny, 2, F->nx, F->ny, 1);
      for (int q = 6; q < 11; ++q)
        inject(src[q], C->m[q], C->nx, C->ny, C->nz, F->nx, F->ny, 0);
      pmgo_buildA_fv(C->nx, C->ny, C->nz, ipkey, NULL, NULL, C->a[0], C->cc,
                     C->fc, C->a[1], C->a[2], C->a[3], C->m[0], C->m[1],
                     C->m[2], C->m[3], C->m[4], C->m[5], C->m[6], C->m[7],
                     C->m[8], C->m[9], C->m[10]);
      continue;
    }
    pmgo_buildG(F->nx, F->ny, F->nz, C->nx, C->ny, C->nz,
                (const double *const *)C->P, &fo, C->a);
    pmgo_restrc2(F->nx, F->ny, F->nz, C->nx, C->ny, C->nz, F->cc, C->cc,
                 (const double *const *)C->P);
    pmgo_restrc2(F->nx, F->ny, F->nz, C->nx, C->ny, C->nz, F->fc, C->fc,
                 (const double *const *)C->P);
  }
  if (mgsolv == 1) { /* Vbuildband on the coarsest level, factored */
    const alevel *C = &lv[nlev];
    const pmgo_op o = aop(C);
    const int mx = C->nx - 2, my = C->ny - 2;
    const int m = C->kind == 7 ? mx * my : mx * my + mx + 1;
    band = calloc((size_t)(m + 1) * mx * my * (C->nz - 2), sizeof(double));
    if (!band) {
      ok = 0;
      goto done;
    }
    pmgo_buildband(C->nx, C->ny, C->nz, &o, &bn, &bm, &blda, band);
    if (pmgo_dpbfa(band, blda, bn, bm) != 0) {
      ok = -1;
      goto done;
    }
  }
  /* u starts from zero (mgdrvd.cc:419) */
  memset(u, 0, sizeof(double) * nf);
  afbound(nx, ny, nz, u, NULL, NULL, NULL);
  /* Vmvcs: the stop test's denominator */
  double rsden = 1.0;
  if (istop == 1)
    rsden = inorm1(nx, ny, nz, lv[1].fc);
  else if (istop == 2)
    rsden = sqrt((double)nx * ny * nz);
  else if (istop == 3)
    rsden = sqrt(idot(nx, ny, nz, tcf, tcf));
  if (rsden == 0.0)
    rsden = 1.0;
  if (istop == 2 || istop == 3) {
    tru = tcf;
  }
  if (nlev == 1) {
    /* direct solve on the only level: 100 CG iterations (mgsolv 0) */
    acoarse(&lv[1], lv[1].fc, mgsolv, band, bn, bm, blda, w1, w2, w3);
    iters = 1;
    rsnrm = astop(&lv[1], istop, u, tru, w1);
  } else {
    do {
      asmooth(&lv[1], lv[1].fc, lv[1].x, nu1, 0, 1, mgsmoo, w1, w2, w3);
      for (int L = 2; L <= nlev; ++L) {
        const alevel *F = &lv[L - 1];
        alevel *C = &lv[L];
        pmgo_restrc2(F->nx, F->ny, F->nz, C->nx, C->ny, C->nz, w1, C->w0,
                     (const double *const *)C->P);
        if (L != nlev) {
          memset(C->x, 0, sizeof(double) * C->nx * C->ny * C->nz);
          asmooth(C, C->w0, C->x, nu1, 0, 1, mgsmoo, w1, w2, w3);
        }
      }
      acoarse(&lv[nlev], lv[nlev].w0, mgsolv, band, bn, bm, blda, w1, w2,
              w3);
      for (int L = nlev - 1; L >= 1; --L) {
        alevel *F = &lv[L];
        const alevel *C = &lv[L + 1];
        const pmgo_op co = aop(C);
        pmgo_matvec(C->nx, C->ny, C->nz, &co, C->cc, C->x, w2);
        const double xdamp = idot(C->nx, C->ny, C->nz, C->x, C->w0) /
                             idot(C->nx, C->ny, C->nz, C->x, w2);
        memset(w1, 0, sizeof(double) * nf);
        pmgo_interp2(C->nx, C->ny, C->nz, F->nx, F->ny, F->nz, C->x, w1,
                     (const double *const *)C->P);
        for (int k = 2; k <= F->nz - 1; ++k)
          for (int j = 2; j <= F->ny - 1; ++j)
            for (int i = 2; i <= F->nx - 1; ++i) {
              const size_t q = IX(F->nx, F->ny, i, j, k);
              F->x[q] = F->x[q] + xdamp * w1[q];
            }
        asmooth(F, L == 1 ? F->fc : F->w0, F->x, nu2, 1, 0, mgsmoo, w1, w2,
                w3);
      }
      ++iters;
      rsnrm = astop(&lv[1], istop, u, tru, w1);
    } while (iters < itmax && rsnrm / rsden > errtol);
  }
  afbound(nx, ny, nz, u, gxcf, gycf, gzcf);
done:
  for (int L = 1; L <= nlev; ++L) {
    alevel *v = &lv[L];
    for (int s = 0; s < 14; ++s)
      free(v->a[s]);
    free(v->cc);
    free(v->fc);
    free(v->w0);
    if (L > 1) {
      free(v->x);
      for (int s = 0; s < 27; ++s)
        free(v->P[s]);
      for (int q = 0; q < 11; ++q)
        free(v->m[q]);
    }
  }
  free(w1);
  free(w2);
  free(w3);
  free(band);
  if (ok == -1)
    return -3;
  if (!ok)
    return -2;
  if (iters_out)
    *iters_out = iters;
  if (ierror_out)
    *ierror_out = iters < itmax ? 0 : 1;
  if (rsnrm_out)
    *rsnrm_out = rsnrm / rsden;
  return 0;
}

int pmgo_cg(int nx, int ny, int nz, const pmgo_op *A, const double *rhs,
            double *x, double thresh) {
  const size_t n = (size_t)nx * ny * nz;
  double *r = calloc(n, sizeof(double));
  double *p = calloc(n, sizeof(double));
  double *ap = calloc(n, sizeof(double));
  int it = 0;
  if (!r || !p || !ap)
    goto done;
  pmgo_defect(nx, ny, nz, A, rhs, x, r);
  memcpy(p, r, n * sizeof(double));
  double rs = 0.0, pap = 0.0;
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        const size_t q = IX(nx, ny, i, j, k);
        rs += r[q] * r[q];
      }
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        pap += apply_at(nx, ny, A, NULL, p, i, j, k) * p[IX(nx, ny, i, j, k)];
  if (pap == 0.0)
    goto done;
  double alpha = rs / pap;
  double res = sqrt(sqrt(rs));
  while (res > thresh && it < 100000) {
    ++it;
    pmgo_matvec(nx, ny, nz, A, NULL, p, ap);
    double rsn = 0.0;
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          const size_t q = IX(nx, ny, i, j, k);
          x[q] += alpha * p[q];
          r[q] -= alpha * ap[q];
        }
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          const size_t q = IX(nx, ny, i, j, k);
          rsn += r[q] * r[q];
        }
    const double beta = rs == 0.0 ? 0.0 : rsn / rs;
    rs = rsn;
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          const size_t q = IX(nx, ny, i, j, k);
          p[q] = r[q] + beta * p[q];
        }
    pap = 0.0;
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i)
          pap +=
              apply_at(nx, ny, A, NULL, p, i, j, k) * p[IX(nx, ny, i, j, k)];
    alpha = pap == 0.0 ? 0.0 : rs / pap;
    res = sqrt(rs);
  }
done:
  free(r);
  free(p);
  free(ap);
  return it;
}

/* ------------------------------------------------------------------------
 * Hierarchy and V-cycle of the class (buildmultilevelops,
 * PBE_pmgc_class.h:351-617; v_cycle :1070-1114)
 * ---------------------------------------------------------------------- */
typedef struct {
  int n;
  double *op[14]; /* level operator; finest uses 4 (7-point) */
  double *P[27];  /* prolongation from this level to the next finer one */
  double *x, *f, *r, *zero;
  pmgo_op A;
} olevel;

typedef struct {
  int nlev;
  olevel lv[16]; /* 1-based: lv[1] coarsest .. lv[nlev] finest */
} ohier;

static void hier_free(ohier *h) {
  for (int L = 1; L <= h->nlev; ++L) {
    olevel *v = &h->lv[L];
    for (int s = 0; s < 14; ++s)
      free(v->op[s]);
    for (int s = 0; s < 27; ++s)
      free(v->P[s]);
    free(v->x);
    free(v->f);
    free(v->r);
    free(v->zero);
  }
}

static int hier_build(ohier *h, int base, int nlev, const double *oC,
                      const double *oE, const double *oN, const double *uC,
                      int trilinear) {
  memset(h, 0, sizeof(*h));
  h->nlev = nlev;
  if (nlev < 2 || nlev > 15)
    return -1;
  for (int L = 1; L <= nlev; ++L) {
    olevel *v = &h->lv[L];
    v->n = base * (1 << L) + 1;
    const size_t n3 = (size_t)v->n * v->n * v->n;
    const int nops = L == nlev ? 4 : 14;
    for (int s = 0; s < nops; ++s)
      if (!(v->op[s] = calloc(n3, sizeof(double))))
        return -1;
    if (L < nlev)
      for (int s = 0; s < 27; ++s)
        if (!(v->P[s] = calloc(n3, sizeof(double))))
          return -1;
    if (!(v->x = calloc(n3, sizeof(double))) ||
        !(v->f = calloc(n3, sizeof(double))) ||
        !(v->r = calloc(n3, sizeof(double))) ||
        !(v->zero = calloc(n3, sizeof(double))))
      return -1;
    v->A.kind = L == nlev ? 7 : 27;
    for (int s = 0; s < 14; ++s)
      v->A.a[s] = v->op[s];
  }
  olevel *fine = &h->lv[nlev];
  const size_t n3 = (size_t)fine->n * fine->n * fine->n;
  memcpy(fine->op[0], oC, n3 * sizeof(double));
  memcpy(fine->op[1], oE, n3 * sizeof(double));
  memcpy(fine->op[2], oN, n3 * sizeof(double));
  memcpy(fine->op[3], uC, n3 * sizeof(double));
  for (int L = nlev; L >= 2; --L) {
    olevel *f = &h->lv[L], *c = &h->lv[L - 1];
    if (trilinear)
      pmgo_buildP_trilin(c->n, c->n, c->n, c->P);
    else
      pmgo_buildP_op(f->n, f->n, f->n, c->n, c->n, c->n, &f->A, c->P);
    pmgo_buildG(f->n, f->n, f->n, c->n, c->n, c->n,
                (const double *const *)c->P, &f->A, c->op);
  }
  return 0;
}

static void smooth(ohier *h, int L, int zero_init) {
  olevel *v = &h->lv[L];
  if (L == h->nlev)
    pmgo_gsrb7x(v->n, v->n, v->n, v->op[0], v->zero, v->f, v->op[1],
                v->op[2], v->op[3], v->x, 1, 0, zero_init);
  else
    pmgo_gsrb27x(v->n, v->n, v->n, (const double *const *)v->op, v->zero,
                 v->f, v->x, 1, 0, zero_init);
}

static void vcycle(ohier *h, int L, int as_preconditioner) {
  olevel *v = &h->lv[L];
  if (L == 1) {
    pmgo_cg(v->n, v->n, v->n, &v->A, v->f, v->x, 1e-8);
    return;
  }
  olevel *c = &h->lv[L - 1];
  int zero_init = (L != h->nlev) || as_preconditioner;
  for (int s = 0; s < 2; ++s) {
    smooth(h, L, zero_init);
    zero_init = 0;
  }
  pmgo_defect(v->n, v->n, v->n, &v->A, v->f, v->x, v->r);
  pmgo_restrc2(v->n, v->n, v->n, c->n, c->n, c->n, v->r, c->f,
               (const double *const *)c->P);
  vcycle(h, L - 1, 0);
  const double omega =
      pmgo_ideal_lambda(c->n, c->n, c->n, &c->A, c->x, c->f);
  pmgo_interp2(c->n, c->n, c->n, v->n, v->n, v->n, c->x, v->r,
               (const double *const *)c->P);
  /* x = x + omega * e over the whole padded array (Domain.h:602-623) */
  const size_t n3 = (size_t)v->n * v->n * v->n;
  for (size_t q = 0; q < n3; ++q)
    v->x[q] = v->x[q] + omega * v->r[q];
  for (int s = 0; s < 2; ++s)
    smooth(h, L, 0);
}

int pmgo_solve(int base, int nlev, const double *oC, const double *oE,
               const double *oN, const double *uC, const double *f,
               const double *x0, double tol, int max_cycles, int trilinear,
               double *x_out, double *hist) {
  ohier h;
  if (hier_build(&h, base, nlev, oC, oE, oN, uC, trilinear) != 0) {
    hier_free(&h);
    return -1;
  }
  olevel *fine = &h.lv[nlev];
  const int n = fine->n;
  const size_t n3 = (size_t)n * n * n;
  memcpy(fine->f, f, n3 * sizeof(double));
  memcpy(fine->x, x0, n3 * sizeof(double));
  const double r0 = pmgo_residual2(n, n, n, &fine->A, fine->f, fine->x);
  if (hist)
    hist[0] = r0;
  int c = 0;
  while (c < max_cycles) {
    vcycle(&h, nlev, 0);
    ++c;
    const double r = pmgo_residual2(n, n, n, &fine->A, fine->f, fine->x);
    if (hist)
      hist[c] = r;
    if (r / r0 < tol)
      break;
  }
  if (x_out)
    memcpy(x_out, fine->x, n3 * sizeof(double));
  hier_free(&h);
  return c;
}

/* MG-preconditioned CG on the finest level: CG_solver (CG_Solver.h:45-242)
 * with the class as preconditioner (PBE_pmgc_class.h:1116-1133: rhs -> the
 * class's finest rhs, one zero-started V-cycle, the class's finest iterate
 * returned), as the app runs it (PBE_pmgc_class_with_non_zero_IS.cc:
 * 118-131). The class's finest iterate has a zero shell there; x0 (with the
 * Dirichlet shell) is the initial guess. Sums run over the interior in
 * (k, j, i) order. Iterates until max_iters or, with tol > 0, until
 * sqrt(sum r^2 / n^3) of the updated residual falls below tol times its
 * initial value; hist[c] holds that norm after c iterations. Returns the
 * iterations run, -1 on allocation failure. */
static double dot_interior(int n, const double *a, const double *b) {
  double s = 0.0;
  for (int k = 2; k <= n - 1; ++k)
    for (int j = 2; j <= n - 1; ++j)
      for (int i = 2; i <= n - 1; ++i) {
        const size_t p = IX(n, n, i, j, k);
        s += a[p] * b[p];
      }
  return s;
}

static void mg_precondition(ohier *h, const double *r, double *s) {
  olevel *fine = &h->lv[h->nlev];
  const size_t n3 = (size_t)fine->n * fine->n * fine->n;
  memcpy(fine->f, r, n3 * sizeof(double));
  memset(fine->x, 0, n3 * sizeof(double));
  vcycle(h, h->nlev, 1);
  memcpy(s, fine->x, n3 * sizeof(double));
}

int pmgo_pcg(int base, int nlev, const double *oC, const double *oE,
             const double *oN, const double *uC, const double *f,
             const double *x0, int max_iters, double tol, double *x_out,
             double *hist) {
  ohier h;
  if (hier_build(&h, base, nlev, oC, oE, oN, uC, 0) != 0) {
    hier_free(&h);
    return -1;
  }
  olevel *fine = &h.lv[nlev];
  const int n = fine->n;
  const size_t n3 = (size_t)n * n * n;
  const pmgo_op *A = &fine->A;
  double *x = malloc(n3 * sizeof(double)), *r = calloc(n3, sizeof(double));
  double *s = calloc(n3, sizeof(double)), *pv = calloc(n3, sizeof(double));
  double *ap = calloc(n3, sizeof(double));
  if (!x || !r || !s || !pv || !ap) {
    free(x); free(r); free(s); free(pv); free(ap);
    hier_free(&h);
    return -1;
  }
  memcpy(x, x0, n3 * sizeof(double));
  pmgo_defect(n, n, n, A, f, x, r);
  const double r0 = sqrt(dot_interior(n, r, r) / (double)n3);
  if (hist)
    hist[0] = r0;
  mg_precondition(&h, r, s);
  memcpy(pv, s, n3 * sizeof(double));
  double rs = dot_interior(n, r, s);
  pmgo_matvec(n, n, n, A, NULL, pv, ap);
  double pap = dot_interior(n, ap, pv);
  int c = 0;
  if (pap != 0.0) {
    double alpha = rs / pap;
    while (c < max_iters) {
      for (int k = 2; k <= n - 1; ++k)
        for (int j = 2; j <= n - 1; ++j)
          for (int i = 2; i <= n - 1; ++i) {
            const size_t q = IX(n, n, i, j, k);
            x[q] += alpha * pv[q];
            r[q] -= alpha * ap[q];
          }
      mg_precondition(&h, r, s);
      const double rs_next = dot_interior(n, r, s);
      const double beta = rs == 0.0 ? 0.0 : rs_next / rs;
      rs = rs_next;
      for (int k = 2; k <= n - 1; ++k)
        for (int j = 2; j <= n - 1; ++j)
          for (int i = 2; i <= n - 1; ++i) {
            const size_t q = IX(n, n, i, j, k);
            pv[q] = s[q] + beta * pv[q];
          }
      pmgo_matvec(n, n, n, A, NULL, pv, ap);
      pap = dot_interior(n, ap, pv);
      alpha = pap == 0.0 ? 0.0 : rs / pap;
      ++c;
      const double rn = sqrt(dot_interior(n, r, r) / (double)n3);
      if (hist)
        hist[c] = rn;
      if (tol > 0.0 && r0 > 0.0 && rn / r0 < tol)
        break;
    }
  }
  if (x_out)
    memcpy(x_out, x, n3 * sizeof(double));
  free(x); free(r); free(s); free(pv); free(ap);
  hier_free(&h);
  return c;
}

long pmgo_hierarchy(int base, int nlev, const double *oC, const double *oE,
                    const double *oN, const double *uC, int trilinear,
                    double *out, long cap) {
  long need = 0;
  for (int L = nlev - 1; L >= 1; --L) {
    const long n = base * (1L << L) + 1;
    need += 41 * n * n * n;
  }
  if (cap < need)
    return -1;
  ohier h;
  if (hier_build(&h, base, nlev, oC, oE, oN, uC, trilinear) != 0) {
    hier_free(&h);
    return -1;
  }
  double *o = out;
  for (int L = nlev - 1; L >= 1; --L) {
    olevel *v = &h.lv[L];
    const size_t n3 = (size_t)v->n * v->n * v->n;
    for (int s = 0; s < 27; ++s, o += n3)
      memcpy(o, v->P[s], n3 * sizeof(double));
    for (int s = 0; s < 14; ++s, o += n3)
      memcpy(o, v->op[s], n3 * sizeof(double));
  }
  hier_free(&h);
  return need;
}
