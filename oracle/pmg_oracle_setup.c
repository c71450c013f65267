/* CPU restatement of the fine-level set-up from atoms (oracle, test
 * infrastructure). Independent C of the set-up that the reference class runs
 * in its constructor (PBE_pmgc_class.h:141-349), with the physical constants
 * as runtime parameters and the optional probe-radius (molecular surface)
 * marking of the PB workloads. It lets the oracle side build its own inputs
 * without the product library, and it is held bit for bit against the
 * product's host set-up by the CPU tests.
 *
 *   dielectric faces : initialize_epsilons, PBE_pmgc_class.h:248-281, with
 *                      the sphere bounds of dot_finder.h:22-87
 *   kappa map / oC   : PBE_pmgc_class.h:283-313 and
 *                      compute_center_domain_with_kappa, :67-100
 *   charges          : add_charges_to_distribution,
 *                      create_charge_distribution.h:16-61
 *   boundary         : Set_boundary_conditions / initialize_boundary_extern,
 *                      PBE_pmgc_class.h:173-242, DH_Sphere,
 *                      Debye_Hueckel_functions.h:10-14
 *   constants        : scientific_quantities.h:7-55 (kappa through the
 *                      reference's Newton square root, :18-25)
 *
 * Array index (i0, i1, i2) -> (i0 n + i1) n + i2: axis 0 is the slowest
 * (pmgc k), axis 2 the fastest (pmgc i); atom coordinate d lies on axis d.
 * The boundary's face sums run on host threads (each face point is
 * independent, so the thread count does not change a bit).
 */
#define _POSIX_C_SOURCE 200809L
#include "pmg_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

static const double K_B = 1.380649e-23;
static const double K_E = 1.60217663e-19;
static const double K_EPS_SI = 8.8541878128e-12;
static const double K_NA = 6.0221408e23;
static const double K_PI = 3.14159265358979323846;
#define PROBE_POINTS 96

/* const_sqrt of scientific_quantities.h:18-25: Heron iteration from 1.0
 * until |g^2 - x| <= 1e-13 x. */
static double heron_sqrt(double x) {
  double g = 1.0;
  int it;
  if (x == 0)
    return 0;
  for (it = 0; it < 2000; ++it) {
    if (fabs(g * g - x) <= x * 1e-13)
      return g;
    g = (g + x / g) / 2;
  }
  return g;
}

void pmgo_physics(double eps_out, double ionic_strength, double temperature,
                  double *kappa, double *eps0) {
  const double beta = 1 / (K_B * temperature);
  /* vacuum permittivity in e^2 / (kT Angstrom) */
  const double e0 = K_EPS_SI * 1e-10 / (K_E * K_E) * K_B * temperature;
  /* Debye_length_inverse_squared (ionic strength in mol/l -> mol/m^3) */
  const double is_si = 1000 * ionic_strength;
  const double inv_sq =
      K_E * K_E * beta * 2 * is_si * K_NA / (eps_out * K_EPS_SI);
  if (kappa)
    *kappa = heron_sqrt(inv_sq) * 1e-10;
  if (eps0)
    *eps0 = e0;
}

typedef struct {
  int n;
  double h;
} grid_t;

static long at3(const grid_t *g, long i0, long i1, long i2) {
  return (i0 * g->n + i1) * g->n + i2;
}

/* Sets mask[q] = 1 for every grid point inside the sphere (c, r): axis-0
 * range ceil((c0 - r)/h) .. trunc((c0 + r)/h), then on axes 1 and 2 the
 * chord half-widths sqrt(r^2 - squared offsets) (dot_finder.h:22-80).
 * Points outside the array are skipped. */
static void mark_sphere(const grid_t *g, const double c[3], double r,
                        char *mask) {
  const double h = g->h;
  const int lo0 = (int)ceil((c[0] - r) / h);
  const int hi0 = (int)((c[0] + r) / h);
  int i0, i1, i2;
  for (i0 = lo0; i0 <= hi0; ++i0) {
    double s1 = r * r - ((c[0] - h * i0) * (c[0] - h * i0));
    double w1;
    int lo1, hi1;
    if (s1 < 0)
      s1 = 0;
    w1 = sqrt(s1);
    lo1 = (int)ceil((c[1] - w1) / h);
    hi1 = (int)((c[1] + w1) / h);
    for (i1 = lo1; i1 <= hi1; ++i1) {
      double s2 = r * r - ((c[0] - h * i0) * (c[0] - h * i0) +
                           (c[1] - h * i1) * (c[1] - h * i1));
      double w2;
      int lo2, hi2;
      if (s2 < 0)
        s2 = 0;
      w2 = sqrt(s2);
      lo2 = (int)ceil((c[2] - w2) / h);
      hi2 = (int)((c[2] + w2) / h);
      for (i2 = lo2; i2 <= hi2; ++i2) {
        if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= g->n || i1 >= g->n ||
            i2 >= g->n)
          continue;
        mask[at3(g, i0, i1, i2)] = 1;
      }
    }
  }
}

/* Probe-sphere directions: a Fibonacci lattice of PROBE_POINTS unit vectors
 * (z, xy radius, cos and sin of the azimuth). */
static void probe_dirs(double (*d)[4]) {
  const double golden = K_PI * (3.0 - sqrt(5.0));
  int s;
  for (s = 0; s < PROBE_POINTS; ++s) {
    const double zz = 1 - 2 * (s + 0.5) / PROBE_POINTS;
    const double t = 1 - zz * zz;
    d[s][0] = zz;
    d[s][1] = sqrt(t > 0.0 ? t : 0.0);
    d[s][2] = cos(golden * s);
    d[s][3] = sin(golden * s);
  }
}

/* Accessible probe centres: the lattice points on each inflated sphere
 * (radius r + probe) that no other inflated sphere contains, atoms in order,
 * directions in order. A uniform cell list (edge 2 (r_max + probe)) limits
 * the containment test to the 27 cells around the atom; any containing
 * sphere lies there, so the result is the all-pairs one. Returns the number
 * of centres written to *out (3 doubles each; malloc'd). */
static long accessible_probes(const double *atoms, int natoms, double probe,
                              double **out) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  double rmax = 0, cell, dirs[PROBE_POINTS][4];
  int nc[3], a, d;
  long ncell, *start, *fill, *members, cap, count = 0;
  double *probes;
  int *cell_of_atom;
  for (a = 0; a < natoms; ++a) {
    for (d = 0; d < 3; ++d) {
      if (atoms[5 * a + d] < lo[d])
        lo[d] = atoms[5 * a + d];
      if (atoms[5 * a + d] > hi[d])
        hi[d] = atoms[5 * a + d];
    }
    if (atoms[5 * a + 3] > rmax)
      rmax = atoms[5 * a + 3];
  }
  cell = 2 * (rmax + probe);
  for (d = 0; d < 3; ++d) {
    nc[d] = (int)((hi[d] - lo[d]) / cell) + 1;
    if (nc[d] < 1)
      nc[d] = 1;
  }
  ncell = (long)nc[0] * nc[1] * nc[2];
  start = calloc((size_t)ncell + 1, sizeof(long));
  fill = calloc((size_t)ncell, sizeof(long));
  members = malloc(sizeof(long) * (size_t)(natoms > 0 ? natoms : 1));
  cell_of_atom = malloc(sizeof(int) * 3 * (size_t)(natoms > 0 ? natoms : 1));
  cap = (long)natoms * PROBE_POINTS * 3 + 3;
  probes = malloc(sizeof(double) * (size_t)cap);
  for (a = 0; a < natoms; ++a) {
    for (d = 0; d < 3; ++d) {
      int ci = (int)((atoms[5 * a + d] - lo[d]) / cell);
      if (ci < 0)
        ci = 0;
      if (ci > nc[d] - 1)
        ci = nc[d] - 1;
      cell_of_atom[3 * a + d] = ci;
    }
    start[((long)cell_of_atom[3 * a + 2] * nc[1] + cell_of_atom[3 * a + 1]) *
              nc[0] +
          cell_of_atom[3 * a] + 1]++;
  }
  for (a = 0; a < ncell; ++a)
    start[a + 1] += start[a];
  for (a = 0; a < natoms; ++a) {
    const long c = ((long)cell_of_atom[3 * a + 2] * nc[1] +
                    cell_of_atom[3 * a + 1]) *
                       nc[0] +
                   cell_of_atom[3 * a];
    members[start[c] + fill[c]++] = a;
  }
  probe_dirs(dirs);
  for (a = 0; a < natoms; ++a) {
    const double R = atoms[5 * a + 3] + probe;
    int s;
    for (s = 0; s < PROBE_POINTS; ++s) {
      const double pc[3] = {atoms[5 * a] + R * dirs[s][1] * dirs[s][2],
                            atoms[5 * a + 1] + R * dirs[s][1] * dirs[s][3],
                            atoms[5 * a + 2] + R * dirs[s][0]};
      int free = 1, dx, dy, dz;
      for (dz = -1; dz <= 1 && free; ++dz)
        for (dy = -1; dy <= 1 && free; ++dy)
          for (dx = -1; dx <= 1 && free; ++dx) {
            const int cx = cell_of_atom[3 * a] + dx;
            const int cy = cell_of_atom[3 * a + 1] + dy;
            const int cz = cell_of_atom[3 * a + 2] + dz;
            long c, m;
            if (cx < 0 || cy < 0 || cz < 0 || cx >= nc[0] || cy >= nc[1] ||
                cz >= nc[2])
              continue;
            c = ((long)cz * nc[1] + cy) * nc[0] + cx;
            for (m = start[c]; m < start[c + 1]; ++m) {
              const long b = members[m];
              const double Rb = atoms[5 * b + 3] + probe;
              double d2 = 0;
              int e;
              if (b == a)
                continue;
              for (e = 0; e < 3; ++e) {
                const double t = pc[e] - atoms[5 * b + e];
                d2 += t * t;
              }
              if (d2 < Rb * Rb * (1 - 1e-12)) {
                free = 0;
                break;
              }
            }
          }
      if (free) {
        probes[3 * count] = pc[0];
        probes[3 * count + 1] = pc[1];
        probes[3 * count + 2] = pc[2];
        ++count;
      }
    }
  }
  free(start);
  free(fill);
  free(members);
  free(cell_of_atom);
  *out = probes;
  return count;
}

/* Solute flags of one staggered grid (offset h/2 along `axis`) for a probe
 * radius > 0: inside an atom, or inside an inflated sphere and not within
 * `probe` of an accessible probe centre (the solvent-excluded volume). */
static void probe_surface(const grid_t *g, const double *atoms, int natoms,
                          double probe, int axis, const double *probes,
                          long nprobes, char *inside) {
  const long n3 = (long)g->n * g->n * g->n;
  char *sas = calloc((size_t)n3, 1);
  char *carved = calloc((size_t)n3, 1);
  long q;
  int a;
  for (a = 0; a < natoms; ++a) {
    double c[3] = {atoms[5 * a], atoms[5 * a + 1], atoms[5 * a + 2]};
    c[axis] -= 0.5 * g->h;
    mark_sphere(g, c, atoms[5 * a + 3], inside);
    mark_sphere(g, c, atoms[5 * a + 3] + probe, sas);
  }
  for (q = 0; q < nprobes; ++q) {
    double c[3] = {probes[3 * q], probes[3 * q + 1], probes[3 * q + 2]};
    c[axis] -= 0.5 * g->h;
    mark_sphere(g, c, probe, carved);
  }
  for (q = 0; q < n3; ++q)
    if (!inside[q] && sas[q] && !carved[q])
      inside[q] = 1;
  free(sas);
  free(carved);
}

/* ---- multiple Debye-Hueckel boundary ------------------------------------ */

typedef struct {
  const grid_t *g;
  const double *atoms;
  int natoms;
  double kappa, pref;
  double *x0;
  long next, total;
  pthread_mutex_t lock;
} dh_job;

static void dh_point(dh_job *j, long i0, long i1, long i2) {
  const double h = j->g->h;
  double acc = 0;
  int a;
  for (a = 0; a < j->natoms; ++a) {
    const double *at = j->atoms + 5 * a;
    const double d0 = i0 * h - at[0];
    const double d1 = i1 * h - at[1];
    const double d2 = i2 * h - at[2];
    const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    const double rad = at[3];
    acc += at[4] / (j->pref * (1 + j->kappa * rad)) *
           exp(-j->kappa * (dist - rad)) / dist;
  }
  j->x0[at3(j->g, i0, i1, i2)] = acc;
}

static void *dh_worker(void *arg) {
  dh_job *j = arg;
  const long n = j->g->n;
  for (;;) {
    long b, e, q;
    pthread_mutex_lock(&j->lock);
    b = j->next;
    j->next += 64;
    pthread_mutex_unlock(&j->lock);
    if (b >= j->total)
      return NULL;
    e = b + 64 < j->total ? b + 64 : j->total;
    for (q = b; q < e; ++q) {
      const long a = q / n, c = q % n;
      dh_point(j, a, c, 0);
      dh_point(j, a, c, n - 1);
      dh_point(j, 0, a, c);
      dh_point(j, n - 1, a, c);
      dh_point(j, a, 0, c);
      dh_point(j, a, n - 1, c);
    }
  }
}

int pmgo_setup_fine(int n, double h, const double *atoms, int natoms,
                    double eps_in, double eps_out, double ionic_strength,
                    double ion_radius, double temperature,
                    double probe_radius, double *oC, double *oE, double *oN,
                    double *uC, double *f, double *x0) {
  grid_t g;
  long n3, i0, i1, i2, s0, s1;
  double kappa, eps0, h2, v_out, v_in, kterm, vol, *face[3], *probes = NULL;
  long nprobes = 0;
  char *mask;
  int a, d, axis;
  if (n < 3 || n > 1025 || !(h > 0) || !atoms || natoms < 0 || !oC || !oE ||
      !oN || !uC || !f || !x0)
    return -1;
  g.n = n;
  g.h = h;
  n3 = (long)n * n * n;
  for (a = 0; a < natoms; ++a) {
    for (d = 0; d < 3; ++d) {
      const double x = atoms[5 * a + d];
      if (!(x >= 0 && x <= h * (n - 1)))
        return -1;
    }
    if (!(atoms[5 * a + 3] >= 0))
      return -1;
  }
  pmgo_physics(eps_out, ionic_strength, temperature, &kappa, &eps0);
  h2 = h * h;
  mask = malloc((size_t)n3);
  if (!mask)
    return -2;

  /* face coefficients eps/h^2 at p + h/2 e_axis: axis 0 -> uC, 1 -> oN,
   * 2 -> oE */
  face[0] = uC;
  face[1] = oN;
  face[2] = oE;
  v_out = eps_out / h2;
  v_in = eps_in / h2;
  if (probe_radius > 0)
    nprobes = accessible_probes(atoms, natoms, probe_radius, &probes);
  for (axis = 0; axis < 3; ++axis) {
    double *m = face[axis];
    long q;
    memset(mask, 0, (size_t)n3);
    if (probe_radius > 0) {
      probe_surface(&g, atoms, natoms, probe_radius, axis, probes, nprobes,
                    mask);
    } else {
      for (a = 0; a < natoms; ++a) {
        double c[3] = {atoms[5 * a], atoms[5 * a + 1], atoms[5 * a + 2]};
        c[axis] -= 0.5 * h;
        mark_sphere(&g, c, atoms[5 * a + 3], mask);
      }
    }
    for (q = 0; q < n3; ++q)
      m[q] = mask[q] ? v_in : v_out;
  }
  free(probes);

  /* ion-exclusion spheres r + ion_radius; kappa^2 eps_out outside them is
   * added to oC = sum over axes of (face(p) + face(p - e_axis)) */
  memset(mask, 0, (size_t)n3);
  for (a = 0; a < natoms; ++a) {
    double c[3] = {atoms[5 * a], atoms[5 * a + 1], atoms[5 * a + 2]};
    mark_sphere(&g, c, atoms[5 * a + 3] + ion_radius, mask);
  }
  kterm = kappa * kappa * eps_out;
  memset(oC, 0, sizeof(double) * (size_t)n3);
  s1 = n;
  s0 = (long)n * n;
  for (i0 = 1; i0 <= n - 2; ++i0)
    for (i1 = 1; i1 <= n - 2; ++i1)
      for (i2 = 1; i2 <= n - 2; ++i2) {
        const long q = at3(&g, i0, i1, i2);
        double c = ((uC[q] + uC[q - s0]) + (oN[q] + oN[q - s1])) +
                   (oE[q] + oE[q - 1]);
        c += mask[q] ? 0.0 : kterm;
        oC[q] = c;
      }
  free(mask);

  /* trilinear charges q / eps0 / h^3, atoms in order */
  memset(f, 0, sizeof(double) * (size_t)n3);
  vol = h * (h * h);
  for (a = 0; a < natoms; ++a) {
    const double charge = atoms[5 * a + 4] / eps0;
    long pt[6];
    double w[6];
    int corner;
    for (d = 0; d < 3; ++d) {
      const double s = atoms[5 * a + d] / h;
      const long lo = (long)s;
      pt[2 * d] = lo;
      pt[2 * d + 1] = lo + 1;
      w[2 * d] = (lo + 1 - s);
      w[2 * d + 1] = (s - lo);
    }
    for (corner = 0; corner < 8; ++corner) {
      double wt = 1;
      long c[3];
      for (d = 0; d < 3; ++d) {
        const int b = (corner >> d) & 1;
        wt *= w[2 * d + b];
        c[d] = pt[2 * d + b];
      }
      if (c[0] >= n || c[1] >= n || c[2] >= n)
        continue;
      f[at3(&g, c[0], c[1], c[2])] += charge * wt / vol;
    }
  }

  /* multiple Debye-Hueckel values on the six faces, zero inside */
  memset(x0, 0, sizeof(double) * (size_t)n3);
  {
    dh_job job;
    long nt = sysconf(_SC_NPROCESSORS_ONLN), t;
    pthread_t th[64];
    if (nt < 1)
      nt = 1;
    if (nt > 64)
      nt = 64;
    job.g = &g;
    job.atoms = atoms;
    job.natoms = natoms;
    job.kappa = kappa;
    job.pref = 4 * K_PI * (eps0 * eps_out);
    job.x0 = x0;
    job.next = 0;
    job.total = (long)n * n;
    pthread_mutex_init(&job.lock, NULL);
    for (t = 0; t < nt; ++t)
      if (pthread_create(&th[t], NULL, dh_worker, &job) != 0)
        break;
    if (t == 0)
      dh_worker(&job);
    while (t-- > 0)
      pthread_join(th[t], NULL);
    pthread_mutex_destroy(&job.lock);
  }
  return 0;
}
