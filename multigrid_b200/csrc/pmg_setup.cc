// Host set-up of the fine PMG level from a list of atoms: dielectric and
// kappa maps, trilinear charges and the multiple-Debye-Hueckel boundary,
// following the reference class's set-up (PBE_pmgc_class.h:141-349) with
// the physical constants as runtime parameters.
//
// With probe_radius = 0 this is the reference's marking (van der Waals union
// at staggered points, dot_finder.h:82-87) and, at the reference's constants
// (eps_in 4, eps_out 78.4, T 298.15), it reproduces the reference set-up
// exactly. With probe_radius > 0 the dielectric boundary is the molecular
// (solvent-excluded) surface instead: a staggered point is solute if it lies
// inside an atom, or inside the probe-inflated spheres but outside every
// probe placed on the accessible surface (see mark_probe_surface).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "../../include/pmg_b200.h"

#include "pmg_physics.h"

namespace {

using pmg::Physics;
using pmg::physics;
using pmg::kPi;

struct Grid {
  int n;
  double h;
  long at(long i0, long i1, long i2) const {
    return (i0 * n + i1) * n + i2;
  }
};

// Marks every grid point inside a sphere (dot_finder.h:22-80): index ranges
// ceil((c - r)/h) .. trunc((c + r)/h) on axis 0, then the chord half-widths
// sqrt(r^2 - sum of squared offsets) on axes 1 and 2. Axis 0 is the slowest
// array axis (pmgc k), axis 2 the fastest (pmgc i); atom coordinate d lies
// on axis d, as in the reference (Position[0] is the slowest axis). Points
// outside the array are skipped.
template <typename F>
void for_dots_in_sphere(const Grid &g, const double c[3], double r, F mark) {
  const double h = g.h;
  const int lo0 = (int)ceil((c[0] - r) / h);
  const int hi0 = (int)((c[0] + r) / h);
  for (int i0 = lo0; i0 <= hi0; ++i0) {
    double s1 = r * r - ((c[0] - h * i0) * (c[0] - h * i0));
    if (s1 < 0)
      s1 = 0;
    const double w1 = sqrt(s1);
    const int lo1 = (int)ceil((c[1] - w1) / h);
    const int hi1 = (int)((c[1] + w1) / h);
    for (int i1 = lo1; i1 <= hi1; ++i1) {
      double s2 = r * r - ((c[0] - h * i0) * (c[0] - h * i0) +
                           (c[1] - h * i1) * (c[1] - h * i1));
      if (s2 < 0)
        s2 = 0;
      const double w2 = sqrt(s2);
      const int lo2 = (int)ceil((c[2] - w2) / h);
      const int hi2 = (int)((c[2] + w2) / h);
      for (int i2 = lo2; i2 <= hi2; ++i2) {
        if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= g.n || i1 >= g.n ||
            i2 >= g.n)
          continue;
        mark(g.at(i0, i1, i2));
      }
    }
  }
}

template <typename F> void parallel_for(long n, F body) {
  unsigned nt = std::thread::hardware_concurrency();
  nt = std::max(1u, std::min(nt, 64u));
  std::atomic<long> next{0};
  std::vector<std::thread> th;
  const long chunk = 256;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&] {
      for (;;) {
        const long b = next.fetch_add(chunk);
        if (b >= n)
          return;
        const long e = std::min(n, b + chunk);
        for (long q = b; q < e; ++q)
          body(q);
      }
    });
  for (auto &t : th)
    t.join();
}

// Molecular-surface marking for probe_radius > 0 on one staggered grid
// (offset along `axis`): solute = inside an atom, or inside an inflated
// sphere (r + probe) and farther than `probe` from every accessible probe
// centre. Probe centres are points of a Fibonacci sphere of radius r + probe
// around each atom that lie outside every other inflated sphere.
void mark_probe_surface(const Grid &g, const double *atoms, int natoms,
                        double probe, int axis, std::vector<char> &inside) {
  const long n3 = (long)g.n * g.n * g.n;
  std::vector<char> sas(n3, 0);
  for (int a = 0; a < natoms; ++a) {
    double c[3] = {atoms[5 * a + 0], atoms[5 * a + 1], atoms[5 * a + 2]};
    if (axis >= 0)
      c[axis] -= 0.5 * g.h;
    for_dots_in_sphere(g, c, atoms[5 * a + 3], [&](long q) { inside[q] = 1; });
    for_dots_in_sphere(g, c, atoms[5 * a + 3] + probe,
                       [&](long q) { sas[q] = 1; });
  }
  // cell list of inflated spheres for the accessibility test
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  double rmax = 0;
  for (int a = 0; a < natoms; ++a) {
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], atoms[5 * a + d]);
      hi[d] = std::max(hi[d], atoms[5 * a + d]);
    }
    rmax = std::max(rmax, atoms[5 * a + 3]);
  }
  const double cell = 2 * (rmax + probe);
  int nc[3];
  for (int d = 0; d < 3; ++d)
    nc[d] = std::max(1, (int)((hi[d] - lo[d]) / cell) + 1);
  std::vector<std::vector<int>> cells((size_t)nc[0] * nc[1] * nc[2]);
  auto cell_of = [&](const double *x, int *ci) {
    for (int d = 0; d < 3; ++d)
      ci[d] = std::min(nc[d] - 1, std::max(0, (int)((x[d] - lo[d]) / cell)));
  };
  for (int a = 0; a < natoms; ++a) {
    int ci[3];
    cell_of(&atoms[5 * a], ci);
    cells[((size_t)ci[2] * nc[1] + ci[1]) * nc[0] + ci[0]].push_back(a);
  }
  pmg::ProbeDir dirs[pmg::kProbePoints];
  pmg::probe_directions(dirs);
  std::vector<double> probes;
  for (int a = 0; a < natoms; ++a) {
    const double R = atoms[5 * a + 3] + probe;
    int ci[3];
    cell_of(&atoms[5 * a], ci);
    for (int s = 0; s < pmg::kProbePoints; ++s) {
      const pmg::ProbeDir &u = dirs[s];
      const double pc[3] = {atoms[5 * a] + R * u.rr * u.c,
                            atoms[5 * a + 1] + R * u.rr * u.s,
                            atoms[5 * a + 2] + R * u.zz};
      bool free = true;
      for (int dz = -1; dz <= 1 && free; ++dz)
        for (int dy = -1; dy <= 1 && free; ++dy)
          for (int dx = -1; dx <= 1 && free; ++dx) {
            const int cx = ci[0] + dx, cy = ci[1] + dy, cz = ci[2] + dz;
            if (cx < 0 || cy < 0 || cz < 0 || cx >= nc[0] || cy >= nc[1] ||
                cz >= nc[2])
              continue;
            for (int b : cells[((size_t)cz * nc[1] + cy) * nc[0] + cx]) {
              if (b == a)
                continue;
              const double Rb = atoms[5 * b + 3] + probe;
              double d2 = 0;
              for (int d = 0; d < 3; ++d) {
                const double t = pc[d] - atoms[5 * b + d];
                d2 += t * t;
              }
              if (d2 < Rb * Rb * (1 - 1e-12)) {
                free = false;
                break;
              }
            }
          }
      if (free)
        probes.insert(probes.end(), {pc[0], pc[1], pc[2]});
    }
  }
  std::vector<char> carved(n3, 0);
  for (size_t q = 0; q < probes.size(); q += 3) {
    double c[3] = {probes[q + 0], probes[q + 1], probes[q + 2]};
    if (axis >= 0)
      c[axis] -= 0.5 * g.h;
    for_dots_in_sphere(g, c, probe, [&](long t) { carved[t] = 1; });
  }
  for (long q = 0; q < n3; ++q)
    if (!inside[q] && sas[q] && !carved[q])
      inside[q] = 1;
}

} // namespace

extern "C" {

int pmg_kappa(const pmg_physics *ph, double *kappa, double *eps0) {
  if (!ph)
    return PMG_ERR_ARG;
  const Physics p = physics(*ph);
  if (kappa)
    *kappa = p.kappa;
  if (eps0)
    *eps0 = p.eps0;
  return PMG_OK;
}

int pmg_setup_fine(int n, double h, const double *atoms, int natoms,
                   const pmg_physics *ph, double *oC, double *oE, double *oN,
                   double *uC, double *f, double *x0) {
  if (n < 3 || n > 1025 || !(h > 0) || !atoms || natoms < 0 || !ph || !oC ||
      !oE || !oN || !uC || !f || !x0)
    return PMG_ERR_ARG;
  const Grid g{n, h};
  const long n3 = (long)n * n * n;
  const Physics p = physics(*ph);
  const double h2 = h * h;
  for (int a = 0; a < natoms; ++a) {
    for (int d = 0; d < 3; ++d) {
      const double x = atoms[5 * a + d];
      if (!(x >= 0 && x <= h * (n - 1)))
        return PMG_ERR_ARG; // atom outside the grid
    }
    if (!(atoms[5 * a + 3] >= 0))
      return PMG_ERR_ARG;
  }

  // Face coefficients eps/h^2 at the staggered points p + h/2 e_axis
  // (initialize_epsilons, PBE_pmgc_class.h:248-281): axis 0 -> uC (z),
  // axis 1 -> oN (y), axis 2 -> oE (x).
  double *face[3] = {uC, oN, oE};
  const double v_out = p.eps_out / h2, v_in = p.eps_in / h2;
  for (int axis = 0; axis < 3; ++axis) {
    double *m = face[axis];
    std::fill(m, m + n3, v_out);
    if (ph->probe_radius > 0) {
      std::vector<char> inside(n3, 0);
      mark_probe_surface(g, atoms, natoms, ph->probe_radius, axis, inside);
      for (long q = 0; q < n3; ++q)
        if (inside[q])
          m[q] = v_in;
    } else {
      for (int a = 0; a < natoms; ++a) {
        // atom (x, y, z) -> grid axes (0: z, 1: y, 2: x)
        double c[3] = {atoms[5 * a + 0], atoms[5 * a + 1], atoms[5 * a + 2]};
        c[axis] -= 0.5 * h;
        for_dots_in_sphere(g, c, atoms[5 * a + 3],
                           [&](long q) { m[q] = v_in; });
      }
    }
  }

  // kappa^2 eps_out outside the ion-accessible spheres r + ion_radius, 0
  // inside (PBE_pmgc_class.h:283-308), added to the centre coefficient
  // oC = sum_axis (face(p) + face(p - e_axis)) on the interior
  // (compute_center_domain_with_kappa, PBE_pmgc_class.h:67-100).
  std::vector<char> ion(n3, 0);
  for (int a = 0; a < natoms; ++a) {
    double c[3] = {atoms[5 * a + 0], atoms[5 * a + 1], atoms[5 * a + 2]};
    for_dots_in_sphere(g, c, atoms[5 * a + 3] + ph->ion_radius,
                       [&](long q) { ion[q] = 1; });
  }
  const double kappa2 = p.kappa * p.kappa;
  const double kterm = kappa2 * p.eps_out;
  std::fill(oC, oC + n3, 0.0);
  const long s1 = n, s0 = (long)n * n;
  for (long i0 = 1; i0 <= n - 2; ++i0)
    for (long i1 = 1; i1 <= n - 2; ++i1)
      for (long i2 = 1; i2 <= n - 2; ++i2) {
        const long q = g.at(i0, i1, i2);
        double c = ((uC[q] + uC[q - s0]) + (oN[q] + oN[q - s1])) +
                   (oE[q] + oE[q - 1]);
        c += ion[q] ? 0.0 : kterm;
        oC[q] = c;
      }

  // Trilinear charges q/eps0/h^3, atoms in order
  // (add_charges_to_distribution, create_charge_distribution.h:16-61).
  std::fill(f, f + n3, 0.0);
  const double vol = h * (h * h);
  for (int a = 0; a < natoms; ++a) {
    const double pos[3] = {atoms[5 * a + 0], atoms[5 * a + 1],
                           atoms[5 * a + 2]};
    const double charge = atoms[5 * a + 4] / p.eps0;
    long pt[6];
    double w[6];
    for (int d = 0; d < 3; ++d) {
      const double s = pos[d] / h;
      const long lo = (long)s;
      pt[2 * d] = lo;
      pt[2 * d + 1] = lo + 1;
      w[2 * d] = (lo + 1 - s);
      w[2 * d + 1] = (s - lo);
    }
    for (int corner = 0; corner < 8; ++corner) {
      double wt = 1;
      long c[3];
      for (int d = 0; d < 3; ++d) {
        const int b = (corner >> d) & 1;
        wt *= w[2 * d + b];
        c[d] = pt[2 * d + b];
      }
      if (c[0] >= n || c[1] >= n || c[2] >= n)
        continue;
      f[g.at(c[0], c[1], c[2])] += charge * wt / vol;
    }
  }

  // Multiple Debye-Hueckel boundary on the six faces, zero inside
  // (Set_boundary_conditions / initialize_boundary_extern,
  // PBE_pmgc_class.h:173-242; DH_Sphere, Debye_Hueckel_functions.h:10-14).
  std::fill(x0, x0 + n3, 0.0);
  const double pref = 4 * kPi * (p.eps0 * p.eps_out);
  auto dh = [&](long i0, long i1, long i2) {
    double acc = 0;
    for (int a = 0; a < natoms; ++a) {
      const double d0 = i0 * h - atoms[5 * a + 0];
      const double d1 = i1 * h - atoms[5 * a + 1];
      const double d2 = i2 * h - atoms[5 * a + 2];
      const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
      const double rad = atoms[5 * a + 3];
      acc += atoms[5 * a + 4] / (pref * (1 + p.kappa * rad)) *
             exp(-p.kappa * (dist - rad)) / dist;
    }
    x0[g.at(i0, i1, i2)] = acc;
  };
  const long faces = (long)n * n;
  parallel_for(faces, [&](long q) {
    const long a = q / n, b = q % n;
    dh(a, b, 0);
    dh(a, b, n - 1);
    dh(0, a, b);
    dh(n - 1, a, b);
    dh(a, 0, b);
    dh(a, n - 1, b);
  });
  return PMG_OK;
}

} // extern "C"
