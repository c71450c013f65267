// Physical constants and derived parameters of the linearized PB set-up,
// shared by the host and the GPU set-up.
#pragma once

#include <math.h>

#include "../../include/pmg_b200.h"

namespace pmg {

// Physical constants of the reference (scientific_quantities.h:7-15).
constexpr double kB = 1.380649e-23;
constexpr double kE = 1.60217663e-19;
constexpr double kEpsSI = 8.8541878128e-12;
constexpr double kNA = 6.0221408e23;
constexpr double kPi = 3.14159265358979323846;

// Heron/Newton square root with the reference's stopping rule
// |g^2 - x| <= 1e-13 x, starting from 1.0 (const_sqrt,
// scientific_quantities.h:18-25); kept so kappa rounds like the reference.
inline double newton_sqrt(double x, double guess = 1.0) {
  if (x == 0)
    return 0;
  for (int it = 0; it < 2000; ++it) {
    if (fabs(guess * guess - x) <= x * 1e-13)
      return guess;
    guess = (guess + x / guess) / 2;
  }
  return guess;
}

struct Physics {
  double eps_in, eps_out, T, kappa, eps0;
};

inline Physics physics(const pmg_physics &ph) {
  Physics p;
  p.eps_in = ph.eps_in;
  p.eps_out = ph.eps_out;
  p.T = ph.temperature;
  const double beta = 1 / (kB * p.T);
  // vacuum permittivity in e^2 / (kT * Angstrom)
  p.eps0 = kEpsSI * 1e-10 / (kE * kE) * kB * p.T;
  // inverse Debye length in 1/Angstrom (Debye_length_inverse_squared,
  // Kappa, KappaA: scientific_quantities.h:38-55); IS in mol/l
  const double is_si = 1000 * ph.ionic_strength;
  const double inv_sq = kE * kE * beta * 2 * is_si * kNA / (p.eps_out * kEpsSI);
  p.kappa = newton_sqrt(inv_sq) * 1e-10;
  return p;
}

// Unit directions of the probe-placement sphere (a Fibonacci lattice of
// kProbePoints points): z, the xy radius and cos / sin of the azimuth, so
// the host and the GPU place probe centres with the same doubles.
constexpr int kProbePoints = 96;
struct ProbeDir {
  double zz, rr, c, s;
};
inline void probe_directions(ProbeDir *out) {
  const double golden = kPi * (3.0 - sqrt(5.0));
  for (int s = 0; s < kProbePoints; ++s) {
    const double zz = 1 - 2 * (s + 0.5) / kProbePoints;
    const double t = 1 - zz * zz;
    out[s].zz = zz;
    out[s].rr = sqrt(t > 0.0 ? t : 0.0);
    out[s].c = cos(golden * s);
    out[s].s = sin(golden * s);
  }
}

} // namespace pmg
