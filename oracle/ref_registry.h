// Registry of the reference PMG class instantiations compiled into the
// oracle library (test infrastructure). PBE_linear_problem takes its grid as
// template parameters <base_length, nlev, box_length>
// (PBE_pmgc_class.h:112), so every grid the tests or the CPU baseline use is
// compiled once (ref_class_inst.cc, one object per configuration) and found
// here at run time by (base, nlev).
#pragma once

#include "ref_api.h"

struct pmgref_entry {
  int base;
  int nlev;
  double box;
  int (*solve)(const pmgref_fine *in, double tol, int max_cycles,
               int trilinear, double *x_out, double *hist, int *cycles);
  int (*cycles)(const pmgref_fine *in, int ncycles, double *x_out);
  long (*hierarchy)(const pmgref_fine *in, int trilinear, double *out,
                    long cap);
  int (*cg_level1)(const double *const *op14, const double *rhs, double *x);
  int (*setup)(const double *atoms, int natoms, double ionic_strength,
               double ion_radius, double *oC, double *oE, double *oN,
               double *uC, double *f, double *x0);
  int (*pcg)(const pmgref_fine *in, int iters, double *x_out);
};

void pmgref_register(const pmgref_entry &e);
