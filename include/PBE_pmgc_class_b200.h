/* C++ drop-in for the reference's solver class on libpmg_b200.
 *
 * pmgc_b200::PBE_linear_problem<base_length, nlev, box_length> keeps the
 * template parameters and the method names of PBE_linear_problem
 * (PBE_pmgc_class.h:112-1174), so host code written against the class
 * changes its include and namespace and passes a CUDA stream where it passed
 * the sycl::queue (PBE_pmgc_class.h:141-148). The hierarchy lives on the GPU
 * behind a pmg_problem handle (pmg_b200.h); failures throw pmg_error with
 * the library's message. Header only, C++20 (the class takes its box length
 * as a floating-point template argument, as the reference does); link with
 * -lpmg_b200.
 *
 *   pmgc_b200::PBE_linear_problem<8, 5, 102.4> pb(0.15, 2.0, stream);
 *   pb.initialize_boundary(atoms);
 *   pb.initialize_epsilons(atoms);
 *   pb.set_up_rhs(atoms);
 *   pb.buildmultilevelops();
 *   const double r0 = pb.compute_residual_2();
 *   while (pb.compute_residual_2() / r0 > 1e-10)
 *     pb.v_cycle();                   // or: pb.solve(1e-10, 100)
 *   std::vector<double> phi = pb.potential();
 */
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "pmg_b200.h"

namespace pmgc_b200 {

/* Atom of the reference (Atom_types.h:11): centre in the grid's frame
 * (Position[0] along the slowest array axis), radius and charge. */
template <typename DataType> struct Atom {
  DataType Position[3];
  DataType radius;
  DataType charge;
};

/* A failed library call: status is the PMG_ERR_* code. */
struct pmg_error : std::runtime_error {
  int status;
  pmg_error(int rc, const std::string &what)
      : std::runtime_error(what), status(rc) {}
};

inline void check(int rc, const char *call) {
  if (rc != PMG_OK)
    throw pmg_error(rc, std::string(call) + ": " + pmg_last_error());
}

/* The class's physical constants (scientific_quantities.h:14-15) with the
 * salt of the constructor; temperature 298.15 K, van der Waals dielectric
 * boundary (no probe), as the reference's set-up. */
inline pmg_physics reference_physics(double ionic_strength,
                                     double ion_radius) {
  pmg_physics ph;
  ph.eps_in = 4.0;
  ph.eps_out = 78.4;
  ph.ionic_strength = ionic_strength;
  ph.ion_radius = ion_radius;
  ph.temperature = 298.15;
  ph.probe_radius = 0.0;
  return ph;
}

/* Result of solve(): cycles run and the final relative residual. */
struct SolveResult {
  int cycles;
  double relres;
};

template <std::size_t base_length, std::size_t nlev, double box_length>
class PBE_linear_problem {
public:
  /* Points per axis of the finest level (the class's length + 2). */
  static constexpr int n = (int)(base_length << nlev) + 1;
  /* box / (base * 2^nlev), PBE_pmgc_class.h:1157-1159 */
  static constexpr double grid_step =
      box_length / ((double)base_length * (double)(1u << nlev));

  /* precision: PMG_PREC_FP64 (the reference's arithmetic) or
   * PMG_PREC_MIXED (float V-cycles inside double refinement). stream may
   * be null (the problem creates its own). */
  PBE_linear_problem(double ionic_strength, double ion_radius,
                     pmg_stream_t stream = nullptr,
                     int precision = PMG_PREC_FP64)
      : physics_(reference_physics(ionic_strength, ion_radius)) {
    check(pmg_problem_create((int)base_length, (int)nlev, box_length,
                             precision, stream, &p_),
          "pmg_problem_create");
  }
  PBE_linear_problem(const PBE_linear_problem &) = delete;
  PBE_linear_problem &operator=(const PBE_linear_problem &) = delete;
  ~PBE_linear_problem() { pmg_problem_destroy(p_); }

  /* The three set-up steps of the class (PBE_pmgc_class.h:191-349). The
   * library builds the whole finest level from the atoms on the GPU in one
   * pass, so the first of them does it and the others, given the same
   * atoms, find it done. */
  void initialize_boundary(const std::vector<Atom<double>> &atoms) {
    load(atoms);
  }
  void initialize_epsilons(const std::vector<Atom<double>> &atoms) {
    load(atoms);
  }
  void set_up_rhs(const std::vector<Atom<double>> &atoms) { load(atoms); }

  /* Prolongations and Galerkin operators of every level
   * (PBE_pmgc_class.h:351-617); trilinear: constant weights. */
  void buildmultilevelops(bool trilinear = false) {
    check(pmg_build_hierarchy(p_, trilinear ? 1 : 0), "pmg_build_hierarchy");
  }

  /* One V-cycle of the class (PBE_pmgc_class.h:1070-1114). FP64 only. */
  void v_cycle() { check(pmg_vcycle(p_, 0), "pmg_vcycle"); }

  /* sqrt(sum over the interior of (f - A x)^2 / n^3) of the finest level
   * (PBE_pmgc_class.h:768-772). */
  double compute_residual_2() {
    double r = 0;
    check(pmg_compute_residual_2(p_, &r), "pmg_compute_residual_2");
    return r;
  }

  /* The apps' loop (PBE_pmgc_class_test.cc:124-146) as one graph launch:
   * cycles until compute_residual_2()/r0 < tol, at most max_cycles. */
  SolveResult solve(double tol = 1e-10, int max_cycles = 100) {
    SolveResult s{0, 0.0};
    check(pmg_solve(p_, tol, max_cycles, &s.cycles, &s.relres, nullptr),
          "pmg_solve");
    return s;
  }

  /* The finest iterate, n^3 values including the shell (x fastest). */
  std::vector<double> potential() {
    std::vector<double> x((std::size_t)n * n * n);
    check(pmg_get_potential(p_, x.data()), "pmg_get_potential");
    return x;
  }

  pmg_problem *handle() { return p_; }

private:
  void load(const std::vector<Atom<double>> &atoms) {
    std::vector<double> rows(5 * atoms.size());
    for (std::size_t a = 0; a < atoms.size(); ++a) {
      for (int d = 0; d < 3; ++d)
        rows[5 * a + d] = atoms[a].Position[d];
      rows[5 * a + 3] = atoms[a].radius;
      rows[5 * a + 4] = atoms[a].charge;
    }
    if (loaded_ && rows == rows_)
      return;
    check(pmg_problem_set_atoms(p_, rows.data(), (int)atoms.size(),
                                &physics_),
          "pmg_problem_set_atoms");
    rows_ = std::move(rows);
    loaded_ = true;
  }

  pmg_problem *p_ = nullptr;
  pmg_physics physics_;
  std::vector<double> rows_;
  bool loaded_ = false;
};

} // namespace pmgc_b200
