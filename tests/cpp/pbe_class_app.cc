// A host program written against the reference's PBE_linear_problem,
// moved to pmgc_b200 (include/PBE_pmgc_class_b200.h): reads atoms, sets up
// the 65^3 problem (base 4, 4 levels, box 32 A), builds the hierarchy and
// runs the class's V-cycle loop to a relative residual of 1e-10, then the
// same problem through solve(). Writes both potentials (n^3 doubles each)
// and the cycle counts.
//   pbe_class_app atoms.bin out.bin   (atoms.bin: rows x y z radius charge)
#include <cstdio>
#include <vector>

#include "PBE_pmgc_class_b200.h"

using Problem = pmgc_b200::PBE_linear_problem<4, 4, 32.0>;

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s atoms.bin out.bin\n", argv[0]);
    return 2;
  }
  std::FILE *f = std::fopen(argv[1], "rb");
  if (!f)
    return 2;
  std::vector<pmgc_b200::Atom<double>> atoms;
  double row[5];
  while (std::fread(row, sizeof(double), 5, f) == 5)
    atoms.push_back({{row[0], row[1], row[2]}, row[3], row[4]});
  std::fclose(f);
  try {
    // the class's loop, cycle by cycle
    Problem pb(0.15, 2.0);
    pb.initialize_boundary(atoms);
    pb.initialize_epsilons(atoms);
    pb.set_up_rhs(atoms);
    pb.buildmultilevelops();
    const double r0 = pb.compute_residual_2();
    int cycles = 0;
    while (pb.compute_residual_2() / r0 >= 1e-10 && cycles < 100) {
      pb.v_cycle();
      ++cycles;
    }
    const std::vector<double> x1 = pb.potential();
    // the same solve in one call
    Problem pb2(0.15, 2.0);
    pb2.initialize_boundary(atoms);
    pb2.initialize_epsilons(atoms);
    pb2.set_up_rhs(atoms);
    pb2.buildmultilevelops();
    const pmgc_b200::SolveResult s = pb2.solve(1e-10, 100);
    const std::vector<double> x2 = pb2.potential();
    std::FILE *o = std::fopen(argv[2], "wb");
    if (!o)
      return 2;
    std::fwrite(x1.data(), sizeof(double), x1.size(), o);
    std::fwrite(x2.data(), sizeof(double), x2.size(), o);
    std::fclose(o);
    std::printf("%d %d %.6e\n", cycles, s.cycles, s.relres);
  } catch (const pmgc_b200::pmg_error &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
