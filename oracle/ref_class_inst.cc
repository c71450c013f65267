// One instantiation of the reference's PMG problem class for the oracle
// (test infrastructure). Compiled once per grid with
//   -DPMG_BASE=<base_length> -DPMG_NLEV=<nlev> -DPMG_BOX=<box_length>
// and registered under (base, nlev). Every function below drives the
// reference's own class methods; the only thing it adds is copying host arrays
// in and out of the class's hierarchies (the shim's "device" memory is host
// memory).
#include "PBE_pmgc_class.h"

#include "ref_registry.h"

#include <cstring>
#include <memory>
#include <utility>
#include <vector>

namespace {

constexpr std::size_t kBase = PMG_BASE;
constexpr std::size_t kNlev = PMG_NLEV;
constexpr ::DataType kBox = PMG_BOX;

using Problem = pmgc_solver::PBE_linear_problem<kBase, kNlev, kBox>;

sycl::queue &oracle_queue() {
  static sycl::queue q;
  return q;
}

template <std::size_t L> constexpr std::size_t npts() {
  const std::size_t n = kBase * (std::size_t(1) << L) + 1;
  return n * n * n;
}

template <typename G> void put(G &grid, const double *src) {
  std::memcpy(grid.values_buff, src, sizeof(double) * grid.num_values);
}
template <typename G> void get(const G &grid, double *dst) {
  std::memcpy(dst, grid.values_buff, sizeof(double) * grid.num_values);
}

std::unique_ptr<Problem> make_problem(const pmgref_fine *in) {
  // The ionic strength / ion radius only matter for the class's own set-up,
  // which the solve entry points replace with the caller's fine arrays.
  auto p = std::make_unique<Problem>(0.0, 0.0, oracle_queue());
  if (in) {
    put(p->epsilon_oC_map.template get_domain<kNlev>(), in->oC);
    put(p->epsilon_oE_map.template get_domain<kNlev>(), in->oE);
    put(p->epsilon_oN_map.template get_domain<kNlev>(), in->oN);
    put(p->epsilon_uC_map.template get_domain<kNlev>(), in->uC);
    put(p->rhs_domain.template get_domain<kNlev>(), in->f);
    put(p->sol.template get_domain<kNlev>(), in->x0);
  }
  return p;
}

void build(Problem &p, int trilinear) {
  if (trilinear)
    p.template buildmultilevelops<std::true_type>();
  else
    p.template buildmultilevelops<std::false_type>();
}

int solve(const pmgref_fine *in, double tol, int max_cycles, int trilinear,
          double *x_out, double *hist, int *cycles) {
  auto p = make_problem(in);
  build(*p, trilinear);
  const double r0 = p->compute_residual_2();
  if (hist)
    hist[0] = r0;
  int c = 0;
  while (c < max_cycles) {
    p->template v_cycle<std::false_type>();
    ++c;
    const double r = p->compute_residual_2();
    if (hist)
      hist[c] = r;
    if (r / r0 < tol)
      break;
  }
  if (cycles)
    *cycles = c;
  if (x_out)
    get(p->sol.template get_domain<kNlev>(), x_out);
  return 0;
}

int cycles_only(const pmgref_fine *in, int ncycles, double *x_out) {
  auto p = make_problem(in);
  build(*p, 0);
  for (int c = 0; c < ncycles; ++c)
    p->template v_cycle<std::false_type>();
  if (x_out)
    get(p->sol.template get_domain<kNlev>(), x_out);
  return 0;
}

template <std::size_t L>
void dump_level(Problem &p, double *&out) {
  auto emit = [&](auto &hier) {
    auto &g = hier.template get_domain<L>();
    get(g, out);
    out += g.num_values;
  };
  emit(p.oPC); emit(p.oPN); emit(p.oPS); emit(p.oPE); emit(p.oPW);
  emit(p.oPNE); emit(p.oPNW); emit(p.oPSE); emit(p.oPSW);
  emit(p.uPC); emit(p.uPN); emit(p.uPS); emit(p.uPE); emit(p.uPW);
  emit(p.uPNE); emit(p.uPNW); emit(p.uPSE); emit(p.uPSW);
  emit(p.dPC); emit(p.dPN); emit(p.dPS); emit(p.dPE); emit(p.dPW);
  emit(p.dPNE); emit(p.dPNW); emit(p.dPSE); emit(p.dPSW);
  emit(p.epsilon_oC_map); emit(p.epsilon_oE_map); emit(p.epsilon_oN_map);
  emit(p.epsilon_uC_map); emit(p.epsilon_oNE_map); emit(p.epsilon_oNW_map);
  emit(p.epsilon_uE_map); emit(p.epsilon_uW_map); emit(p.epsilon_uN_map);
  emit(p.epsilon_uS_map); emit(p.epsilon_uNE_map); emit(p.epsilon_uNW_map);
  emit(p.epsilon_uSE_map); emit(p.epsilon_uSW_map);
}

template <std::size_t... I>
void dump_all(Problem &p, double *out, std::index_sequence<I...>) {
  // I = 0 .. nlev-2  ->  level nlev-1-I (finest coarse level first)
  (dump_level<kNlev - 1 - I>(p, out), ...);
}

template <std::size_t... I>
constexpr long hierarchy_size(std::index_sequence<I...>) {
  return (0L + ... + (41L * (long)npts<kNlev - 1 - I>()));
}

long hierarchy(const pmgref_fine *in, int trilinear, double *out, long cap) {
  constexpr auto seq = std::make_index_sequence<kNlev - 1>{};
  constexpr long need = hierarchy_size(seq);
  if (cap < need)
    return -1;
  auto p = make_problem(in);
  build(*p, trilinear);
  dump_all(*p, out, seq);
  return need;
}

int cg_level1(const double *const *op14, const double *rhs, double *x) {
  auto p = make_problem(nullptr);
  put(p->epsilon_oC_map.template get_domain<1>(), op14[0]);
  put(p->epsilon_oE_map.template get_domain<1>(), op14[1]);
  put(p->epsilon_oN_map.template get_domain<1>(), op14[2]);
  put(p->epsilon_uC_map.template get_domain<1>(), op14[3]);
  put(p->epsilon_oNE_map.template get_domain<1>(), op14[4]);
  put(p->epsilon_oNW_map.template get_domain<1>(), op14[5]);
  put(p->epsilon_uE_map.template get_domain<1>(), op14[6]);
  put(p->epsilon_uW_map.template get_domain<1>(), op14[7]);
  put(p->epsilon_uN_map.template get_domain<1>(), op14[8]);
  put(p->epsilon_uS_map.template get_domain<1>(), op14[9]);
  put(p->epsilon_uNE_map.template get_domain<1>(), op14[10]);
  put(p->epsilon_uNW_map.template get_domain<1>(), op14[11]);
  put(p->epsilon_uSE_map.template get_domain<1>(), op14[12]);
  put(p->epsilon_uSW_map.template get_domain<1>(), op14[13]);
  put(p->rhs_domain.template get_domain<1>(), rhs);
  put(p->sol.template get_domain<1>(), x);
  p->template solve_by_cg<1>(Float<(::DataType)1e-8>{});
  get(p->sol.template get_domain<1>(), x);
  return 0;
}

int setup(const double *atoms, int natoms, double ionic_strength,
          double ion_radius, double *oC, double *oE, double *oN, double *uC,
          double *f, double *x0) {
  std::vector<Atom<::DataType>> list(static_cast<std::size_t>(natoms));
  for (int a = 0; a < natoms; ++a) {
    list[a].Position = {atoms[5 * a + 0], atoms[5 * a + 1], atoms[5 * a + 2]};
    list[a].radius = atoms[5 * a + 3];
    list[a].charge = atoms[5 * a + 4];
  }
  auto p = std::make_unique<Problem>(ionic_strength, ion_radius,
                                     oracle_queue());
  p->initialize_boundary(list);
  p->initialize_epsilons(list);
  p->set_up_rhs(list);
  get(p->epsilon_oC_map.template get_domain<kNlev>(), oC);
  get(p->epsilon_oE_map.template get_domain<kNlev>(), oE);
  get(p->epsilon_oN_map.template get_domain<kNlev>(), oN);
  get(p->epsilon_uC_map.template get_domain<kNlev>(), uC);
  get(p->rhs_domain.template get_domain<kNlev>(), f);
  get(p->sol.template get_domain<kNlev>(), x0);
  return 0;
}

// The app's MG-preconditioned CG (PBE_pmgc_class_with_non_zero_IS.cc:
// 118-131): general CG solver over the class's finest map, the class itself
// as preconditioner, counting criterion.
int pcg(const pmgref_fine *in, int iters, double *x_out) {
  auto p = make_problem(in);
  build(*p, 0);
  auto &sol = p->sol.template get_domain<kNlev>();
  using D = std::remove_reference_t<decltype(sol)>;
  D init_guess(Paddings::PERIODIC, oracle_queue(), 1),
      rhs(Paddings::PERIODIC, oracle_queue(), 1);
  put(init_guess, in->x0);
  put(rhs, in->f);
  // the app's class never gets a boundary: its finest iterate is zero
  std::memset(sol.values_buff, 0, sizeof(::DataType) * sol.num_values);
  auto main_solver = cg_solver::make_general_solver<::DataType>(sol);
  cg_solver::counting_criterion counter((std::size_t)iters);
  auto map = p->get_map();
  main_solver(init_guess, rhs, map, counter, *p, false);
  get(init_guess, x_out);
  return 0;
}

struct registrar {
  registrar() {
    pmgref_register(pmgref_entry{(int)kBase, (int)kNlev, (double)kBox, solve,
                                 cycles_only, hierarchy, cg_level1, setup,
                                 pcg});
  }
} the_registrar;

} // namespace
