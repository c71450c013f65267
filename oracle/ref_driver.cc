// extern "C" entry points of the reference-built oracle (test
// infrastructure): dispatch to the registered class instantiations and thin
// wrappers over the reference's pmgc kernels. See ref_api.h.
#include "ref_registry.h"

#include "pmgc/buildAd.h"
#include "pmgc/buildBd.h"
#include "pmgc/buildGd.h"
#include "pmgc/buildPd.h"
#include "pmgc/gsd.h"
#include "pmgc/matvecd.h"
#include "pmgc/mlinpckd.h"

#include <iostream>
#include <vector>

namespace {

std::vector<pmgref_entry> &registry() {
  static std::vector<pmgref_entry> r;
  return r;
}

const pmgref_entry *find(int base, int nlev) {
  for (const auto &e : registry())
    if (e.base == base && e.nlev == nlev)
      return &e;
  return nullptr;
}

// The reference prints progress to std::cout from inside its set-up and
// kernels; callers of the oracle (tests, the bench's JSON line) need a clean
// stdout, so every entry point mutes it for its duration.
struct quiet_cout {
  std::streambuf *old;
  quiet_cout() : old(std::cout.rdbuf(nullptr)) {}
  ~quiet_cout() {
    std::cout.rdbuf(old);
    std::cout.clear();
  }
};

sycl::queue &kq() {
  static sycl::queue q;
  return q;
}

using D = double;
D *m(const D *p) { return const_cast<D *>(p); }

} // namespace

void pmgref_register(const pmgref_entry &e) { registry().push_back(e); }

extern "C" {

int pmgref_configs(int *base, int *nlev, double *box, int cap) {
  const auto &r = registry();
  for (int i = 0; i < (int)r.size() && i < cap; ++i) {
    base[i] = r[i].base;
    nlev[i] = r[i].nlev;
    box[i] = r[i].box;
  }
  return (int)r.size();
}

int pmgref_solve(int base, int nlev, const pmgref_fine *in, double tol,
                 int max_cycles, int trilinear, double *x_out, double *hist,
                 int *cycles) {
  const pmgref_entry *e = find(base, nlev);
  if (!e)
    return -1;
  quiet_cout q;
  return e->solve(in, tol, max_cycles, trilinear, x_out, hist, cycles);
}

int pmgref_cycles(int base, int nlev, const pmgref_fine *in, int ncycles,
                  double *x_out) {
  const pmgref_entry *e = find(base, nlev);
  if (!e)
    return -1;
  quiet_cout q;
  return e->cycles(in, ncycles, x_out);
}

long pmgref_hierarchy(int base, int nlev, const pmgref_fine *in,
                      int trilinear, double *out, long cap) {
  const pmgref_entry *e = find(base, nlev);
  if (!e)
    return -1;
  quiet_cout q;
  return e->hierarchy(in, trilinear, out, cap);
}

int pmgref_cg_level1(int base, int nlev, const double *const *op14,
                     const double *rhs, double *x) {
  const pmgref_entry *e = find(base, nlev);
  if (!e)
    return -1;
  quiet_cout q;
  return e->cg_level1(op14, rhs, x);
}

int pmgref_setup(int base, int nlev, const double *atoms, int natoms,
                 double ionic_strength, double ion_radius, double *oC,
                 double *oE, double *oN, double *uC, double *f, double *x0) {
  const pmgref_entry *e = find(base, nlev);
  if (!e)
    return -1;
  quiet_cout q;
  return e->setup(atoms, natoms, ionic_strength, ion_radius, oC, oE, oN, uC,
                  f, x0);
}

int pmgref_pcg(int base, int nlev, const pmgref_fine *in, int iters,
               double *x_out) {
  const pmgref_entry *e = find(base, nlev);
  if (!e)
    return -1;
  quiet_cout q;
  return e->pcg(in, iters, x_out);
}

int pmgref_Vgsrb7x(int nx, int ny, int nz, const double *oC, const double *cc,
                   const double *fc, const double *oE, const double *oN,
                   const double *uC, double *x, int itmax, int iadjoint,
                   int zero_init) {
  quiet_cout q;
  pmgc::Vgsrb7x<D>(nx, ny, nz, m(oC), m(cc), m(fc), m(oE), m(oN), m(uC), x,
                   &itmax, iadjoint, kq(), zero_init != 0);
  return 0;
}

int pmgref_Vgsrb27x(int nx, int ny, int nz, const double *const *a,
                    const double *cc, const double *fc, double *x, int itmax,
                    int iadjoint, int zero_init) {
  quiet_cout q;
  pmgc::Vgsrb27x<D>(nx, ny, nz, m(a[0]), m(cc), m(fc), m(a[1]), m(a[2]),
                    m(a[3]), m(a[4]), m(a[5]), m(a[6]), m(a[7]), m(a[8]),
                    m(a[9]), m(a[10]), m(a[11]), m(a[12]), m(a[13]), x, &itmax,
                    kq(), zero_init != 0, iadjoint);
  return 0;
}

int pmgref_Vmatvec7_1s(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *oE, const double *oN,
                       const double *uC, const double *x, double *y) {
  quiet_cout q;
  pmgc::Vmatvec7_1s<D>(&nx, &ny, &nz, nullptr, nullptr, m(oC), m(cc), m(oE),
                       m(oN), m(uC), m(x), y, kq());
  return 0;
}

int pmgref_Vmatvec27_1s(int nx, int ny, int nz, const double *const *a,
                        const double *cc, const double *x, double *y) {
  quiet_cout q;
  pmgc::Vmatvec27_1s<D>(&nx, &ny, &nz, nullptr, nullptr, m(a[0]), m(cc),
                        m(a[1]), m(a[2]), m(a[3]), m(a[4]), m(a[5]), m(a[6]),
                        m(a[7]), m(a[8]), m(a[9]), m(a[10]), m(a[11]),
                        m(a[12]), m(a[13]), m(x), y, kq());
  return 0;
}

int pmgref_Vmresid7_1s(int nx, int ny, int nz, const double *oC,
                       const double *cc, const double *fc, const double *oE,
                       const double *oN, const double *uC, const double *x,
                       double *r) {
  quiet_cout q;
  pmgc::Vmresid7_1s<D>(&nx, &ny, &nz, nullptr, nullptr, m(oC), m(cc), m(fc),
                       m(oE), m(oN), m(uC), m(x), r, kq());
  return 0;
}

int pmgref_Vmresid27_1s(int nx, int ny, int nz, const double *const *a,
                        const double *cc, const double *fc, const double *x,
                        double *r) {
  quiet_cout q;
  pmgc::Vmresid27_1s<D>(&nx, &ny, &nz, nullptr, nullptr, m(a[0]), m(cc),
                        m(fc), m(a[1]), m(a[2]), m(a[3]), m(a[4]), m(a[5]),
                        m(a[6]), m(a[7]), m(a[8]), m(a[9]), m(a[10]), m(a[11]),
                        m(a[12]), m(a[13]), m(x), r, kq());
  return 0;
}

#define P27(p)                                                                 \
  m(p[0]), m(p[1]), m(p[2]), m(p[3]), m(p[4]), m(p[5]), m(p[6]), m(p[7]),     \
      m(p[8]), m(p[9]), m(p[10]), m(p[11]), m(p[12]), m(p[13]), m(p[14]),      \
      m(p[15]), m(p[16]), m(p[17]), m(p[18]), m(p[19]), m(p[20]), m(p[21]),    \
      m(p[22]), m(p[23]), m(p[24]), m(p[25]), m(p[26])

int pmgref_Vrestrc2(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                    const double *xin, double *xout,
                    const double *const *p) {
  quiet_cout q;
  pmgc::Vrestrc2<D>(nxf, nyf, nzf, nxc, nyc, nzc, m(xin), xout, P27(p), kq());
  return 0;
}

int pmgref_VinterpPMG2(int nxc, int nyc, int nzc, int nxf, int nyf, int nzf,
                       const double *xin, double *xout,
                       const double *const *p) {
  quiet_cout q;
  pmgc::VinterpPMG2<D>(nxc, nyc, nzc, nxf, nyf, nzf, m(xin), xout, P27(p),
                       kq());
  return 0;
}

int pmgref_VbuildPb_op7(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                        const double *oC, const double *oE, const double *oN,
                        const double *uC, double *const *p) {
  quiet_cout q;
  pmgc::VbuildPb_op7<D>(nxf, nyf, nzf, nxc, nyc, nzc, m(oC), m(oE), m(oN),
                        m(uC), P27(p), kq());
  return 0;
}

int pmgref_VbuildPb_op27(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                         const double *const *a, double *const *p) {
  quiet_cout q;
  pmgc::VbuildPb_op27<D>(nxf, nyf, nzf, nxc, nyc, nzc, m(a[0]), m(a[1]),
                         m(a[2]), m(a[3]), m(a[4]), m(a[5]), m(a[6]), m(a[7]),
                         m(a[8]), m(a[9]), m(a[10]), m(a[11]), m(a[12]),
                         m(a[13]), P27(p), kq());
  return 0;
}

int pmgref_VbuildPb_trilin(int nxf, int nyf, int nzf, int nxc, int nyc,
                           int nzc, double *const *p) {
  quiet_cout q;
  pmgc::VbuildPb_trilin<D>(nxf, nyf, nzf, nxc, nyc, nzc, P27(p), kq());
  return 0;
}

int pmgref_VbuildG_7(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                     const double *const *p, const double *oC,
                     const double *oE, const double *oN, const double *uC,
                     double *const *o) {
  quiet_cout q;
  pmgc::VbuildG_7<D>(nxf, nyf, nzf, nxc, nyc, nzc, P27(p), m(oC), m(oE),
                     m(oN), m(uC), o[0], o[1], o[2], o[3], o[4], o[5], o[6],
                     o[7], o[8], o[9], o[10], o[11], o[12], o[13], kq());
  return 0;
}

int pmgref_VbuildG_27(int nxf, int nyf, int nzf, int nxc, int nyc, int nzc,
                      const double *const *p, const double *const *a,
                      double *const *o) {
  quiet_cout q;
  pmgc::VbuildG_27<D>(nxf, nyf, nzf, nxc, nyc, nzc, P27(p), m(a[0]), m(a[1]),
                      m(a[2]), m(a[3]), m(a[4]), m(a[5]), m(a[6]), m(a[7]),
                      m(a[8]), m(a[9]), m(a[10]), m(a[11]), m(a[12]), m(a[13]),
                      o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8],
                      o[9], o[10], o[11], o[12], o[13], kq());
  return 0;
}

int pmgref_VbuildA_fv(int nx, int ny, int nz, int ipkey, int *numdia,
                      int *ipc, double *oC, double *cc, double *fc,
                      double *oE, double *oN, double *uC, const double *xf,
                      const double *yf, const double *zf, const double *gxcf,
                      const double *gycf, const double *gzcf,
                      const double *a1cf, const double *a2cf,
                      const double *a3cf, const double *ccf,
                      const double *fcf) {
  quiet_cout q;
  pmgc::VbuildA_fv<D>(&nx, &ny, &nz, &ipkey, numdia, ipc, nullptr, oC, cc,
                      fc, oE, oN, uC, m(xf), m(yf), m(zf), m(gxcf), m(gycf),
                      m(gzcf), m(a1cf), m(a2cf), m(a3cf), m(ccf), m(fcf),
                      kq());
  return 0;
}

int pmgref_Vbuildband(int nx, int ny, int nz, int numdia, double *ac,
                      int *ipcB, double *acB) {
  quiet_cout q;
  int ipc[12] = {0};
  ipc[10] = numdia;
  int key = -1;
  pmgc::Vbuildband<D>(&key, &nx, &ny, &nz, ipc, nullptr, ac, ipcB, nullptr,
                      acB, kq());
  return key;
}

int pmgref_Vdpbfa(double *abd, int lda, int n, int m) {
  int info = -1;
  pmgc::Vdpbfa<D>(abd, &lda, &n, &m, &info);
  return info;
}

int pmgref_Vdpbsl(double *abd, int lda, int n, int m, double *b) {
  pmgc::Vdpbsl<D>(abd, &lda, &n, &m, b);
  return 0;
}

} // extern "C"
