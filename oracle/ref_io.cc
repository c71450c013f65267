// The reference's PQR reader and OpenDX writer behind a C interface (test
// infrastructure). read_pqr_file (fileio.cc:10-53) is compiled from the
// reference's own fileio.cc; print_dx_to_stream (Domain.h:136-185) is the
// member of the reference's domain::Grid, instantiated here on two grid
// shapes. Nothing is added but copying values in and text out.
#include "Domain.h"
#include "fileio.h"

#include <cstring>
#include <list>
#include <sstream>
#include <string>

#include "ref_api.h"

namespace {

sycl::queue &io_queue() {
  static sycl::queue q;
  return q;
}

template <std::size_t A, std::size_t B, std::size_t C>
long write_dx(const double *values, double xmin, double ymin, double zmin,
              double box, char *out, long cap) {
  domain::Grid<double, 3, A, B, C> g(Paddings::ZERO, io_queue(), 1);
  std::memcpy(g.values_buff, values, sizeof(double) * g.num_values);
  std::ostringstream os;
  g.print_dx_to_stream(os, xmin, ymin, zmin, box);
  sycl::free(g.values_buff, io_queue()); // the Grid itself does not free
  const std::string s = os.str();
  if ((long)s.size() + 1 > cap)
    return -(long)s.size() - 1;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return (long)s.size();
}

} // namespace

extern "C" {

int pmgref_read_pqr(const char *path, double *atoms, int cap, int *count) {
  std::string name(path);
  std::list<Atom<DataType>> list;
  read_pqr_file(name, list);
  int n = 0;
  for (const auto &a : list) {
    if (n < cap) {
      atoms[5 * n + 0] = a.Position[0];
      atoms[5 * n + 1] = a.Position[1];
      atoms[5 * n + 2] = a.Position[2];
      atoms[5 * n + 3] = a.radius;
      atoms[5 * n + 4] = a.charge;
    }
    ++n;
  }
  *count = n;
  return n > cap ? -1 : 0;
}

long pmgref_write_dx(int shape, const double *values, double xmin,
                     double ymin, double zmin, double box, char *out,
                     long cap) {
  // interior lengths (slowest axis first) plus a one-point padding
  switch (shape) {
  case 0:
    return write_dx<4, 5, 6>(values, xmin, ymin, zmin, box, out, cap);
  case 1:
    return write_dx<7, 7, 7>(values, xmin, ymin, zmin, box, out, cap);
  default:
    return 0;
  }
}

} // extern "C"
