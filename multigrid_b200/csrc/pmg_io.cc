// File formats around the solve: PQR atoms in, OpenDX potential out.
//
// read: the reference's PQR reader (read_pqr_file, fileio.cc:10-53) takes
// every line with exactly ten whitespace-separated fields that is not a
// REMARK and reads x y z from fields 6-8, the charge from field 9 and the
// radius from field 10 (1-based). Blank lines are skipped (the reference
// indexes an empty field list there).
//
// write: the reference's OpenDX writer (Grid::print_dx_to_stream,
// Domain.h:136-185): gridpositions header with the counts slowest axis
// first (nz ny nx, OpenDX's order: the last count varies fastest), origin,
// and the three axis deltas box / (nz - 1) (the reference's spacing of its
// first, slowest axis), then the values in array order, three per line,
// each formatted as a left-aligned, explicitly signed, 13-wide exponent
// number followed by a space, then the field trailer.
#include <stdio.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pmg_b200.h"

namespace {

void put_value(FILE *f, double v) { fprintf(f, "%-+13e ", v); }

} // namespace

extern "C" {

int pmg_read_pqr(const char *path, double *atoms, int cap, int *count) {
  if (!path || !count || cap < 0 || (cap > 0 && !atoms))
    return PMG_ERR_ARG;
  std::ifstream file(path);
  if (!file.is_open())
    return PMG_ERR_ARG;
  int n = 0;
  std::string line;
  while (std::getline(file, line)) {
    std::istringstream iss(line);
    std::vector<std::string> li;
    for (std::string s; iss >> s;)
      li.push_back(s);
    if (li.empty() || li[0] == "REMARK" || li.size() != 10)
      continue;
    double v[5];
    try {
      v[0] = std::stod(li[5]);
      v[1] = std::stod(li[6]);
      v[2] = std::stod(li[7]);
      v[4] = std::stod(li[8]); // charge
      v[3] = std::stod(li[9]); // radius
    } catch (...) {
      return PMG_ERR_ARG;
    }
    if (atoms && n < cap)
      memcpy(atoms + 5 * (size_t)n, v, sizeof(v));
    ++n;
  }
  *count = n;
  return (atoms && n > cap) ? PMG_ERR_ARG : PMG_OK;
}

int pmg_write_dx(const char *path, const double *values, int nx, int ny,
                 int nz, double xmin, double ymin, double zmin,
                 double box_length) {
  if (!path || !values || nx < 2 || ny < 2 || nz < 2)
    return PMG_ERR_ARG;
  FILE *f = fopen(path, "w");
  if (!f)
    return PMG_ERR_ARG;
  const double delta = box_length / (double)(nz - 1);
  const long count = (long)nx * ny * nz;
  fprintf(f, "object 1 class gridpositions counts %d %d %d\n", nz, ny, nx);
  fprintf(f, "origin ");
  put_value(f, xmin);
  put_value(f, ymin);
  put_value(f, zmin);
  fprintf(f, "\n");
  for (int axis = 0; axis < 3; ++axis) {
    fprintf(f, "delta ");
    for (int c = 0; c < 3; ++c)
      put_value(f, c == axis ? delta : 0.0);
    fprintf(f, "\n");
  }
  fprintf(f, "object 2 class gridconnections count %d %d %d\n", nz, ny, nx);
  fprintf(f, "object 3 class array type double rank 0 items %ld data follows\n",
          count);
  for (long i = 0; i < count; ++i) {
    if (i % 3 == 0 && i != 0)
      fprintf(f, "\n");
    put_value(f, values[i]);
  }
  fprintf(f, "\n");
  fprintf(f, "attribute \"dep\" string \"positions\"\n");
  fprintf(f, "object \"regular positions regular connections\" class field\n");
  fprintf(f, "component \"positions\" value 1\n");
  fprintf(f, "component \"connections\" value 2\n");
  fprintf(f, "component \"data\" value 3\n");
  const int bad = ferror(f);
  fclose(f);
  return bad ? PMG_ERR_ARG : PMG_OK;
}

} // extern "C"
