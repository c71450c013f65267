// Command-line front end of the reference's OpenDX writer (test
// infrastructure): reads a little-endian double array from a file and
// prints the reference's print_dx_to_stream text (pmgref_write_dx) to
// stdout. A separate process keeps the reference's iostream and std::format
// use away from the interpreter that runs the tests.
//
//   ref_dx <shape> <values.bin> <xmin> <ymin> <zmin> <box>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ref_api.h"

int main(int argc, char **argv) {
  if (argc != 7)
    return 2;
  std::FILE *f = std::fopen(argv[2], "rb");
  if (!f)
    return 3;
  std::vector<double> v;
  double x;
  while (std::fread(&x, sizeof x, 1, f) == 1)
    v.push_back(x);
  std::fclose(f);
  std::vector<char> out(64 * v.size() + 4096);
  const long n = pmgref_write_dx(std::atoi(argv[1]), v.data(),
                                 std::atof(argv[3]), std::atof(argv[4]),
                                 std::atof(argv[5]), std::atof(argv[6]),
                                 out.data(), (long)out.size());
  if (n <= 0)
    return 4;
  std::fwrite(out.data(), 1, (size_t)n, stdout);
  return 0;
}
