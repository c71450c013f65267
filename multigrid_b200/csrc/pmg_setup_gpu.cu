// Fine-level set-up from atoms on the GPU: the host set-up of pmg_setup.cc
// (the reference class's initialize_epsilons, set_up_rhs and
// initialize_boundary, PBE_pmgc_class.h:141-349) restated as kernels, so a
// request only moves its atoms to the device instead of six n^3 arrays.
//
//   marking   every sphere (atom, inflated atom, probe) marks the grid points
//             the host's sphere walk marks (same index bounds, same chord
//             square roots); marks are idempotent, so any order gives the
//             host's masks bit for bit.
//   probes    the accessibility test of each probe centre is an OR over all
//             other inflated spheres (the host's cell list only skips atoms
//             that cannot contain the point); probe centres use the host's
//             direction table, so they are the same doubles.
//   oC        the host's per-point sum, same order.
//   charges   the trilinear contributions are sorted by grid point with a
//             stable sort over records generated in atom order, and each
//             point sums its run in that order: the host's serial sum, bit
//             for bit.
//   boundary  the multiple Debye-Hueckel sum over atoms in order on the six
//             faces; exp() is CUDA's, so values agree with the host's to a
//             few ulp.
// All work is stream-ordered on the caller's stream; scratch comes from the
// library's stream-ordered pool.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pmg_common.cuh"
#include "pmg_physics.h"

namespace pmg {
namespace {

constexpr int kSetupThreads = 256;

struct SphereSet {
  const double *centers; // rows of `stride` doubles, x y z first
  int stride;
  int count;
  const double *radius; // radius of row q at radius[q * stride] or null
  double radius_add;    // added to the row radius (or the radius if null)
  const unsigned char *use; // row q used only when use[q] != 0 (or null)
  int axis;                 // centre shifted by -h/2 along this axis (-1: no)
};

// Marks the grid points of every sphere of a set (for_dots_in_sphere of the
// host set-up): axis-0 range ceil((c0 - r)/h) .. trunc((c0 + r)/h), chord
// half-widths from sqrt of the clamped squared remainders on axes 1 and 2.
// One block per sphere; threads over the (i0, i1) bounding rectangle.
template <typename M>
__global__ void __launch_bounds__(kSetupThreads)
    mark_spheres_kernel(int n, double h, SphereSet set, M *mask, M value) {
  const int q = blockIdx.x;
  if (q >= set.count || (set.use && !set.use[q]))
    return;
  const double *row = set.centers + (size_t)q * set.stride;
  double c[3] = {row[0], row[1], row[2]};
  if (set.axis >= 0)
    c[set.axis] -= 0.5 * h;
  const double r = set.radius ? set.radius[(size_t)q * set.stride] +
                                    set.radius_add
                              : set.radius_add;
  const int lo0 = (int)ceil((c[0] - r) / h);
  const int hi0 = (int)((c[0] + r) / h);
  const int blo1 = (int)ceil((c[1] - r) / h) - 1;
  const int bhi1 = (int)((c[1] + r) / h) + 1;
  const int w0 = hi0 - lo0 + 1, w1 = bhi1 - blo1 + 1;
  if (w0 <= 0 || w1 <= 0)
    return;
  for (int t = threadIdx.x; t < w0 * w1; t += blockDim.x) {
    const int i0 = lo0 + t / w1, i1 = blo1 + t % w1;
    double s1 = r * r - ((c[0] - h * i0) * (c[0] - h * i0));
    if (s1 < 0)
      s1 = 0;
    const double ww1 = sqrt(s1);
    const int lo1 = (int)ceil((c[1] - ww1) / h);
    const int hi1 = (int)((c[1] + ww1) / h);
    if (i1 < lo1 || i1 > hi1)
      continue;
    double s2 = r * r - ((c[0] - h * i0) * (c[0] - h * i0) +
                         (c[1] - h * i1) * (c[1] - h * i1));
    if (s2 < 0)
      s2 = 0;
    const double ww2 = sqrt(s2);
    const int lo2 = (int)ceil((c[2] - ww2) / h);
    const int hi2 = (int)((c[2] + ww2) / h);
    if (i0 < 0 || i1 < 0 || i0 >= n || i1 >= n)
      continue;
    for (int i2 = lo2 < 0 ? 0 : lo2; i2 <= hi2 && i2 < n; ++i2)
      mask[((size_t)i0 * n + i1) * n + i2] = value;
  }
}

__global__ void face_from_masks_kernel(long count, const unsigned char *inside,
                                       const unsigned char *sas,
                                       const unsigned char *carved,
                                       double v_in, double v_out,
                                       double *face) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < count;
       q += (long)gridDim.x * blockDim.x) {
    const bool solute = inside[q] || (sas && sas[q] && !carved[q]);
    face[q] = solute ? v_in : v_out;
  }
}

// oC = sum of the six faces (+ kappa^2 eps_out outside the ion-exclusion
// spheres) on the interior, 0 on the shell; the host's summation order.
__global__ void centre_kernel(int n, const double *uC, const double *oN,
                              const double *oE, const unsigned char *ion,
                              double kterm, double *oC) {
  const long n3 = (long)n * n * n;
  const long s1 = n, s0 = (long)n * n;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n3;
       q += (long)gridDim.x * blockDim.x) {
    const long i0 = q / s0, i1 = (q / s1) % n, i2 = q % n;
    if (i0 < 1 || i1 < 1 || i2 < 1 || i0 > n - 2 || i1 > n - 2 ||
        i2 > n - 2) {
      oC[q] = 0.0;
      continue;
    }
    double c = ((uC[q] + uC[q - s0]) + (oN[q] + oN[q - s1])) +
               (oE[q] + oE[q - 1]);
    c += ion[q] ? 0.0 : kterm;
    oC[q] = c;
  }
}

// Trilinear charge records in atom order: key = grid point (or INT_MAX when
// the corner is outside the grid), value = 8 * atom + corner.
__global__ void charge_records_kernel(const double *atoms, int natoms, int n,
                                      double h, int *keys, int *vals) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= 8 * natoms)
    return;
  const int a = r >> 3, corner = r & 7;
  long c[3];
  for (int d = 0; d < 3; ++d) {
    const double s = atoms[5 * a + d] / h;
    const long lo = (long)s;
    c[d] = lo + ((corner >> d) & 1);
  }
  const bool in = c[0] < n && c[1] < n && c[2] < n;
  keys[r] = in ? (int)((c[0] * n + c[1]) * n + c[2]) : 0x7fffffff;
  vals[r] = r;
}

// Sums every run of equal keys in record order (= atom order):
// f[q] = ((0 + t_1) + t_2) + ..., t = charge * wt / vol as on the host.
__global__ void charge_sum_kernel(const double *atoms, int nrec, double h,
                                  double eps0, double vol,
                                  const int *keys, const int *vals,
                                  double *f) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec || keys[r] == 0x7fffffff)
    return;
  if (r > 0 && keys[r - 1] == keys[r])
    return; // not the head of its run
  double acc = 0.0;
  for (int t = r; t < nrec && keys[t] == keys[r]; ++t) {
    const int a = vals[t] >> 3, corner = vals[t] & 7;
    const double charge = atoms[5 * a + 4] / eps0;
    double wt = 1;
    for (int d = 0; d < 3; ++d) {
      const double s = atoms[5 * a + d] / h;
      const long lo = (long)s;
      const double w = ((corner >> d) & 1) ? (s - lo) : (lo + 1 - s);
      wt *= w;
    }
    acc += charge * wt / vol;
  }
  f[keys[r]] = acc;
}

// Probe centres on the sphere of radius r_a + probe around every atom; a
// centre is kept when no other inflated sphere contains it
// (d^2 < R_b^2 (1 - 1e-12), the host's test). Output rows (x, y, z). The
// atoms are found through a cell list: a centre lies within the largest
// inflated radius (<= the cell edge) of any sphere containing it, so only
// the 27 cells around it are searched; "kept" is an AND over atoms, so the
// order of the atoms within a cell does not matter.
__global__ void __launch_bounds__(kSetupThreads)
    probe_centres_cells_kernel(const double *atoms, int natoms, double probe,
                               const ProbeDir *dirs, double cell, int dim,
                               const int *cell_start, const int *cell_atoms,
                               double *centres, unsigned char *free_flag) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= (long)natoms * kProbePoints)
    return;
  const int a = (int)(g / kProbePoints), s = (int)(g % kProbePoints);
  const double R = atoms[5 * a + 3] + probe;
  const ProbeDir u = dirs[s];
  double pc[3];
  pc[0] = atoms[5 * a] + R * u.rr * u.c;
  pc[1] = atoms[5 * a + 1] + R * u.rr * u.s;
  pc[2] = atoms[5 * a + 2] + R * u.zz;
  int cc[3];
  for (int d = 0; d < 3; ++d)
    cc[d] = (int)floor(pc[d] / cell);
  bool free = true;
  for (int dz = -1; dz <= 1 && free; ++dz)
    for (int dy = -1; dy <= 1 && free; ++dy)
      for (int dx = -1; dx <= 1 && free; ++dx) {
        const int c0 = cc[0] + dx, c1 = cc[1] + dy, c2 = cc[2] + dz;
        if (c0 < 0 || c1 < 0 || c2 < 0 || c0 >= dim || c1 >= dim ||
            c2 >= dim)
          continue;
        const int cid = (c2 * dim + c1) * dim + c0;
        for (int q = cell_start[cid]; q < cell_start[cid + 1]; ++q) {
          const int b = cell_atoms[q];
          if (b == a)
            continue;
          const double Rb = atoms[5 * b + 3] + probe;
          double d2 = 0;
          for (int d = 0; d < 3; ++d) {
            const double e = pc[d] - atoms[5 * b + d];
            d2 += e * e;
          }
          if (d2 < Rb * Rb * (1 - 1e-12)) {
            free = false;
            break;
          }
        }
      }
  centres[3 * g + 0] = pc[0];
  centres[3 * g + 1] = pc[1];
  centres[3 * g + 2] = pc[2];
  free_flag[g] = free ? 1 : 0;
}

// Cell list of the atoms: cell of each atom and per-cell counts
__global__ void atom_cells_kernel(const double *atoms, int natoms, double cell,
                                  int dim, int *cid, int *count) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms)
    return;
  int c[3];
  for (int d = 0; d < 3; ++d)
    c[d] = min((int)floor(atoms[5 * a + d] / cell), dim - 1);
  cid[a] = (c[2] * dim + c[1]) * dim + c[0];
  atomicAdd(&count[cid[a]], 1);
}

// atoms into their cells' ranges (fill: a copy of the ranges' starts)
__global__ void atom_scatter_kernel(int natoms, const int *cid, int *fill,
                                    int *cell_atoms) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < natoms)
    cell_atoms[atomicAdd(&fill[cid[a]], 1)] = a;
}

// Multiple Debye-Hueckel values on the six faces (atoms in order); faces
// share their edges, which get the same value from each.
__global__ void __launch_bounds__(kSetupThreads)
    boundary_kernel(const double *atoms, int natoms, int n, double h,
                    double pref, double kappa, double *x0) {
  __shared__ double sa[kSetupThreads * 5];
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long face_pts = (long)n * n;
  const bool active = g < 6 * face_pts;
  long i0 = 0, i1 = 0, i2 = 0;
  if (active) {
    const int face = (int)(g / face_pts);
    const long q = g % face_pts;
    const long a = q / n, b = q % n;
    switch (face) {
    case 0: i0 = a; i1 = b; i2 = 0; break;
    case 1: i0 = a; i1 = b; i2 = n - 1; break;
    case 2: i0 = 0; i1 = a; i2 = b; break;
    case 3: i0 = n - 1; i1 = a; i2 = b; break;
    case 4: i0 = a; i1 = 0; i2 = b; break;
    default: i0 = a; i1 = n - 1; i2 = b; break;
    }
  }
  double acc = 0;
  for (int b0 = 0; b0 < natoms; b0 += kSetupThreads) {
    __syncthreads();
    const int b = b0 + threadIdx.x;
    if (b < natoms) {
      for (int d = 0; d < 4; ++d)
        sa[5 * threadIdx.x + d] = atoms[5 * b + d];
      // the atom's factor q / (pref (1 + kappa r)), once per atom: the
      // same operations as inside the sum, so the same bits
      sa[5 * threadIdx.x + 4] =
          atoms[5 * b + 4] / (pref * (1 + kappa * atoms[5 * b + 3]));
    }
    __syncthreads();
    const int nb = natoms - b0 < kSetupThreads ? natoms - b0 : kSetupThreads;
    if (active)
      for (int t = 0; t < nb; ++t) {
        const double *at = &sa[5 * t];
        const double d0 = i0 * h - at[0];
        const double d1 = i1 * h - at[1];
        const double d2 = i2 * h - at[2];
        const double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        acc += at[4] * exp(-kappa * (dist - at[3])) / dist;
      }
  }
  if (active)
    x0[((size_t)i0 * n + i1) * n + i2] = acc;
}

unsigned grid_for(long count) {
  const long b = (count + kSetupThreads - 1) / kSetupThreads;
  return (unsigned)(b < 1 ? 1 : (b > 148L * 32 ? 148L * 32 : b));
}

// Stream-ordered scratch freed at scope exit (after the work queued on the
// stream, by stream order).
struct Scratch {
  cudaStream_t s;
  std::vector<void *> ptrs;
  explicit Scratch(cudaStream_t st) : s(st) {}
  ~Scratch() {
    for (void *p : ptrs)
      scratch_free(p, s);
  }
  template <typename T> cudaError_t take(T **p, size_t count) {
    void *q = nullptr;
    const cudaError_t e = scratch_alloc(&q, sizeof(T) * (count ? count : 1),
                                        s);
    if (e == cudaSuccess)
      ptrs.push_back(q);
    *p = (T *)q;
    return e;
  }
};

} // namespace

// Device set-up into device arrays; atoms are host rows (validated here).
int setup_fine_device(int n, double h, const double *atoms_host, int natoms,
                      const pmg_physics *ph, double *oC, double *oE,
                      double *oN, double *uC, double *f, double *x0,
                      cudaStream_t st) {
  if (n < 3 || n > 1025 || !(h > 0) || (natoms > 0 && !atoms_host) ||
      natoms < 0 || !ph || !oC || !oE || !oN || !uC || !f || !x0) {
    set_last_message("setup_fine_device: bad argument");
    return PMG_ERR_ARG;
  }
  for (int a = 0; a < natoms; ++a) {
    for (int d = 0; d < 3; ++d) {
      const double x = atoms_host[5 * a + d];
      if (!(x >= 0 && x <= h * (n - 1))) {
        set_last_message("setup_fine_device: atom outside the grid");
        return PMG_ERR_ARG;
      }
    }
    if (!(atoms_host[5 * a + 3] >= 0)) {
      set_last_message("setup_fine_device: negative radius");
      return PMG_ERR_ARG;
    }
  }
  const long n3 = (long)n * n * n;
  const Physics p = physics(*ph);
  const double h2 = h * h;
  const double v_out = p.eps_out / h2, v_in = p.eps_in / h2;
  const bool probe = ph->probe_radius > 0;
  Scratch sc(st);
  double *d_atoms = nullptr;
  unsigned char *inside = nullptr, *sas = nullptr, *carved = nullptr,
                *ion = nullptr, *free_flag = nullptr;
  double *centres = nullptr;
  ProbeDir *d_dirs = nullptr;
  PMG_CUDA_TRY(sc.take(&d_atoms, 5 * (size_t)natoms));
  PMG_CUDA_TRY(sc.take(&inside, n3));
  PMG_CUDA_TRY(sc.take(&ion, n3));
  if (natoms > 0)
    PMG_CUDA_TRY(cudaMemcpyAsync(d_atoms, atoms_host,
                                 sizeof(double) * 5 * natoms,
                                 cudaMemcpyHostToDevice, st));
  if (probe && natoms > 0) {
    ProbeDir dirs[kProbePoints];
    probe_directions(dirs);
    PMG_CUDA_TRY(sc.take(&sas, n3));
    PMG_CUDA_TRY(sc.take(&carved, n3));
    PMG_CUDA_TRY(sc.take(&free_flag, (size_t)natoms * kProbePoints));
    PMG_CUDA_TRY(sc.take(&centres, 3 * (size_t)natoms * kProbePoints));
    PMG_CUDA_TRY(sc.take(&d_dirs, kProbePoints));
    PMG_CUDA_TRY(cudaMemcpyAsync(d_dirs, dirs, sizeof(dirs),
                                 cudaMemcpyHostToDevice, st));
    const long np = (long)natoms * kProbePoints;
    const unsigned pgrid = (unsigned)((np + kSetupThreads - 1) / kSetupThreads);
    // cell list of the atoms, built on the stream: edge >= the largest
    // inflated radius, at most 64 cells per axis of the grid's extent
    const double extent = h * (n - 1);
    double cell = 0;
    for (int a = 0; a < natoms; ++a)
      cell = std::max(cell, atoms_host[5 * a + 3]);
    cell = std::max(cell + ph->probe_radius, extent / 63);
    const int dim = (int)(extent / cell) + 1;
    const int ncells = dim * dim * dim;
    int *d_cid = nullptr, *d_count = nullptr, *d_cstart = nullptr,
        *d_fill = nullptr, *d_cat = nullptr;
    PMG_CUDA_TRY(sc.take(&d_cid, (size_t)natoms));
    PMG_CUDA_TRY(sc.take(&d_count, (size_t)ncells + 1));
    PMG_CUDA_TRY(sc.take(&d_cstart, (size_t)ncells + 1));
    PMG_CUDA_TRY(sc.take(&d_fill, (size_t)ncells + 1));
    PMG_CUDA_TRY(sc.take(&d_cat, (size_t)natoms));
    PMG_CUDA_TRY(
        cudaMemsetAsync(d_count, 0, sizeof(int) * (ncells + 1), st));
    atom_cells_kernel<<<(natoms + 255) / 256, 256, 0, st>>>(
        d_atoms, natoms, cell, dim, d_cid, d_count);
    size_t scan_bytes = 0;
    PMG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_count,
                                               d_cstart, ncells + 1, st));
    unsigned char *scan_tmp = nullptr;
    PMG_CUDA_TRY(sc.take(&scan_tmp, scan_bytes));
    PMG_CUDA_TRY(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, d_count,
                                               d_cstart, ncells + 1, st));
    PMG_CUDA_TRY(cudaMemcpyAsync(d_fill, d_cstart,
                                 sizeof(int) * (ncells + 1),
                                 cudaMemcpyDeviceToDevice, st));
    atom_scatter_kernel<<<(natoms + 255) / 256, 256, 0, st>>>(
        natoms, d_cid, d_fill, d_cat);
    probe_centres_cells_kernel<<<pgrid, kSetupThreads, 0, st>>>(
        d_atoms, natoms, ph->probe_radius, d_dirs, cell, dim, d_cstart, d_cat,
        centres, free_flag);
    PMG_LAUNCH_CHECK();
  }

  // face coefficients, axis 0 -> uC, 1 -> oN, 2 -> oE
  double *face[3] = {uC, oN, oE};
  for (int axis = 0; axis < 3; ++axis) {
    PMG_CUDA_TRY(cudaMemsetAsync(inside, 0, n3, st));
    if (natoms > 0) {
      SphereSet atoms_set{d_atoms, 5, natoms, d_atoms + 3, 0.0, nullptr,
                          axis};
      mark_spheres_kernel<unsigned char>
          <<<natoms, kSetupThreads, 0, st>>>(n, h, atoms_set, inside, 1);
    }
    if (probe && natoms > 0) {
      PMG_CUDA_TRY(cudaMemsetAsync(sas, 0, n3, st));
      PMG_CUDA_TRY(cudaMemsetAsync(carved, 0, n3, st));
      SphereSet inflated{d_atoms, 5, natoms, d_atoms + 3, ph->probe_radius,
                         nullptr, axis};
      mark_spheres_kernel<unsigned char>
          <<<natoms, kSetupThreads, 0, st>>>(n, h, inflated, sas, 1);
      const int np = natoms * kProbePoints;
      SphereSet probes{centres, 3, np, nullptr, ph->probe_radius, free_flag,
                       axis};
      mark_spheres_kernel<unsigned char>
          <<<np, kSetupThreads, 0, st>>>(n, h, probes, carved, 1);
    }
    face_from_masks_kernel<<<grid_for(n3), kSetupThreads, 0, st>>>(
        n3, inside, probe && natoms > 0 ? sas : nullptr, carved, v_in, v_out,
        face[axis]);
    PMG_LAUNCH_CHECK();
  }

  // ion-exclusion mask and the centre coefficient
  PMG_CUDA_TRY(cudaMemsetAsync(ion, 0, n3, st));
  if (natoms > 0) {
    SphereSet ions{d_atoms, 5, natoms, d_atoms + 3, ph->ion_radius, nullptr,
                   -1};
    mark_spheres_kernel<unsigned char>
        <<<natoms, kSetupThreads, 0, st>>>(n, h, ions, ion, 1);
  }
  centre_kernel<<<grid_for(n3), kSetupThreads, 0, st>>>(
      n, uC, oN, oE, ion, p.kappa * p.kappa * p.eps_out, oC);
  PMG_LAUNCH_CHECK();

  // charges
  PMG_CUDA_TRY(cudaMemsetAsync(f, 0, sizeof(double) * n3, st));
  if (natoms > 0) {
    const int nrec = 8 * natoms;
    int *k_in, *k_out, *v_in_, *v_out_;
    PMG_CUDA_TRY(sc.take(&k_in, nrec));
    PMG_CUDA_TRY(sc.take(&k_out, nrec));
    PMG_CUDA_TRY(sc.take(&v_in_, nrec));
    PMG_CUDA_TRY(sc.take(&v_out_, nrec));
    charge_records_kernel<<<(nrec + 255) / 256, 256, 0, st>>>(
        d_atoms, natoms, n, h, k_in, v_in_);
    PMG_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    PMG_CUDA_TRY(cub::DeviceRadixSort::SortPairs(
        nullptr, tmp_bytes, k_in, k_out, v_in_, v_out_, nrec, 0, 32, st));
    unsigned char *tmp = nullptr;
    PMG_CUDA_TRY(sc.take(&tmp, tmp_bytes));
    PMG_CUDA_TRY(cub::DeviceRadixSort::SortPairs(
        tmp, tmp_bytes, k_in, k_out, v_in_, v_out_, nrec, 0, 32, st));
    charge_sum_kernel<<<(nrec + 255) / 256, 256, 0, st>>>(
        d_atoms, nrec, h, p.eps0, h * (h * h), k_out, v_out_, f);
    PMG_LAUNCH_CHECK();
  }

  // Debye-Hueckel boundary
  PMG_CUDA_TRY(cudaMemsetAsync(x0, 0, sizeof(double) * n3, st));
  if (natoms > 0) {
    const long pts = 6L * n * n;
    boundary_kernel<<<(unsigned)((pts + kSetupThreads - 1) / kSetupThreads),
                      kSetupThreads, 0, st>>>(
        d_atoms, natoms, n, h, 4 * kPi * (p.eps0 * p.eps_out), p.kappa, x0);
    PMG_LAUNCH_CHECK();
  }
  return PMG_OK;
}

} // namespace pmg

extern "C" int pmg_setup_fine_d(int n, double h, const double *atoms,
                                int natoms, const pmg_physics *phys,
                                double *oC, double *oE, double *oN,
                                double *uC, double *f, double *x0,
                                pmg_stream_t stream) {
  return pmg::setup_fine_device(n, h, atoms, natoms, phys, oC, oE, oN, uC, f,
                                x0, (cudaStream_t)stream);
}
