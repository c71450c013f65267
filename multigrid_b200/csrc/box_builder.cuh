// Box-method (finite volume) fine operator of the APBS driver, built from
// the coefficient maps on a tensor mesh: VbuildA_fv, pmgc/buildAd.cc:63-212.
//
// One thread per interior point. The point's six face weights are the two
// transverse cell widths over four times the normal width, its control
// volume the three widths over eight; the diagonal is the weighted sum of
// the six face coefficients, the upper couplings vanish on the high faces,
// and a boundary neighbour's Dirichlet value moves into the source in the
// order E, N, U, W, S, D. The expressions keep the reference's operand
// order (compiled with --fmad=false: the same bits as the reference).
#pragma once

#include "stencil_kernels.cuh"

namespace pmg {

// Inputs: mesh lines (1-based per axis), boundary values gx(j,k,side) on
// ny x nz x 2, gy(i,k,side) on nx x nz x 2, gz(i,j,side) on nx x ny x 2
// (side 1 low, 2 high), face maps a1 (x faces) a2 (y) a3 (z), kappa and
// source maps.
struct BoxMaps {
  const double *xf, *yf, *zf, *gx, *gy, *gz, *a1, *a2, *a3, *cc, *fc;
};
// Outputs: the 7-point operator, the scaled kappa term and the source.
struct BoxOps {
  double *oC, *cc, *fc, *oE, *oN, *uC;
};

__global__ void __launch_bounds__(256)
    buildA_fv_kernel(Dims d, BoxMaps m, BoxOps o) {
  const Interior t = interior_point(d);
  if (!t.ok)
    return;
  const int i = t.i, j = t.j, k = t.k;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int p = d.at(i, j, k), pw = p - 1, ps = p - d.sy(), pd = p - d.sz();
  const double hzm1 = m.zf[k - 1] - m.zf[k - 2], hz = m.zf[k] - m.zf[k - 1];
  const double hym1 = m.yf[j - 1] - m.yf[j - 2], hy = m.yf[j] - m.yf[j - 1];
  const double hxm1 = m.xf[i - 1] - m.xf[i - 2], hx = m.xf[i] - m.xf[i - 1];
  const double diag = 1.0;
  const double wE = diag * (hym1 + hy) * (hzm1 + hz) / (4.0 * hx);
  const double wW = diag * (hym1 + hy) * (hzm1 + hz) / (4.0 * hxm1);
  const double wN = diag * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hy);
  const double wS = diag * (hxm1 + hx) * (hzm1 + hz) / (4.0 * hym1);
  const double wU = diag * (hxm1 + hx) * (hym1 + hy) / (4.0 * hz);
  const double wD = diag * (hxm1 + hx) * (hym1 + hy) / (4.0 * hzm1);
  const double vol = diag * (hxm1 + hx) * (hym1 + hy) * (hzm1 + hz) / 8.0;
  const double a1 = m.a1[p], a1w = m.a1[pw];
  const double a2 = m.a2[p], a2s = m.a2[ps];
  const double a3 = m.a3[p], a3d = m.a3[pd];
  double f = vol * m.fc[p];
  o.cc[p] = vol * m.cc[p];
  o.oC[p] = wE * a1 + wW * a1w + wN * a2 + wS * a2s + wU * a3 + wD * a3d;
  // 1 inside, 0 where the neighbour is on the shell
  const int e = i != nx - 1, n = j != ny - 1, u = k != nz - 1;
  const int w = i != 2, s = j != 2, dn = k != 2;
  o.oE[p] = e * wE * a1;
  f += (1 - e) * wE * a1 * m.gx[ny * nz + (k - 1) * ny + (j - 1)];
  o.oN[p] = n * wN * a2;
  f += (1 - n) * wN * a2 * m.gy[nx * nz + (k - 1) * nx + (i - 1)];
  o.uC[p] = u * wU * a3;
  f += (1 - u) * wU * a3 * m.gz[nx * ny + (j - 1) * nx + (i - 1)];
  f += (1 - w) * wW * a1w * m.gx[(k - 1) * ny + (j - 1)];
  f += (1 - s) * wS * a2s * m.gy[(k - 1) * nx + (i - 1)];
  f += (1 - dn) * wD * a3d * m.gz[(j - 1) * nx + (i - 1)];
  o.fc[p] = f;
}

} // namespace pmg
