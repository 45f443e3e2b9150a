// Cardinal B-spline stencil of one coordinate on an EES grid, shared by the
// nonlocal (eesAtmBsplineRgrp, cp_ees_nonlocal.C:256-593) and the local
// (eesAtmBsplineRgrp, cp_hart_ext.C:641-900) paths, which use the same
// recursion: fractional coordinate u = x / L wrapped onto [0, 1), scaled by
// the grid size, split into it + frac; for j = 1..order the grid point
// it - (j - 2) wrapped onto [0, ngrid), the weight M_n(frac + j - 1), and
// (dm not null) dM_n = M_{n-1}(u) - M_{n-1}(u - 1) taken at n = order - 1.
#pragma once

__device__ __forceinline__ void ees_bspline_axis(double x, double box, int ngrid, int order, int* idx, double* m,
                                                 double* dm) {
  double u0 = x / box;
  u0 -= rint(u0 - 0.5);
  if (u0 == 1.0) u0 = 0.0;
  u0 *= (double)ngrid;
  const int it = (int)u0;
  const double frac = u0 - (double)it;
  double w[17];
  for (int j = 0; j <= order; ++j) w[j] = 0.0;
  w[1] = 1.0 - fabs(frac - 1.0);
  w[2] = 1.0 - fabs(frac + 1.0 - 1.0);
  for (int n = 3; n <= order; ++n) {
    const double rn1 = 1.0 / (double)(n - 1);
    for (int j = n; j >= 2; --j) {
      const double u = frac + (double)(j - 1);
      w[j] = (u * w[j] + ((double)n - u) * w[j - 1]) * rn1;
    }
    w[1] = frac * w[1] * rn1;
    if (n == order - 1 && dm) {
      dm[0] = w[1];
      for (int j = 2; j <= order; ++j) dm[j - 1] = w[j] - w[j - 1];
    }
  }
  for (int j = 1; j <= order; ++j) {
    int g = it - (j - 2);
    g = g > 0 ? g : ngrid + g;
    g = g <= ngrid ? g : g - ngrid;
    idx[j - 1] = g - 1;
    m[j - 1] = w[j];
  }
}
