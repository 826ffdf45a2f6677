// Device helpers shared by the stress kernels (internal points and boundary nodes).
#pragma once

#include "common.cuh"

namespace bem {

// calc_principal_and_vm (stress_mod.f90:299-359): von Mises stress and the principal
// stresses (descending) by the closed-form (Cardano) solution of the cubic.
__device__ __forceinline__ void principal_vm(const double* s, double* pr, double* vm) {
  const double sxx = s[0], syy = s[1], szz = s[2], sxy = s[3], syz = s[4], szx = s[5];
  *vm = sqrt(0.5 * ((sxx - syy) * (sxx - syy) + (syy - szz) * (syy - szz) + (szz - sxx) * (szz - sxx) +
                    6.0 * (sxy * sxy + syz * syz + szx * szx)));
  const double i1 = sxx + syy + szz, q = i1 / 3.0;
  const double pxx = sxx - q, pyy = syy - q, pzz = szz - q;
  const double j2 = 0.5 * (pxx * pxx + pyy * pyy + pzz * pzz) + sxy * sxy + syz * syz + szx * szx;
  if (j2 <= 1.0e-20 * (i1 * i1 + 1.0)) {
    pr[0] = pr[1] = pr[2] = q;
    return;
  }
  const double j3 = pxx * (pyy * pzz - syz * syz) - sxy * (sxy * pzz - syz * szx) + szx * (sxy * syz - pyy * szx);
  const double r = sqrt(4.0 * j2 / 3.0);
  double c3 = 4.0 * j3 / (r * r * r);
  c3 = fmin(1.0, fmax(-1.0, c3));
  const double phi = acos(c3) / 3.0;
  double a = q + r * cos(phi);
  double cc = q + r * cos(phi + 2.0 * kPi / 3.0);
  double b = 3.0 * q - a - cc, t;
  if (a < b) { t = a; a = b; b = t; }
  if (b < cc) { t = b; b = cc; cc = t; }
  if (a < b) { t = a; a = b; b = t; }
  pr[0] = a;
  pr[1] = b;
  pr[2] = cc;
}

}  // namespace bem
