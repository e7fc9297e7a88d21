// vset.cuh -- phys_get_vset_point (mod_Phys.F90:757-954) on the device:
// the fixed-point drag-law iteration of the seven settling-velocity models.
// Included by translation units compiled with --fmad=false, so each model
// keeps the reference's separately rounded operations.
#pragma once
#include <cuda_runtime.h>

namespace f3d {

// Iteration limit of phys_get_vset_point (mod_Phys.F90:794: maxit = 1000) for
// the next settling-velocity launches; f3d_set_vset_maxit (f3d_capi.cu)
// lowers it to force the non-convergence path (flag 2) in tests.
constexpr int kVsetMaxit = 1000;
int vset_maxit();

// Bin constants of the drag laws (mod_Phys.F90:817-819, 868-870).
struct VsetConst {
  double rk1, rk2, a, b;
};

__device__ __forceinline__ VsetConst vset_const(int model, double psi) {
  VsetConst k{0.0, 0.0, 0.0, 0.0};
  if (model == 2) {
    k.rk1 = 3.0 / (1.0 + 2.0 / sqrt(psi));
    k.rk2 = pow(10.0, 1.8148 * pow(-log10(psi), 0.5743));
  }
  if (model == 5) {
    double cd100 = 0.24 * pow(psi, -0.828) + 2.0 * sqrt(1.07 - psi);
    k.a = (1.0 - cd100) / 900.0;
    k.b = 1.0 - 1000.0 * k.a;
  }
  return k;
}

// Drag coefficient Cd(Re) of the iterative models 1,2,3,5,6,7
// (mod_Phys.F90:800-940), in the reference's operation order.
__device__ __forceinline__ double vset_cd(int model, double rey, double psi, const VsetConst& k,
                                          double cd) {
  switch (model) {
    case 1:
      if (rey <= 988.947) cd = 24.0 / rey * (1.0 + 0.15 * pow(rey, 0.687));
      else cd = 0.44;
      break;
    case 2:
      cd = 24.0 / (rey * k.rk1) * (1.0 + 0.1118 * pow(rey * k.rk1 * k.rk2, 0.6567)) +
           0.4305 * k.rk2 / (1.0 + 3305.0 / (rey * k.rk1 * k.rk2));
      break;
    case 3:
      cd = 24.0 / rey * pow(psi, -0.828) + 2.0 * sqrt(1.07 - psi);
      break;
    case 5:
      if (rey <= 100.0) cd = 24.0 / rey * pow(psi, -0.828) + 2.0 * sqrt(1.07 - psi);
      else if (rey > 100.0 && rey < 1000.0) cd = k.a * rey + k.b;
      else cd = 1.0;
      break;
    case 6:
      cd = 24.0 * (1.0 + 0.15 * pow(rey, 0.687)) / rey + 0.42 / (1.0 + 42500.0 / pow(rey, 1.16));
      cd = 0.74533 * pow(rey, 0.146012) * cd / pow(psi, 0.5134 / pow(fmax(rey, 0.01), 0.2));
      break;
    case 7:
      cd = 24.0 / rey * (pow((1.0 - psi) / rey + 1.0, 0.25) +
                         (0.1806 * pow(rey, 0.6459)) * pow(psi, -pow(rey, 0.08))) +
           0.4251 / (1.0 + 6880.95 / rey * pow(psi, 5.03));
      break;
  }
  return cd;
}

__device__ __forceinline__ int vset_point_dev(double diam, double rhop, double psi, double rhoa, double visc,
                              int model, double* vset_out, int* iters, int maxit = kVsetMaxit) {
  const double GI = 9.81, atol = 1e-12, rtol = 1e-6;
  double cd = 1.0, vset = 0.0, vold, rey;
  *iters = 0;
  if (model == 4) {  // Dellino: closed form
    double d3 = diam * diam * diam;
    vset = pow(d3 * GI * rhop * rhoa * pow(psi, 1.6) / (visc * visc), 0.5206);
    vset = 1.2065 * visc * vset / (diam * rhoa);
    *vset_out = vset;
    return 0;
  }
  if (model < 1 || model > 7) {
    *vset_out = 0.0;
    return 1;
  }
  const VsetConst kc = vset_const(model, psi);
  vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
  vold = vset;
  for (int it = 1; it <= maxit; ++it) {
    rey = rhoa * vset * diam / visc;
    cd = vset_cd(model, rey, psi, kc, cd);
    vset = sqrt(4.0 * GI * diam * rhop / (3.0 * cd * rhoa));
    *iters = it;
    if (fabs(vset - vold) <= atol + rtol * fabs(vset)) {
      *vset_out = vset;
      return 0;
    }
    vold = vset;
  }
  *vset_out = vset;
  return 2;
}

// One application of the fixed-point map v -> sqrt(4 g d rhop / (3 Cd(Re(v)) rhoa)).
__device__ __forceinline__ double vset_map(int model, double v, double diam, double rhop, double psi,
                                           double rhoa, double visc, const VsetConst& k) {
  const double rey = rhoa * v * diam / visc;
  const double cd = vset_cd(model, rey, psi, k, 1.0);
  return sqrt(4.0 * 9.81 * diam * rhop / (3.0 * cd * rhoa));
}

// Steffensen (Aitken delta-squared) correction of a starting value v0 towards
// the fixed point of vset_map: two map evaluations, quadratic convergence for
// the linearly contracting drag-law iteration.  Falls back to the second map
// iterate when the extrapolation is degenerate or leaves a 1% neighbourhood.
__device__ __forceinline__ double vset_steffensen(int model, double v0, double diam, double rhop,
                                                  double psi, double rhoa, double visc,
                                                  const VsetConst& k) {
  const double v1 = vset_map(model, v0, diam, rhop, psi, rhoa, visc, k);
  const double v2 = vset_map(model, v1, diam, rhop, psi, rhoa, visc, k);
  const double den = (v2 - v1) - (v1 - v0);
  double v = v2;
  if (den != 0.0) {
    const double t = v0 - (v1 - v0) * (v1 - v0) / den;
    if (t > 0.0 && fabs(t - v2) <= 0.01 * v2) v = t;
  }
  return v;
}

}  // namespace f3d
