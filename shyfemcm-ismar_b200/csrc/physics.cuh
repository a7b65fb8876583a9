// physics.cuh -- device helpers shared by the step kernels: error status,
// UNESCO equation of state, level boundary values.
#pragma once
#include "common.cuh"
#include "../../include/shygpu.h"

namespace shy {

__device__ __forceinline__ void set_status(BasinOut *o, int code) {
  atomicCAS(&o->status, 0, code);
}

// UNESCO 1981 equation of state (Millero & Poisson 1981; Fofonoff & Millard
// 1983), the formulation of sigma_stp (eq_state.f90:154-230): density at one
// atmosphere and secant bulk modulus; p in bar; returns rho - 1000.
__device__ inline double sigma_stp_d(double s, double t, double p) {
  double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  double s32 = sqrt(s * s * s);
  double rw = 999.842594 + 6.793952e-2 * t - 9.095290e-3 * t2 + 1.001685e-4 * t3
              - 1.120083e-6 * t4 + 6.536332e-9 * t5;
  double a = 8.24493e-1 - 4.0899e-3 * t + 7.6438e-5 * t2 - 8.2467e-7 * t3 + 5.3875e-9 * t4;
  double b = -5.72466e-3 + 1.0227e-4 * t - 1.6546e-6 * t2;
  double rho0 = rw + a * s + b * s32 + 4.8314e-4 * s * s;
  double kw = 19652.21 + 148.4206 * t - 2.327105 * t2 + 1.360477e-2 * t3 - 5.155288e-5 * t4;
  double aw = 3.239908 + 1.43713e-3 * t + 1.16092e-4 * t2 - 5.77905e-7 * t3;
  double bw = 8.50935e-5 - 6.12293e-6 * t + 5.2787e-8 * t2;
  double k0 = kw + (54.6746 - 0.603459 * t + 1.09987e-2 * t2 - 6.1670e-5 * t3) * s
              + (7.944e-2 + 1.6483e-2 * t - 5.3009e-4 * t2) * s32;
  double aa = aw + (2.2838e-3 - 1.0981e-5 * t - 1.6078e-6 * t2) * s + 1.91075e-4 * s32;
  double bb = bw + (-9.9348e-7 + 2.0816e-8 * t + 9.1697e-10 * t2) * s;
  double kk = k0 + aa * p + bb * p * p;
  return rho0 / (1. - p / kk) - 1000.;
}

// level boundary value at time t: get_oscil (bnd_admin.f90:1304-1320), the
// constituents summed; single-precision pi and a real result like the reference.
__device__ __forceinline__ double level_bc(const Dev &d, const BasinPar &P, int kb, double t) {
  const double pi = 3.141592653;
  double z = 0.;
  const float *tb = d.tide + P.tide_off + (size_t)(kb - 1) * P.ntide * 4;
  for (int c = 0; c < P.ntide; c++) {
    double ampli = tb[4 * c], period = tb[4 * c + 1], phase = tb[4 * c + 2], zref = tb[4 * c + 3];
    if (period == 0.) continue;
    z += zref + ampli * sin(2. * pi * (t + phase) / period);
  }
  return (double)(float)z;
}

}  // namespace shy
