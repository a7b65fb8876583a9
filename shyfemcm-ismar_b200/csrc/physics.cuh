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

// z-adaptive (z-star) surface layers of z-layer basins with nzadapt > 1
// (zadaptutil.f90).  compute_nadapt_info (:212-240): the lowest layer that
// follows the level z (1-based; 0: none) in a column of lmax layers.
__device__ __forceinline__ int zad_levmax(double z, const float *hlv, int lmax, double rzmov) {
  int nad = 0;
  for (int l = 1; l <= lmax - 1; l++) {
    const double hl = hlv[l - 1], hp = l > 1 ? (double)hlv[l - 2] : 0.;
    if (z <= -hl + rzmov * (hl - hp)) nad = l + 1;
    else break;
  }
  return nad;
}

// layer l (0-based) at an element vertex of level z and depth htot (setdepth,
// elems_dealing.f90:1014-1055, with compute_zadaptive_info :321-380): the
// layers down to levmax share the column hadapt + z in proportion to their
// nominal thickness (hadapt = hlv(levmax), or htot when levmax is the bottom
// layer); below them z-layers, the first plus z when no layer follows z
__device__ __forceinline__ double zad_vertex_h(int l, double z, double htot, int lmax, int levmax, const float *hlv,
                                               const float *hld) {
  const int l1 = l + 1;
  if (levmax > 0 && l1 <= levmax) {
    const double had = levmax == lmax ? htot : (double)hlv[levmax - 1];
    const double htop = l1 == 1 ? 0. : (double)hlv[l1 - 2], hbot = l1 == lmax ? htot : (double)hlv[l1 - 1];
    return -(had + z) * ((htop - hbot) / had);
  }
  if (lmax == 1) return htot + z;
  if (l1 < lmax) return (double)hld[l] + (levmax == 0 && l1 == 1 ? z : 0.);
  return htot - (double)hlv[lmax - 2];
}

// layer l (0-based) of an element: down to the deepest levmax of its
// vertices the mean of the vertex values, below z-layers of its mean depth
// hev and mean level zmed (setdepth :1087-1110)
__device__ __forceinline__ double zad_elem_h(int l, const double (&z)[3], const float4 hm, int lmax,
                                             const int (&lev)[3], const float *hlv, const float *hld, double zmed) {
  const int lad = max(lev[0], max(lev[1], lev[2]));
  const int l1 = l + 1;
  if (lad > 0 && l1 <= lad)
    return (zad_vertex_h(l, z[0], hm.x, lmax, lev[0], hlv, hld) + zad_vertex_h(l, z[1], hm.y, lmax, lev[1], hlv, hld) +
            zad_vertex_h(l, z[2], hm.z, lmax, lev[2], hlv, hld)) / 3.;
  if (lmax == 1) return (double)hm.w + zmed;
  if (l1 < lmax) return (double)hld[l] + (lad == 0 && l1 == 1 ? zmed : 0.);
  return (double)hm.w - (double)hlv[lmax - 2];
}

// set_barocl_new_interface with bsigadjust (explicit.f90:1346-1440): the
// density of node column k at depth `dep` below the rest level, for an
// interface of sigma layers that does not lie on a horizontal surface.  The
// column's interfaces are at -zo + the old layer thicknesses hk summed from
// the top (hkko); the layer ll holding `dep` brackets it, with the layer
// above or below, between their mid-layer depths (hkkom), and the density
// is interpolated there; above the first mid-layer it is the first layer's
// (ld = 1), below the last it is the last layer's and *below is set (nb).
// The reference looks for ll from layer l up or down; for a column whose
// interfaces increase with depth that finds the same layer as this scan
// from the top.
__device__ __forceinline__ float sigma_rho_at(const float *hk, const float *rho, double z0, int lkmax, double dep,
                                              bool *below) {
  *below = false;
  int ll = lkmax;
  double ho = z0;
  for (int j = 1; j <= lkmax; j++) {
    ho += hk[j - 1];
    if (dep < ho) { ll = j; break; }
  }
  // hkkom of layers ll-1, ll and ll+1
  double top = z0;
  for (int j = 1; j < ll - 1; j++) top += hk[j - 1];
  const double hop = ll >= 2 ? top + hk[ll - 2] : z0;            // hkko(ll-1)
  const double hmm = ll >= 2 ? 0.5 * (top + hop) : z0;            // hkkom(ll-1)
  const double hoc = hop + hk[ll - 1];                           // hkko(ll)
  const double hmc = 0.5 * (hop + hoc);                          // hkkom(ll)
  const double hmp = ll < lkmax ? 0.5 * (hoc + hoc + hk[ll]) : 0.;   // hkkom(ll+1)
  int lu, ld;
  double hu, hd;
  if (dep < hmc) { lu = ll == 1 ? 1 : ll - 1; ld = ll; hu = ll == 1 ? hmc : hmm; hd = hmc; }
  else { lu = ll; ld = ll == lkmax ? lkmax : ll + 1; hu = hmc; hd = ll == lkmax ? hmc : hmp; }
  if (ld == 1) return rho[0];
  if (lu >= lkmax) { *below = true; return rho[lkmax - 1]; }
  const double alpha = (dep - hu) / (hd - hu);
  return (float)(alpha * (double)rho[ld - 1] + (1. - alpha) * (double)rho[lu - 1]);
}

}  // namespace shy
