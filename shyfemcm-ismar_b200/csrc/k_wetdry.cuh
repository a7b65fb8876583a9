// k_wetdry.cuh -- wetting and drying of elements on z-layers (wetdry.f90,
// topo_update.f90), for basins with shy_params::wetdry.
//
// An element leaves the system (iweg > 0, the number of its vertices below
// the limit) when a vertex's total depth falls below hzoff at the start of
// a step (setweg 2) or below hzmin after a zeta solve (setweg 1, which makes
// the zeta kernel assemble and solve again); it returns once its vertices
// reach hzon, or their mean does and it has been dry for more than iwait
// steps (setweg 3).  iwet counts the steps an element has been wet (> 0) or
// dry (< 0) (wetdry.f90:322-331).  Dry elements carry a Laplacian in the
// zeta system (hydrodynamic.f90:710-727, in k_zeta_global.cuh), their level
// and barotropic transport follow from continuity (setuvd, in
// k_final.cuh), and their transport is spread over the layers by
// thickness (baro2l).  Included by step.cu and step_zeta.cu.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace shy {

constexpr int kWetWait = 5;            // iwait: dry steps before the mean-depth rule may add (:176)
constexpr int kWetDryRepeats = 64;     // solves of one step at most (the domain can only shrink)

__device__ __forceinline__ bool wd_basin(const BasinPar &P) { return P.wetdry && P.nsigma == 0; }

// the step counter of an element after a setweg pass (:322-331)
__device__ __forceinline__ int wd_count(int iweg, int iwet, bool bnewtime) {
  return (bnewtime || iwet == 0) ? iwet + (iweg == 0 ? 1 : -1) : iwet;
}

// set_dry at the start of a step (shyfem_subs.f90:578): setweg(2) then
// setweg(3) on the level of the step's start, neither at a new time
static __global__ void k_wd_set(Dev d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.NEL) return;
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  if (!wd_basin(P)) return;
  const float4 hm = d.hm3v[e];
  const double hz[3] = {(double)d.zo[en.x] + (double)hm.x, (double)d.zo[en.y] + (double)hm.y,
                        (double)d.zo[en.z] + (double)hm.z};
  int iweg = d.iweg[e], iwet = d.iwet[e];
  // setweg 2: take away below hzoff (:265-290)
  if (iweg == 0) {
    int cnt = 0;
    for (int ii = 0; ii < 3; ii++) cnt += hz[ii] < (double)P.hzoff;
    if (cnt > 0) { iweg = cnt; iwet = 0; }
  }
  iwet = wd_count(iweg, iwet, false);
  // setweg 3: add back (:291-320, the new algorithm)
  if (iweg > 0) {
    int cnt = 0;
    double hztot = 0.;
    for (int ii = 0; ii < 3; ii++) { hztot += hz[ii]; cnt += hz[ii] < (double)P.hzon; }
    hztot /= 3.;
    if (hztot >= (double)P.hzon && -iwet > kWetWait) cnt = 0;
    if (cnt == 0) { iweg = 0; iwet = 0; }
  }
  iwet = wd_count(iweg, iwet, false);
  d.iweg[e] = iweg;
  d.iwet[e] = iwet;
}

// initial state (sp111 init, bnd_routines.f90:413-415): zenv from znv
// (init_z), then setweg(0) -- elements with a vertex below hzoff leave, and
// vertex levels below the minimum depth zmin are raised to it
// (wetdry.f90:232-252) -- for basins with wetting and drying
static __global__ void k_wd_init(Dev d, int basin) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.NEL) return;
  const int4 en = d.enode[e];
  if (basin >= 0 && en.w != basin) return;
  const BasinPar &P = d.par[en.w];
  const int kn[3] = {en.x, en.y, en.z};
  double z[3];
  for (int ii = 0; ii < 3; ii++) z[ii] = d.zn[kn[ii]];
  if (P.wetdry) {
    const float4 hm = d.hm3v[e];
    const double h[3] = {hm.x, hm.y, hm.z};
    const double aomega = d.ev8[(size_t)e * 8 + 6];
    double zmin = (double)P.hzmin + (double)P.volmin / (4. * aomega);
    if (zmin > (double)P.hzoff) zmin = (double)P.hzmin + 0.5 * ((double)P.hzmin + (double)P.hzoff);
    int iweg = 0;
    for (int ii = 0; ii < 3; ii++) {
      const double hzg = z[ii] + h[ii];
      if (hzg < (double)P.hzoff) iweg++;
      if (hzg < zmin) z[ii] = zmin - h[ii];
    }
    if (P.nsigma > 0) iweg = 0;
    const int iwet = iweg == 0 ? 1 : 0;
    d.iweg[e] = iweg;
    d.iwet[e] = wd_count(iweg, iwet, true);
  } else if (d.iweg) {
    d.iweg[e] = 0;
    d.iwet[e] = 0;
  }
  for (int ii = 0; ii < 3; ii++) d.zen[3 * e + ii] = (float)z[ii];
}

// setznv (wetdry.f90:619-712) for basins with wetting and drying: a node's
// level from its wet elements (the largest vertex level), else the
// area-weighted mean over its dry elements
static __global__ void k_wd_znv(Dev d, const int *kbas, int basin) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.NKN) return;
  if (basin >= 0 && kbas[k] != basin) return;
  const BasinPar &P = d.par[kbas[k]];
  if (!P.wetdry) return;
  bool wet = false;
  double zw = 0., v1 = 0., v2 = 0.;
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
    const int4 ix = d.incx[p];
    const int e = ix.x, ii = ix.y & 3;
    const double z = d.zen[3 * e + ii];
    if (d.iweg[e] == 0) {
      zw = wet ? fmax(zw, z) : z;
      wet = true;
    } else {
      const double area = 4. * (double)d.ev8[(size_t)e * 8 + 6];
      v1 += z * area;
      v2 += area;
    }
  }
  d.zn[k] = (float)(wet ? zw : v1 / v2);
}

// setnod (topo_update.f90:166-260) for the rows of one basin: a node is
// internal when all elements of a closed fan are wet, out of the system
// when none is, else on the boundary of the wet domain; a level-boundary
// node must be on that boundary.  Returns false for a dry open boundary.
__device__ __forceinline__ bool wd_setnod(const Dev &d, int k) {
  int n = 0, wet = 0;
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
    n++;
    wet += __ldcg(&d.iweg[d.incx[p].x]) == 0;
  }
  int kind = wet == 0 ? -2 : (wet == n && d.kfull[k] ? 0 : -1);
  bool ok = true;
  if (d.kbnd[k] > 0) {
    ok = kind == -1;
    kind = d.kbnd[k];
  }
  d.inod[k] = kind;
  return ok;
}

// the zeta system of a dry element (hydrodynamic.f90:710-727): a Laplacian,
// no right-hand side, and no equation from it for vertices on the boundary
// of the wet domain
__device__ __forceinline__ void wd_dry_system(const Dev &d, int e) {
  const int4 en = d.enode[e];
  const int kn[3] = {en.x, en.y, en.z};
  const float *evp = d.ev8 + (size_t)e * 8;
  double b[3], c[3];
  for (int i = 0; i < 3; i++) { b[i] = evp[i]; c[i] = evp[3 + i]; }
  const double hh999 = 12. * (double)evp[6];
  double hia[3][3], hik[3];
  for (int n = 0; n < 3; n++) {
    const int in = __ldcg(&d.inod[kn[n]]);
    const bool keep = in == 0 || in == -2;
    for (int m = 0; m < 3; m++) hia[n][m] = keep ? hh999 * (b[n] * b[m] + c[n] * c[m]) : 0.;
    hik[n] = 0.;
  }
  store_elem_system(d, e, hia, hik);
}

// setweg(1) for one element after a solve (:265-290): out when a vertex is
// below hzmin; returns whether it changed
__device__ __forceinline__ bool wd_take_away(const Dev &d, const BasinPar &P, int e) {
  if (__ldcg(&d.iweg[e]) != 0) return false;
  const int4 en = d.enode[e];
  const float4 hm = d.hm3v[e];
  const int cnt = ((double)__ldcg(&d.zn[en.x]) + (double)hm.x < (double)P.hzmin) +
                  ((double)__ldcg(&d.zn[en.y]) + (double)hm.y < (double)P.hzmin) +
                  ((double)__ldcg(&d.zn[en.z]) + (double)hm.z < (double)P.hzmin);
  if (cnt == 0) return false;
  d.iweg[e] = cnt;
  d.iwet[e] = 0;
  return true;
}

// setuvd (wetdry.f90:350-590) for one dry element: the new vertex levels zz
// and the barotropic transport (u, v) that keep the element's volume and no
// vertex below hzmin, from its old vertex levels zn and old transport
// (uo, vo).  Returns false where the reference stops with an error.
__device__ __forceinline__ bool wd_setuvd(const BasinPar &P, const float *evp, const float4 hm,
                                          const double zn[3], double uo, double vo, double zz[3],
                                          double &u, double &v) {
  const double dt = P.dt, hzmin = P.hzmin, az = P.az, azt = 1. - az, eps = 1.e-5;
  const double axdt = 3. * dt, adt = 1. / axdt;
  const double h[3] = {hm.x, hm.y, hm.z};
  double b[3], c[3], z[3];
  double zm = 0.;
  for (int ii = 0; ii < 3; ii++) { zm += zn[ii]; b[ii] = evp[ii]; c[ii] = evp[3 + ii]; }
  const double zmed = zm / 3.;
  int itot = 0, isum = 0;
  for (int ii = 0; ii < 3; ii++) {
    if (zmed + h[ii] < hzmin) { z[ii] = hzmin - h[ii]; itot++; isum += ii + 1; }
    else z[ii] = zmed;
    zm -= z[ii];
  }
  if (itot == 1) {
    const int i1 = isum % 3, i2 = (i1 + 1) % 3, is = isum - 1;
    if (z[i1] + zm * 0.5 + h[i1] < hzmin) {
      z[i1] = hzmin - h[i1];
      z[i2] = 3. * zmed - z[i1] - z[is];
    } else if (z[i2] + zm * 0.5 + h[i2] < hzmin) {
      z[i2] = hzmin - h[i2];
      z[i1] = 3. * zmed - z[i2] - z[is];
    } else {
      z[i1] += 0.5 * zm;
      z[i2] += 0.5 * zm;
    }
  } else if (itot == 2) {
    z[6 - isum - 1] += zm;
  } else if (itot == 3) {
    return false;
  }
  zm = 0.;
  for (int ii = 0; ii < 3; ii++) {
    zm += z[ii];
    if (z[ii] + h[ii] < hzmin - eps) return false;
  }
  if (fabs(zm - 3. * zmed) > eps) return false;
  double d1 = (z[0] - zn[0]) * adt - azt * (b[0] * uo + c[0] * vo);
  double d2 = (z[1] - zn[1]) * adt - azt * (b[1] * uo + c[1] * vo);
  double det = 1. / (b[0] * c[1] - b[1] * c[0]);
  u = det * (c[1] * d1 - c[0] * d2);
  v = det * (-b[1] * d1 + b[0] * d2);
  itot = 0;
  for (int ii = 0; ii < 3; ii++) {
    const double t = axdt * (b[ii] * (azt * uo + az * u) + c[ii] * (azt * vo + az * v)) + zn[ii];
    if (t + h[ii] < hzmin - eps) itot++;
  }
  if (itot > 0) {                      // a vertex is drying: the transport that keeps z
    if (az == 0.) return false;
    det = 1. / (az * (b[0] * c[1] - b[1] * c[0]));
    u = det * (c[1] * d1 - c[0] * d2);
    v = det * (-b[1] * d1 + b[0] * d2);
  }
  itot = 0;
  zm = 0.;
  for (int ii = 0; ii < 3; ii++) {
    zz[ii] = axdt * (b[ii] * (azt * uo + az * u) + c[ii] * (azt * vo + az * v)) + zn[ii];
    if (zz[ii] + h[ii] < hzmin - eps) itot++;
    zm += zz[ii];
  }
  return fabs(zm - 3. * zmed) <= eps && itot == 0;
}

}  // namespace shy
