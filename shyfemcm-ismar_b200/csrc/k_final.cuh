// k_final.cuh -- hydro_transports_final, setzev, element layer thickness
// Included by step.cu.
#pragma once
#include "common.cuh"
#include "k_wetdry.cuh"
#include "physics.cuh"

namespace shy {

// ===========================================================================
// k_final: hydro_transports_final + setzev + element layer thickness
// ===========================================================================
template <int S, bool COR>
__global__ void __launch_bounds__(256) k_final(Dev d, int init_only) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int e0 = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const bool valid = e0 < d.NEL;
  const int e = valid ? e0 : d.NEL - 1;
  const int NLV = d.NLV;
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  const int kn[3] = {en.x, en.y, en.z};
  const int ilevel = d.ilhv[e];
  const bool act = lane < ilevel;
  const size_t o = (size_t)e * NLV + lane;
  const float *evp = d.ev8 + (size_t)e * 8;
  double zn3[3];
#pragma unroll
  for (int ii = 0; ii < 3; ii++) zn3[ii] = d.zn[kn[ii]];
  if (!init_only) {
    const double beta = P.dt * (double)P.grav * P.am;
    double bz = 0., cz = 0.;
#pragma unroll
    for (int ii = 0; ii < 3; ii++) {
      double dz = zn3[ii] - (double)d.zeo[3 * e + ii];
      bz += dz * evp[ii];
      cz += dz * evp[3 + ii];
    }
    double u = 0., v = 0.;
    if (act) {
      double re = d.ddx[o], im = COR ? (double)d.ddxi[o] : 0.;
      double du = beta * (re * bz - im * cz);
      double dv = beta * (im * bz + re * cz);
      u = (double)(float)((double)d.un[o] - du);
      v = (double)(float)((double)d.vn[o] - dv);
      if (valid) { d.un[o] = (float)u; d.vn[o] = (float)v; }
    }
    // the time-weighted transports az*U^{n+1} + (1-az)*U^n that hydro_vertical,
    // conzstab and conz3d use (hydrodynamic.f90:1681-1683, concentration_omp.f90:566)
    if (valid && lane < d.NLV) {
      const double az = P.az;
      d.usv[o] = act ? (float)(az * u + (1. - az) * (double)d.uo[o]) : 0.f;
      d.vsv[o] = act ? (float)(az * v + (1. - az) * (double)d.vo[o]) : 0.f;
    }
    double um = seg_sum<S>(u), vm = seg_sum<S>(v);
    if (lane == 0 && valid) { d.unv[e] = (float)um; d.vnv[e] = (float)vm; }
  }
  // setzev and the element part of setdepth (z-layers or pure sigma layers)
  if (lane == 0 && valid) {
#pragma unroll
    for (int ii = 0; ii < 3; ii++) d.zen[3 * e + ii] = (float)zn3[ii];
  }
  const float4 hm = d.hm3v[e];
  double zmed = (zn3[0] + zn3[1] + zn3[2]) / 3.;
  const float *hld = d.hldv + (size_t)en.w * NLV;
  const float *hlv = d.hlv + (size_t)en.w * NLV;
  double h = 0.;
  if (act) {
    if (P.nzadapt > 1) {                 // z-adaptive surface layers
      const int lev[3] = {zad_levmax(zn3[0], hlv, ilevel, P.rzmov), zad_levmax(zn3[1], hlv, ilevel, P.rzmov),
                          zad_levmax(zn3[2], hlv, ilevel, P.rzmov)};
      h = zad_elem_h(lane, zn3, hm, ilevel, lev, hlv, hld, zmed);
    }
    else if (lane < P.nsigma) h = -(fmin((double)hm.w, (double)P.hsigma) + zmed) * (double)hld[lane];   // :1079-1083
    else if (ilevel == 1) h = hm.w + zmed;
    else if (lane < ilevel - 1) h = (double)hld[lane] + (lane == 0 ? zmed : 0.);
    else h = (double)hm.w - hlv[ilevel - 2];
    if (!(h > 0.) && valid) set_status(&d.out[en.w], SHY_EDEPTH);
  }
  if (valid && lane < NLV) d.hen[o] = (float)h;
}

// ===========================================================================
// k_final_t: the same with one thread per element column (shallow columns):
// the per-element FP64 terms once per element, the layers in a loop
// ===========================================================================
template <bool COR>
__global__ void __launch_bounds__(256) k_final_t(Dev d, int init_only) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.NEL) return;
  const int NLV = d.NLV;
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  const int kn[3] = {en.x, en.y, en.z};
  const int ilevel = d.ilhv[e];
  const size_t o = (size_t)e * NLV;
  const float *evp = d.ev8 + (size_t)e * 8;
  const float4 hm = d.hm3v[e];
  const bool dry = wd_basin(P) && d.iweg[e] > 0;   // out of the system (wetting and drying)
  double zn3[3], zv[3];
#pragma unroll
  for (int ii = 0; ii < 3; ii++) { zn3[ii] = d.zn[kn[ii]]; zv[ii] = zn3[ii]; }
  if (!init_only && dry) {
    // setuvd: the element's new vertex levels and barotropic transport from
    // continuity; baro2l: that transport over the layers by their thickness
    double zo3[3], ub = 0., vb = 0.;
#pragma unroll
    for (int ii = 0; ii < 3; ii++) zo3[ii] = d.zeo[3 * e + ii];
    if (!wd_setuvd(P, evp, hm, zo3, (double)d.unv[e], (double)d.vnv[e], zv, ub, vb))
      set_status(&d.out[en.w], SHY_EDEPTH);
    double htot = 0.;
    for (int l = 0; l < ilevel; l++) htot += d.heo[o + l];
    const double az = P.az;
    for (int l = 0; l < NLV; l++) {
      const bool act = l < ilevel;
      const double w = act ? (double)d.heo[o + l] / htot : 0.;
      const float u = (float)(ub * w), v = (float)(vb * w);
      d.un[o + l] = u;
      d.vn[o + l] = v;
      d.usv[o + l] = act ? (float)(az * u + (1. - az) * (double)d.uo[o + l]) : 0.f;
      d.vsv[o + l] = act ? (float)(az * v + (1. - az) * (double)d.vo[o + l]) : 0.f;
    }
    d.unv[e] = (float)ub;
    d.vnv[e] = (float)vb;
  } else if (!init_only) {
    const double beta = P.dt * (double)P.grav * P.am;
    double bz = 0., cz = 0.;
#pragma unroll
    for (int ii = 0; ii < 3; ii++) {
      const double dz = zn3[ii] - (double)d.zeo[3 * e + ii];
      bz += dz * evp[ii];
      cz += dz * evp[3 + ii];
    }
    const double az = P.az;
    double um = 0., vm = 0.;
#pragma unroll 4
    for (int l = 0; l < NLV; l++) {
      const bool act = l < ilevel;
      double u = 0., v = 0.;
      if (act) {
        const double re = d.ddx[o + l], im = COR ? (double)d.ddxi[o + l] : 0.;
        const double du = beta * (re * bz - im * cz);
        const double dv = beta * (im * bz + re * cz);
        u = (double)(float)((double)d.un[o + l] - du);
        v = (double)(float)((double)d.vn[o + l] - dv);
        d.un[o + l] = (float)u;
        d.vn[o + l] = (float)v;
      }
      // az*U^{n+1} + (1-az)*U^n for hydro_vertical, conzstab and conz3d
      d.usv[o + l] = act ? (float)(az * u + (1. - az) * (double)d.uo[o + l]) : 0.f;
      d.vsv[o + l] = act ? (float)(az * v + (1. - az) * (double)d.vo[o + l]) : 0.f;
      um += u; vm += v;
    }
    d.unv[e] = (float)um;
    d.vnv[e] = (float)vm;
  } else {
    // the initial state: barotropic transports; a dry element keeps the
    // vertex levels the set-up gave it
    double um = 0., vm = 0.;
    for (int l = 0; l < ilevel; l++) { um += d.un[o + l]; vm += d.vn[o + l]; }
    d.unv[e] = (float)um;
    d.vnv[e] = (float)vm;
    if (dry)
#pragma unroll
      for (int ii = 0; ii < 3; ii++) zv[ii] = d.zen[3 * e + ii];
  }
  // setzev (elements in the system) and the element part of setdepth
  // (z-layers or pure sigma layers) from the vertex levels
#pragma unroll
  for (int ii = 0; ii < 3; ii++) d.zen[3 * e + ii] = (float)zv[ii];
  const double zmed = (zv[0] + zv[1] + zv[2]) / 3.;
  const float *hld = d.hldv + (size_t)en.w * NLV;
  const float *hlv = d.hlv + (size_t)en.w * NLV;
  bool bad = false;
  int lev[3] = {0, 0, 0};
  if (P.nzadapt > 1)
    for (int ii = 0; ii < 3; ii++) lev[ii] = zad_levmax(zv[ii], hlv, ilevel, P.rzmov);
  for (int l = 0; l < NLV; l++) {
    double h = 0.;
    if (l < ilevel) {
      if (P.nzadapt > 1) h = zad_elem_h(l, zv, hm, ilevel, lev, hlv, hld, zmed);   // z-adaptive surface layers
      else if (l < P.nsigma) h = -(fmin((double)hm.w, (double)P.hsigma) + zmed) * (double)hld[l];   // sigma layers (:1079-1083)
      else if (ilevel == 1) h = hm.w + zmed;
      else if (l < ilevel - 1) h = (double)hld[l] + (l == 0 ? zmed : 0.);
      else h = (double)hm.w - hlv[ilevel - 2];
      if (!(h > 0.)) bad = true;
    }
    d.hen[o + l] = (float)h;
  }
  if (bad) set_status(&d.out[en.w], SHY_EDEPTH);
}

// ===========================================================================
// k_final_w: k_final_t without Coriolis, with the layer arrays of a warp's
// 32 element columns (one contiguous run of 32*NLV values, since a column
// is contiguous and the elements are consecutive) moved between global and
// shared memory by the whole warp in coalesced passes; each thread then
// works its own column in shared memory as k_final_t does.  ZA: the
// instance with z-adaptive layers; without them (every basin with
// nzadapt <= 1) the element thickness needs no FP64 adaptive-layer terms
// and the kernel keeps 80 registers, six CTAs per SM.
// ===========================================================================
template <int L, bool ZA = true>
__global__ void __launch_bounds__(128, ZA ? 1 : 6) k_final_w(Dev d, int init_only) {
  __shared__ float sb[4][5][32 * L];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * 4 + warp) * 32;         // first element of this warp
  if (w0 >= d.NEL) return;                              // whole warps only
  const int nw = min(32, d.NEL - w0);
  const int NLV = d.NLV, cnt = nw * NLV;
  const size_t base = (size_t)w0 * NLV;
  float *bA = sb[warp][0], *bU = sb[warp][1], *bV = sb[warp][2], *bUo = sb[warp][3], *bVo = sb[warp][4];
  const bool valid = lane < nw;
  const int e = w0 + (valid ? lane : 0);
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  const int kn[3] = {en.x, en.y, en.z};
  const int ilevel = d.ilhv[e];
  const int ol = lane * NLV;                            // this thread's column in the buffers
  const float *evp = d.ev8 + (size_t)e * 8;
  double zn3[3];
#pragma unroll
  for (int ii = 0; ii < 3; ii++) zn3[ii] = d.zn[kn[ii]];
  if (!init_only) {
    for (int j = lane; j < cnt; j += 32) {
      bA[j] = d.ddx[base + j];
      bU[j] = d.un[base + j];
      bV[j] = d.vn[base + j];
      bUo[j] = d.uo[base + j];
      bVo[j] = d.vo[base + j];
    }
    __syncwarp();
    if (valid) {
      const double beta = P.dt * (double)P.grav * P.am;
      double bz = 0., cz = 0.;
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const double dz = zn3[ii] - (double)d.zeo[3 * e + ii];
        bz += dz * evp[ii];
        cz += dz * evp[3 + ii];
      }
      const double az = P.az;
      double um = 0., vm = 0.;
      for (int l = 0; l < NLV; l++) {
        const bool act = l < ilevel;
        double u = 0., v = 0.;
        if (act) {
          const double re = bA[ol + l];
          const double du = beta * (re * bz);
          const double dv = beta * (re * cz);
          u = (double)(float)((double)bU[ol + l] - du);
          v = (double)(float)((double)bV[ol + l] - dv);
          bU[ol + l] = (float)u;
          bV[ol + l] = (float)v;
        }
        // az*U^{n+1} + (1-az)*U^n for hydro_vertical, conzstab and conz3d
        bUo[ol + l] = act ? (float)(az * u + (1. - az) * (double)bUo[ol + l]) : 0.f;
        bVo[ol + l] = act ? (float)(az * v + (1. - az) * (double)bVo[ol + l]) : 0.f;
        um += u; vm += v;
      }
      d.unv[e] = (float)um;
      d.vnv[e] = (float)vm;
    }
    __syncwarp();
    for (int j = lane; j < cnt; j += 32) {
      d.un[base + j] = bU[j];
      d.vn[base + j] = bV[j];
      d.usv[base + j] = bUo[j];
      d.vsv[base + j] = bVo[j];
    }
    __syncwarp();
  }
  // setzev and the element part of setdepth (z-layers or pure sigma layers)
  if (valid) {
#pragma unroll
    for (int ii = 0; ii < 3; ii++) d.zen[3 * e + ii] = (float)zn3[ii];
    const float4 hm = d.hm3v[e];
    const double zmed = (zn3[0] + zn3[1] + zn3[2]) / 3.;
    const float *hld = d.hldv + (size_t)en.w * NLV;
    const float *hlv = d.hlv + (size_t)en.w * NLV;
    bool bad = false;
    int lev[3] = {0, 0, 0};
    if (ZA && P.nzadapt > 1)
      for (int ii = 0; ii < 3; ii++) lev[ii] = zad_levmax(zn3[ii], hlv, ilevel, P.rzmov);
    for (int l = 0; l < NLV; l++) {
      double h = 0.;
      if (l < ilevel) {
        if (ZA && P.nzadapt > 1) h = zad_elem_h(l, zn3, hm, ilevel, lev, hlv, hld, zmed);   // z-adaptive surface layers
        else if (l < P.nsigma) h = -(fmin((double)hm.w, (double)P.hsigma) + zmed) * (double)hld[l];   // sigma layers (:1079-1083)
        else if (ilevel == 1) h = hm.w + zmed;
        else if (l < ilevel - 1) h = (double)hld[l] + (l == 0 ? zmed : 0.);
        else h = (double)hm.w - hlv[ilevel - 2];
        if (!(h > 0.)) bad = true;
      }
      bA[ol + l] = (float)h;
    }
    if (bad) set_status(&d.out[en.w], SHY_EDEPTH);
  }
  __syncwarp();
  for (int j = lane; j < cnt; j += 32) d.hen[base + j] = bA[j];
}

}  // namespace shy
