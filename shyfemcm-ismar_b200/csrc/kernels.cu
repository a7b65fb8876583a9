// kernels.cu -- the semi-implicit step on sm_100a.
//
// Per time step, for all basins of a model at once:
//   k_column  hydro_transports + hydro_intern + hydro_zeta element part
//             (hydrodynamic.f90:758-864, 868-1416, 488-733): one warp segment per
//             element column, vertical system by PCR across lanes, 3x3 element
//             system of the zeta equation written per element.
//   k_zeta    system_init/assemble/add_rhs/solve/get (simsys_spkaux.f90:137-705,
//             sparskit_admin.f90:115-334): one thread-block cluster per basin;
//             atomic-free gather assembly into CSR in element order (FP64), then
//             FP32 preconditioned Krylov iterations inside FP64 residual
//             refinement, all in one persistent launch.
//   k_final   hydro_transports_final + setzev + element part of setdepth
//             (hydrodynamic.f90:1468-1578, wetdry.f90:594, elems_dealing.f90:1063-1097).
//   k_node    nodal part of setdepth + hydro_vertical + per-node volume
//             (elems_dealing.f90:1010-1137, hydrodynamic.f90:1582-1781).
//   k_stab    conzstab (concentration.f90:1573-2080): transport stability index.
//   k_reduce  per basin: total volume (vol_mass), sub-step counts, model time.
//   k_conz    conz3d_omp (concentration_omp.f90:65-888) for all scalars of a
//             node column, vertical system by PCR, bndo_impbc, and rhoset
//             (baroclinic.f90:654-710) after the last sub-step.
#include <cooperative_groups.h>
#include <cstdint>
#include <cstdio>

#include "../../include/shygpu.h"
#include "common.cuh"
#include "launch.h"

namespace cg = cooperative_groups;

namespace shy {

__device__ __forceinline__ void set_status(BasinOut *o, int code) {
  atomicCAS(&o->status, 0, code);
}

// UNESCO 1981 equation of state (Millero & Poisson 1981; Fofonoff & Millard
// 1983), the formulation of sigma_stp (eq_state.f90:154-230): density at one
// atmosphere and secant bulk modulus; p in bar; returns rho - 1000.
__device__ double sigma_stp_d(double s, double t, double p) {
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

// ===========================================================================
// k_column: hydro_transports / hydro_intern / hydro_zeta (element part)
// ===========================================================================
template <int S, bool COR>
__global__ void __launch_bounds__(256) k_column(Dev d) {
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
  const double dt = P.dt;
  const float *evp = d.ev8 + (size_t)e * 8;
  double b[3], c[3];
#pragma unroll
  for (int i = 0; i < 3; i++) { b[i] = evp[i]; c[i] = evp[3 + i]; }
  const double aj = evp[6];

  // barotropic terms (hydro_intern :1011-1041), FP64 like the reference
  double bz = 0., cz = 0., bpres = 0., cpres = 0., tx = 0., ty = 0.;
#pragma unroll
  for (int ii = 0; ii < 3; ii++) {
    double zz = d.zeo[3 * e + ii];
    bz += zz * b[ii]; cz += zz * c[ii];
    double pp = d.ppv[kn[ii]];
    bpres += pp * b[ii]; cpres += pp * c[ii];
    tx += d.taux[kn[ii]]; ty += d.tauy[kn[ii]];
  }
  const double drittl = 1. / 3.;
  tx *= drittl; ty *= drittl;
  const double gammat = COR ? (double)d.fcorv[e] : 0.;
  const double gamma = (double)P.af * dt * gammat;

  // column values
  const size_t o = (size_t)e * NLV + lane;
  const bool inl = lane < NLV;
  double hhi = act ? (double)d.heo[o] : 0.;
  double uui = act ? (double)d.uo[o] : 0.;
  double vvi = act ? (double)d.vo[o] : 0.;
  double hhip = seg_down<S>(hhi, 1), hhim = seg_up<S>(hhi, 1);
  double uuip = seg_down<S>(uui, 1), uuim = seg_up<S>(uui, 1);
  double vvip = seg_down<S>(vvi, 1), vvim = seg_up<S>(vvi, 1);
  if (lane + 1 >= ilevel) { hhip = 0.; uuip = uui; vvip = vvi; }
  if (lane == 0) { hhim = 0.; uuim = uui; vvim = vvi; }
  double rhact = hhi > 0. ? 1. / hhi : 0.;
  double rhactp = hhip > 0. ? 1. / hhip : 0.;
  double rhactm = hhim > 0. ? 1. / hhim : 0.;
  // element viscosity at the top (lane) and bottom (lane+1) interfaces (:1098-1104)
  double alev_t = P.vismol, alev_b = P.vismol;
  if (act) {
    const int I = NLV + 1;
    alev_t += ((double)d.visv[(size_t)kn[0] * I + lane] + d.visv[(size_t)kn[1] * I + lane] +
               d.visv[(size_t)kn[2] * I + lane]) / 3.;
    alev_b += ((double)d.visv[(size_t)kn[0] * I + lane + 1] + d.visv[(size_t)kn[1] * I + lane + 1] +
               d.visv[(size_t)kn[2] * I + lane + 1]) / 3.;
  }
  double rhp = 0., rhm = 0.;
  if (hhi > 0.) {
    if (hhip > 0.) rhp = 2.0 * alev_b / (hhi + hhip);
    if (hhim > 0.) rhm = 2.0 * alev_t / (hhi + hhim);
  }
  const double aux = dt * P.at;
  double aa = aux * rhact * (rhm + rhp);
  double aat = rhact * (rhm + rhp);
  const double bb = aux * rhactp * rhp, bbt = rhactp * rhp;
  const double cc = aux * rhactm * rhm, cct = rhactm * rhm;
  const bool bfirst = lane == 0, blast = lane == ilevel - 1;
  double ppx = 0., ppy = 0.;
  if (bfirst) { ppx -= tx; ppy -= ty; }
  if (blast) {
    // bottom_friction (chezy.f90:239-398), ireib 5: rr = cd |U_b| / h^2
    double uv = sqrt(uui * uui + vvi * vvi);
    double hzg = hhi < P.hzoff ? (double)P.hzoff : hhi;
    double rr = 0.;
    if (P.ireib == 5) rr = (double)d.czv[e] * uv / (hzg * hzg);
    aa += dt * rr;
    aat += rr;
  }

  // explicit terms fxv/fyv (set_explicit, explicit.f90:123-213)
  double fx = 0., fy = 0.;
  if (P.ahpar > 0.f && act) {            // set_diff_horizontal (:389-493)
    const double area = 12. * aj;
    for (int ii = 0; ii < 3; ii++) {
      int iei = d.ieltv[3 * e + ii];
      if (iei < 0) iei = e;
      if (lane >= d.ilhv[iei]) continue;
      const double areai = 12. * (double)d.ev8[(size_t)iei * 8 + 6];
      double ui = d.uo[(size_t)iei * NLV + lane], vi = d.vo[(size_t)iei * NLV + lane];
      double anu = (double)P.ahpar * d.difhv[o];
      double ai = 2. * anu / (area + areai);
      fx -= ai * (ui - uui);
      fy -= ai * (vi - vvi);
    }
  }
  if (P.ibarcl > 0 && P.ibarcl != 3 && P.ibarcl != 5) {
    // set_barocl_new_interface for z-layers (explicit.f90:1226-1530)
    double br = 0., cr = 0.;
    if (act) {
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        double rp = d.rho[(size_t)kn[ii] * NLV + lane];
        br += b[ii] * rp; cr += c[ii] * rp;
      }
    }
    const float *hld = d.hldv + (size_t)en.w * NLV;
    double hlayer = inl ? (double)hld[lane] : 0.;
    double hh = 0.5 * hlayer;
    double brup = seg_up<S>(br, 1), crup = seg_up<S>(cr, 1), hhup = seg_up<S>(hh, 1);
    if (lane == 0) { brup = br; crup = cr; hhup = 0.; }
    double hint = hh + hhup;
    double px = act ? hint * 0.5 * (br + brup) : 0.;
    double py = act ? hint * 0.5 * (cr + crup) : 0.;
    px = seg_scan_down<S>(px, lane);
    py = seg_scan_down<S>(py, lane);
    const double raux = (double)P.grav / P.rowass;
    if (act) { fx += raux * hlayer * px; fy += raux * hlayer * py; }
  }

  ppx += aat * uui - bbt * uuip - cct * uuim - gammat * vvi + P.grav * hhi * bz +
         (hhi / P.rowass) * bpres + fx;
  ppy += aat * vvi - bbt * vvip - cct * vvim + gammat * uui + P.grav * hhi * cz +
         (hhi / P.rowass) * cpres + fy;

  // vertical system and its solution (hydrodynamic.f90:1270-1343)
  double lo = (act && !bfirst) ? -cc : 0.;
  double up = (act && !blast) ? -bb : 0.;
  double dg = act ? 1. + aa : 1.;
  double solu, solv, hre, him = 0.;
  if (!COR) {
    double rr[3] = {act ? ppx : 0., act ? ppy : 0., act ? hhi : 0.};
    pcr_solve<S, 3>(lo, dg, up, rr, lane);
    solu = rr[0]; solv = rr[1]; hre = rr[2];
  } else {
    double2 rr[2] = {make_double2(act ? ppx : 0., act ? ppy : 0.), make_double2(act ? hhi : 0., 0.)};
    pcr_solve_c<S, 2>(lo, make_double2(dg, act ? gamma : 0.), up, rr, lane);
    solu = rr[0].x; solv = rr[0].y; hre = rr[1].x; him = rr[1].y;
  }
  float uhat = act ? (float)(uui - dt * solu) : 0.f;
  float vhat = act ? (float)(vvi - dt * solv) : 0.f;
  if (valid && inl) {
    d.un[o] = uhat;
    d.vn[o] = vhat;
    d.ddx[o] = act ? (float)hre : 0.f;
    if (COR) d.ddxi[o] = act ? (float)him : 0.f;
  }

  // hydro_zeta (hydrodynamic.f90:604-733): layer sums and the element system
  // ddxv(ju) = Re, ddxv(jv) = Im, ddyv(ju) = -Im, ddyv(jv) = Re
  double dbb = seg_sum<S>(act ? hre : 0.);
  double dcb = seg_sum<S>(act ? him : 0.);
  double dbc = -dcb, dcc = dbb;
  double uold = seg_sum<S>(uui), vold = seg_sum<S>(vvi);
  double uh = seg_sum<S>((double)uhat), vh = seg_sum<S>((double)vhat);
  if (lane == 0 && valid) {
    const double az = P.az, am = P.am;
    const double ut = az * uh + (1. - az) * uold;
    const double vt = az * vh + (1. - az) * vold;
    const double delta = dt * dt * az * am * (double)P.grav;
    double z[3], hia[3][3], hik[3];
#pragma unroll
    for (int i = 0; i < 3; i++) z[i] = d.zeo[3 * e + i];
#pragma unroll
    for (int n = 0; n < 3; n++) {
#pragma unroll
      for (int m = 0; m < 3; m++) {
        double abn = b[n] * (b[m] * dbb + c[m] * dbc);
        double acn = c[n] * (b[m] * dcb + c[m] * dcc);
        hia[n][m] = aj * ((n == m ? 4. : 0.) + 12. * delta * (abn + acn));
      }
      hik[n] = hia[n][0] * z[0] + hia[n][1] * z[1] + hia[n][2] * z[2] +
               12. * aj * dt * (ut * b[n] + vt * c[n]);
    }
    // level boundary conditions (:688-704), rzv at the new time (sp111)
    const double tnew = d.out[en.w].dtime + dt;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      int kb = d.kbnd[kn[i]];
      if (kb > 0) {
        double rw = level_bc(d, P, kb, tnew);
        int j1 = (i + 1) % 3, j2 = (i + 2) % 3;
        hik[j1] -= rw * hia[j1][i];
        hik[j2] -= rw * hia[j2][i];
        hia[i][j1] = 0.; hia[i][j2] = 0.; hia[j1][i] = 0.; hia[j2][i] = 0.;
        hik[i] = rw * hia[i][i];
      }
    }
#pragma unroll
    for (int n = 0; n < 3; n++) {
#pragma unroll
      for (int m = 0; m < 3; m++) d.hia[(size_t)(3 * n + m) * d.NEL + e] = (float)hia[n][m];
      d.hik[(size_t)n * d.NEL + e] = (float)hik[n];
    }
  }
}

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
    double um = seg_sum<S>(u), vm = seg_sum<S>(v);
    if (lane == 0 && valid) { d.unv[e] = (float)um; d.vnv[e] = (float)vm; }
  }
  // setzev and the element part of setdepth (z-layers)
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
    if (ilevel == 1) h = hm.w + zmed;
    else if (lane < ilevel - 1) h = (double)hld[lane] + (lane == 0 ? zmed : 0.);
    else h = (double)hm.w - hlv[ilevel - 2];
    if (!(h > 0.) && valid) set_status(&d.out[en.w], SHY_EDEPTH);
  }
  if (valid && lane < NLV) d.hen[o] = (float)h;
}

// ===========================================================================
// k_node: nodal layer thickness, vertical velocity, node volume
// ===========================================================================
template <int S>
__global__ void __launch_bounds__(256) k_node(Dev d, const int *kbas, int init_only) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const bool valid = k0 < d.NKN;
  const int k = valid ? k0 : d.NKN - 1;
  const int NLV = d.NLV;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  const int lmax = d.ilhkv[k];
  const bool act = lane < lmax;
  const double z = d.zn[k];
  const double az = P.az, azt = 1. - az;
  const float *hld = d.hldv + (size_t)b * NLV;
  const float *hlv = d.hlv + (size_t)b * NLV;
  const double hldl = lane < NLV ? (double)hld[lane] : 0.;
  double hsum = 0., vf = 0., va = 0.;
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
    const int q = d.inc[p];
    const int e = q / 3, ii = q - 3 * e;
    const int le = d.ilhv[e];
    if (lane >= le) continue;
    const float *evp = d.ev8 + (size_t)e * 8;
    const double aj = evp[6];
    const double areafv = 4. * aj;            // 12*aj/3
    const float4 hm = d.hm3v[e];
    const double htot = ii == 0 ? hm.x : (ii == 1 ? hm.y : hm.z);
    double hl;
    if (le == 1) hl = htot + z;
    else if (lane < le - 1) hl = hldl + (lane == 0 ? z : 0.);
    else hl = htot - hlv[le - 2];
    hsum += areafv * hl;
    if (!init_only) {
      const double bb = evp[ii], cc = evp[3 + ii];
      const size_t oe = (size_t)e * NLV + lane;
      double ffn = (double)d.un[oe] * bb + (double)d.vn[oe] * cc;
      double ffo = (double)d.uo[oe] * bb + (double)d.vo[oe] * cc;
      double ff = ffn * az + ffo * azt;
      const double aj4 = 4. * aj;
      vf += 3. * aj4 * ff;
      va += aj4;
    }
  }
  const size_t o = (size_t)k * NLV + lane;
  const double area = act ? (double)d.areakv[o] : 0.;
  double hk = act && area > 0. ? hsum / area : 0.;
  float hkf = (float)hk;
  if (act && !(hkf > 0.f) && valid) set_status(&d.out[b], SHY_EDEPTH);
  if (valid && lane < NLV) d.hkn[o] = act ? hkf : 0.f;
  // node volume (masscont: sum of real hdknv*areakv in double)
  double vol = act ? (double)(hkf * (float)area) : 0.;
  vol = seg_sum<S>(vol);
  if (lane == 0 && valid) d.vol_node[k] = vol;
  if (init_only) return;
  // hydro_vertical: w from continuity, bottom-up (hydrodynamic.f90:1711-1771)
  const int I = NLV + 1;
  double dv = 0.;
  if (act && P.nlv > 1) {
    double voln = (double)(hkf * (float)area), volo = (double)(d.hko[o] * (float)area);
    dv = vf - (voln - volo) / P.dt;
  }
  double wtop = seg_scan_up<S>(dv, lane);      // flux through the top interface of layer lane
  if (lane == 0) wtop = 0.;                     // wlnv(lmin-1) = 0
  if (lane >= 1 && act && va > 0.) wtop /= va;
  if (!act || P.nlv == 1 || d.kbnd[k] > 0) wtop = 0.;
  if (valid) {
    if (lane < I) d.wl[(size_t)k * I + lane] = (float)wtop;
    if (lane == 0 && S < I) d.wl[(size_t)k * I + S] = 0.f;
    if (lane == 0 && S == NLV) d.wl[(size_t)k * I + NLV] = 0.f;
  }
}

// ===========================================================================
// k_stab: conzstab stability index per node, max-reduced per basin/scalar
// ===========================================================================
template <int S>
__global__ void __launch_bounds__(256) k_stab(Dev d, const int *kbas) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const bool valid = k0 < d.NKN;
  const int k = valid ? k0 : d.NKN - 1;
  const int NLV = d.NLV, I = NLV + 1;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  if (P.nsc == 0) return;
  const int lmax = d.ilhkv[k];
  const bool act = lane < lmax;
  const double az = P.az, azt = 1. - az, adt = 1. - (double)P.ad, aat = 1. - (double)P.aa;
  const size_t o = (size_t)k * NLV + lane;
  const double hold = act ? (double)d.hko[o] : 0., hnew = act ? (double)d.hkn[o] : 0.;
  const double rvptop = act ? (double)d.difv[(size_t)k * I + lane] + P.difmol : 0.;
  const double rvpbot = act ? (double)d.difv[(size_t)k * I + lane + 1] + P.difmol : 0.;
  float rk_prev = -1.f;
  float stab = 0.f;
  for (int s = 0; s < P.nsc; s++) {
    const float rkpar = P.rkpar[s];
    if (rkpar != rk_prev) {
      rk_prev = rkpar;
      double chigh = 0., clow = 0., cn = 0., cdiag = 0.;
      if (act) {
        for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
          const int q = d.inc[p];
          const int e = q / 3, ii = q - 3 * e;
          const int le = d.ilhv[e];
          if (lane >= le) continue;
          const int4 en = d.enode[e];
          const int kn[3] = {en.x, en.y, en.z};
          const float *evp = d.ev8 + (size_t)e * 8;
          const double aj4 = 4. * (double)evp[6];
          const size_t oe = (size_t)e * NLV + lane;
          const double us = az * d.un[oe] + azt * d.uo[oe];
          const double vs = az * d.vn[oe] + azt * d.vo[oe];
          double coadv = 0., ciadv = 0.;
          for (int jj = 0; jj <= ii; jj++) {
            const double f = us * evp[jj] + vs * evp[3 + jj];
            double wt = lane == 0 ? 0. : (double)d.wl[(size_t)kn[jj] * I + lane];
            double wb = lane + 1 == le ? 0. : (double)d.wl[(size_t)kn[jj] * I + lane + 1];
            double fwin = 0., fwout = 0.;
            if (wt > 0.) fwout += aat * wt; else fwin -= aat * wt;
            if (wb > 0.) fwin += aat * wb; else fwout -= aat * wb;
            const double chadv = aj4 * 3. * f;
            if (chadv < 0.) coadv = aj4 * fwout - chadv;
            else ciadv = aj4 * fwin + chadv;
          }
          chigh += fmax(coadv, ciadv);
          const double rk3 = 3. * (double)rkpar * d.difhv[oe];
          clow += aj4 * rk3 * hold * (double)d.wdif[(size_t)e * 9 + 4 * ii];
          const double hdv = d.heo[oe];
          const double hdvm = lane > 0 ? (double)d.heo[oe - 1] : 0.;
          const double hdvp = lane + 1 < le ? (double)d.heo[oe + 1] : 0.;
          const double hmtop = lane > 0 ? 2. * rvptop / (hdvm + hdv) : 0.;
          const double hmbot = lane + 1 < le ? 2. * rvpbot / (hdv + hdvp) : 0.;
          cn += aj4 * adt * (hmtop + hmbot);
          cdiag += aj4 * fmin(hold, hnew);
        }
      }
      double r = (act && cdiag > 0.) ? (chigh + clow + cn) / cdiag : 0.;
      stab = seg_max<S>((float)r);
    }
    if (lane == 0 && valid && d.kbnd[k] == 0) atomic_max_pos(&d.out[b].stab[s], stab);
  }
}

// ===========================================================================
// k_reduce: per basin (one block each): volume, sub-step counts, time
// ===========================================================================
__global__ void __launch_bounds__(256) k_reduce(Dev d, int nsub, int advance) {
  const int b = blockIdx.x;
  const BasinPar &P = d.par[b];
  BasinOut &O = d.out[b];
  __shared__ double part[256];
  double s = 0.;
  for (int k = threadIdx.x; k < P.nk; k += blockDim.x) s += d.vol_node[P.k0 + k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    O.volume = part[0];
    if (advance) {
      int mx = 1;
      for (int sc = 0; sc < P.nsc; sc++) {
        // scal3sh: sindex = stabind/rstol, rindex = dt*sindex, istot = 1 + rindex
        float sindex = O.stab[sc] / P.rstol;
        float rindex = (float)P.dt * sindex;
        int ist = 1 + (int)rindex;
        O.stab[sc] = (float)ist;       // now holds the sub-step count of scalar sc
        mx = ist > mx ? ist : mx;
        if (ist > P.istot_max) set_status(&O, SHY_EISTOT);

      }
      O.istot = mx;
      atomicMax(d.imax, mx);
      O.dtime += P.dt;
    }
  }
}

// ===========================================================================
// k_conz: one transport sub-step of every scalar of a node column
// ===========================================================================
template <int S>
__device__ __forceinline__ double clip_load(const float *a, size_t i, bool is_temp) {
  float v = a[i];
  if (!is_temp && v < 1.e-15f) v = 0.f;     // scal3sh: where(cnv < 1e-15) cnv = 0
  return v;
}

template <int S>
__global__ void __launch_bounds__(256) k_conz(Dev d, const int *kbas, int j_arg) {
  const int j = j_arg >= 0 ? j_arg : *d.subj;   // sub-step index: argument or device counter
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const bool valid = k0 < d.NKN;
  const int k = valid ? k0 : d.NKN - 1;
  const int NLV = d.NLV, I = NLV + 1;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  const BasinOut &O = d.out[b];
  const int lmax = d.ilhkv[k];
  const bool act = lane < lmax;
  const size_t o = (size_t)k * NLV + lane;
  const size_t SN = (size_t)d.NKN * NLV;
  const double az = P.az, azt = 1. - az, ad = P.ad, adt = 1. - ad, aa = P.aa, aat = 1. - aa;
  const double hko = act ? (double)d.hko[o] : 0., hkn = act ? (double)d.hkn[o] : 0.;
  const double rvptop = act ? (double)d.difv[(size_t)k * I + lane] + P.difmol : 0.;
  const double rvpbot = act ? (double)d.difv[(size_t)k * I + lane + 1] + P.difmol : 0.;
  const double wtop_k = act ? (double)d.wl[(size_t)k * I + lane] : 0.;
  const double wbot_k = act ? (double)d.wl[(size_t)k * I + lane + 1] : 0.;
  // Buffers: sub-step 1 reads the step's input d.sc_in, the last sub-step
  // (isact == istot) writes the step's output d.sc_out, intermediate sub-steps
  // go through two scratch buffers.  A launch j beyond a scalar's istot does
  // nothing for it, so the number of launches may exceed the sub-steps.
  double tnew = 0., snew = 0.;
  const int sT = P.itemp ? 0 : -1, sS = P.isalt ? (P.itemp ? 1 : 0) : -1;
  int ist_ts = 1;
  if (sT >= 0) ist_ts = max(ist_ts, (int)O.stab[sT]);
  if (sS >= 0) ist_ts = max(ist_ts, (int)O.stab[sS]);
  for (int s = 0; s < P.nsc; s++) {
    const bool is_temp = P.is_temp[s] != 0;
    const int istot = (int)O.stab[s];
    const int isact = j + 1;
    if (isact > istot) {                 // finished in an earlier launch
      if ((s == sT || s == sS) && lane < NLV) {
        const float cv = d.sc_out[s * SN + o];
        if (s == sT) tnew = cv; else snew = cv;
      }
      continue;
    }
    const float *cin = (isact == 1 ? d.sc_in : (isact & 1 ? d.scr1 : d.scr0)) + s * SN;
    float *cout = (isact == istot ? d.sc_out : (isact & 1 ? d.scr0 : d.scr1)) + s * SN;
    const double rstot = istot;
    const double rso = (isact - 1) / rstot, rsn = isact / rstot, rsot = 1. - rso, rsnt = 1. - rsn;
    const double dt = P.dt / rstot;
    const double rkpar = P.rkpar[s];
    double cl = act ? clip_load<S>(cin, o, is_temp) : 0.;
    double clm1 = seg_up<S>(cl, 1), clp1 = seg_down<S>(cl, 1);
    if (lane == 0) clm1 = 0.;
    if (lane + 1 >= lmax) clp1 = 0.;
    const double hold = rso * hkn + rsot * hko, hnew = rsn * hkn + rsnt * hko;
    double holdm = seg_up<S>(hold, 1), holdp = seg_down<S>(hold, 1);
    double hnewm = seg_up<S>(hnew, 1), hnewp = seg_down<S>(hnew, 1);
    if (lane == 0) { holdm = 0.; hnewm = 0.; }
    double cn = 0., cdg = 0., clo = 0., chi = 0.;
    if (act) {
      for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
        const int q = d.inc[p];
        const int e = q / 3, ii = q - 3 * e;
        const int le = d.ilhv[e];
        if (lane >= le) continue;
        const int4 en = d.enode[e];
        const int kn[3] = {en.x, en.y, en.z};
        const float *evp = d.ev8 + (size_t)e * 8;
        const double aj4 = 4. * (double)evp[6];
        const size_t oe = (size_t)e * NLV + lane;
        const bool hasp = lane + 1 < le;           // presentl(l+1)
        // vertical: w at the element's bottom interface is zero (wl(ilevel)=0)
        const double wt = wtop_k;
        const double wb = hasp ? wbot_k : 0.;
        const double cnext = hasp ? clp1 : 0.;
        double vtop = 0., vbot = 0.;
        if (lane > 0) vtop = wt * (wt > 0. ? cl : clm1);
        if (hasp) vbot = wb * (wb > 0. ? cnext : cl);
        const double fw = aat * (vtop - vbot);
        double clc = 0., clmm = 0., clpp = 0.;
        const double hmotop = lane > 0 ? 2. * rvptop / (holdm + hold) : 0.;
        const double hmobot = hasp ? 2. * rvpbot / (hold + holdp) : 0.;
        const double hmntop = lane > 0 ? 2. * rvptop / (hnewm + hnew) : 0.;
        const double hmnbot = hasp ? 2. * rvpbot / (hnew + hnewp) : 0.;
        const double fd = adt * ((cl - cnext) * hmobot - (clm1 - cl) * hmotop);
        clc += ad * (hmntop + hmnbot);
        clmm -= ad * hmntop;
        clpp -= ad * hmnbot;
        double w = lane == 0 ? 0. : wt;
        if (w >= 0.) clc += aa * w; else clmm += aa * w;
        w = hasp ? wb : 0.;
        if (w > 0.) clpp -= aa * w; else clc -= aa * w;
        // horizontal upwind advection (concentration_omp.f90:566-673)
        const double us = az * d.un[oe] + azt * d.uo[oe];
        const double vs = az * d.vn[oe] + azt * d.vo[oe];
        double c3[3], f3[3];
        int itot = 0, isum = 0;
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          c3[jj] = jj == ii ? cl : clip_load<S>(cin, (size_t)kn[jj] * NLV + lane, is_temp);
          f3[jj] = us * evp[jj] + vs * evp[3 + jj];
          if (f3[jj] < 0.) { itot++; isum += jj + 1; }
        }
        double fl;
        if (itot == 1) fl = f3[ii] * c3[isum - 1];
        else if (itot == 2) {
          const int is = 6 - isum - 1;
          if (ii == is) fl = -(f3[(is + 1) % 3] * c3[(is + 1) % 3] + f3[(is + 2) % 3] * c3[(is + 2) % 3]);
          else fl = f3[ii] * c3[ii];
        } else fl = 0.;
        double wdiff = 0.;
        if (rkpar != 0.) {
#pragma unroll
          for (int iii = 0; iii < 3; iii++) wdiff += (double)d.wdif[(size_t)e * 9 + 3 * iii + ii] * c3[iii];
        }
        const double rk3 = 3. * rkpar * d.difhv[oe];
        const double hmed = rso * d.hen[oe] + rsot * d.heo[oe];
        cn += aj4 * (hold * cl + dt * (3. * fl - fw - rk3 * hmed * wdiff - fd));
        clo += aj4 * dt * clmm;
        chi += aj4 * dt * clpp;
        cdg += aj4 * dt * clc + aj4 * hnew;
      }
    }
    // conz3d_nodes: vertical system (concentration_omp.f90:841-868)
    double cres;
    if ((P.aa == 0.f && P.ad == 0.f) || P.nlv == 1) {
      cres = (act && cdg != 0.) ? cn / cdg : cn;
    } else {
      double rr[1] = {act ? cn : 0.};
      if (act && cdg == 0. && valid) set_status(&d.out[b], SHY_ESINGULAR);
      pcr_solve<S, 1>(act ? clo : 0., act ? cdg : 1., act ? chi : 0., rr, lane);
      cres = rr[0];
    }
    // bndo_impbc: scalar value imposed on level-boundary nodes
    if (act && d.kbnd[k] > 0) cres = d.cbnd[s * SN + o];
    if (!act) cres = 0.;
    float cf = (float)cres;
    if (valid && lane < NLV) cout[o] = cf;
    if (s == sT) tnew = cf;
    else if (s == sS) snew = cf;
  }
  // rhoset once T and S have their final values (baroclinic.f90:654-710), z-layers
  if (j + 1 == ist_ts && P.ibarcl > 0 && P.itemp && P.isalt) {
    const float *hld = d.hldv + (size_t)b * NLV;
    const double hh = lane < NLV ? 0.5 * (double)hld[lane] : 0.;
    const double rold = act ? (double)d.rho[o] : 0.;
    const double dpresc = rold * P.grav * hh;
    // depth to mid-layer and baroclinic pressure at mid-layer
    double depth = seg_scan_down<S>(act ? 2. * hh : 0., lane) - hh;
    double pbc = seg_scan_down<S>(act ? 2. * dpresc : 0., lane) - dpresc;
    if (act && valid) {
      const double rho0 = P.rowass, sigma0 = rho0 - 1000.;
      double pres = 1.e-5 * (rho0 * P.grav * depth + pbc);
      double salt = snew > 0.f ? (double)snew : 0.;
      d.rho[o] = (float)(sigma_stp_d(salt, (double)tnew, (double)(float)pres) - sigma0);
    }
  }
}

// rhoset for the initial state (barocl(0): rhov = 0, then rhoset_shell(3)),
// temperature and salinity taken from the scalar buffer d.sc_in
template <int S>
__global__ void __launch_bounds__(256) k_rhoset(Dev d, const int *kbas) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const bool valid = k0 < d.NKN;
  const int k = valid ? k0 : d.NKN - 1;
  const int NLV = d.NLV;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  const int lmax = d.ilhkv[k];
  const bool act = lane < lmax;
  const size_t o = (size_t)k * NLV + lane;
  if (!(P.ibarcl > 0 && P.itemp && P.isalt)) {
    if (valid && lane < NLV) d.rho[o] = 0.f;
    return;
  }
  const size_t SN = (size_t)d.NKN * NLV;
  const float *tv = d.sc_in, *sv = d.sc_in + SN;     // T is scalar 0, S scalar 1
  const float *hld = d.hldv + (size_t)b * NLV;
  const double hh = lane < NLV ? 0.5 * (double)hld[lane] : 0.;
  const double depth = seg_scan_down<S>(act ? 2. * hh : 0., lane) - hh;
  double r = 0.;
  const double t = act ? (double)tv[o] : 0., sal = act ? (double)sv[o] : 0.;
  for (int it = 0; it < 3; it++) {
    const double dpresc = r * P.grav * hh;
    double pbc = seg_scan_down<S>(act ? 2. * dpresc : 0., lane) - dpresc;
    const double rho0 = P.rowass, sigma0 = rho0 - 1000.;
    double pres = 1.e-5 * (rho0 * P.grav * depth + pbc);
    r = act ? (double)(float)(sigma_stp_d(sal > 0. ? sal : 0., t, (double)(float)pres) - sigma0) : 0.;
  }
  if (valid && lane < NLV) d.rho[o] = (float)r;
}

// ===========================================================================
// k_zeta: assembly + Krylov solve, one thread-block cluster per basin
// ===========================================================================


template <int NV>
__device__ __forceinline__ void cluster_sum(cg::cluster_group &cl, double (&v)[NV], double *wbuf,
                                            double *slots, double *bc, int &par, int CL) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double x = v[i];
#pragma unroll
    for (int dd = 16; dd > 0; dd >>= 1) x += __shfl_xor_sync(0xffffffffu, x, dd);
    if (lane == 0) wbuf[i * 32 + warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double x = lane < nw ? wbuf[i * 32 + lane] : 0.;
#pragma unroll
      for (int dd = 16; dd > 0; dd >>= 1) x += __shfl_xor_sync(0xffffffffu, x, dd);
      if (lane == 0) slots[par * 4 + i] = x;
    }
  }
  cl.sync();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double t = 0.;
      for (int q = 0; q < CL; q++) t += *cl.map_shared_rank(&slots[par * 4 + i], q);
      bc[i] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = bc[i];
  par ^= 1;
}

__global__ void __launch_bounds__(1024) k_zeta(Dev d, ZetaArgs za, int CL, int b_first) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int b = b_first + (int)(blockIdx.x / CL);
  const BasinPar &P = d.par[b];
  BasinOut &O = d.out[b];
  __shared__ double wbuf[4 * 32];
  __shared__ double slots[2 * 4];
  __shared__ double bcast[4];
  int par = 0;
  const int chunk = (P.nk + CL - 1) / CL;
  const int r0 = P.k0 + rank * chunk;
  const int r1 = min(P.k0 + P.nk, r0 + chunk);
  const int tid = threadIdx.x, nth = blockDim.x;
  if (rank == 0 && tid < kMaxScal) O.stab[tid] = 0.f;   // reset for k_stab max
  if (blockIdx.x == 0 && tid == 0 && d.imax) { *d.imax = 0; *d.subj = 0; }
  const float dtf = (float)P.dt;

  // ---- assembly (system_init + hydro_zeta scatter + system_add_rhs) ----
  for (int i = r0 + tid; i < r1; i += nth) {
    double diag = 0.;
    for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) {
      double v = 0.;
      for (int t = d.slot_ptr[s]; t < d.slot_ptr[s + 1]; t++) {
        const int src = d.slot_src[t];
        const int e = src / 9, c = src - 9 * e;
        v += (double)za.hia[(size_t)c * za.cs + (size_t)e * za.es];
      }
      d.val64[s] = v;
      d.val32[s] = (float)v;
      if (d.col[s] == i) diag = v;
    }
    double rhs = 0.;
    for (int p = d.inc_ptr[i]; p < d.inc_ptr[i + 1]; p++) {
      const int q = d.inc[p];
      const int e = q / 3, ii = q - 3 * e;
      rhs += (double)za.hik[(size_t)ii * za.cs + (size_t)e * za.es];
    }
    rhs += (double)(dtf * d.rqv[i]);
    d.rhs64[i] = rhs;
    d.dinv32[i] = diag != 0. ? (float)(1. / diag) : 1.f;
    d.x64[i] = za.explicit_mode ? (diag != 0. ? rhs / diag : 0.) : (double)za.zguess[i];
  }
  if (za.explicit_mode) {
    for (int i = r0 + tid; i < r1; i += nth) d.zn[i] = (float)d.x64[i];
    if (rank == 0 && tid == 0) { O.iters = 0; O.refinements = 0; O.resid0 = 0.; O.resid = 0.; }
    return;
  }
  cl.sync();

  // ---- FP64 residual refinement around FP32 Krylov iterations ----
  double tol = 0., rn = 0.;
  int iters = 0, outer = 0;
  bool conv = false;
  for (outer = 0; outer < za.max_outer; outer++) {
    double acc[1] = {0.};
    for (int i = r0 + tid; i < r1; i += nth) {
      double t = d.rhs64[i];
      for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) t -= d.val64[s] * __ldcg(&d.x64[d.col[s]]);
      d.r32[i] = (float)t;
      acc[0] += t * t;
    }
    cluster_sum<1>(cl, acc, wbuf, slots, bcast, par, CL);
    rn = sqrt(acc[0]);
    if (outer == 0) {
      tol = (double)P.rtol * rn + (double)P.atol;
      if (rank == 0 && tid == 0) O.resid0 = rn;
    }
    if (rn <= tol) { conv = true; break; }
    const double itol = fmax((double)za.inner_rtol * rn, 0.25 * tol);
    if (za.sym) {
      // preconditioned CG (Jacobi), p computed on the fly from z and p_prev so
      // that one cluster barrier per reduction suffices
      double a2[1] = {0.};
      for (int i = r0 + tid; i < r1; i += nth) {
        float r = d.r32[i], z = d.dinv32[i] * r;
        d.z32[i] = z; d.e32[i] = 0.f; d.p32[i] = 0.f;
        a2[0] += (double)r * z;
      }
      cluster_sum<1>(cl, a2, wbuf, slots, bcast, par, CL);
      double rz = a2[0], beta = 0.;
      float *pprev = d.p32, *pcur = d.q32 + 0;   // q32 doubles as the second p buffer
      for (int it = 0; it < P.maxit; it++) {
        double pq[1] = {0.};
        const float fb = (float)beta;
        for (int i = r0 + tid; i < r1; i += nth) {
          float q = 0.f;
          for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) {
            const int j = d.col[s];
            q += d.val32[s] * (__ldcg(&d.z32[j]) + fb * __ldcg(&pprev[j]));
          }
          const float p = d.z32[i] + fb * pprev[i];
          pcur[i] = p;
          d.t32[i] = q;
          pq[0] += (double)p * q;
        }
        cluster_sum<1>(cl, pq, wbuf, slots, bcast, par, CL);
        const float alpha = (float)(rz / pq[0]);
        double a3[2] = {0., 0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          const float p = pcur[i];
          d.e32[i] += alpha * p;
          float r = d.r32[i] - alpha * d.t32[i];
          d.r32[i] = r;
          float z = d.dinv32[i] * r;
          d.z32[i] = z;
          a3[0] += (double)r * z;
          a3[1] += (double)r * r;
        }
        cluster_sum<2>(cl, a3, wbuf, slots, bcast, par, CL);
        iters++;
        if (sqrt(a3[1]) <= itol || !(a3[0] == a3[0])) break;
        beta = a3[0] / rz;
        rz = a3[0];
        float *tmp = pprev; pprev = pcur; pcur = tmp;
      }
    } else {
      // BiCGStab (van der Vorst 1992), right preconditioned (Jacobi), FP32
      double a1[1] = {0.};
      for (int i = r0 + tid; i < r1; i += nth) {
        float r = d.r32[i];
        d.rh32[i] = r; d.p32[i] = 0.f; d.v32[i] = 0.f; d.e32[i] = 0.f;
        a1[0] += (double)r * r;
      }
      cluster_sum<1>(cl, a1, wbuf, slots, bcast, par, CL);
      double rho = 1., alpha = 1., omega = 1.;
      for (int it = 0; it < P.maxit; it++) {
        double g1[1] = {0.};
        for (int i = r0 + tid; i < r1; i += nth) g1[0] += (double)d.rh32[i] * d.r32[i];
        cluster_sum<1>(cl, g1, wbuf, slots, bcast, par, CL);
        const double rho1 = g1[0];
        const double beta = (rho1 / rho) * (alpha / omega);
        rho = rho1;
        const float fb = (float)beta, fo = (float)omega;
        for (int i = r0 + tid; i < r1; i += nth) {
          float p = d.r32[i] + fb * (d.p32[i] - fo * d.v32[i]);
          d.p32[i] = p;
          d.z32[i] = d.dinv32[i] * p;         // phat
        }
        cl.sync();
        double g2[1] = {0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          float v = 0.f;
          for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) v += d.val32[s] * __ldcg(&d.z32[d.col[s]]);
          d.v32[i] = v;
          g2[0] += (double)d.rh32[i] * v;
        }
        cluster_sum<1>(cl, g2, wbuf, slots, bcast, par, CL);
        alpha = rho / g2[0];
        const float fa = (float)alpha;
        for (int i = r0 + tid; i < r1; i += nth) {
          float s = d.r32[i] - fa * d.v32[i];
          d.s32[i] = s;
          d.q32[i] = d.dinv32[i] * s;         // shat
        }
        cl.sync();
        double g3[2] = {0., 0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          float t = 0.f;
          for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) t += d.val32[s] * __ldcg(&d.q32[d.col[s]]);
          d.t32[i] = t;
          g3[0] += (double)t * d.s32[i];
          g3[1] += (double)t * t;
        }
        cluster_sum<2>(cl, g3, wbuf, slots, bcast, par, CL);
        omega = g3[1] > 0. ? g3[0] / g3[1] : 0.;
        const float fw = (float)omega;
        double g4[1] = {0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          d.e32[i] += fa * d.z32[i] + fw * d.q32[i];
          float r = d.s32[i] - fw * d.t32[i];
          d.r32[i] = r;
          g4[0] += (double)r * r;
        }
        cluster_sum<1>(cl, g4, wbuf, slots, bcast, par, CL);
        iters++;
        if (sqrt(g4[0]) <= itol || omega == 0. || !(g4[0] == g4[0])) break;
      }
    }
    for (int i = r0 + tid; i < r1; i += nth) d.x64[i] += (double)d.e32[i];
    cl.sync();
  }
  for (int i = r0 + tid; i < r1; i += nth) d.zn[i] = (float)d.x64[i];
  if (rank == 0 && tid == 0) {
    O.iters = iters;
    O.refinements = outer;
    O.resid = rn;
    if (!conv) set_status(&O, SHY_ENOCONV);
  }
}

}  // namespace shy

// ---------------------------------------------------------------------------
// launch wrappers (host side)
// ---------------------------------------------------------------------------
namespace shy {

template <int S>
static void launch_elem_S(const Dev &d, int which, int init_only, cudaStream_t st, bool cor) {
  const int threads = 256;
  const long long nt = (long long)d.NEL * S;
  const int blocks = (int)((nt + threads - 1) / threads);
  if (which == 0) {
    if (cor) k_column<S, true><<<blocks, threads, 0, st>>>(d);
    else k_column<S, false><<<blocks, threads, 0, st>>>(d);
  } else {
    if (cor) k_final<S, true><<<blocks, threads, 0, st>>>(d, init_only);
    else k_final<S, false><<<blocks, threads, 0, st>>>(d, init_only);
  }
}

template <int S>
static void launch_node_S(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st) {
  const int threads = 256;
  const long long nt = (long long)d.NKN * S;
  const int blocks = (int)((nt + threads - 1) / threads);
  switch (which) {
    case 0: k_node<S><<<blocks, threads, 0, st>>>(d, kbas, a); break;
    case 1: k_stab<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 2: k_conz<S><<<blocks, threads, 0, st>>>(d, kbas, a); break;
    case 3: k_rhoset<S><<<blocks, threads, 0, st>>>(d, kbas); break;
  }
}

void launch_elem(const Dev &d, int which, int init_only, cudaStream_t st, bool cor) {
  switch (d.S) {
    case 1: launch_elem_S<1>(d, which, init_only, st, cor); break;
    case 2: launch_elem_S<2>(d, which, init_only, st, cor); break;
    case 4: launch_elem_S<4>(d, which, init_only, st, cor); break;
    case 8: launch_elem_S<8>(d, which, init_only, st, cor); break;
    case 16: launch_elem_S<16>(d, which, init_only, st, cor); break;
    default: launch_elem_S<32>(d, which, init_only, st, cor); break;
  }
}

void launch_node(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st) {
  switch (d.S) {
    case 1: launch_node_S<1>(d, kbas, which, a, b, st); break;
    case 2: launch_node_S<2>(d, kbas, which, a, b, st); break;
    case 4: launch_node_S<4>(d, kbas, which, a, b, st); break;
    case 8: launch_node_S<8>(d, kbas, which, a, b, st); break;
    case 16: launch_node_S<16>(d, kbas, which, a, b, st); break;
    default: launch_node_S<32>(d, kbas, which, a, b, st); break;
  }
}

// control of the device-driven transport sub-step loop (body of a CUDA-graph
// WHILE node): advance the sub-step index and keep looping while any basin
// has sub-steps left (scal3sh's isact = 1..istot, concentration.f90:728).
__global__ void k_subctl(Dev d, cudaGraphConditionalHandle h) {
  const int nj = *d.subj + 1;
  *d.subj = nj;
  *d.nsub_launched += 2;
  cudaGraphSetConditional(h, nj < *d.imax ? 1u : 0u);
}

void launch_subctl(const Dev &d, cudaGraphConditionalHandle h, cudaStream_t st) {
  k_subctl<<<1, 1, 0, st>>>(d, h);
}

void launch_reduce(const Dev &d, int nsub, int advance, cudaStream_t st) {
  k_reduce<<<d.nbasin, 256, 0, st>>>(d, nsub, advance);
}

cudaError_t launch_zeta(const Dev &d, const ZetaArgs &za, int CL, int threads, int b_first,
                        int nb, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nb * CL, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_zeta, d, za, CL, b_first);
}

cudaError_t zeta_kernel_setup(int CL) {
  if (CL > 8) return cudaFuncSetAttribute(k_zeta, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return cudaSuccess;
}

int zeta_max_active_clusters(int CL, int threads) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CL, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_zeta, &cfg) != cudaSuccess) return -1;
  return n;
}

}  // namespace shy
