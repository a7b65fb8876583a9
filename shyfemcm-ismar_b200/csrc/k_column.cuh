// k_column.cuh -- hydro_transports / hydro_intern / hydro_zeta element part
// Included by step.cu.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace shy {

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
  // single precision like the reference's real locals (hact, alev, aa..cct)
  const float hhi = act ? d.heo[o] : 0.f;
  const float uui = act ? d.uo[o] : 0.f;
  const float vvi = act ? d.vo[o] : 0.f;
  float hhip = seg_down<S>(hhi, 1), hhim = seg_up<S>(hhi, 1);
  float uuip = seg_down<S>(uui, 1), uuim = seg_up<S>(uui, 1);
  float vvip = seg_down<S>(vvi, 1), vvim = seg_up<S>(vvi, 1);
  if (lane + 1 >= ilevel) { hhip = 0.f; uuip = uui; vvip = vvi; }
  if (lane == 0) { hhim = 0.f; uuim = uui; vvim = vvi; }
  const float rhact = hhi > 0.f ? 1.f / hhi : 0.f;
  const float rhactp = hhip > 0.f ? 1.f / hhip : 0.f;
  const float rhactm = hhim > 0.f ? 1.f / hhim : 0.f;
  // element viscosity at the top (lane) and bottom (lane+1) interfaces (:1098-1104)
  float alev_t = P.vismol, alev_b = P.vismol;
  if (act) {
    const int I = NLV + 1;
    alev_t += (d.visv[(size_t)kn[0] * I + lane] + d.visv[(size_t)kn[1] * I + lane] +
               d.visv[(size_t)kn[2] * I + lane]) * (1.f / 3.f);
    alev_b += (d.visv[(size_t)kn[0] * I + lane + 1] + d.visv[(size_t)kn[1] * I + lane + 1] +
               d.visv[(size_t)kn[2] * I + lane + 1]) * (1.f / 3.f);
  }
  float rhp = 0.f, rhm = 0.f;
  if (hhi > 0.f) {
    if (hhip > 0.f) rhp = 2.f * alev_b / (hhi + hhip);
    if (hhim > 0.f) rhm = 2.f * alev_t / (hhi + hhim);
  }
  const float aux = (float)dt * P.at;
  float aa = aux * rhact * (rhm + rhp);
  float aat = rhact * (rhm + rhp);
  const float bb = aux * rhactp * rhp, bbt = rhactp * rhp;
  const float cc = aux * rhactm * rhm, cct = rhactm * rhm;
  const bool bfirst = lane == 0, blast = lane == ilevel - 1;
  float ppx = 0.f, ppy = 0.f;
  if (bfirst) { ppx -= (float)tx; ppy -= (float)ty; }
  if (blast) {
    // bottom_friction (chezy.f90:239-398), ireib 5: rr = cd |U_b| / h^2
    const float uv = sqrtf(uui * uui + vvi * vvi);
    const float hzg = hhi < P.hzoff ? P.hzoff : hhi;
    float rr = 0.f;
    if (P.ireib == 5) rr = d.czv[e] * uv / (hzg * hzg);
    aa += (float)dt * rr;
    aat += rr;
  }

  // explicit terms fxv/fyv (set_explicit, explicit.f90:123-213)
  float fx = 0.f, fy = 0.f;
  if (P.ahpar > 0.f && act) {            // set_diff_horizontal (:389-493)
    const float area = 12.f * (float)aj;
    for (int ii = 0; ii < 3; ii++) {
      int iei = d.ieltv[3 * e + ii];
      if (iei < 0) iei = e;
      if (lane >= d.ilhv[iei]) continue;
      const float areai = 12.f * d.ev8[(size_t)iei * 8 + 6];
      const float ui = d.uo[(size_t)iei * NLV + lane], vi = d.vo[(size_t)iei * NLV + lane];
      const float anu = P.ahpar * d.difhv[o];
      const float ai = 2.f * anu / (area + areai);
      fx -= ai * (ui - uui);
      fy -= ai * (vi - vvi);
    }
  }
  // vertical advection of momentum: w at the bottom of each lane's layer,
  // and from the lane above at its top (shuffles by the whole segment)
  float adv_wb = 0.f, adv_wt = 0.f;
  if (P.adv && P.ihwadv > 0) {
    const int I1 = NLV + 1;
    if (act && lane + 1 < ilevel)
      adv_wb = (d.wl[(size_t)kn[0] * I1 + lane + 1] + d.wl[(size_t)kn[1] * I1 + lane + 1] +
                d.wl[(size_t)kn[2] * I1 + lane + 1]) * (1.f / 3.f);
    adv_wt = seg_up<S>(adv_wb, 1);
    if (lane == 0) adv_wt = 0.f;
  }
  if (P.adv && act) {                    // set_advective (:685-861)
    const float uc = uui / hhi, vc = vvi / hhi;
    float xadv = 0.f, yadv = 0.f;
#pragma unroll
    for (int ii = 0; ii < 3; ii++) {
      const float f = uui * (float)b[ii] + vvi * (float)c[ii];
      if (f < 0.f) {                     // flux out of the node, into the element
        const float2 mk = d.mom[(size_t)kn[ii] * NLV + lane];
        xadv += f * (mk.x / hhi - uc);
        yadv += f * (mk.y / hhi - vc);
      }
    }
    if (P.ihwadv > 0) {                  // vertical advection of momentum (:776-833)
      const bool has_up = lane > 0, has_dn = lane + 1 < ilevel;
      const float2 z = vert_momentum_adv(P.ihwadv, adv_wt, adv_wb, has_up, has_dn, uui / hhi, vvi / hhi, hhi,
                                         has_up ? uuim / hhim : 0.f, has_up ? vvim / hhim : 0.f, hhim,
                                         has_dn ? uuip / hhip : 0.f, has_dn ? vvip / hhip : 0.f, hhip);
      xadv += z.x;
      yadv += z.y;
    }
    fx += P.rlin * xadv;
    fy += P.rlin * yadv;
  }
  if (P.ibarcl > 0 && P.ibarcl != 3 && P.ibarcl != 5) {
    // set_barocl_new_interface (explicit.f90:1226-1530): on z-layers the mean
    // of the density gradients of the layers above and below an interface;
    // on sigma layers the gradient on the horizontal surface at the
    // element's mean depth of the interface (bsigadjust), with the cases of
    // one or two vertices below the bottom.  Lane = layer.
    const bool bsig = lane < P.nsigma;
    float br = 0.f, cr = 0.f, brl = 0.f, crl = 0.f;
    int nb = 0, nn = 0;
    double helei = 0.;
    if (P.nsigma > 0) {
      // each vertex's depth of the layer's top interface (hkko): the old
      // level and the old node thickness of the layers above
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const double hk = act ? (double)d.hko[(size_t)kn[ii] * NLV + lane] : 0.;
        helei += -(double)d.zo[kn[ii]] + seg_scan_down<S>(hk, lane) - hk;
      }
      helei /= 3.;
    }
    if (act) {
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const int k = kn[ii];
        float rp = d.rho[(size_t)k * NLV + lane];
        if (lane + 1 == P.nsigma) { brl += (float)b[ii] * rp; crl += (float)c[ii] * rp; }
        if (bsig) {
          bool below;
          rp = sigma_rho_at(d.hko + (size_t)k * NLV, d.rho + (size_t)k * NLV, -(double)d.zo[k], d.ilhkv[k], helei,
                            &below);
          if (below) { nb++; nn += ii + 1; }
        }
        br += (float)b[ii] * rp; cr += (float)c[ii] * rp;
      }
    }
    const float *hld = d.hldv + (size_t)en.w * NLV;
    const float hlayer = bsig ? hhi : (inl ? hld[lane] : 0.f);
    const float hh = 0.5f * hlayer;
    // the layer above passes its gradient on (at layer nsigma the one
    // before the interpolation); the first layer sees zero
    const float brn = lane + 1 == P.nsigma ? brl : br, crn = lane + 1 == P.nsigma ? crl : cr;
    float brup = seg_up<S>(brn, 1), crup = seg_up<S>(crn, 1), hhup = seg_up<S>(hh, 1);
    if (lane == 0) { brup = 0.f; crup = 0.f; hhup = 0.f; }
    const float hint = hh + hhup;
    float brint, crint;
    if (bsig) {
      if (nb == 2) { brint = brup; crint = crup; }
      else if (nb == 1) {
        const float b3 = (float)b[nn - 1], c3 = (float)c[nn - 1];
        const float aux = 1.f / (c3 * c3 + b3 * b3);
        const float pu = aux * (brup * b3 + crup * c3), pc = aux * (br * b3 + cr * c3);
        brint = pu * b3 + (br - pc * b3);
        crint = pu * c3 + (cr - pc * c3);
      } else { brint = br; crint = cr; }
    } else if (lane == 0) { brint = br; crint = cr; }
    else { brint = 0.5f * (br + brup); crint = 0.5f * (cr + crup); }
    float px = act ? hint * brint : 0.f;
    float py = act ? hint * crint : 0.f;
    px = seg_scan_down<S>(px, lane);
    py = seg_scan_down<S>(py, lane);
    const float raux = P.grav / P.rowass;
    if (act) { fx += raux * hlayer * px; fy += raux * hlayer * py; }
  }
  if (P.inohyd && act) {
    // nonhydro_set_explicit (nohydro.f90:526-586): the old pressure's
    // gradient times the old thickness, weight 1 - aqpar
    float qx = 0.f, qy = 0.f;
#pragma unroll
    for (int ii = 0; ii < 3; ii++) {
      const float q = d.qdist[kn[ii]] * d.qp[(size_t)kn[ii] * NLV + lane];
      qx += (float)b[ii] * q; qy += (float)c[ii] * q;
    }
    fx += (1.f - P.aqpar) * hhi * qx;
    fy += (1.f - P.aqpar) * hhi * qy;
  }

  ppx += aat * uui - bbt * uuip - cct * uuim - (float)gammat * vvi + (float)(P.grav * hhi * bz) +
         (hhi / P.rowass) * (float)bpres + fx;
  ppy += aat * vvi - bbt * vvip - cct * vvim + (float)gammat * uui + (float)(P.grav * hhi * cz) +
         (hhi / P.rowass) * (float)cpres + fy;

  // vertical system and its solution (hydrodynamic.f90:1270-1343)
  double lo = (act && !bfirst) ? -cc : 0.;
  double up = (act && !blast) ? -bb : 0.;
  double dg = act ? 1. + aa : 1.;
  // single-precision PCR across the segment (the matrix is the identity plus
  // small viscous/friction terms, well conditioned)
  double solu, solv, hre, him = 0.;
  if (!COR) {
    float rr[3] = {act ? (float)ppx : 0.f, act ? (float)ppy : 0.f, act ? (float)hhi : 0.f};
    pcr_solve_f<S, 3>((float)lo, (float)dg, (float)up, rr, lane);
    solu = rr[0]; solv = rr[1]; hre = rr[2];
  } else {
    float2 rr[2] = {make_float2(act ? (float)ppx : 0.f, act ? (float)ppy : 0.f),
                    make_float2(act ? (float)hhi : 0.f, 0.f)};
    pcr_solve_cf<S, 2>((float)lo, make_float2((float)dg, act ? (float)gamma : 0.f), (float)up, rr, lane);
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
  double uold = seg_sum<S>((double)uui), vold = seg_sum<S>((double)vvi);
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
      // the nudging term 4 aj dt andgzv (hydrodynamic.f90:677-679), where set
      const double andg = d.andg ? 4. * aj * dt * (double)d.andg[kn[n]] : 0.;
      hik[n] = hia[n][0] * z[0] + hia[n][1] * z[1] + hia[n][2] * z[2] + andg +
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
    store_elem_system(d, e, hia, hik);
  }
}


}  // namespace shy
