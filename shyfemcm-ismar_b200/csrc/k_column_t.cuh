// k_column_t.cuh -- the column kernel with one thread per element column,
// for shallow columns (at most L layers): hydro_transports / hydro_intern /
// hydro_zeta element part (hydrodynamic.f90:758-864, 868-1416, 488-733).
//
// The same arithmetic as k_column (k_column.cuh), which spreads a column's
// layers over the lanes of a warp segment and solves the vertical system
// by parallel cyclic reduction.  For short columns most of k_column's work
// is per element (the FP64 barotropic terms, the 3x3 element system, the
// level boundary), done once per segment while the other lanes idle, and a
// 10-layer column leaves 6 of 16 lanes empty.  Here each thread walks its
// column top to bottom: the layer coefficients of hydro_intern
// (:1098-1304) on a sliding window of the layer above and below, a Thomas
// sweep for the tridiagonal system (the reference's tria_multi,
// penta.f90:333-372; FP32 here as k_column's PCR), and the element system
// with all 32 lanes of a warp busy on 32 elements.
// Included by step.cu.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace shy {

//
// W (staged, no Coriolis): the layer arrays of a warp's 32 element columns
// (one contiguous run of 32*NLV values) move between global and shared
// memory in coalesced passes of the whole warp, as k_final_w does; each
// thread then reads and writes its own column in shared memory.  Without
// it each load of layer l touches 32 sectors, one per column.
//
// XT: the instance with the explicit terms that only some basins use
// (horizontal viscosity, baroclinic pressure, the old non-hydrostatic
// pressure); without them the plain barotropic column keeps fewer registers
// and runs six CTAs per SM (measured faster than five, where it has no
// spills, on the 10-layer ensemble).
template <int L, bool COR, bool ADV, bool W = false, bool XT = true>
__global__ void __launch_bounds__(128, W ? (XT ? 4 : 6) : 3) k_column_t(Dev d) {
  static_assert(!(W && COR), "the staged form has no Coriolis instance");
  __shared__ float sbuf[W ? 4 : 1][W ? 3 : 1][W ? 32 * L : 1];
  const int e0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if constexpr (!W) {
    if (e0 >= d.NEL) return;
  } else {
    if (e0 - lane >= d.NEL) return;                   // whole warps only
  }
  const int w0 = e0 - lane;                           // first element of the warp
  const int nw = W ? min(32, d.NEL - w0) : 32;
  const bool valid = !W || lane < nw;
  const int e = valid ? e0 : w0;                      // spare lanes work a copy of the first column
  const int NLV = d.NLV;
  float *bH = sbuf[warp][0], *bU = sbuf[warp][1], *bV = sbuf[warp][2];
  const int ol = lane * NLV;                          // this thread's column in the buffers
  if constexpr (W) {
    const size_t base = (size_t)w0 * NLV;
    const int cnt = nw * NLV;
    for (int j = lane; j < 32 * NLV; j += 32) {      // spare lanes' columns read as zero
      const bool in = j < cnt;
      bH[j] = in ? d.heo[base + j] : 0.f;
      bU[j] = in ? d.uo[base + j] : 0.f;
      bV[j] = in ? d.vo[base + j] : 0.f;
    }
    __syncwarp();
  }
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  const int kn[3] = {en.x, en.y, en.z};
  const int ilevel = d.ilhv[e];
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
    const double zz = d.zeo[3 * e + ii];
    bz += zz * b[ii]; cz += zz * c[ii];
    const double pp = d.ppv[kn[ii]];
    bpres += pp * b[ii]; cpres += pp * c[ii];
    tx += d.taux[kn[ii]]; ty += d.tauy[kn[ii]];
  }
  const double drittl = 1. / 3.;
  tx *= drittl; ty *= drittl;
  const double gammat = COR ? (double)d.fcorv[e] : 0.;
  const double gamma = (double)P.af * dt * gammat;

  // the column (inactive layers read as zero)
  const size_t o = (size_t)e * NLV;
  // W: the layer values stay in shared memory (read where used, which
  // frees the registers of three layer arrays); else in registers
  float h[W ? 1 : L], u[W ? 1 : L], v[W ? 1 : L];
  if constexpr (!W) {
#pragma unroll
    for (int l = 0; l < L; l++) {
      const bool act = l < ilevel;
      h[l] = act ? d.heo[o + l] : 0.f;
      u[l] = act ? d.uo[o + l] : 0.f;
      v[l] = act ? d.vo[o + l] : 0.f;
    }
  }
#define COL_H(i) (W ? ((i) < ilevel ? bH[ol + (i)] : 0.f) : h[W ? 0 : (i)])
#define COL_U(i) (W ? ((i) < ilevel ? bU[ol + (i)] : 0.f) : u[W ? 0 : (i)])
#define COL_V(i) (W ? ((i) < ilevel ? bV[ol + (i)] : 0.f) : v[W ? 0 : (i)])
  const int I = NLV + 1;
  const float aux = (float)dt * P.at;
  const bool explicit_visc = XT && P.ahpar > 0.f;
  const bool barocl = XT && P.ibarcl > 0 && P.ibarcl != 3 && P.ibarcl != 5;
  const float area = 12.f * (float)aj;
  const float *hld = d.hldv + (size_t)en.w * NLV;
  const float raux = P.grav / P.rowass;

  // forward Thomas sweep as the layer coefficients are formed
  float cp[L];
  float dp0[L], dp1[L], dp2[L];            // real: rhs ppx, ppy, h
  float2 cpc[COR ? L : 1], dq0[COR ? L : 1], dq1[COR ? L : 1];   // complex: ppx+i ppy, h
  float adv_wtop = 0.f;                    // vertical momentum advection: w at the layer's top
  float alev_t = P.vismol;
  if (0 < ilevel)
    alev_t += (d.visv[(size_t)kn[0] * I] + d.visv[(size_t)kn[1] * I] + d.visv[(size_t)kn[2] * I]) * (1.f / 3.f);
  float brm = 0.f, crm = 0.f, hhm = 0.f;   // baroclinic values of the layer above
  // sigma layers: each vertex's depth of the current layer's top interface
  // (hkko: the old level and the old node thickness summed from the top)
  double hoi[3] = {0., 0., 0.};
  if (barocl && P.nsigma > 0)
#pragma unroll
    for (int ii = 0; ii < 3; ii++) hoi[ii] = -(double)d.zo[kn[ii]];
  float pxs = 0.f, pys = 0.f;              // their running sums from the surface
#pragma unroll
  for (int l = 0; l < L; l++) {
    if (l >= ilevel) break;
    const bool bfirst = l == 0, blast = l == ilevel - 1;
    const float hhi = COL_H(l), uui = COL_U(l), vvi = COL_V(l);
    float hhip = blast ? 0.f : COL_H(l + 1 < L ? l + 1 : l);
    float uuip = blast ? uui : COL_U(l + 1 < L ? l + 1 : l);
    float vvip = blast ? vvi : COL_V(l + 1 < L ? l + 1 : l);
    const float hhim = bfirst ? 0.f : COL_H(l > 0 ? l - 1 : 0);
    const float uuim = bfirst ? uui : COL_U(l > 0 ? l - 1 : 0);
    const float vvim = bfirst ? vvi : COL_V(l > 0 ? l - 1 : 0);
    const float rhact = hhi > 0.f ? 1.f / hhi : 0.f;
    const float rhactp = hhip > 0.f ? 1.f / hhip : 0.f;
    const float rhactm = hhim > 0.f ? 1.f / hhim : 0.f;
    // element viscosity at the bottom interface (:1098-1104)
    const float alev_b = P.vismol + (d.visv[(size_t)kn[0] * I + l + 1] + d.visv[(size_t)kn[1] * I + l + 1] +
                                     d.visv[(size_t)kn[2] * I + l + 1]) * (1.f / 3.f);
    float rhp = 0.f, rhm = 0.f;
    if (hhi > 0.f) {
      if (hhip > 0.f) rhp = 2.f * alev_b / (hhi + hhip);
      if (hhim > 0.f) rhm = 2.f * alev_t / (hhi + hhim);
    }
    alev_t = alev_b;
    float aa = aux * rhact * (rhm + rhp);
    float aat = rhact * (rhm + rhp);
    const float bb = aux * rhactp * rhp, bbt = rhactp * rhp;
    const float cc = aux * rhactm * rhm, cct = rhactm * rhm;
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
    if (explicit_visc) {                 // set_diff_horizontal (:389-493)
      for (int ii = 0; ii < 3; ii++) {
        int iei = d.ieltv[3 * e + ii];
        if (iei < 0) iei = e;
        if (l >= d.ilhv[iei]) continue;
        const float areai = 12.f * d.ev8[(size_t)iei * 8 + 6];
        const float ui = d.uo[(size_t)iei * NLV + l], vi = d.vo[(size_t)iei * NLV + l];
        const float anu = P.ahpar * d.difhv[o + l];
        const float ai = 2.f * anu / (area + areai);
        fx -= ai * (ui - uui);
        fy -= ai * (vi - vvi);
      }
    }
    if (ADV && P.adv) {                  // set_advective (:685-861), ihwadv 0
      const float uc = uui / hhi, vc = vvi / hhi;
      float xadv = 0.f, yadv = 0.f;
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const float f = uui * (float)b[ii] + vvi * (float)c[ii];
        if (f < 0.f) {                   // flux out of the node, into the element
          const float2 mk = d.mom[(size_t)kn[ii] * NLV + l];
          xadv += f * (mk.x / hhi - uc);
          yadv += f * (mk.y / hhi - vc);
        }
      }
      if (P.ihwadv > 0) {                // vertical advection of momentum (:776-833)
        const int I1 = NLV + 1;
        float wb = 0.f;
        if (!blast)
          wb = (d.wl[(size_t)kn[0] * I1 + l + 1] + d.wl[(size_t)kn[1] * I1 + l + 1] +
                d.wl[(size_t)kn[2] * I1 + l + 1]) * (1.f / 3.f);
        const float2 z = vert_momentum_adv(P.ihwadv, adv_wtop, wb, !bfirst, !blast, uui / hhi, vvi / hhi, hhi,
                                           bfirst ? 0.f : uuim / hhim, bfirst ? 0.f : vvim / hhim, hhim,
                                           blast ? 0.f : uuip / hhip, blast ? 0.f : vvip / hhip, hhip);
        xadv += z.x;
        yadv += z.y;
        adv_wtop = wb;
      }
      fx += P.rlin * xadv;
      fy += P.rlin * yadv;
    }
    if (barocl) {
      // set_barocl_new_interface (explicit.f90:1226-1530): on z-layers the
      // mean of the density gradients of the layers above and below an
      // interface; on sigma layers the gradient on the horizontal surface
      // at the element's mean depth of the interface (bsigadjust), with the
      // cases of one or two vertices below the bottom
      const bool bsig = l < P.nsigma;
      float br = 0.f, cr = 0.f, brl = 0.f, crl = 0.f;
      int nb = 0, nn = 0;
      const double helei = (hoi[0] + hoi[1] + hoi[2]) / 3.;
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const int k = kn[ii];
        float rp = d.rho[(size_t)k * NLV + l];
        if (l + 1 == P.nsigma) { brl += (float)b[ii] * rp; crl += (float)c[ii] * rp; }
        if (bsig) {
          bool below;
          rp = sigma_rho_at(d.hko + (size_t)k * NLV, d.rho + (size_t)k * NLV, -(double)d.zo[k], d.ilhkv[k], helei,
                            &below);
          if (below) { nb++; nn += ii + 1; }
        }
        br += (float)b[ii] * rp; cr += (float)c[ii] * rp;
      }
      const float hlayer = bsig ? hhi : hld[l];
      const float hh = 0.5f * hlayer;
      const float hhup = bfirst ? 0.f : hhm;
      const float hint = hh + hhup;
      float brint, crint;
      if (bsig) {
        if (nb == 2) { brint = brm; crint = crm; }
        else if (nb == 1) {                // the gradient along the bottom side kept from above
          const float b3 = (float)b[nn - 1], c3 = (float)c[nn - 1];
          const float aux = 1.f / (c3 * c3 + b3 * b3);
          const float pu = aux * (brm * b3 + crm * c3), pc = aux * (br * b3 + cr * c3);
          brint = pu * b3 + (br - pc * b3);
          crint = pu * c3 + (cr - pc * c3);
        } else { brint = br; crint = cr; }
      } else if (bfirst) { brint = br; crint = cr; }
      else { brint = 0.5f * (br + brm); crint = 0.5f * (cr + crm); }
      pxs += hint * brint;
      pys += hint * crint;
      brm = br; crm = cr;
      if (l + 1 == P.nsigma) { brm = brl; crm = crl; }
      hhm = hh;
      if (P.nsigma > 0)
#pragma unroll
        for (int ii = 0; ii < 3; ii++) hoi[ii] += (double)d.hko[(size_t)kn[ii] * NLV + l];
      fx += raux * hlayer * pxs;
      fy += raux * hlayer * pys;
    }
    if (XT && P.inohyd) {
      // nonhydro_set_explicit (nohydro.f90:526-586): the old pressure's
      // gradient times the old thickness, weight 1 - aqpar
      float qx = 0.f, qy = 0.f;
#pragma unroll
      for (int ii = 0; ii < 3; ii++) {
        const float q = d.qdist[kn[ii]] * d.qp[(size_t)kn[ii] * NLV + l];
        qx += (float)b[ii] * q; qy += (float)c[ii] * q;
      }
      fx += (1.f - P.aqpar) * hhi * qx;
      fy += (1.f - P.aqpar) * hhi * qy;
    }
    ppx += aat * uui - bbt * uuip - cct * uuim - (float)gammat * vvi + (float)(P.grav * hhi * bz) +
           (hhi / P.rowass) * (float)bpres + fx;
    ppy += aat * vvi - bbt * vvip - cct * vvim + (float)gammat * uui + (float)(P.grav * hhi * cz) +
           (hhi / P.rowass) * (float)cpres + fy;
    // vertical system (hydrodynamic.f90:1270-1343): -cc, 1+aa (+ i gamma), -bb
    const float lo = bfirst ? 0.f : -cc;
    const float up = blast ? 0.f : -bb;
    const float dg = 1.f + aa;
    if constexpr (!COR) {
      const float cprev = bfirst ? 0.f : cp[l > 0 ? l - 1 : 0];
      const float rden = 1.f / (dg - lo * cprev);
      cp[l] = up * rden;
      dp0[l] = (ppx - (bfirst ? 0.f : lo * dp0[l > 0 ? l - 1 : 0])) * rden;
      dp1[l] = (ppy - (bfirst ? 0.f : lo * dp1[l > 0 ? l - 1 : 0])) * rden;
      dp2[l] = (hhi - (bfirst ? 0.f : lo * dp2[l > 0 ? l - 1 : 0])) * rden;
    } else {
      const float2 cprev = bfirst ? make_float2(0.f, 0.f) : cpc[l > 0 ? l - 1 : 0];
      const float2 den = make_float2(dg - lo * cprev.x, (float)gamma - lo * cprev.y);
      const float2 one = make_float2(1.f, 0.f);
      const float2 rden = cdivf(one, den);
      cpc[l] = make_float2(up * rden.x, up * rden.y);
      float2 r0 = make_float2(ppx, ppy), r1 = make_float2(hhi, 0.f);
      if (!bfirst) {
        const float2 p0 = dq0[l > 0 ? l - 1 : 0], p1 = dq1[l > 0 ? l - 1 : 0];
        r0.x -= lo * p0.x; r0.y -= lo * p0.y;
        r1.x -= lo * p1.x; r1.y -= lo * p1.y;
      }
      dq0[l] = cmulf(r0, rden);
      dq1[l] = cmulf(r1, rden);
    }
  }

  // back substitution, new transports, layer sums of hydro_zeta
  double dbb = 0., dcb = 0., uold = 0., vold = 0., uh = 0., vh = 0.;
  float x0 = 0.f, x1 = 0.f, x2 = 0.f;
  float2 y0 = make_float2(0.f, 0.f), y1 = make_float2(0.f, 0.f);
#pragma unroll
  for (int l = L - 1; l >= 0; l--) {
    if (l >= NLV) continue;
    const bool act = l < ilevel;
    float solu = 0.f, solv = 0.f, hre = 0.f, him = 0.f;
    if (act) {
      const bool blast = l == ilevel - 1;
      if constexpr (!COR) {
        x0 = dp0[l] - (blast ? 0.f : cp[l] * x0);
        x1 = dp1[l] - (blast ? 0.f : cp[l] * x1);
        x2 = dp2[l] - (blast ? 0.f : cp[l] * x2);
        solu = x0; solv = x1; hre = x2;
      } else {
        if (blast) { y0 = dq0[l]; y1 = dq1[l]; }
        else {
          const float2 t0 = cmulf(cpc[l], y0), t1 = cmulf(cpc[l], y1);
          y0 = make_float2(dq0[l].x - t0.x, dq0[l].y - t0.y);
          y1 = make_float2(dq1[l].x - t1.x, dq1[l].y - t1.y);
        }
        solu = y0.x; solv = y0.y; hre = y1.x; him = y1.y;
      }
    }
    const float ul = COL_U(l), vl = COL_V(l);
    const float uhat = act ? (float)(ul - dt * solu) : 0.f;
    const float vhat = act ? (float)(vl - dt * solv) : 0.f;
    if constexpr (W) {
      bU[ol + l] = uhat;                              // spare lanes write past the warp's run
      bV[ol + l] = vhat;
      bH[ol + l] = act ? hre : 0.f;
    } else {
      d.un[o + l] = uhat;
      d.vn[o + l] = vhat;
      d.ddx[o + l] = act ? hre : 0.f;
    }
    if (COR) d.ddxi[o + l] = act ? him : 0.f;
    if (act) {
      dbb += (double)hre; dcb += (double)him;
      uold += (double)ul; vold += (double)vl;
      uh += (double)uhat; vh += (double)vhat;
    }
  }

  if constexpr (W) {
    __syncwarp();
    const size_t base = (size_t)w0 * NLV;
    const int cnt = nw * NLV;
    for (int j = lane; j < cnt; j += 32) {
      d.un[base + j] = bU[j];
      d.vn[base + j] = bV[j];
      d.ddx[base + j] = bH[j];
    }
  }

  // hydro_zeta (hydrodynamic.f90:604-733): the element system
  // ddxv(ju) = Re, ddxv(jv) = Im, ddyv(ju) = -Im, ddyv(jv) = Re
  const double dbc = -dcb, dcc = dbb;
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
      const double abn = b[n] * (b[m] * dbb + c[m] * dbc);
      const double acn = c[n] * (b[m] * dcb + c[m] * dcc);
      hia[n][m] = aj * ((n == m ? 4. : 0.) + 12. * delta * (abn + acn));
    }
    // the nudging term 4 aj dt andgzv (hydrodynamic.f90:677-679), where set
    const double andg = d.andg ? 4. * aj * dt * (double)d.andg[kn[n]] : 0.;
    hik[n] = hia[n][0] * z[0] + hia[n][1] * z[1] + hia[n][2] * z[2] + andg + 12. * aj * dt * (ut * b[n] + vt * c[n]);
  }
  // level boundary conditions (:688-704), rzv at the new time (sp111)
  const double tnew = d.out[en.w].dtime + dt;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int kb = d.kbnd[kn[i]];
    if (kb > 0) {
      const double rw = level_bc(d, P, kb, tnew);
      const int j1 = (i + 1) % 3, j2 = (i + 2) % 3;
      hik[j1] -= rw * hia[j1][i];
      hik[j2] -= rw * hia[j2][i];
      hia[i][j1] = 0.; hia[i][j2] = 0.; hia[j1][i] = 0.; hia[j2][i] = 0.;
      hik[i] = rw * hia[i][i];
    }
  }
  if (valid) store_elem_system(d, e, hia, hik);
#undef COL_H
#undef COL_U
#undef COL_V
}

}  // namespace shy
