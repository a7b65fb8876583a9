// k_conz.cuh -- one sub-step of 3D scalar transport for every scalar of a
// node column: conz3d_omp (concentration_omp.f90:65-350) with the element
// part conz3d_element (:355-755, vertical fluxes of vertical_flux_ie,
// tvd_admin.f90:930-1019, without vertical TVD) gathered per node in element
// order, the node part conz3d_nodes (:757-888: vertical tridiagonal system),
// the level-boundary values of bndo_impbc (bndo.f90:700-760); and rhoset
// (baroclinic.f90:654-710) once temperature and salinity are final.
//
// Two kernels per sub-step.  k_conz_el, one warp segment per element column
// (lane = layer), computes each element's horizontal fluxes (upwind or TVD)
// and horizontal diffusion into each of its three vertices for every scalar
// of the sub-step and writes them per element vertex (Dev::cz_ef).  k_conz,
// one warp segment per node column, sums them over the node's elements in
// element order and does the rest.  In conz3d_element the storage,
// vertical-diffusion and vertical-advection terms of node k depend on an
// element e only through its weight aj4 = 4*aj and through whether layer
// l+1 exists in e (presentl(l+1), and wl(ilevel) = 0 at the element's
// bottom).  Their sum over the elements of k is therefore the node's own
// column terms weighted by two static sums, A_t = sum of aj4 over elements
// that continue below layer l and A_f = sum over elements whose bottom layer
// is l (Dev::avol).  Scalars with the same sub-step count share one PCR
// solve of the vertical system.  FP32.
//
// Increment form.  The node layer's system M c' = M_old c + dt F(c) is
// solved for the increment d = c' - c: every flux is evaluated on the
// concentrations shifted by the node's own value (c_j - c), which gives the
// same flux minus c times the flow (the schemes, upwind and superbee TVD, are
// shift-equivariant), and c times the continuity residual of the node layer,
// r = A (h_old - h_new) + dt (sum of flows), is added back.  In exact
// arithmetic this is the conservative update of conz3d; in FP32 it rounds
// relative to the increment instead of relative to the mass A h c, so a
// uniform field stays uniform and the drift against the FP64 reference
// stays at the rounding of the stored values.
// Included by node_launch.cuh.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace shy {

// v[i] for a run-time i in 0..2 through selects (no local-memory array)
__device__ __forceinline__ float sel3(const float (&v)[3], int i) {
  return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]);
}

__device__ __forceinline__ float clipc(float v, bool is_temp) {
  return (!is_temp && v < 1.e-15f) ? 0.f : v;   // scal3sh: where(cnv < 1e-15) cnv = 0
}

// the sub-step's input columns of every scalar (sub-step isact, 1-based)
__device__ __forceinline__ const float *conz_input(const Dev &d, int isact) {
  return isact == 1 ? d.sc_in : (isact & 1 ? d.scr1 : d.scr0);
}

// ===========================================================================
// k_tvdgrad: node gradients of the sub-step's scalars for the horizontal TVD
// scheme (tvd_grad_3d, tvd_admin.f90:478-550, itvd = 1): per node layer the
// area-weighted mean of the gradients of the incident elements that have
// the layer, from the clipped input (scal3sh clips before it,
// concentration.f90:736-744).  One warp segment per node column, lane =
// layer; FP32 sums in element order.
// ===========================================================================
template <int S>
__global__ void __launch_bounds__(256) k_tvdgrad(Dev d, const int *kbas, int j_arg) {
  const int j = j_arg >= 0 ? j_arg : *d.subj;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const int NLV = d.NLV;
  if (k >= d.NKN || lane >= NLV) return;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  if (P.itvd != 1) return;
  const BasinOut &O = d.out[b];
  const int isact = j + 1;
  const float *cin = conz_input(d, isact);
  const size_t SN = (size_t)d.NKN * NLV, o = (size_t)k * NLV + lane;
  const int pbeg = d.inc_ptr[k], pend = d.inc_ptr[k + 1];
  for (int s = 0; s < P.nsc; s++) {
    if (isact > (int)O.stab[s]) continue;        // no sub-step of this scalar
    const bool istmp = P.is_temp[s] != 0;
    const float *cs = cin + s * SN;
    const float cown = clipc(cs[o], istmp);
    float gx = 0.f, gy = 0.f, ar = 0.f;
    for (int p = pbeg; p < pend; p++) {
      const int4 ix = d.incx[p];
      const int e = ix.x, ii = ix.y & 3;
      if (lane >= (ix.y >> 2)) continue;
      const float *evp = d.ev8 + (size_t)e * 8;
      const float ca = clipc(cs[(size_t)ix.z * NLV + lane], istmp);
      const float cb = clipc(cs[(size_t)ix.w * NLV + lane], istmp);
      const float c3[3] = {ii == 0 ? cown : ca, ii == 1 ? cown : (ii == 0 ? ca : cb), ii == 2 ? cown : cb};
      const float ggx = c3[0] * evp[0] + c3[1] * evp[1] + c3[2] * evp[2];
      const float ggy = c3[0] * evp[3] + c3[1] * evp[4] + c3[2] * evp[5];
      const float area = evp[6];
      gx += ggx * area;
      gy += ggy * area;
      ar += area;
    }
    d.tgrad[s * SN + o] = ar > 0.f ? make_float2(gx / ar, gy / ar) : make_float2(0.f, 0.f);
  }
}

// tvd_fluxes (tvd_admin.f90:673-838), itvd 1 or 2: the horizontal flux of
// vertex `own` (0..2) of an element layer, replacing the upwind one.  The
// pairs (ic, id) of the one vertex with outflow (itot 1) or inflow (itot 2)
// and each other vertex carry the concentration of ic corrected towards id
// by the superbee limiter of the ratio of the upwind difference to the
// difference along the side: the node gradient at ic (g, itvd 1), or the
// value at the point beyond ic opposite id interpolated in the element
// holding it (Dev::tvdup, itvd 2).  kv: node of each vertex,
// u, v: the element's velocity, aj24 = 24 ev(10) (twice the area); the side
// length is aj24 |(b, c)| of the opposite vertex (ev(17..19)).
__device__ __forceinline__ float tvd_flux_own(int own, int itot, int isum, const float (&f3)[3],
                                              const float (&c3)[3], const float (&bb)[3],
                                              const float (&cc)[3], const int (&kv)[3], float aj24,
                                              float u, float v, float dt, const float2 *g, int NLV,
                                              int lane, const Dev &d, int e, int itvd, const float *cs,
                                              bool istmp, float csh) {
  if (itot < 1 || itot > 2) return 0.f;
  const int itot2 = itot - 1, itot1 = 2 - itot;
  const int ip = itot2 * (6 - isum) + itot1 * isum;          // 1-based
  const float fact = (float)(itot1 - itot2);
  float fl = 0.f;
#pragma unroll
  for (int ii = 1; ii <= 3; ii++) {
    if (ii == ip) continue;
    const int ic = itot2 * ii + itot1 * ip, id = itot2 * ip + itot1 * ii;
    if (ic != own + 1 && id != own + 1) continue;            // no share of vertex own
    const float conc = sel3(c3, ic - 1), cond = sel3(c3, id - 1);
    const int iop = 6 - (id + ic);                           // the vertex opposite side ic-id
    const int tet1 = 1 + iop % 3;
    const float bo = sel3(bb, iop - 1), co = sel3(cc, iop - 1);
    float dx = aj24 * co;
    if (tet1 == id) dx = -dx;
    float dy = aj24 * bo;
    if (tet1 == ic) dy = -dy;
    const float dis = aj24 * sqrtf(bo * bo + co * co);
    const float vel = fabsf(u * dx + v * dy) / dis;
    const float alfa = dt * vel / dis;
    float grad;
    if (itvd == 1) {
      const int kc = ic == 1 ? kv[0] : (ic == 2 ? kv[1] : kv[2]);
      const float2 gc = g[(size_t)kc * NLV + lane];
      grad = 2.f * (gc.x * dx + gc.y * dy);
    } else {
      // itvd 2: the value at the point beyond ic opposite id
      // (tvd_get_upwind_c, tvd_admin.f90:608-671), cond where it has no layer;
      // shifted by csh like c3 (the interpolation weights sum to one)
      float conu = cond;
      const int4 t = d.tvdup[(size_t)e * 6 + 2 * (ic - 1) + ((id - ic + 3) % 3 - 1)];
      if (t.x >= 0 && lane < d.ilhv[t.x]) {
        const int4 tn = d.enode[t.x];
        conu = __int_as_float(t.y) * (clipc(cs[(size_t)tn.x * NLV + lane], istmp) - csh) +
               __int_as_float(t.z) * (clipc(cs[(size_t)tn.y * NLV + lane], istmp) - csh) +
               __int_as_float(t.w) * (clipc(cs[(size_t)tn.z * NLV + lane], istmp) - csh);
      }
      grad = cond - conu;
    }
    const float rf = fabsf(conc - cond) < 1.e-8f ? -1.f : grad / (cond - conc) - 1.f;
    const float psi = fmaxf(0.f, fmaxf(fminf(1.f, 2.f * rf), fminf(2.f, rf)));   // superbee
    const float conf = conc + 0.5f * psi * (cond - conc) * (1.f - alfa);
    const float term = fact * conf * sel3(f3, ii - 1);
    fl += (ic == own + 1) ? -term : term;
  }
  return fl;
}

// the interface value of vertical TVD (vertical_flux_ie,
// tvd_admin.f90:976-1004): from the upwind layer towards the downwind one,
// limited by superbee of the ratio to the far-upwind difference
__device__ __forceinline__ float tvd_v(float conc, float cond, float conu, float alfa) {
  const float rf = fabsf(conc - cond) < 1.e-8f ? -1.f : (cond - conu) / (cond - conc) - 1.f;
  const float psi = fmaxf(0.f, fmaxf(fminf(1.f, 2.f * rf), fminf(2.f, rf)));
  return conc + 0.5f * psi * (cond - conc) * (1.f - alfa);
}

// ===========================================================================
// k_conz_el: the element part of a sub-step (conz3d_element,
// concentration_omp.f90:355-755, the horizontal terms :620-690): per element
// layer and scalar with a sub-step now, the upwind flux (one vertex of
// outflow, itot 1, or of inflow, itot 2) or the TVD flux (itvd 1, 2; not
// where a vertex is on an open boundary) into each vertex, and horizontal
// diffusion through wdifhv, all on concentrations shifted by that vertex's
// own (the increment form, see k_conz), times 4aj; and the flux of a unit
// field.  Zero on the layers the element lacks.
// ===========================================================================
template <int S, bool TVD>
__global__ void __launch_bounds__(256) k_conz_el(Dev d, int j_arg) {
  const int j = j_arg >= 0 ? j_arg : *d.subj;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const int NLV = d.NLV;
  if (e >= d.NEL || lane >= NLV) return;       // no shuffles in this kernel
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  const BasinOut &O = d.out[en.w];
  const int nsc = P.nsc, isact = j + 1;
  bool any = false;
  for (int s = 0; s < nsc; s++) any |= isact <= (int)O.stab[s];
  if (!any) return;
  const bool act = lane < d.ilhv[e];
  const size_t oe = (size_t)e * NLV + lane, e3 = (size_t)e * 3;
  const size_t SN = (size_t)d.NKN * NLV;
  const int NSCM = d.nsc_max;
  const float4 e0 = *reinterpret_cast<const float4 *>(d.ev8 + (size_t)e * 8);
  const float4 e1 = *reinterpret_cast<const float4 *>(d.ev8 + (size_t)e * 8 + 4);
  const float bb[3] = {e0.x, e0.y, e0.z}, cc[3] = {e0.w, e1.x, e1.y};
  const float aj4 = 4.f * e1.z;
  const float us = act ? d.usv[oe] : 0.f, vs = act ? d.vsv[oe] : 0.f;
  float f3[3];
  int itot = 0, isum = 0;
#pragma unroll
  for (int jj = 0; jj < 3; jj++) {
    f3[jj] = us * bb[jj] + vs * cc[jj];
    if (f3[jj] < 0.f) { itot++; isum += jj + 1; }
  }
  // the flux of a unit field into each vertex (the same for TVD on a
  // divergence-free element)
#pragma unroll
  for (int ii = 0; ii < 3; ii++) {
    const float fii = f3[ii];
    const float fl1 = itot == 1 ? fii : (itot == 2 ? ((ii == 5 - isum) ? fii - (f3[0] + f3[1] + f3[2]) : fii) : 0.f);
    d.cz_ef1[(e3 + ii) * NLV + lane] = act ? aj4 * 3.f * fl1 : 0.f;
  }
  const int kv[3] = {en.x, en.y, en.z};
  // TVD (the instance for models where a basin uses it): not where a vertex
  // is on an open boundary
  const bool tvd = TVD && P.itvd >= 1 && d.kbnd[kv[0]] <= 0 && d.kbnd[kv[1]] <= 0 && d.kbnd[kv[2]] <= 0;
  float ue = 0.f, ve = 0.f;
  if (tvd && act) {
    const float hn = d.hen[oe];
    if (hn > 0.f) { ue = d.un[oe] / hn; ve = d.vn[oe] / hn; }
  }
  const float *cin_base = conz_input(d, isact);
  for (int s = 0; s < nsc; s++) {
    if (isact > (int)O.stab[s]) continue;        // no sub-step of this scalar now
    const float rstot = O.stab[s];
    const float rso = (isact - 1) / rstot, rsot = 1.f - rso;
    const float dt = (float)P.dt / rstot;
    const bool istmp = P.is_temp[s] != 0;
    const float rk = P.rkpar[s];
    const float *cs = cin_base + s * SN;
    float c3[3];
#pragma unroll
    for (int ii = 0; ii < 3; ii++) c3[ii] = act ? clipc(cs[(size_t)kv[ii] * NLV + lane], istmp) : 0.f;
    float hmed = 0.f, dfh = 0.f;
    if (rk != 0.f && act) {
      hmed = rso * d.hen[oe] + rsot * d.heo[oe];
      dfh = d.difhv[oe];
    }
#pragma unroll
    for (int ii = 0; ii < 3; ii++) {
      // concentrations shifted by vertex ii's own
      const float c3s[3] = {c3[0] - c3[ii], c3[1] - c3[ii], c3[2] - c3[ii]};
      float fl;
      if (itot == 1) fl = f3[ii] * sel3(c3s, isum - 1);
      else if (itot == 2)   // flux into the vertex with f >= 0 balances the two outflows
        fl = (ii == 5 - isum) ? -(f3[0] * c3s[0] + f3[1] * c3s[1] + f3[2] * c3s[2]) : 0.f;
      else fl = 0.f;
      if constexpr (TVD) {
        if (tvd && act)
          fl = tvd_flux_own(ii, itot, isum, f3, c3s, bb, cc, kv, 24.f * e1.z, ue, ve, dt, d.tgrad + s * SN, NLV,
                            lane, d, e, P.itvd, cs, istmp, c3[ii]);
      }
      float hdif = 0.f;
      if (rk != 0.f) {
        float wdiff = 0.f;
#pragma unroll
        for (int iii = 0; iii < 3; iii++) wdiff += d.wdif[(size_t)e * 9 + 3 * iii + ii] * c3s[iii];
        hdif = 3.f * rk * dfh * hmed * wdiff;
      }
      d.cz_ef[((e3 + ii) * NSCM + s) * NLV + lane] = act ? aj4 * (3.f * fl - hdif) : 0.f;
    }
  }
}

// EX: the instance of shygpu_conz3d with conz3d_omp's source terms (one
// scalar): settling lowers the interface velocities by wsink*wsinkv
// (concentration_omp.f90:496); nudging adds dt*aj4*hold*robs*rtau*(cobs - c)
// per element (:694-709; an = 0, so nothing implicit); loading acts on the
// assembled mass before the vertical solve (conz3d_nodes :816-833).
// TV: the instance with vertical TVD (models where a basin uses itvdv = 1)
template <int S, int NR, bool EX, bool TV>
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
  const int nsc = P.nsc;
  const int lmax = d.ilhkv[k];
  const bool act = lane < lmax;
  const size_t o = (size_t)k * NLV + lane;
  const size_t SN = (size_t)d.NKN * NLV;
  const int isact = j + 1;
  unsigned todo = 0;
  for (int s = 0; s < nsc; s++)
    if (isact <= (int)O.stab[s]) todo |= 1u << s;
  if (todo == 0) return;                        // the whole segment skips together
  const float ad = P.ad, adt = 1.f - ad, aa = P.aa, aat = 1.f - aa;
  const float hko = act ? d.hko[o] : 0.f, hkn = act ? d.hkn[o] : 0.f;
  const float rvptop = act ? d.difv[(size_t)k * I + lane] + P.difmol : 0.f;
  const float rvpbot = act ? d.difv[(size_t)k * I + lane + 1] + P.difmol : 0.f;
  float wt = act ? d.wl[(size_t)k * I + lane] : 0.f;
  float wb = act ? d.wl[(size_t)k * I + lane + 1] : 0.f;
  if constexpr (EX) {
    if (act && d.cz_wsink != 0.f) {
      wt -= d.cz_wsink * d.cz_wsv[(size_t)k * I + lane];
      wb -= d.cz_wsink * d.cz_wsv[(size_t)k * I + lane + 1];
    }
  }
  const float2 av = act ? d.avol[o] : make_float2(0.f, 0.f);
  const float At = av.x, A = av.x + av.y;      // continuing elements, all elements
  // vertical TVD: the far-upwind layer of an element's column exists only
  // where the element continues, so the bottom interface splits At into the
  // elements continuing below layer l+1 and those ending at it
  const bool tvdv = TV && P.itvdv == 1;
  float2 avn = make_float2(0.f, 0.f);
  if (tvdv) { avn.x = seg_down<S>(av.x, 1); avn.y = seg_down<S>(av.y, 1); }
  const bool isbnd = d.kbnd[k] > 0;
  // the node layer's share of the node's discharge (mfluxv, set_mass_flux)
  const float qf = mflux_layer<S>(d, k, act, o, P.wetdry != 0);
  const int pbeg = d.inc_ptr[k], pend = d.inc_ptr[k + 1];
  const bool up_ok = lane > 0, dn_ok = lane + 1 < lmax;
  while (todo) {
    // a group: scalars with the sub-step count of the first pending one
    const int s0 = __ffs(todo) - 1;
    const int istot = (int)O.stab[s0];
    int sidx[NR];
    int nm = 0;
#pragma unroll
    for (int r = 0; r < NR; r++) sidx[r] = -1;
    for (int s = s0; s < nsc && nm < NR; s++)
      if ((todo >> s & 1u) && (int)O.stab[s] == istot) { sidx[nm++] = s; todo &= ~(1u << s); }
    const float rstot = istot;
    const float rso = (isact - 1) / rstot, rsn = isact / rstot, rsot = 1.f - rso, rsnt = 1.f - rsn;
    const float dt = (float)P.dt / rstot;
    const float *cin_base = conz_input(d, isact);
    float *cout_base = isact == istot ? d.sc_out : (isact & 1 ? d.scr0 : d.scr1);
    // node column: thickness, vertical diffusion conductances
    const float hold = rso * hkn + rsot * hko, hnew = rsn * hkn + rsnt * hko;
    const float holdm = seg_up<S>(hold, 1), holdp = seg_down<S>(hold, 1);
    const float hnewm = seg_up<S>(hnew, 1), hnewp = seg_down<S>(hnew, 1);
    const float hmotop = up_ok ? 2.f * rvptop / (holdm + hold) : 0.f;
    const float hmobot = dn_ok ? 2.f * rvpbot / (hold + holdp) : 0.f;
    const float hmntop = up_ok ? 2.f * rvptop / (hnewm + hnew) : 0.f;
    const float hmnbot = dn_ok ? 2.f * rvpbot / (hnew + hnewp) : 0.f;
    float cl[NR], cm1[NR], cp1[NR], hs[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
      const int s = sidx[r] < 0 ? 0 : sidx[r];
      const bool istmp = P.is_temp[s] != 0;
      const float v = (act && sidx[r] >= 0) ? clipc(cin_base[s * SN + o], istmp) : 0.f;
      cl[r] = v;
      cm1[r] = seg_up<S>(v, 1);
      cp1[r] = seg_down<S>(v, 1);
      if (!up_ok) cm1[r] = 0.f;
      if (!dn_ok) cp1[r] = 0.f;
      hs[r] = 0.f;
    }
    // horizontal fluxes: the element part's values of this node's vertex in
    // each incident element, summed in element order
    float hs1 = 0.f;
    if (act) {
      const int NSCM = d.nsc_max;
#pragma unroll 4
      for (int p = pbeg; p < pend; p++) {
        const int4 ix = __ldg(&d.incx[p]);   // element, vertex | layers, other two nodes
        if (lane >= (ix.y >> 2)) continue;
        const size_t ev = (size_t)ix.x * 3 + (ix.y & 3);
        hs1 += d.cz_ef1[ev * NLV + lane];
#pragma unroll
        for (int r = 0; r < NR; r++)
          if (sidx[r] >= 0) hs[r] += d.cz_ef[(ev * NSCM + sidx[r]) * NLV + lane];
      }
    }
    // storage, vertical diffusion and vertical advection, summed over the
    // elements through A_t (layer l+1 present) and A (all elements)
    const float w0 = up_ok ? wt : 0.f;               // top interface (0 at the surface)
    float clc_b = ad * hmntop, clmm = -ad * hmntop;  // parts every element has
    if (w0 >= 0.f) clc_b += aa * w0; else clmm += aa * w0;
    float clc_x = ad * hmnbot, clpp = -ad * hmnbot;  // parts of elements that continue below
    if (wb > 0.f) clpp -= aa * wb; else clc_x -= aa * wb;
    const float clo = A * dt * clmm;
    const float chi = At * dt * clpp;
    const float cdg = A * (dt * clc_b + hnew) + At * dt * clc_x;
    // continuity residual of the node layer: A (h_old - h_new) + dt (flow
    // in); h_new - h_old = (hkn - hko) / istot, the difference exact in FP32
    const float rcont = act ? -A * ((hkn - hko) / rstot) + dt * (hs1 + qf - (A * w0 - At * wb)) : 0.f;
    float res[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) {
      const float c = cl[r];
      const float cm = up_ok ? cm1[r] - c : 0.f, cp = dn_ok ? cp1[r] - c : 0.f;   // shifted
      float topw, botw;                               // interface fluxes times their element weights
      if (!TV || !tvdv) {
        const float vtop = up_ok ? wt * (wt > 0.f ? 0.f : cm) : 0.f;
        const float vbot = wb * (wb > 0.f ? cp : 0.f);
        topw = A * vtop;
        botw = At * vbot;
      } else {
        const float cm2r = seg_up<S>(c, 2), cp2r = seg_down<S>(c, 2);   // every lane shuffles
        const float cm2 = (lane >= 2 ? cm2r : c) - c, cp2 = cp2r - c;
        topw = 0.f;
        if (up_ok) {
          const float alfa = dt * fabsf(wt) / (0.5f * (holdm + hold));
          if (wt > 0.f)
            topw = wt * (At * tvd_v(0.f, cm, cp, alfa) + av.y * tvd_v(0.f, cm, cm, alfa));
          else
            topw = A * wt * tvd_v(cm, 0.f, cm2, alfa);
        }
        botw = 0.f;
        if (dn_ok) {
          const float alfa = dt * fabsf(wb) / (0.5f * (hold + holdp));
          if (wb > 0.f)
            botw = wb * (avn.x * tvd_v(cp, 0.f, cp2, alfa) + avn.y * tvd_v(cp, 0.f, 0.f, alfa));
          else
            botw = At * wb * tvd_v(0.f, cp, up_ok ? cm : cp, alfa);
        }
      }
      const float fw = aat * (topw - botw);
      const float fd = adt * (-At * cp * hmobot - A * cm * hmotop);
      const float fi = A * clmm * cm + At * clpp * cp;   // implicit vertical terms on the shifted values
      float q = hs[r] - fw - fd - fi;
      // boundary mass flux (conz3d_nodes :805-813): an inflow brings the
      // boundary concentration, an outflow takes the node's own (no change)
      if (qf > 0.f && sidx[r] >= 0) {
        const float cb = d.cbnd[sidx[r] * SN + o];
        q += qf * (cb - c);
      }
      if constexpr (EX)                               // nudging, summed over the elements
        if (act && d.cz_robs != 0.f) q += A * hold * (d.cz_robs * d.cz_tau[o] * (d.cz_obs[o] - c));
      res[r] = act ? c * rcont + dt * q : 0.f;        // right-hand side of the increment
    }
    if constexpr (EX) {
      // loading on the node layer's mass M = A h_old c + dt q: a source adds
      // dt*loading; a sink removes at most what an exponential decay over dt
      // would, and the load is cut to what it removed
      if (act && valid && d.cz_rload != 0.f) {
        const float c = cl[0];
        const float mass = res[0] + (up_ok ? clo * cm1[0] : 0.f) + cdg * c + (dn_ok ? chi * cp1[0] : 0.f);
        float loading = d.cz_rload * d.cz_load[o];
        if (loading < 0.f) {
          float cload = 0.f;
          if (mass > 0.f) cload = mass * (1.f - expf(dt * loading / mass));
          else if (mass < 0.f) res[0] -= mass;
          loading = -cload / dt;
          if (d.cz_rload > 0.f) d.cz_load[o] = loading / d.cz_rload;
        }
        res[0] += dt * loading;
      }
    }
    // vertical system of the node column (conz3d_nodes :841-868)
    if ((P.aa == 0.f && P.ad == 0.f) || P.nlv == 1) {
#pragma unroll
      for (int r = 0; r < NR; r++) res[r] = (act && cdg != 0.f) ? res[r] / cdg : res[r];
    } else {
      if (act && cdg == 0.f && valid) set_status(&d.out[b], SHY_ESINGULAR);
#pragma unroll
      for (int r = 0; r < NR; r++) res[r] = act ? res[r] : 0.f;
      pcr_solve_f<S, NR>(act ? clo : 0.f, act ? cdg : 1.f, act ? chi : 0.f, res, lane);
    }
#pragma unroll
    for (int r = 0; r < NR; r++) {
      if (sidx[r] < 0) continue;
      const int s = sidx[r];
      float cf = act ? cl[r] + res[r] : 0.f;         // old value plus increment
      if (act && isbnd && !d.conz_free_bnd) cf = d.cbnd[s * SN + o];      // bndo_impbc
      if (valid && lane < NLV) cout_base[s * SN + o] = cf;
    }
  }
}

// rhoset (baroclinic.f90:654-710) once temperature and salinity are final:
// one pass, the pressure from the previous rho' (rhoset_shell(1)), z-layers
// (hlayer = hldv).  d.sc_out holds the step's final scalars.
template <int S>
__global__ void __launch_bounds__(256) k_rho(Dev d, const int *kbas) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = gt / S;
  const int lane = threadIdx.x & (S - 1);
  const bool valid = k0 < d.NKN;
  const int k = valid ? k0 : d.NKN - 1;
  const int NLV = d.NLV;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  if (!(P.ibarcl > 0 && P.itemp && P.isalt)) return;
  const int lmax = d.ilhkv[k];
  const bool act = lane < lmax;
  const size_t o = (size_t)k * NLV + lane;
  const size_t SN = (size_t)d.NKN * NLV;
  const float *hld = d.hldv + (size_t)b * NLV;
  // sigma layers: the old thickness of the step (hdkov); z-layers: nominal
  const double hh = lane < NLV ? 0.5 * (lane < P.nsigma ? (act ? (double)d.hko[o] : 0.) : (double)hld[lane]) : 0.;
  const double rold = act ? (double)d.rho[o] : 0.;
  const double dpresc = rold * P.grav * hh;
  const double depth = seg_scan_down<S>(act ? 2. * hh : 0., lane) - hh;
  const double pbc = seg_scan_down<S>(act ? 2. * dpresc : 0., lane) - dpresc;
  if (act && valid) {
    const double t = d.sc_out[o], s = d.sc_out[SN + o];    // T is scalar 0, S scalar 1
    const double rho0 = P.rowass, sigma0 = rho0 - 1000.;
    const double pres = 1.e-5 * (rho0 * P.grav * depth + pbc);
    d.rho[o] = (float)(sigma_stp_d(s > 0. ? s : 0., t, (double)(float)pres) - sigma0);
  }
}

}  // namespace shy
