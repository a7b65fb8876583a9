// k_node.cuh -- nodal layer thickness, vertical velocity, stability index, reductions, initial rho
// Included by node_launch.cuh.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace shy {

// The FP64 volume budget of a node column: every step adds dt times the flow
// into it, the element fluxes 3 * 4aj * (U b + V c) of the zeta equation
// (az-weighted transports summed over the element's layers) and the node's
// discharge.  The gradients come from the element's FP32 b, c with the last
// vertex's taken as minus the sum of the other two, so that each element's
// three fluxes cancel exactly and a closed basin's summed budget moves by
// FP64 round-off only.  A level-boundary node has no continuity equation
// (its level is imposed), so its budget is its volume at that level.
__device__ __forceinline__ double2 budget_grad(const float *evp, int ii) {
  if (ii < 2) return make_double2((double)evp[ii], (double)evp[3 + ii]);
  return make_double2(-((double)evp[0] + (double)evp[1]), -((double)evp[3] + (double)evp[4]));
}

__device__ __forceinline__ double budget_discharge(const Dev &d, const BasinPar &P, int k) {
  return (P.wetdry && d.inod[k] == -2) ? 0. : (double)d.rqv[k];
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
  const float *hld = d.hldv + (size_t)b * NLV;
  const float *hlv = d.hlv + (size_t)b * NLV;
  const double hldl = lane < NLV ? (double)hld[lane] : 0.;
  double hsum = 0., vf = 0., va = 0.;
  double bud = 0.;                            // FP64 budget: this layer's flow into the node
  double hsig_h = 0.;                         // sigma: depth of the last incident element's vertex
#pragma unroll 2
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
    const int4 ix = d.incx[p];
    const int e = ix.x, ii = ix.y & 3, le = ix.y >> 2;
    if (lane >= le) continue;
    const float *evp = d.ev8 + (size_t)e * 8;
    const double aj = evp[6];
    const double areafv = 4. * aj;            // 12*aj/3
    const float4 hm = d.hm3v[e];
    const double htot = ii == 0 ? hm.x : (ii == 1 ? hm.y : hm.z);
    hsig_h = htot;
    double hl;
    if (P.nzadapt > 1) hl = zad_vertex_h(lane, z, htot, le, zad_levmax(z, hlv, le, P.rzmov), hlv, hld);
    else if (le == 1) hl = htot + z;
    else if (lane < le - 1) hl = hldl + (lane == 0 ? z : 0.);
    else hl = htot - hlv[le - 2];
    hsum += areafv * hl;
    if (!init_only) {
      const double bb = evp[ii], cc = evp[3 + ii];
      const size_t oe = (size_t)e * NLV + lane;
      double ff = (double)d.usv[oe] * bb + (double)d.vsv[oe] * cc;   // az*ffn + azt*ffo
      const double aj4 = 4. * aj;
      vf += 3. * aj4 * ff;
      va += aj4;
      const double2 g = budget_grad(evp, ii);
      bud += 3. * aj4 * ((double)d.usv[oe] * g.x + (double)d.vsv[oe] * g.y);
    }
  }
  const size_t o = (size_t)k * NLV + lane;
  const double area = act ? (double)d.areakv[o] : 0.;
  double hk = act && area > 0. ? hsum / area : 0.;
  if (lane < P.nsigma && act) hk = -(fmin(hsig_h, (double)P.hsigma) + z) * hldl;   // sigma layers (:1019-1025)
  float hkf = (float)hk;
  if (act && !(hkf > 0.f) && valid) set_status(&d.out[b], SHY_EDEPTH);
  if (valid && lane < NLV) d.hkn[o] = act ? hkf : 0.f;
  // node volume (masscont: sum of real hdknv*areakv in double)
  double vol = act ? (double)(hkf * (float)area) : 0.;
  vol = seg_sum<S>(vol);
  if (lane == 0 && valid) d.vol_node[k] = vol;
  bud = seg_sum<S>(act ? bud : 0.);
  if (lane == 0 && valid) {
    if (init_only || d.kbnd[k] > 0) d.vbud_node[k] = vol;   // level boundary: the imposed level's volume
    else d.vbud_node[k] += P.dt * (bud + budget_discharge(d, P, k));
  }
  if (init_only) return;
  // hydro_vertical: w from continuity, bottom-up (hydrodynamic.f90:1711-1771),
  // with the layer's share of the node's discharge (mfluxv, :1727)
  const int I = NLV + 1;
  const float q = mflux_layer<S>(d, k, act, o, P.wetdry != 0);
  double dv = 0.;
  if (act && P.nlv > 1) {
    double voln = (double)(hkf * (float)area), volo = (double)(d.hko[o] * (float)area);
    // a sigma layer's thickness moves with the level alone, -hldv (zn - zo):
    // taken so, its change carries no rounding of the two FP32 thicknesses,
    // which at short time steps would be most of the change
    if (lane < P.nsigma) { voln = -hldl * (z - (double)d.zo[k]) * (double)(float)area; volo = 0.; }
    dv = vf + (double)q - (voln - volo) / P.dt;
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
// k_node_t: the same with one thread per node column (shallow columns): the
// incident elements are walked once, each adding to the FP64 sums of all
// its layers (in element order, as k_node); then the node's layers in turn
// ===========================================================================
//
// ZA: the instance with z-adaptive layers; without them (every basin with
// nzadapt <= 1) the thickness of a layer is a sum of nominal values and
// the level, and the kernel keeps fewer registers.
template <int L, bool PF = false, bool ZA = true>
__global__ void __launch_bounds__(128, ZA ? 6 : 8) k_node_t(Dev d, const int *kbas, int init_only) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.NKN) return;
  const int NLV = d.NLV, I = NLV + 1;
  const int b = kbas[k];
  const BasinPar &P = d.par[b];
  const int lmax = d.ilhkv[k];
  const double z = d.zn[k];
  const float *hld = d.hldv + (size_t)b * NLV;
  const float *hlv = d.hlv + (size_t)b * NLV;
  // sums in FP32 in element order, as the reference's real hdkn and vf
  // (setdepth, hydro_vertical); va, the area of the elements with the layer,
  // is static (Dev::avol)
  float hsum[L], vf[L];
  double bud = 0.;                            // FP64 budget: the flow into the node column
  double hsig_h = 0.;                         // sigma: depth of the last incident element's vertex
#pragma unroll
  for (int l = 0; l < L; l++) { hsum[l] = 0.f; vf[l] = 0.f; }
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
    const int4 ix = d.incx[p];
    const int e = ix.x, ii = ix.y & 3, le = ix.y >> 2;
    const float *evp = d.ev8 + (size_t)e * 8;
    const float aj = evp[6];
    const float areafv = 4.f * aj;            // 12*aj/3
    const float4 hm = d.hm3v[e];
    const float htot = ii == 0 ? hm.x : (ii == 1 ? hm.y : hm.z);
    const float bb = evp[ii], cc = evp[3 + ii];
    const size_t oe = (size_t)e * NLV;
    const float hbot = le >= 2 ? htot - hlv[le - 2] : 0.f;
    hsig_h = htot;
    // setdepth takes the element's vertex level (a dry element's differs)
    const float ze = P.wetdry ? d.zen[3 * e + ii] : (float)z;
    double us = 0., vs = 0.;                  // the element's transports summed over its layers
    const int lev = ZA && P.nzadapt > 1 ? zad_levmax((double)ze, hlv, le, P.rzmov) : 0;
    // PF: the element's transports of every layer loaded at once (the
    // layers below its bottom hold zeros), so their loads are in flight
    // together; else each layer's as the loop reaches it
    float ue[PF ? L : 1], ve[PF ? L : 1];
    if constexpr (PF) {
#pragma unroll
      for (int l = 0; l < L; l++) {
        const bool in = !init_only && l < NLV;
        ue[l] = in ? d.usv[oe + l] : 0.f;
        ve[l] = in ? d.vsv[oe + l] : 0.f;
      }
    }
#pragma unroll
    for (int l = 0; l < L; l++) {
      if (l >= le) break;
      float hl;
      if (ZA && P.nzadapt > 1) hl = (float)zad_vertex_h(l, (double)ze, (double)htot, le, lev, hlv, hld);
      else if (le == 1) hl = htot + ze;
      else if (l < le - 1) hl = hld[l] + (l == 0 ? ze : 0.f);
      else hl = hbot;
      hsum[l] += areafv * hl;
      if (!init_only) {
        const float ul = PF ? ue[PF ? l : 0] : d.usv[oe + l], vl = PF ? ve[PF ? l : 0] : d.vsv[oe + l];
        const float ff = ul * bb + vl * cc;   // az*ffn + azt*ffo
        vf[l] += 3.f * areafv * ff;
        us += (double)ul;
        vs += (double)vl;
      }
    }
    if (!init_only) {
      const double2 g = budget_grad(evp, ii);
      bud += 3. * (4. * (double)aj) * (us * g.x + vs * g.y);
    }
  }
  const size_t o = (size_t)k * NLV;
  double vol = 0.;
  float hkf[L];                               // the new thickness; the areas are read again below
  bool bad = false;
#pragma unroll
  for (int l = 0; l < L; l++) {
    hkf[l] = 0.f;
    if (l >= NLV) continue;
    const bool act = l < lmax;
    const float areal = act ? d.areakv[o + l] : 0.f;
    double hk = act && areal > 0.f ? (double)(hsum[l] / areal) : 0.;
    if (l < P.nsigma && act) hk = -(fmin(hsig_h, (double)P.hsigma) + z) * (double)hld[l];   // sigma layers (:1019-1025)
    hkf[l] = (float)hk;
    if (act && !(hkf[l] > 0.f)) bad = true;
    d.hkn[o + l] = act ? hkf[l] : 0.f;
    // node volume (masscont: sum of real hdknv*areakv in double)
    vol += act ? (double)(hkf[l] * areal) : 0.;
  }
  if (bad) set_status(&d.out[b], SHY_EDEPTH);
  d.vol_node[k] = vol;
  if (init_only || d.kbnd[k] > 0) d.vbud_node[k] = vol;     // level boundary: the imposed level's volume
  else d.vbud_node[k] += P.dt * (bud + budget_discharge(d, P, k));
  if (init_only) return;
  // hydro_vertical: w from continuity, bottom-up (hydrodynamic.f90:1711-1771),
  // with each layer's share of the node's discharge (set_mass_flux: by the
  // layers' volumes at the start of the step; mfluxv, :1727)
  const bool wzero = P.nlv == 1 || d.kbnd[k] > 0;
  const float rq = (P.wetdry && d.inod[k] == -2) ? 0.f : d.rqv[k];
  double vtot = 0.;
  if (rq != 0.f)
    for (int l = 0; l < lmax; l++) vtot += (double)(d.hko[o + l] * d.areakv[o + l]);
  double acc = 0.;                             // flux through the top of layer l
#pragma unroll
  for (int l = L - 1; l >= 0; l--) {
    if (l >= NLV) continue;
    const bool act = l < lmax;
    double dv = 0.;
    if (act && P.nlv > 1) {
      const float areal = d.areakv[o + l];
      double voln = (double)(hkf[l] * areal);
      double volo = (double)(d.hko[o + l] * areal);
      // a sigma layer's thickness moves with the level alone, -hldv (zn -
      // zo): taken so, its change carries no rounding of the two FP32
      // thicknesses, which at short time steps would be most of the change
      if (l < P.nsigma) { voln = -(double)hld[l] * (z - (double)d.zo[k]) * (double)areal; volo = 0.; }
      const float q = vtot > 0. ? (float)((double)rq * ((double)(d.hko[o + l] * d.areakv[o + l]) / vtot)) : 0.f;
      dv = (double)vf[l] + (double)q - (voln - volo) / P.dt;
    }
    acc += dv;
    double wtop = acc;
    if (l == 0) wtop = 0.;                     // wlnv(lmin-1) = 0
    if (l >= 1 && act) {
      const float2 av = d.avol[o + l];         // aj4 over the elements with layer l
      const double va = (double)av.x + (double)av.y;
      if (va > 0.) wtop /= va;
    }
    if (!act || wzero) wtop = 0.;
    d.wl[(size_t)k * I + l] = (float)wtop;
  }
  d.wl[(size_t)k * I + NLV] = 0.f;
}

// ===========================================================================
// k_moment: the node momentum of the step's advective terms (set_momentum_flux,
// explicit.f90:588-683), for basins with ilin = 0, from the old level at
// the start of the step.  Per node layer (one lane each): the momentum that
// flows in, weighted by the inflow f = U b + V c > 0 of each incident element
// layer; with outflow only, the node's velocity times its thickness, the
// velocity (uprv) being the area-weighted mean of U/h over the incident
// elements in the system (uvtopr, transforms.f90:214-270, computed by the
// reference at the end of the last step, which these old arrays hold).
// Launched before the set_dry pass, so the wet marks are the last step's.
// Sums in FP32 in element order, as the reference's real arrays.
// ===========================================================================
template <int S>
__global__ void __launch_bounds__(256) k_moment(Dev d, const int *kbas) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = gt / S;
  const int lane = threadIdx.x & (S - 1);
  if (k >= d.NKN) return;
  const int NLV = d.NLV;
  const BasinPar &P = d.par[kbas[k]];
  if (!P.adv) return;
  const bool wd = P.wetdry && P.nsigma == 0;
  float saux = 0.f, mx = 0.f, my = 0.f, vv = 0.f, up = 0.f, vp = 0.f;
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {
    const int4 ix = d.incx[p];
    const int e = ix.x, ii = ix.y & 3, le = ix.y >> 2;
    if (lane >= le) continue;
    const size_t oe = (size_t)e * NLV + lane;
    const float ut = d.uo[oe], vt = d.vo[oe];
    const float *evp = d.ev8 + (size_t)e * 8;
    const float f = ut * evp[ii] + vt * evp[3 + ii];       // > 0: flux into the node
    if (f > 0.f) { saux += f; mx += f * ut; my += f * vt; }
    if (!wd || d.iweg[e] == 0) {
      const float aj = evp[6], h = d.heo[oe];
      vv += aj;
      up += aj * (h > 0.f ? ut / h : 0.f);
      vp += aj * (h > 0.f ? vt / h : 0.f);
    }
  }
  if (lane >= NLV) return;
  const size_t o = (size_t)k * NLV + lane;
  float2 m = make_float2(0.f, 0.f);
  if (lane < d.ilhkv[k]) {
    if (saux > 0.f) m = make_float2(mx / saux, my / saux);
    else if (vv > 0.f) {
      const float h = d.hko[o];
      m = make_float2(up / vv * h, vp / vv * h);
    }
  }
  d.mom[o] = m;
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
  const double adt = 1. - (double)P.ad, aat = 1. - (double)P.aa;
  const size_t o = (size_t)k * NLV + lane;
  const double hold = act ? (double)d.hko[o] : 0., hnew = act ? (double)d.hkn[o] : 0.;
  const double rvptop = act ? (double)d.difv[(size_t)k * I + lane] + P.difmol : 0.;
  const double rvpbot = act ? (double)d.difv[(size_t)k * I + lane + 1] + P.difmol : 0.;
  // point sources: the inflow of the node layer (conzstab co, concentration.f90:1801)
  const float qin = fmaxf(mflux_layer<S>(d, k, act, o, P.wetdry != 0), 0.f);
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
          const double us = d.usv[oe], vs = d.vsv[oe];
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
      double r = (act && cdiag > 0.) ? (chigh + clow + cn + (double)qin) / cdiag : 0.;
      stab = seg_max<S>((float)r);
    }
    if (lane == 0 && valid && d.kbnd[k] == 0) atomic_max_pos(&d.out[b].stab[s], stab);
  }
}

// ===========================================================================
// k_reduce: per basin (one block each): volume, sub-step counts, time
// ===========================================================================
static __global__ void __launch_bounds__(1024) k_reduce(Dev d, int nsub, int advance) {
  const int b = blockIdx.x;
  const BasinPar &P = d.par[b];
  BasinOut &O = d.out[b];
  __shared__ double part[1024], partb[1024];
  double s = 0., sb = 0.;
  for (int k = threadIdx.x; k < P.nk; k += blockDim.x) {
    s += d.vol_node[P.k0 + k];
    sb += d.vbud_node[P.k0 + k];
  }
  part[threadIdx.x] = s;
  partb[threadIdx.x] = sb;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      part[threadIdx.x] += part[threadIdx.x + w];
      partb[threadIdx.x] += partb[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    O.volume = part[0];
    O.vbudget = partb[0];
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
      O.steps += 1;
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
  // sigma layers: the initial thickness (hdkov = hdknv at the start); z-layers: nominal
  const double hh = lane < NLV ? 0.5 * (lane < P.nsigma ? (act ? (double)d.hkn[o] : 0.) : (double)hld[lane]) : 0.;
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


}  // namespace shy
