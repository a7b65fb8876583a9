// nonhydro.cu -- the non-hydrostatic pressure (nohydro.f90) on the device,
// and the device-wide sparse solver of its 3D system, which the 3D simsys
// entries (system_solve_3d_) share.
//
// After the hydrostatic part of the step (k_final: transports, element
// levels and thickness) the basins with inohyd = 1 run
//   k_nh_w        sp256wnh (nohydro.f90:205-524): w from the vertical
//                 momentum equation, one tridiagonal system per node over
//                 its interfaces, the element terms gathered in element order;
//   k_nh_sys      nonhydro_prepare_matrix + system_assemble_3d (nohydro.f90:
//                 589-753, simsys_spkaux.f90:597-635): one thread per row of
//                 the 3D system, the element-layer contributions summed in
//                 element order in FP64, as the reference's COO sums them;
//   k_nh_solve    system_solve_3d (simsys_spkaux.f90:495-530): BiCGStab in
//                 FP32 with Jacobi preconditioning inside FP64 residual
//                 refinement, on the reference's stop test, one cooperative
//                 launch over the device per basin;
//   k_nh_node     nonhydro_correct_uveta's level correction (:785-792) and
//                 the pressure the next step reads, its first layer zeroed
//                 (nonhydro_adjust :168-176);
//   k_nh_elem     nonhydro_correct_uveta's transport correction (:805-827),
//                 the time-weighted transports, setzev and the element part
//                 of make_new_depth.
// k_node then builds the node thickness and w from the corrected state, as
// hydro_vertical follows nonhydro_adjust in hydro (hydrodynamic.f90:435-441).
//
// The 3D system keeps one unknown per active node layer (k, l), l <
// ilhkv(k).  The reference's system also holds the padding layers 0 and
// nlv+1 of every node and the layers below a node's deepest element, all
// identity rows with a zero right-hand side that no other row couples to,
// so their unknowns stay zero and the solution is the same.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "../../include/shygpu.h"
#include "launch.h"
#include "physics.cuh"

namespace shy {

// ---------------------------------------------------------------------------
// sp256wnh: one thread per node column of a non-hydrostatic basin
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_nh_w(Dev d, NhSys s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.NKN || s.roff[k] < 0) return;
  const int NLV = d.NLV, I = NLV + 1;
  const BasinPar &P = d.par[s.kbas[k]];
  const float dt = (float)P.dt, aq = P.aqpar, aqt = 1.f - aq, az = P.az, azt = 1.f - az;
  float wd[SHY_MAX_LAYERS + 1], wt[SHY_MAX_LAYERS + 1], wbt[SHY_MAX_LAYERS + 1], wr[SHY_MAX_LAYERS + 1];
  for (int l = 0; l <= NLV; l++) { wd[l] = 0.f; wt[l] = 0.f; wbt[l] = 0.f; wr[l] = 0.f; }
  const float qd = d.qdist[k];
  const float *wlo = d.wl + (size_t)k * I;
  for (int p = d.inc_ptr[k]; p < d.inc_ptr[k + 1]; p++) {   // incident elements, in element order
    const int v = d.inc[p];
    const int e = v / 3, ii = v - 3 * e;
    const int4 en = d.enode[e];
    const int kn[3] = {en.x, en.y, en.z};
    const float *evp = d.ev8 + (size_t)e * 8;
    const float b[3] = {evp[0], evp[1], evp[2]}, c[3] = {evp[3], evp[4], evp[5]};
    const float aj4 = 4.f * evp[6];
    const int ilevel = d.ilhv[e];
    const size_t o = (size_t)e * NLV;
    for (int l = 1; l <= ilevel; l++) {
      const bool blast = l == ilevel;
      const float hdn = d.hen[o + l - 1], hdo = d.heo[o + l - 1];
      const float utn = d.un[o + l - 1], uto = d.uo[o + l - 1], vtn = d.vn[o + l - 1], vto = d.vo[o + l - 1];
      float hdpn = 0.f, hdpo = 0.f, ubn = 0.f, ubo = 0.f, vbn = 0.f, vbo = 0.f, anu;
      if (blast) anu = 0.5f * P.ahpar * d.difhv[o + l - 1];
      else {
        hdpn = d.hen[o + l]; hdpo = d.heo[o + l];
        ubn = d.un[o + l]; ubo = d.uo[o + l]; vbn = d.vn[o + l]; vbo = d.vo[o + l];
        anu = 0.5f * P.ahpar * (d.difhv[o + l - 1] + d.difhv[o + l]);
      }
      const float dzn = 0.5f * (hdn + hdpn), dzo = 0.5f * (hdo + hdpo);
      const float us = 0.5f * (az * (utn + ubn) / dzn + azt * (uto + ubo) / dzo);
      const float vs = 0.5f * (az * (vtn + vbn) / dzn + azt * (vto + vbo) / dzo);
      float wl[3], f[3], wb = 0.f, wc = 0.f, wsum = 0.f;
      int itot = 0, isum = 0;
#pragma unroll
      for (int jj = 0; jj < 3; jj++) {
        wl[jj] = d.wl[(size_t)kn[jj] * I + l];
        f[jj] = us * b[jj] + vs * c[jj];
        if (f[jj] < 0.f) { itot++; isum += jj + 1; }
        wb += b[jj] * wl[jj]; wc += c[jj] * wl[jj]; wsum += wl[jj];
      }
      float fli = 0.f;                     // inhflx = 1: this vertex's upwind flux of w
      if (P.inhflx == 1) {
        if (itot == 1) fli = f[ii] * wl[isum - 1];
        else if (itot == 2) {
          const int iz = 6 - isum - 1;     // the vertex the flow does not leave
          if (ii != iz) fli = f[ii] * wl[ii];
          else {
            float fs = 0.f;
#pragma unroll
            for (int jj = 0; jj < 3; jj++) if (jj != iz) fs += f[jj] * wl[jj];
            fli = -fs;
          }
        }
      }
      const float wq = blast ? 0.f : -aqt * qd * (d.qp[(size_t)k * NLV + l - 1] - d.qp[(size_t)k * NLV + l]) / dzo;
      float wadvv = 0.f;
      if (P.ivwadv == 1 && !blast) {
        const float wplus = 0.5f * (wlo[l] + wlo[l - 1]) / dzo;
        wadvv = wplus > 0.f ? wplus * wlo[l] : wplus * wlo[l - 1];
        const float wminus = 0.5f * (wlo[l] + wlo[l + 1]) / dzo;
        wadvv -= wminus > 0.f ? wminus * wlo[l + 1] : wminus * wlo[l];
      } else if (P.ivwadv >= 2 && !blast) {
        wadvv = 0.5f * wlo[l] * (wlo[l - 1] - wlo[l + 1]) / dzo;
      }
      const float wdifh = -3.f * anu * (wb * b[ii] + wc * c[ii]);
      const float wadvh = P.inhflx == 1 ? -3.f * fli : -(b[ii] * us + c[ii] * vs) * wsum;
      const float wrr = dzn * (wlo[l] + dt * (wq + wdifh - wadvh - wadvv));
      wr[l] += aj4 * wrr;
      if (blast) {                         // the element's bottom: w = 0 (an identity row)
        wd[l] = 1.f; wt[l] = 0.f; wbt[l] = 0.f; wr[l] = 0.f;
      } else {
        const float rnu = d.visv[(size_t)k * I + l];
        wd[l] += dzn * aj4 + dt * aj4 * rnu * (1.f / hdn + 1.f / hdpn);
        wt[l] -= dt * aj4 * rnu / hdn;
        wbt[l] -= dt * aj4 * rnu / hdpn;
      }
    }
  }
  // tridag (keps_util.f90:82-111) over the interfaces 1..lmax-1
  const int lmax = d.ilhkv[k];
  float *wn = s.wnh + (size_t)k * I;
  for (int l = 0; l <= NLV; l++) wn[l] = 0.f;
  if (lmax > 2) {
    const int n = lmax - 1;
    float gam[SHY_MAX_LAYERS + 1];
    float bet = wd[1];
    if (bet == 0.f) { set_status(&d.out[s.kbas[k]], SHY_ESINGULAR); return; }
    wn[1] = wr[1] / bet;
    for (int j = 2; j <= n; j++) {
      gam[j] = wbt[j - 1] / bet;
      bet = wd[j] - wt[j] * gam[j];
      if (bet == 0.f) { set_status(&d.out[s.kbas[k]], SHY_ESINGULAR); return; }
      wn[j] = (wr[j] - wt[j] * wn[j - 1]) / bet;
    }
    for (int j = n - 1; j >= 1; j--) wn[j] -= gam[j + 1] * wn[j + 1];
  }
}

// ---------------------------------------------------------------------------
// nonhydro_prepare_matrix + system_assemble_3d: one thread per 3D row
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_nh_sys(Dev d, NhSys s) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= s.nrow) return;
  const int k = s.rnode[r], l = r - s.roff[k] + 1;   // layer l = 1..ilhkv(k)
  const int NLV = d.NLV, I = NLV + 1;
  const BasinPar &P = d.par[s.kbas[k]];
  const double dt = P.dt, aq = P.aqpar, az = P.az, azt = 1. - az, grav = P.grav;
  const int lmaxk = d.ilhkv[k];
  int q = s.rowptr[r];
  double rhs = 0.;
  for (int sl = d.rowptr[k]; sl < d.rowptr[k + 1]; sl++) {   // the 2D row's slots, columns ascending
    const int kj = d.col[sl];
    if (kj != k) {
      if (d.ilhkv[kj] < l) continue;
      double v = 0.;
      for (int t = d.slot_ptr[sl]; t < d.slot_ptr[sl + 1]; t++) {   // element entries, element order
        const int src = d.slot_src[t];
        const int e = src / 9, cc = src - 9 * e, i = cc / 3, j = cc - 3 * i;
        if (d.ilhv[e] < l) continue;
        const float *evp = d.ev8 + (size_t)e * 8;
        const double aj12 = 12. * (double)evp[6];
        const double hd = d.hen[(size_t)e * NLV + l - 1];
        v += -aj12 * hd * dt * aq * az * ((double)evp[i] * evp[j] + (double)evp[3 + i] * evp[3 + j]);
      }
      s.val[q++] = v;
    } else {
      double vm = 0., v0 = 0., vp = 0.;
      for (int t = d.slot_ptr[sl]; t < d.slot_ptr[sl + 1]; t++) {   // every element of node k
        const int src = d.slot_src[t];
        const int e = src / 9, i = (src - 9 * e) / 3;
        const int lmax = d.ilhv[e];
        if (lmax < l) continue;
        const float *evp = d.ev8 + (size_t)e * 8;
        const double aj = evp[6], aj4 = 4. * aj, aj12 = 12. * aj;
        const double bi = evp[i], ci = evp[3 + i];
        const size_t o = (size_t)e * NLV + l - 1;
        const double hd = d.hen[o];
        const double hdm = l > 1 ? (double)d.hen[o - 1] : 0.;
        const double hdp = l < NLV ? (double)d.hen[o + 1] : 0.;
        double rhm = 2. / (hd + hdm), rhp = 2. / (hd + hdp);
        if (l == 1) rhm = 0.;
        if (l == lmax) rhp = 0.;
        const double rhc = rhm + rhp;
        double m0 = -aj12 * hd * dt * aq * az * (bi * bi + ci * ci);
        m0 -= aj4 * dt * aq * rhc;
        const double fhn = (double)d.un[o] * bi + (double)d.vn[o] * ci;
        const double fho = (double)d.uo[o] * bi + (double)d.vo[o] * ci;
        const double fvn = (double)s.wnh[(size_t)k * I + l - 1] - (double)s.wnh[(size_t)k * I + l];
        const double ffh = -(az * fhn + azt * fho);
        double re = aj4 * (3. * ffh + fvn);
        if (l == 1) {                      // the free surface
          m0 -= aj4 / (grav * dt);
          re += aj4 * ((double)d.zn[k] - (double)d.zo[k]) / dt;
        }
        vm += aj4 * dt * aq * rhm;
        v0 += m0;
        vp += aj4 * dt * aq * rhp;
        rhs += re;
      }
      if (l > 1) s.val[q++] = vm;
      s.val[q++] = v0;
      if (l < lmaxk) s.val[q++] = vp;
    }
  }
  s.rhs[r] = rhs;
}

// ---------------------------------------------------------------------------
// The device-wide CSR solver: BiCGStab (van der Vorst 1992) with right Jacobi
// preconditioning in FP32 on the correction of an FP64 iterate; the FP64
// residual is recomputed after every inner solve and the call ends when it
// meets ||r|| <= rtol ||r0|| + atol (the reference's stopbis test).  One
// cooperative launch of G CTAs over rows [r0, r1); CTA c works a contiguous
// share.  Sums are taken per CTA, published, and added by every CTA in CTA
// order after a grid barrier, so every CTA gets the same bits and the result
// does not depend on timing.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned nh_ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// bar-th grid barrier: arrivals count up in ctr[0], the last arrival
// publishes bar in ctr[1] (release), the others poll it (acquire) at most
// spin_limit times; a wait that gives up sets ctr[2], which ends every
// other wait too.  Returns false after a timeout.
__device__ __forceinline__ bool nh_barrier(const CsrGrid &a, unsigned bar, int *s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(a.ctr) : "memory");
    if (old + 1u == bar * gridDim.x) {
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.ctr + 1), "r"(bar) : "memory");
    } else {
      long long spins = 0;
      while (nh_ld_acquire(a.ctr + 1) < bar) {
        if (nh_ld_acquire(a.ctr + 2) != 0u || ++spins > a.spin_limit) {
          atomicExch(a.ctr + 2, 1u);
          ok = 0;
          break;
        }
        if (spins > 256) __nanosleep(32);
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// shared scratch of the sums; the barrier count and the parity of the
// partial-sum slots are kept by every thread in its own registers (all
// threads take the same barriers), so no thread updates them for another
struct NhRed {
  double wsum[4 * 32];
  double bc[4];
  int ok;
};

template <int NV>
__device__ __forceinline__ bool nh_gsum(const CsrGrid &a, double (&v)[NV], NhRed &sm, unsigned &bar, int &par) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sm.wsum[i * 32 + warp] = x;
  }
  __syncthreads();
  const int G = gridDim.x;
  double *part = a.part + (size_t)par * G * 4;
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double x = lane < nw ? sm.wsum[i * 32 + lane] : 0.;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) part[(size_t)blockIdx.x * 4 + i] = x;
    }
  }
  if (!nh_barrier(a, ++bar, &sm.ok)) return false;
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double x = 0.;
      for (int c = lane; c < G; c += 32) x += __ldcg(&part[(size_t)c * 4 + i]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) sm.bc[i] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = sm.bc[i];
  par ^= 1;
  return true;
}

__device__ __forceinline__ float nh_spmv(const CsrGrid &a, int i, const float *u) {
  float w = 0.f;
  for (int k = a.rowptr[i]; k < a.rowptr[i + 1]; k++) w += a.val32[k] * __ldcg(&u[a.col[k]]);
  return w;
}

__global__ void __launch_bounds__(512) k_nh_solve(CsrGrid a) {
  __shared__ NhRed sm;
  unsigned bar = 0;     // grid barriers taken so far (the same in every thread)
  int par = 0;          // slot set of the next partial sums
  if (threadIdx.x == 0) sm.ok = 1;
  __syncthreads();
  const int n = a.r1 - a.r0, G = gridDim.x;
  const int chunk = (n + G - 1) / G;
  const int c0 = a.r0 + min(n, (int)blockIdx.x * chunk), c1 = a.r0 + min(n, ((int)blockIdx.x + 1) * chunk);
  const int tid = threadIdx.x, nth = blockDim.x;
  bool aborted = false;

  for (int i = c0 + tid; i < c1; i += nth) {
    double diag = 0.;
    for (int k = a.rowptr[i]; k < a.rowptr[i + 1]; k++) {
      const double w = a.val[k];
      a.val32[k] = (float)w;
      if (a.col[k] == i) diag += w;
    }
    a.dinv[i] = diag != 0. ? (float)(1. / diag) : 1.f;
    a.x64[i] = (double)a.x[i];
  }
  if (!nh_barrier(a, ++bar, &sm.ok)) aborted = true;

  double tol = 0., rn = 0., rn0 = 0.;
  int iters = 0, outer = 0;
  bool conv = false;
  for (outer = 0; !aborted; outer++) {
    double acc[1] = {0.};
    for (int i = c0 + tid; i < c1; i += nth) {
      double res = a.rhs[i];
      for (int k = a.rowptr[i]; k < a.rowptr[i + 1]; k++) res -= a.val[k] * __ldcg(&a.x64[a.col[k]]);
      a.r[i] = (float)res;
      a.rh[i] = (float)res;
      a.p[i] = 0.f; a.v[i] = 0.f; a.e[i] = 0.f;
      acc[0] += res * res;
    }
    if (!nh_gsum<1>(a, acc, sm, bar, par)) { aborted = true; break; }
    rn = sqrt(acc[0]);
    if (outer == 0) { tol = a.rtol * rn + a.atol; rn0 = rn; }
    if (rn <= tol) { conv = true; break; }
    if (outer == a.max_outer || iters >= a.maxit) break;
    const double itol = fmax((double)a.inner_rtol * rn, 0.25 * tol);
    double rho = 1., alpha = 1., omega = 1., rho1 = acc[0];
    while (iters < a.maxit) {
      const double beta = (rho1 / rho) * (alpha / omega);
      rho = rho1;
      const float fb = (float)beta, fo = (float)omega;
      for (int i = c0 + tid; i < c1; i += nth) {
        const float pp = a.r[i] + fb * (a.p[i] - fo * a.v[i]);
        a.p[i] = pp;
        a.z[i] = a.dinv[i] * pp;
      }
      if (!nh_barrier(a, ++bar, &sm.ok)) { aborted = true; break; }
      double g1[1] = {0.};
      for (int i = c0 + tid; i < c1; i += nth) {
        const float vv = nh_spmv(a, i, a.z);
        a.v[i] = vv;
        g1[0] += (double)a.rh[i] * vv;
      }
      if (!nh_gsum<1>(a, g1, sm, bar, par)) { aborted = true; break; }
      alpha = g1[0] != 0. ? rho / g1[0] : 0.;
      const float fa = (float)alpha;
      for (int i = c0 + tid; i < c1; i += nth) {
        const float ss = a.r[i] - fa * a.v[i];
        a.s[i] = ss;
        a.q[i] = a.dinv[i] * ss;
      }
      if (!nh_barrier(a, ++bar, &sm.ok)) { aborted = true; break; }
      double g2[2] = {0., 0.};
      for (int i = c0 + tid; i < c1; i += nth) {
        const float tt = nh_spmv(a, i, a.q);
        a.t[i] = tt;
        g2[0] += (double)tt * a.s[i];
        g2[1] += (double)tt * tt;
      }
      if (!nh_gsum<2>(a, g2, sm, bar, par)) { aborted = true; break; }
      omega = g2[1] > 0. ? g2[0] / g2[1] : 0.;
      const float fw = (float)omega;
      double g3[2] = {0., 0.};
      for (int i = c0 + tid; i < c1; i += nth) {
        a.e[i] += fa * a.z[i] + fw * a.q[i];
        const float rr = a.s[i] - fw * a.t[i];
        a.r[i] = rr;
        g3[0] += (double)rr * rr;
        g3[1] += (double)a.rh[i] * rr;
      }
      if (!nh_gsum<2>(a, g3, sm, bar, par)) { aborted = true; break; }
      iters++;
      rho1 = g3[1];
      if (sqrt(g3[0]) <= itol || omega == 0. || alpha == 0. || !(g3[0] == g3[0])) break;
    }
    if (aborted) break;
    for (int i = c0 + tid; i < c1; i += nth) a.x64[i] += (double)a.e[i];
    if (!nh_barrier(a, ++bar, &sm.ok)) { aborted = true; break; }
  }
  for (int i = c0 + tid; i < c1; i += nth) a.x[i] = (float)a.x64[i];
  if (blockIdx.x == 0 && tid == 0) {
    a.out->nh_iters = iters;
    a.out->nh_refinements = outer;
    a.out->nh_resid0 = rn0;
    a.out->nh_resid = rn;
    if (aborted) set_status(a.out, SHY_ECUDA);
    else if (!conv) set_status(a.out, SHY_ENOCONV);
  }
}

// ---------------------------------------------------------------------------
// nonhydro_correct_uveta and what follows it
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_nh_node(Dev d, NhSys s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.NKN || s.roff[k] < 0) return;
  const BasinPar &P = d.par[s.kbas[k]];
  const int NLV = d.NLV, lmax = d.ilhkv[k];
  const float *x = s.x + s.roff[k];
  const float zq = d.qdist[k] * x[0] / P.grav;
  d.zn[k] = d.zn[k] + zq;
  // qpnv(l,k) - qpnv(1,k) over l = 1..lmax zeroes the first layer and then
  // subtracts that zero from the others (nohydro.f90:168-176)
  for (int l = 0; l < NLV; l++) d.qp[(size_t)k * NLV + l] = (l == 0 || l >= lmax) ? 0.f : x[l];
}

__global__ void __launch_bounds__(256) k_nh_elem(Dev d, NhSys s) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.NEL) return;
  const int4 en = d.enode[e];
  const BasinPar &P = d.par[en.w];
  if (!P.inohyd) return;
  const int NLV = d.NLV;
  const int kn[3] = {en.x, en.y, en.z};
  const int ilevel = d.ilhv[e];
  const float *evp = d.ev8 + (size_t)e * 8;
  const size_t o = (size_t)e * NLV;
  const double adt = (double)P.aqpar * P.dt, az = P.az;
  float qd[3];
  const float *xk[3];
#pragma unroll
  for (int ii = 0; ii < 3; ii++) { qd[ii] = d.qdist[kn[ii]]; xk[ii] = s.x + s.roff[kn[ii]]; }
  for (int l = 0; l < ilevel; l++) {
    double uq = 0., vq = 0.;
#pragma unroll
    for (int ii = 0; ii < 3; ii++) {
      const double q = (double)qd[ii] * xk[ii][l];
      uq += (double)evp[ii] * q;
      vq += (double)evp[3 + ii] * q;
    }
    const double h = d.hen[o + l];
    const float u = (float)((double)d.un[o + l] - adt * uq * h);
    const float v = (float)((double)d.vn[o + l] - adt * vq * h);
    d.un[o + l] = u;
    d.vn[o + l] = v;
    d.usv[o + l] = (float)(az * u + (1. - az) * (double)d.uo[o + l]);
    d.vsv[o + l] = (float)(az * v + (1. - az) * (double)d.vo[o + l]);
  }
  // setzev and the element part of make_new_depth (z, sigma or hybrid layers)
  double zv[3];
#pragma unroll
  for (int ii = 0; ii < 3; ii++) { zv[ii] = d.zn[kn[ii]]; d.zen[3 * e + ii] = (float)zv[ii]; }
  const double zmed = (zv[0] + zv[1] + zv[2]) / 3.;
  const float4 hm = d.hm3v[e];
  const float *hld = d.hldv + (size_t)en.w * NLV;
  const float *hlv = d.hlv + (size_t)en.w * NLV;
  bool bad = false;
  for (int l = 0; l < NLV; l++) {
    double h = 0.;
    if (l < ilevel) {
      if (l < P.nsigma) h = -(fmin((double)hm.w, (double)P.hsigma) + zmed) * (double)hld[l];
      else if (ilevel == 1) h = hm.w + zmed;
      else if (l < ilevel - 1) h = (double)hld[l] + (l == 0 ? zmed : 0.);
      else h = (double)hm.w - hlv[ilevel - 2];
      if (!(h > 0.)) bad = true;
    }
    d.hen[o + l] = (float)h;
  }
  if (bad) set_status(&d.out[en.w], SHY_EDEPTH);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int nh_solve_threads() { return 512; }

int nh_solve_capacity() {
  int dev = 0, nsm = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_nh_solve, nh_solve_threads(), 0) != cudaSuccess)
    return 0;
  return nsm * std::min(per, 2);
}

cudaError_t launch_nh_solve(const CsrGrid &a, int G, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(a.ctr, 0, 4 * sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  CsrGrid aa = a;
  void *args[] = {&aa};
  return cudaLaunchCooperativeKernel((const void *)k_nh_solve, dim3(G), dim3(nh_solve_threads()), args, 0, st);
}

void launch_nh(const Dev &d, const NhSys &s, int which, cudaStream_t st) {
  switch (which) {
    case 0: k_nh_w<<<(d.NKN + 127) / 128, 128, 0, st>>>(d, s); break;
    case 1: k_nh_sys<<<(s.nrow + 127) / 128, 128, 0, st>>>(d, s); break;
    case 2: k_nh_node<<<(d.NKN + 255) / 256, 256, 0, st>>>(d, s); break;
    default: k_nh_elem<<<(d.NEL + 255) / 256, 256, 0, st>>>(d, s); break;
  }
}

}  // namespace shy
