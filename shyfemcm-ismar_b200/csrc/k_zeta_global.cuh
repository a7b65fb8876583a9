// k_zeta_global.cuh -- zeta assembly + solve with the Krylov vectors in
// global memory (any basin size; CG, or BiCGStab for non-symmetric systems
// such as those with Coriolis).  Shares cluster_sum and assemble_row with
// k_zeta.cuh.  Included by step_zeta.cu after k_zeta.cuh.
#pragma once
#include "k_zeta.cuh"

namespace shy {

// ---------------------------------------------------------------------------
// global-memory variant
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_zeta(Dev d, ZetaArgs za, int CL) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int b = za.blist[blockIdx.x / CL];
  const BasinPar &P = d.par[b];
  BasinOut &O = d.out[b];
  __shared__ double wbuf[4 * 32];
  __shared__ double slots[2 * 4];
  __shared__ double bcast[4];
  int par = 0;
  const int chunk = (P.nk + CL - 1) / CL;
  const int r0 = P.k0 + rank * chunk;
  const int r1 = min(P.k0 + P.nk, r0 + chunk);
  const int echunk = (P.ne + CL - 1) / CL;        // this CTA's elements (wetting and drying)
  const int ea = P.e0 + min(P.ne, rank * echunk), eb = min(P.e0 + P.ne, ea + echunk);
  const int tid = threadIdx.x, nth = blockDim.x;
  if (rank == 0 && tid < kMaxScal) O.stab[tid] = 0.f;   // reset for k_stab's max
  if (blockIdx.x == 0 && tid == 0 && d.imax) { *d.imax = 0; *d.subj = 0; }
  const float dtf = (float)P.dt;
  // wetting and drying: the loop over a changing domain (hydrodynamic.f90:374-404)
  const bool wd = wd_basin(P) && !za.explicit_mode;

  double tol = 0., rn = 0., resid0 = 0.;
  int iters = 0, outer = 0, refine = 0;
  bool conv = false;
  for (int rep = 0;; rep++) {
    if (wd) {
      bool ok = true;
      for (int i = r0 + tid; i < r1; i += nth) ok &= wd_setnod(d, i);
      if (!ok) set_status(&O, SHY_EDEPTH);           // the open boundary dried (setnod :245)
      cl.sync();
      for (int e = ea + tid; e < eb; e += nth)
        if (__ldcg(&d.iweg[e]) != 0) wd_dry_system(d, e);
      cl.sync();
    }
    for (int i = r0 + tid; i < r1; i += nth) {
      double diag, rhs;
      assemble_row(d, za, i, dtf, diag, rhs, wd);
      d.dinv32[i] = diag != 0. ? (float)(1. / diag) : 1.f;
      // the guess: the old level, then (repeats) the last solution
      if (rep == 0) d.x64[i] = za.explicit_mode ? (diag != 0. ? rhs / diag : 0.) : (double)za.zguess[i];
    }
    if (za.explicit_mode) {
      for (int i = r0 + tid; i < r1; i += nth) d.zn[i] = (float)d.x64[i];
      if (rank == 0 && tid == 0) { O.iters = 0; O.refinements = 0; O.resid0 = 0.; O.resid = 0.; }
      return;
    }
    cl.sync();

    conv = false;
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
        if (rep == 0) resid0 = rn;
      }
      if (rn <= tol) { conv = true; break; }
      const double itol = fmax((double)za.inner_rtol * rn, tfrac(za) * tol);
      if (za.sym) {
        // Chronopoulos-Gear CG with vectors in global memory
        for (int i = r0 + tid; i < r1; i += nth) {
          d.z32[i] = d.dinv32[i] * d.r32[i];
          d.e32[i] = 0.f; d.p32[i] = 0.f; d.s32[i] = 0.f;
        }
        cl.sync();
        double g2[2] = {0., 0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          float w = 0.f;
          for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) w += d.val32[s] * __ldcg(&d.z32[d.col[s]]);
          d.t32[i] = w;
          g2[0] += (double)d.r32[i] * d.z32[i];
          g2[1] += (double)w * d.z32[i];
        }
        cluster_sum<2>(cl, g2, wbuf, slots, bcast, par, CL);
        double gamma = g2[0], alpha = gamma / g2[1], beta = 0.;
        for (int it = 0; it < P.maxit; it++) {
          const float fa = (float)alpha, fb = (float)beta;
          for (int i = r0 + tid; i < r1; i += nth) {
            const float p = d.z32[i] + fb * d.p32[i];
            const float s = d.t32[i] + fb * d.s32[i];
            d.p32[i] = p; d.s32[i] = s;
            d.e32[i] += fa * p;
            const float r = d.r32[i] - fa * s;
            d.r32[i] = r;
            d.z32[i] = d.dinv32[i] * r;
          }
          cl.sync();
          double g3[3] = {0., 0., 0.};
          for (int i = r0 + tid; i < r1; i += nth) {
            float w = 0.f;
            for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) w += d.val32[s] * __ldcg(&d.z32[d.col[s]]);
            d.t32[i] = w;
            const float r = d.r32[i], u = d.z32[i];
            g3[0] += (double)r * u;
            g3[1] += (double)w * u;
            g3[2] += (double)r * r;
          }
          cluster_sum<3>(cl, g3, wbuf, slots, bcast, par, CL);
          iters++;
          if (sqrt(g3[2]) <= itol || !(g3[0] == g3[0])) break;
          beta = g3[0] / gamma;
          alpha = g3[0] / (g3[1] - beta * g3[0] / alpha);
          gamma = g3[0];
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
    refine += outer;
    for (int i = r0 + tid; i < r1; i += nth) d.zn[i] = (float)d.x64[i];
    if (!wd) break;
    cl.sync();                                       // the new levels of every row
    // setweg(1): elements with a vertex below hzmin leave; then the step
    // counters, every element on the first pass of the step (a new time)
    double chg[1] = {0.};
    for (int e = ea + tid; e < eb; e += nth) chg[0] += wd_take_away(d, P, e) ? 1. : 0.;
    cluster_sum<1>(cl, chg, wbuf, slots, bcast, par, CL);
    for (int e = ea + tid; e < eb; e += nth) d.iwet[e] = wd_count(d.iweg[e], d.iwet[e], rep == 0);
    if (chg[0] == 0.) break;
    if (rep + 1 >= kWetDryRepeats) { if (rank == 0 && tid == 0) set_status(&O, SHY_ENOCONV); break; }
    cl.sync();
  }
  if (rank == 0 && tid == 0) {
    O.iters = iters;
    O.refinements = refine;
    O.resid0 = resid0;
    O.resid = rn;
    if (!conv) set_status(&O, SHY_ENOCONV);
  }
  // no CTA leaves while a peer may still read its shared memory (the last
  // cluster_sum reads every rank's partial after its barrier)
  cl.sync();
}

}  // namespace shy
