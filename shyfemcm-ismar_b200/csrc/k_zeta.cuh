// k_zeta.cuh -- the zeta system of one basin per thread-block cluster:
// system_init + the element scatter of system_assemble + system_add_rhs
// (simsys_spkaux.f90:137-154, 533-594, 687-705) as an atomic-free gather in
// element order (FP64 sums, as the reference's c2coo), then system_solve
// (sparskit_admin.f90:115-334): Krylov iterations in FP32 inside FP64
// residual refinement, stopped on the reference's test
// ||r|| <= rtol*||r0|| + atol (stopbis, spk_iters.f90:3304-3360), with r0 the
// residual of the reference's guess (the old water level).  All iterations
// run inside one launch; the CTAs of a cluster meet only at cluster barriers.
//
// This file holds the shared helpers and the shared-memory variant
// k_zeta_sm: each CTA keeps its rows of the matrix (FP32, local column
// indices) and the Krylov vectors in shared memory.  Values of rows that a
// neighbouring CTA needs are pushed into that CTA's halo slots through
// distributed shared memory as soon as they are computed, so the
// matrix-vector product reads only local shared memory.  Chronopoulos-Gear
// CG: one fused reduction per iteration, the iteration scalars computed once
// per CTA.  The global-memory variant is in k_zeta_global.cuh.
// Included by step_zeta.cu.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "launch.h"
#include "physics.cuh"

namespace cg = cooperative_groups;

namespace shy {

// Sum of NV values over all threads of a cluster.  Fixed reduction order
// (warp shuffles, then warps, then cluster ranks in a shuffle tree), so every
// CTA obtains the same bits.  Uses one cluster barrier.
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
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double x = lane < CL ? *cl.map_shared_rank(&slots[par * 4 + i], lane) : 0.;
#pragma unroll
      for (int dd = 16; dd > 0; dd >>= 1) x += __shfl_xor_sync(0xffffffffu, x, dd);
      if (lane == 0) bc[i] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = bc[i];
  par ^= 1;
}

// Cluster sum of NV FP32 per-thread partials; the totals (FP64) land in
// warp 0 only (every lane of warp 0 holds them).  The caller's warp 0 turns
// them into what all threads need and publishes it after its own barrier.
template <int NV>
__device__ __forceinline__ void cluster_sum_w0(cg::cluster_group &cl, const float (&v)[NV], double *wbuf,
                                               double *slots, double (&tot)[NV], int &par, int CL) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    float x = v[i];
#pragma unroll
    for (int dd = 16; dd > 0; dd >>= 1) x += __shfl_xor_sync(0xffffffffu, x, dd);
    if (lane == 0) wbuf[i * 32 + warp] = (double)x;
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
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double x = lane < CL ? *cl.map_shared_rank(&slots[par * 4 + i], lane) : 0.;
#pragma unroll
      for (int dd = 16; dd > 0; dd >>= 1) x += __shfl_xor_sync(0xffffffffu, x, dd);
      tot[i] = x;
    }
  }
  par ^= 1;
}

// the fraction of the outer target the FP32 inner solve goes down to
__device__ __forceinline__ double tfrac(const ZetaArgs &za) {
  return za.tol_frac > 0.f ? (double)za.tol_frac : 0.25;
}

// one row of the assembly: FP64 gather of the element entries of every slot
// (element order), the rhs, the diagonal
__device__ __forceinline__ void assemble_row(const Dev &d, const ZetaArgs &za, int i, float dtf,
                                             double &diag, double &rhs, bool wd = false, bool w32 = true) {
  diag = 0.;
  for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) {
    double v = 0.;
    for (int t = d.slot_ptr[s]; t < d.slot_ptr[s + 1]; t++) {
      const int src = d.slot_src[t];
      const int e = src / 9, c = src - 9 * e;
      const float *ph = &za.hia[(size_t)c * za.cs + (size_t)e * za.es];
      v += (double)(wd ? __ldcg(ph) : *ph);      // dry systems are written in this launch
    }
    d.val64[s] = v;
    if (w32) d.val32[s] = (float)v;            // the FP32 copy the cluster solvers iterate on
    if (d.col[s] == i) diag = v;
  }
  rhs = 0.;
  for (int p = d.inc_ptr[i]; p < d.inc_ptr[i + 1]; p++) {
    const int q = d.inc[p];
    const int e = q / 3, ii = q - 3 * e;
    const float *pk = &za.hik[(size_t)ii * za.cs + (size_t)e * za.es];
    rhs += (double)(wd ? __ldcg(pk) : *pk);
  }
  // adjust_mass_flux (bnd_routines.f90:1185-1210): with wetting and drying
  // (wd) no flux enters a node out of the system
  if (!(wd && d.inod[i] == -2)) rhs += (double)(dtf * d.rqv[i]);
  d.rhs64[i] = rhs;
}

// FP64 residual of the rows r0..r1 for the iterate in d.x64
__device__ __forceinline__ double residual_rows(const Dev &d, int r0, int r1, float *rout) {
  double acc = 0.;
  for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    double t = d.rhs64[i];
    for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) t -= d.val64[s] * __ldcg(&d.x64[d.col[s]]);
    rout[i - r0] = (float)t;
    acc += t * t;
  }
  return acc;
}

// ---------------------------------------------------------------------------
// shared-memory variant
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_zeta_sm(Dev d, ZetaArgs za, ZetaShape zs, ZetaMaps zm) {
  cg::cluster_group cl = cg::this_cluster();
  const int CL = zs.CL, chunk = zs.chunk;
  const int rank = (int)cl.block_rank();
  const int b = za.blist[blockIdx.x / CL];
  const BasinPar &P = d.par[b];
  BasinOut &O = d.out[b];
  extern __shared__ __align__(16) unsigned char smem[];
  int *srow = reinterpret_cast<int *>(smem);                       // chunk+1
  int *scol = srow + (chunk + 1);                                  // nnzcap (local indices)
  float *sval = reinterpret_cast<float *>(scol + zs.nnzcap);       // nnzcap
  float *su = sval + zs.nnzcap;                                    // chunk + halocap
  float *sr = su + chunk + zs.halocap, *sw = sr + chunk, *sp = sw + chunk;
  float *ss = sp + chunk, *se = ss + chunk, *sdv = se + chunk;
  __shared__ double wbuf[4 * 32];
  __shared__ double slots[2 * 4];
  __shared__ double bcast[4];
  int par = 0;
  const int tid = threadIdx.x, nth = blockDim.x, warp = tid >> 5, lane = tid & 31;
  const int cb = (P.nk + CL - 1) / CL;        // this basin's rows per CTA (<= chunk)
  const int r0 = P.k0 + min(P.nk, rank * cb);
  const int r1 = min(P.k0 + P.nk, r0 + cb);
  const int nloc = max(0, r1 - r0);
  if (rank == 0 && tid < kMaxScal) O.stab[tid] = 0.f;   // reset for k_stab's max
  if (blockIdx.x == 0 && tid == 0 && d.imax) { *d.imax = 0; *d.subj = 0; }
  const float dtf = (float)P.dt;
  const int base = nloc > 0 ? d.rowptr[r0] : 0;

  // ---- assembly into global FP64 (for the residual) and local FP32 rows ----
  for (int li = tid; li < nloc; li += nth) {
    const int i = r0 + li;
    double diag, rhs;
    assemble_row(d, za, i, dtf, diag, rhs);
    srow[li] = d.rowptr[i] - base;
    for (int s = d.rowptr[i]; s < d.rowptr[i + 1]; s++) {
      scol[s - base] = zm.loc[s];
      sval[s - base] = d.val32[s];
    }
    sdv[li] = diag != 0. ? (float)(1. / diag) : 1.f;
    d.x64[i] = za.explicit_mode ? (diag != 0. ? rhs / diag : 0.) : (double)za.zguess[i];
  }
  if (tid == 0) srow[nloc] = nloc > 0 ? d.rowptr[r1] - base : 0;
  if (za.explicit_mode) {
    for (int li = tid; li < nloc; li += nth) d.zn[r0 + li] = (float)d.x64[r0 + li];
    if (rank == 0 && tid == 0) { O.iters = 0; O.refinements = 0; O.resid0 = 0.; O.resid = 0.; }
    return;
  }
  cl.sync();

  // ---- stop target from the reference's guess, then a better start ----
  double acc[1] = {residual_rows(d, r0, r1, sr)};
  cluster_sum<1>(cl, acc, wbuf, slots, bcast, par, CL);
  double rn = sqrt(acc[0]);
  const double tol = (double)P.rtol * rn + (double)P.atol;
  if (rank == 0 && tid == 0) O.resid0 = rn;
  const bool extrap = za.zprev != nullptr && O.steps > 0 && rn > tol;
  if (extrap) {
    // z_guess = 2 z^n - z^{n-1}: smooth in time, a smaller starting residual
    for (int li = tid; li < nloc; li += nth) {
      const int i = r0 + li;
      d.x64[i] = 2. * (double)za.zguess[i] - (double)za.zprev[i];
    }
    cl.sync();
  }

  int iters = 0, outer = 0;
  bool conv = false;
  for (outer = 0; outer < za.max_outer; outer++) {
    if (outer > 0 || extrap) {
      acc[0] = residual_rows(d, r0, r1, sr);
      cluster_sum<1>(cl, acc, wbuf, slots, bcast, par, CL);
      rn = sqrt(acc[0]);
    }
    if (rn <= tol) { conv = true; break; }
    const double itol2 = fmax((double)za.inner_rtol * rn, tfrac(za) * tol) * fmax((double)za.inner_rtol * rn, tfrac(za) * tol);
    // Chronopoulos-Gear CG, Jacobi preconditioner (u = D^-1 r, w = A u)
    for (int li = tid; li < nloc; li += nth) {
      const float u = sdv[li] * sr[li];
      su[li] = u; se[li] = 0.f; sp[li] = 0.f; ss[li] = 0.f;
      for (int t = zm.push_ptr[r0 + li]; t < zm.push_ptr[r0 + li + 1]; t++) {
        const int pk = zm.push[t];
        *cl.map_shared_rank(&su[pk & 0xffffff], pk >> 24) = u;
      }
    }
    cl.sync();
    float g2[2] = {0.f, 0.f};
    for (int li = tid; li < nloc; li += nth) {
      float w = 0.f;
      for (int t = srow[li]; t < srow[li + 1]; t++) w += sval[t] * su[scol[t]];
      sw[li] = w;
      g2[0] += sr[li] * su[li];
      g2[1] += w * su[li];
    }
    double t2[2];
    cluster_sum_w0<2>(cl, g2, wbuf, slots, t2, par, CL);
    // warp 0 keeps the iteration scalars, all threads read them from bcast
    double gamma = 0., alpha = 0.;
    if (warp == 0) {
      gamma = t2[0];
      alpha = gamma / t2[1];
      if (lane == 0) { bcast[0] = alpha; bcast[1] = 0.; bcast[2] = 0.; }
    }
    __syncthreads();
    float fa = (float)bcast[0], fb = 0.f;
    for (int it = 0; it < P.maxit; it++) {
      for (int li = tid; li < nloc; li += nth) {
        const float p = su[li] + fb * sp[li];
        const float s = sw[li] + fb * ss[li];
        sp[li] = p; ss[li] = s;
        se[li] += fa * p;
        const float r = sr[li] - fa * s;
        sr[li] = r;
        const float u = sdv[li] * r;
        su[li] = u;
        for (int t = zm.push_ptr[r0 + li]; t < zm.push_ptr[r0 + li + 1]; t++) {
          const int pk = zm.push[t];
          *cl.map_shared_rank(&su[pk & 0xffffff], pk >> 24) = u;
        }
      }
      cl.sync();                                   // u and the pushed halo visible
      float g3[3] = {0.f, 0.f, 0.f};
      for (int li = tid; li < nloc; li += nth) {
        float w = 0.f;
        for (int t = srow[li]; t < srow[li + 1]; t++) w += sval[t] * su[scol[t]];
        sw[li] = w;
        const float r = sr[li], u = su[li];
        g3[0] += r * u;
        g3[1] += w * u;
        g3[2] += r * r;
      }
      double t3[3];
      cluster_sum_w0<3>(cl, g3, wbuf, slots, t3, par, CL);
      if (warp == 0) {
        const bool stop = !(t3[2] > itol2) || !(t3[0] == t3[0]);
        const double beta = t3[0] / gamma;
        alpha = t3[0] / (t3[1] - beta * t3[0] / alpha);
        gamma = t3[0];
        if (lane == 0) { bcast[0] = alpha; bcast[1] = beta; bcast[2] = stop ? 1. : 0.; }
      }
      __syncthreads();
      iters++;
      if (bcast[2] != 0.) break;
      fa = (float)bcast[0];
      fb = (float)bcast[1];
    }
    for (int li = tid; li < nloc; li += nth) d.x64[r0 + li] += (double)se[li];
    cl.sync();
  }
  for (int li = tid; li < nloc; li += nth) d.zn[r0 + li] = (float)d.x64[r0 + li];
  if (rank == 0 && tid == 0) {
    O.iters = iters;
    O.refinements = outer;
    O.resid = rn;
    if (!conv) set_status(&O, SHY_ENOCONV);
  }
  // no CTA leaves while a peer may still read its shared memory (the last
  // cluster_sum reads every rank's partial after its barrier)
  cl.sync();
}

}  // namespace shy
