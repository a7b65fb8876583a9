// k_zeta_grid.cuh -- zeta assembly + solve for basins larger than one
// thread-block cluster can hold: one persistent cooperative launch over the
// whole device for every basin of the model.
//
// Each basin's rows are cut into tiles of 1024 rows, dealt to the CTAs so
// that each has about the same rows and a basin's tiles spread over many
// CTAs, so the work of the few basins still iterating late in a solve is
// shared out.
// The solver is the one of k_zeta_sm (system_solve,
// sparskit_admin.f90:115-334, with the reference's stop test
// ||r|| <= rtol*||r0|| + atol, spk_iters.f90:3304-3360): FP64 residual
// refinement around Jacobi-preconditioned Chronopoulos-Gear CG in FP32, the
// extrapolated start 2 z^n - z^(n-1).  The FP32 iterations run on the
// symmetrically scaled system S A S (S = D^-1/2), which is Jacobi-
// preconditioned CG in another basis: its diagonal is one, so a row stores
// only its off-diagonal entries, in a fixed-width block of eight (16-bit
// column offsets where every offset fits, a CSR tail for rows with more)
// that a thread reads with three independent vector loads, and no
// preconditioner; a row's record is {r, w, s, p} with the correction e
// beside it: 88 bytes per row and iteration instead of 108, and one level
// of dependent loads (row pointers) fewer.  Every basin runs its own state
// machine; all basins advance in lock step through "super-steps" separated
// by one grid barrier.  One CG iteration is one super-step: a row needs its
// neighbours' new residual r_j - a (w_j + b s_j) for the product, and
// computes it from their values of the previous iteration (kept in a
// second generation of the vectors) with the iteration scalars a, b that
// every row of the basin shares, so no barrier separates the vector update
// from the matrix-vector product.  In a super-step each
// tile does the work of its basin's stage and writes its partial sums; after
// the barrier every CTA that holds a tile of the basin sums that basin's
// partials in tile order (the same bits in every CTA, and the same alone or
// in any batch) and takes the same stage decision.  A basin that has
// finished idles until every basin has.
//
// The grid barrier is an arrival counter with a bounded wait: a CTA that
// waits longer than the plan's poll limit (kGridSpinLimit by default) marks every basin of the launch
// with SHY_ECUDA and leaves, and so do the others when they see the abort
// flag.  The launch is cooperative, so all CTAs are resident together.
// Vectors written by other CTAs are read with ordinary (L1-cached) loads:
// no CTA reads, in a super-step, what another writes in the same one, and
// the barrier's acquire makes the previous super-step's writes visible.
// Included by step_zeta.cu.
#pragma once
#include "k_zeta.cuh"

namespace shy {

constexpr int kGridMaxSlots = 32;                // basins per CTA
constexpr int kGridMaxTiles = 32;                // tiles per CTA
constexpr int kGridTileRows = 1024;              // rows per tile
constexpr long long kMbarSpinLimit = 1LL << 22;  // try_wait polls before a staged copy counts as lost
constexpr long long kGridSpinLimit = 1LL << 24;  // default poll limit: ~ seconds with the back-off below
constexpr int kGridPartialUnroll = 8;           // partial sums a lane loads at once

enum GridStage : int { G_RES = 0, G_XTRP, G_SPMV0, G_ITER, G_FIX, G_FINISH, G_DONE };

// per-basin solver state, one copy in each CTA holding a segment of it
struct GridState {
  int stage, first, conv, outer, inner, iters, basin, owner, cur;
  double tol, itol2, rn, resid0, alpha, beta, gamma;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// bar-th grid barrier (bar = 1, 2, ...).  Arrivals count up in ctr[0]; the
// CTA that completes a barrier reads the active-basin count ctr[act_idx]
// (when act_idx != 0) and publishes 2*bar + (count == 0) in ctr[5] with a
// release store, which the others poll with acquire loads (read-only
// polling keeps the counter's atomics uncontended, and nobody reads the
// count after the barrier).  The CTA barriers on both sides extend the
// release and the acquire to every thread of the CTA.  Returns false on
// timeout/abort (ctr[4]).  *s_act receives 0 when no basin is active.
__device__ __forceinline__ bool grid_barrier(const GridPlan &gp, unsigned bar, int *s_ok, unsigned act_idx,
                                             unsigned *s_act) {
  unsigned *ctr = gp.ctr;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned old, flag = 0u;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(ctr) : "memory");
    if (old + 1u == bar * (gridDim.x + gp.phantom)) {
      const unsigned none = act_idx != 0u && ld_acquire_u32(ctr + act_idx) == 0u ? 1u : 0u;
      flag = 2u * bar + none;
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(ctr + 5), "r"(flag) : "memory");
    } else {
      long long spins = 0;
      while (((flag = ld_acquire_u32(ctr + 5)) >> 1) < bar) {
        if (ld_acquire_u32(ctr + 4) != 0u || ++spins > gp.spin_limit) {
          atomicExch(ctr + 4, 1u);
          ok = 0;
          break;
        }
        if (spins > 256) __nanosleep(32);
      }
    }
    if (s_act) *s_act = (flag & 1u) ? 0u : 1u;
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// the new residual of a row from its record of the previous iteration q =
// {r, w, s, p}: s' = w + b s, r' = r - a s'.  Rows and their neighbours
// evaluate the same expression, so the same bits.
__device__ __forceinline__ float cg_rnext(const float4 q, float fa, float fb, float &s_new) {
  s_new = q.y + fb * q.z;
  return q.x - fa * s_new;
}

// columns of the eight entries of row i's block (padding: i)
template <bool C16>
__device__ __forceinline__ void ell_cols(const GridPlan &gp, int i, int (&c)[8]) {
  if constexpr (C16) {
    const int4 p = __ldg(reinterpret_cast<const int4 *>(gp.ecol16) + i);   // eight 16-bit offsets
    const int w[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      c[2 * k] = i + (int)(short)(w[k] & 0xffff);
      c[2 * k + 1] = i + (w[k] >> 16);            // arithmetic shift: the signed high half
    }
  } else {
    const int4 p0 = __ldg(reinterpret_cast<const int4 *>(gp.ecol32) + 2 * i);
    const int4 p1 = __ldg(reinterpret_cast<const int4 *>(gp.ecol32) + 2 * i + 1);
    c[0] = p0.x; c[1] = p0.y; c[2] = p0.z; c[3] = p0.w;
    c[4] = p1.x; c[5] = p1.y; c[6] = p1.z; c[7] = p1.w;
  }
}

// one row of (S A S) r' in FP32: the unit diagonal times the row's own new
// residual, then the entries in slot order (the block, then the tail) with
// r' of each entry's row from the previous generation (fa = fb = 0: r' =
// r).  The block's columns and values come in three vector loads and its
// eight neighbour records are all requested before the products; padding
// entries point at the row itself with value 0.
template <bool C16>
__device__ __forceinline__ float grid_spmv_row(const GridPlan &gp, int i, const float4 *qg, float fa, float fb,
                                               float own) {
  int c[8];
  ell_cols<C16>(gp, i, c);
  const float4 va = reinterpret_cast<const float4 *>(gp.eval)[2 * i];
  const float4 vb = reinterpret_cast<const float4 *>(gp.eval)[2 * i + 1];
  float4 x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = qg[c[k]];
  const float v[8] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
  float w = own, sn;
#pragma unroll
  for (int k = 0; k < 8; k++) w += v[k] * cg_rnext(x[k], fa, fb, sn);
  if (gp.nx)
    for (int k = gp.xptr[i]; k < gp.xptr[i + 1]; k++) w += gp.xval[k] * cg_rnext(qg[gp.xcol[k]], fa, fb, sn);
  return w;
}

// the first residual pass of a solve: the scaled FP32 entries of row i,
// a_ij s_i s_j (0 on padding)
template <bool C16>
__device__ __forceinline__ void grid_scale_row(const Dev &d, const GridPlan &gp, int i) {
  int c[8];
  ell_cols<C16>(gp, i, c);
  const double sdi = (double)gp.sd[i];
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int slot = __ldg(&gp.eslot[8 * i + k]);
    v[k] = slot >= 0 ? (float)(d.val64[slot] * sdi * (double)gp.sd[c[k]]) : 0.f;
  }
  reinterpret_cast<float4 *>(gp.eval)[2 * i] = make_float4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<float4 *>(gp.eval)[2 * i + 1] = make_float4(v[4], v[5], v[6], v[7]);
  if (gp.nx)
    for (int k = gp.xptr[i]; k < gp.xptr[i + 1]; k++)
      gp.xval[k] = (float)(d.val64[gp.xslot[k]] * sdi * (double)gp.sd[gp.xcol[k]]);
}

// FP64 residual of one row: rhs - A*x
__device__ __forceinline__ double grid_resid_row(const Dev &d, int i) {
  const int s0 = d.rowptr[i], s1 = d.rowptr[i + 1];
  double t = d.rhs64[i];
  for (int s = s0; s < s1; s += 8) {
    int c[8];
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const bool ok = s + k < s1;
      c[k] = ok ? d.col[s + k] : i;
      v[k] = ok ? d.val64[s + k] : 0.;
    }
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = d.x64[c[k]];
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (s + k < s1) t -= v[k] * x[k];
  }
  return t;
}

// ---------------------------------------------------------------------------
// TMA staging of a tile (the staged form): one bulk copy each of the tile's
// row pointers, its CSR column indices and FP32 values, its {r, w, s, 1/diag}
// rows and its {p, e} rows into a shared-memory buffer, completing on that
// buffer's mbarrier.  Every copy starts 16-byte aligned (ranges rounded out
// to 16 bytes; the arrays carry the slack) and moves a multiple of 16 bytes.
// ---------------------------------------------------------------------------
struct StageLayout {   // byte offsets inside one buffer
  int col, val, q4, ev, bytes;
};

// cb: bytes of one row's column block (16 for 16-bit offsets, 32 absolute)
__host__ __device__ inline StageLayout stage_layout(int cb) {
  StageLayout L;
  L.col = 0;
  L.val = L.col + kGridTileRows * cb;
  L.q4 = L.val + kGridTileRows * 32;
  L.ev = L.q4 + kGridTileRows * 16;
  L.bytes = (L.ev + (kGridTileRows + 8) * 4 + 127) & ~127;
  return L;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, int bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

// thread 0: copy the blocks of tile rows [a,e) into the buffer at sbuf:
// the column and value blocks and the {r, w, s, p} records are whole
// 16-byte units per row, the corrections are widened to 16-byte boundaries
// (the array carries the slack), so each copy starts aligned and moves
// whole 16 bytes.  Tail entries are read from global memory.
template <bool C16>
__device__ __forceinline__ void stage_issue(const GridPlan &gp, const StageLayout &L, uint32_t sbuf, uint32_t mbar,
                                            int a, int e, const float4 *qg) {
  constexpr int CB = C16 ? 16 : 32;
  const int ea = a & ~3, ec = ((e - ea) + 3) & ~3;
  const int bytes = (e - a) * (CB + 32 + 16) + ec * 4;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  if constexpr (C16) bulk_g2s(sbuf + L.col, gp.ecol16 + (size_t)8 * a, (e - a) * CB, mbar);
  else bulk_g2s(sbuf + L.col, gp.ecol32 + (size_t)8 * a, (e - a) * CB, mbar);
  bulk_g2s(sbuf + L.val, gp.eval + (size_t)8 * a, (e - a) * 32, mbar);
  bulk_g2s(sbuf + L.q4, qg + a, (e - a) * 16, mbar);
  bulk_g2s(sbuf + L.ev, gp.ecor + ea, ec * 4, mbar);
}

// bounded wait for an mbarrier phase; false when it did not complete
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < kMbarSpinLimit; it++) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// (S A S) r' for one row from a staged tile: the row's block, and r' of
// rows inside the tile, from shared memory; r' of rows outside it and the
// tail entries from global memory
template <bool C16>
__device__ __forceinline__ float staged_spmv_row(const GridPlan &gp, const unsigned char *buf, const StageLayout &L,
                                                 int i, int j, int a, int R, const float4 *sq, const float4 *qg,
                                                 float fa, float fb, float own) {
  int c[8];
  if constexpr (C16) {
    const short *sc = reinterpret_cast<const short *>(buf + L.col) + 8 * j;
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = i + (int)sc[k];
  } else {
    const int *sc = reinterpret_cast<const int *>(buf + L.col) + 8 * j;
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = sc[k];
  }
  const float *sv = reinterpret_cast<const float *>(buf + L.val) + 8 * j;
  float w = own, sn;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const float4 x = (unsigned)(c[k] - a) < (unsigned)R ? sq[c[k] - a] : qg[c[k]];
    w += sv[k] * cg_rnext(x, fa, fb, sn);
  }
  if (gp.nx)
    for (int k = gp.xptr[i]; k < gp.xptr[i + 1]; k++) w += gp.xval[k] * cg_rnext(qg[gp.xcol[k]], fa, fb, sn);
  return w;
}

// the stage decision of one basin after the sums tot of its partials (the
// same inputs, so the same decision, in every CTA holding a tile of it)
__device__ __forceinline__ void grid_transition(GridState &g, const double (&tot)[3], const Dev &d,
                                                const ZetaArgs &za) {
  const int st = g.stage;
  const BasinPar &P = d.par[g.basin];
  if (st == G_RES) {
    const double rn = sqrt(tot[0]);
    bool next = true;
    if (g.first) {
      g.first = 0;
      g.tol = (double)P.rtol * rn + (double)P.atol;
      g.resid0 = rn;
      if (za.zprev != nullptr && d.out[g.basin].steps > 0 && rn > g.tol) { g.stage = G_XTRP; next = false; }
    }
    if (next) {
      g.rn = rn;
      if (rn <= g.tol) { g.conv = 1; g.stage = G_FINISH; }
      else if (g.outer >= za.max_outer) g.stage = G_FINISH;
      else {
        // the FP32 sweep's target, moved into the norm of the scaled residual
        // (tot[1] = ||S r||^2) by the ratio of the two norms at its start
        const double it = fmax((double)za.inner_rtol * rn, tfrac(za) * g.tol);
        g.itol2 = tot[0] > 0. ? it * it * (tot[1] / tot[0]) : 0.;
        g.stage = G_SPMV0;
      }
    }
  } else if (st == G_SPMV0) {
    g.cur ^= 1;
    g.gamma = tot[0];
    g.alpha = g.gamma / tot[1];
    g.beta = 0.;
    g.inner = 0;
    g.stage = G_ITER;
  } else {   // G_ITER
    g.cur ^= 1;
    g.iters++;
    g.inner++;
    const bool stop = !(tot[2] > g.itol2) || !(tot[0] == tot[0]) || g.inner >= P.maxit;
    if (stop) g.stage = G_FIX;
    else {
      const double beta = tot[0] / g.gamma;
      g.alpha = tot[0] / (tot[1] - beta * tot[0] / g.alpha);
      g.beta = beta;
      g.gamma = tot[0];
    }
  }
}

// NT threads per CTA.  STAGED: the CG products read each tile's data from
// TMA-staged shared memory (two buffers, the next tile's copy in flight
// while one is worked; one CTA of 1024 threads per SM); otherwise straight
// from global memory (two CTAs of 512 threads per SM).
template <int NT, bool STAGED, bool C16>
__global__ void __launch_bounds__(NT, STAGED ? 1 : 2) k_zeta_grid(Dev d, ZetaArgs za, GridPlan gp) {
  constexpr int NW = NT / 32;
  __shared__ GridState gs[kGridMaxSlots];
  __shared__ int4 s_tile[kGridMaxTiles];
  __shared__ int s_tid[kGridMaxTiles];
  __shared__ double wred[kGridMaxTiles * NW * 3];
  __shared__ int s_ok;
  __shared__ unsigned s_act;
  extern __shared__ __align__(128) unsigned char dsm[];
  const int tid = threadIdx.x, nth = blockDim.x;
  const int c = blockIdx.x;
  const int nslot = gp.cnslot[c];
  const int t0 = gp.cptr[c], ntl = gp.cptr[c + 1] - t0;   // this CTA's tiles: clist[t0 ..]
  unsigned bar = 0;
  const StageLayout SL = stage_layout(C16 ? 16 : 32);
  uint32_t mbar[2] = {0u, 0u}, sbuf[2] = {0u, 0u}, phase[2] = {0u, 0u};
  if (STAGED) {
    mbar[0] = smem_u32(dsm); mbar[1] = mbar[0] + 8;
    sbuf[0] = smem_u32(dsm + 128); sbuf[1] = sbuf[0] + SL.bytes;
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar[0]) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar[1]) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }

  __shared__ int2 s_bt[kGridMaxSlots];
  if (tid < nslot) {
    GridState &g = gs[tid];
    g.stage = G_RES; g.first = 1; g.conv = 0; g.outer = 0; g.inner = 0; g.iters = 0; g.cur = 0;
    g.basin = gp.cslot[c * kGridMaxSlots + tid];
    g.owner = (gp.cowner[c] >> tid) & 1;
    s_bt[tid] = gp.btile[g.basin];
    g.tol = g.itol2 = g.rn = g.resid0 = g.alpha = g.beta = g.gamma = 0.;
  }
  if (tid < ntl) {
    const int t = gp.clist[t0 + tid];
    s_tid[tid] = t;
    s_tile[tid] = gp.tile[t];
  }
  if (blockIdx.x == 0 && tid == 0 && d.imax) { *d.imax = 0; *d.subj = 0; }
  __syncthreads();

  // ---- assembly (FP64 gather in element order), Jacobi diagonal, start ----
  for (int q = 0; q < ntl; q++) {
    const int4 tl = s_tile[q];
    const BasinPar &P = d.par[tl.z];
    if (tl.x == P.k0 && tid < kMaxScal) d.out[tl.z].stab[tid] = 0.f;   // reset for k_stab's max
    const float dtf = (float)P.dt;
    for (int i = tl.x + tid; i < tl.y; i += nth) {
      double diag, rhs;
      assemble_row(d, za, i, dtf, diag, rhs, false, false);   // no FP32 copy of the full rows
      gp.sd[i] = diag > 0. ? (float)(1. / sqrt(diag)) : 1.f;
      const double x0 = za.explicit_mode ? (diag != 0. ? rhs / diag : 0.) : (double)za.zguess[i];
      d.x64[i] = x0;
      if (za.explicit_mode) d.zn[i] = (float)x0;
    }
  }
  if (za.explicit_mode) {   // system_set_explicit: no coupling between rows, no barrier
    if (tid < nslot && gs[tid].owner) {
      BasinOut &O = d.out[gs[tid].basin];
      O.iters = 0; O.refinements = 0; O.resid0 = 0.; O.resid = 0.;
    }
    return;
  }
  if (STAGED) asm volatile("fence.proxy.async.global;" ::: "memory");
  if (!grid_barrier(gp, ++bar, &s_ok, 0, nullptr)) goto aborted;

  for (unsigned k = 0;; k++) {
    const int par = (int)(k & 1u);
    // ---- the work of each tile's stage ----
    int iq = 0;                                     // thread 0: next tile to stage
    auto staged_stage = [&](int st) { return STAGED && (st == G_SPMV0 || st == G_ITER); };
    auto issue_next = [&](int b) {                  // thread 0 only
      while (iq < ntl && !staged_stage(gs[s_tile[iq].w].stage)) iq++;
      if (iq < ntl) {
        const int4 tl = s_tile[iq];
        stage_issue<C16>(gp, SL, sbuf[b], mbar[b], tl.x, tl.y, d.cg4[gs[tl.w].cur]);
        iq++;
      }
    };
    if (STAGED && tid == 0) {
      asm volatile("fence.proxy.async.global;" ::: "memory");
      issue_next(0);
      issue_next(1);
    }
    int js = 0;                                     // staged tiles worked so far
    for (int q = 0; q < ntl; q++) {
      const int4 tl = s_tile[q];
      const int a = tl.x, e = tl.y;
      GridState &g = gs[tl.w];
      const int stage = g.stage;
      double v[3] = {0., 0., 0.};
      if (staged_stage(stage)) {
        const int b = js & 1;
        if (tid == 0) s_ok = mbar_wait(mbar[b], phase[b]) ? 1 : 0;
        __syncthreads();
        if (!s_ok) {
          if (tid == 0) {
            atomicExch(gp.ctr + 4, 1u);
            mbar_wait(mbar[b], phase[b]);           // let the copies in flight land
            mbar_wait(mbar[b ^ 1], phase[b ^ 1]);
          }
          __syncthreads();
          goto aborted;
        }
        phase[b] ^= 1u;
        const unsigned char *buf = dsm + 128 + (size_t)b * SL.bytes;
        const float4 *sq = reinterpret_cast<const float4 *>(buf + SL.q4);
        const float *sev = reinterpret_cast<const float *>(buf + SL.ev) + (a - (a & ~3));
        const float4 *qi = d.cg4[g.cur];
        float4 *qo = d.cg4[g.cur ^ 1];
        const int R = e - a;
        const float fa = stage == G_ITER ? (float)g.alpha : 0.f;
        const float fb = stage == G_ITER ? (float)g.beta : 0.f;
        for (int j = tid; j < R; j += nth) {
          const int i = a + j;
          const float4 me = sq[j];
          if (stage == G_SPMV0) {
            // w = (S A S) r (fa = fb = 0 leave r)
            const float w = staged_spmv_row<C16>(gp, buf, SL, i, j, a, R, sq, qi, 0.f, 0.f, me.x);
            qo[i] = make_float4(me.x, w, 0.f, 0.f);
            v[0] += (double)me.x * me.x;
            v[1] += (double)w * me.x;
          } else {
            // p = r + b p, s = w + b s, e += a p, r -= a s, w = (S A S) r
            const float p = me.x + fb * me.w;
            float sn;
            const float rn = cg_rnext(me, fa, fb, sn);
            const float w = staged_spmv_row<C16>(gp, buf, SL, i, j, a, R, sq, qi, fa, fb, rn);
            qo[i] = make_float4(rn, w, sn, p);
            gp.ecor[i] = sev[j] + fa * p;
            v[0] += (double)rn * rn;
            v[1] += (double)w * rn;
          }
          v[2] = v[0];
        }
        __syncthreads();                            // buffer b read by every thread
        if (tid == 0) issue_next(b);
        js++;
      } else if (stage == G_RES) {
        // the FP64 residual t (its norm is the stop test's), the scaled S t
        // the FP32 sweep starts from, a zero correction; the first pass of
        // a solve also writes the scaled off-diagonal entries of its rows
        float4 *qo = d.cg4[g.cur];
        const bool scale = g.first != 0;
        for (int i = a + tid; i < e; i += nth) {
          const double t = grid_resid_row(d, i);
          const double sdi = (double)gp.sd[i];
          if (scale) grid_scale_row<C16>(d, gp, i);
          const float rs = (float)(sdi * t);
          qo[i] = make_float4(rs, 0.f, 0.f, 0.f);
          gp.ecor[i] = 0.f;
          v[0] += t * t;
          v[1] += (double)rs * rs;
        }
      } else if (stage == G_XTRP) {
        // z_guess = 2 z^n - z^{n-1}: smooth in time, a smaller starting residual
        for (int i = a + tid; i < e; i += nth) d.x64[i] = 2. * (double)za.zguess[i] - (double)za.zprev[i];
      } else if (stage == G_SPMV0) {
        // w = (S A S) r (fa = fb = 0 leave r); p = s = 0
        const float4 *qi = d.cg4[g.cur];
        float4 *qo = d.cg4[g.cur ^ 1];
        for (int i = a + tid; i < e; i += nth) {
          const float4 me = qi[i];
          const float w = grid_spmv_row<C16>(gp, i, qi, 0.f, 0.f, me.x);
          qo[i] = make_float4(me.x, w, 0.f, 0.f);
          v[0] += (double)me.x * me.x;
          v[1] += (double)w * me.x;
        }
        v[2] = v[0];
      } else if (stage == G_ITER) {
        // p = r + b p, s = w + b s, e += a p, r -= a s, w = (S A S) r
        const float fa = (float)g.alpha, fb = (float)g.beta;
        const float4 *qi = d.cg4[g.cur];
        float4 *qo = d.cg4[g.cur ^ 1];
        for (int i = a + tid; i < e; i += nth) {
          const float4 me = qi[i];
          const float p = me.x + fb * me.w;
          float sn;
          const float rn = cg_rnext(me, fa, fb, sn);
          const float w = grid_spmv_row<C16>(gp, i, qi, fa, fb, rn);
          qo[i] = make_float4(rn, w, sn, p);
          gp.ecor[i] += fa * p;
          v[0] += (double)rn * rn;
          v[1] += (double)w * rn;
        }
        v[2] = v[0];
      } else if (stage == G_FIX) {
        for (int i = a + tid; i < e; i += nth) d.x64[i] += (double)gp.sd[i] * (double)gp.ecor[i];
      } else if (stage == G_FINISH) {
        for (int i = a + tid; i < e; i += nth) d.zn[i] = (float)d.x64[i];
      }
      if (stage == G_RES || stage == G_SPMV0 || stage == G_ITER) {
        // warp sums now, the sum over warps once all tiles are done (no CTA
        // barrier between tiles, so warps run ahead into the next tile)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v[cc] += __shfl_xor_sync(0xffffffffu, v[cc], o);
        }
        if ((tid & 31) == 0) {
          double *w = wred + ((size_t)q * NW + (tid >> 5)) * 3;
          w[0] = v[0]; w[1] = v[1]; w[2] = v[2];
        }
      }
    }
    __syncthreads();
    // tile partials: warp w sums the warp sums of tiles w, w+NW, ... in a fixed tree
    {
      const int warp = tid >> 5, lane = tid & 31;
      for (int q = warp; q < ntl; q += NW) {
        const int stage = gs[s_tile[q].w].stage;
        if (stage != G_RES && stage != G_SPMV0 && stage != G_ITER) continue;
        double x[3];
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
          x[cc] = lane < NW ? wred[((size_t)q * NW + lane) * 3 + cc] : 0.;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) x[cc] += __shfl_xor_sync(0xffffffffu, x[cc], o);
        }
        if (lane == 0) {
          double *pp = gp.partial + ((size_t)par * gp.ntile + s_tid[q]) * 4;
          __stcg(pp + 0, x[0]); __stcg(pp + 1, x[1]); __stcg(pp + 2, x[2]);
        }
      }
    }
    __syncthreads();
    // ---- finished basins leave the machine; count the active ones ----
    if (tid == 0) {
      unsigned nact = 0;
      for (int q = 0; q < nslot; q++) {
        GridState &g = gs[q];
        if (g.stage == G_FINISH) {
          if (g.owner) {
            BasinOut &O = d.out[g.basin];
            O.iters = g.iters;
            O.refinements = g.outer;
            O.resid0 = g.resid0;
            O.resid = g.rn;
            if (!g.conv) set_status(&O, SHY_ENOCONV);
          }
          g.stage = G_DONE;
        }
        if (g.owner && g.stage != G_DONE) nact++;
      }
      if (nact) atomicAdd(gp.ctr + 1 + k % 3, nact);
      if (blockIdx.x == 0) gp.ctr[1 + (k + 1) % 3] = 0u;   // the counter of super-step k+3
    }
    // the next super-step may read these writes through the async proxy
    if (STAGED) asm volatile("fence.proxy.async.global;" ::: "memory");
    if (!grid_barrier(gp, ++bar, &s_ok, 1 + k % 3, &s_act)) goto aborted;
    if (s_act == 0u) break;
    // ---- per-basin sums over its tiles, the same in every CTA; next stage ----
    for (int sl = tid >> 5; sl < nslot; sl += NW) {
      const int lane = tid & 31;
      {
        GridState &g = gs[sl];
        const int st = g.stage;
        if (st == G_RES || st == G_SPMV0 || st == G_ITER) {
          const int2 bt = s_bt[sl];
          double tot[3] = {0., 0., 0.};
          // up to 32*kGridPartialUnroll partials per round, all loads issued first
          for (int s0 = bt.x; s0 < bt.y; s0 += 32 * kGridPartialUnroll) {
            double pv[kGridPartialUnroll][3];
#pragma unroll
            for (int u = 0; u < kGridPartialUnroll; u++) {
              const int sx = s0 + u * 32 + lane;
              const double *pp = gp.partial + ((size_t)par * gp.ntile + (sx < bt.y ? sx : bt.x)) * 4;
              pv[u][0] = __ldcg(pp + 0); pv[u][1] = __ldcg(pp + 1); pv[u][2] = __ldcg(pp + 2);
            }
#pragma unroll
            for (int u = 0; u < kGridPartialUnroll; u++)
              if (s0 + u * 32 + lane < bt.y) { tot[0] += pv[u][0]; tot[1] += pv[u][1]; tot[2] += pv[u][2]; }
          }
#pragma unroll
          for (int cc = 0; cc < 3; cc++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) tot[cc] += __shfl_xor_sync(0xffffffffu, tot[cc], o);
          if (lane == 0) grid_transition(g, tot, d, za);
        } else if (lane == 0) {
          if (st == G_XTRP) g.stage = G_RES;
          else if (st == G_FIX) { g.outer++; g.stage = G_RES; }
        }
      }
    }
    __syncthreads();
  }
  return;

aborted:
  if (tid < nslot && gs[tid].owner) set_status(&d.out[gs[tid].basin], SHY_ECUDA);
}

}  // namespace shy
