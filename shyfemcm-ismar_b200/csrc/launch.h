// launch.h -- host-side launch interface of the kernels in step.cu.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace shy {

// arguments of the zeta assembly + solve kernel
struct ZetaArgs {
  const int *blist;     // basin of each cluster of the launch (cluster c solves blist[c])
  const float *zguess;  // initial guess (the old water level, system_solve's z)
  const float *zprev;   // the level one step earlier (for the extrapolated start), or null
  const float *hia;     // element matrices: hia[c*cs + e*es], c = 3*i + j
  const float *hik;     // element right-hand sides: hik[i*cs + e*es]
  int cs, es;
  int explicit_mode;    // system_set_explicit: diagonal (lumped) solve
  float inner_rtol;     // FP32 inner iterations reduce the residual by this factor
  float tol_frac;       // ... or reach this fraction of the outer target (0: 0.25)
  int max_outer;        // FP64 refinement sweeps
  int sym;              // 1: CG (symmetric system), 0: BiCGStab
};

// which: 0 k_column, 1 k_final
void launch_elem(const Dev &d, int which, int init_only, cudaStream_t st, bool cor);
// which: 0 k_node(init_only=a), 1 k_stab, 2 k_conz(j=a, nsub=b), 3 k_rhoset,
// 4 k_rho, 5 k_moment, 6 k_tvdgrad(j=a), 7 k_conz with conz3d_omp's source
// terms (j=a, one scalar)
void launch_node(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st);
void launch_reduce(const Dev &d, int nsub, int advance, cudaStream_t st);
// wetting and drying: 0 set_dry at the step's start, 1 the initial state's
// setweg(0) (and zenv from znv), 2 setznv; basin >= 0 limits 1 and 2 to it
void launch_wetdry(const Dev &d, const int *kbas, int which, int basin, cudaStream_t st);
void launch_subctl(const Dev &d, cudaGraphConditionalHandle h, cudaStream_t st);
// the 3D system of the non-hydrostatic pressure over the basins with
// inohyd = 1: one unknown per active node layer, row of node k and layer l
// (1-based) roff[k] + l - 1; CSR with the rows of a basin contiguous
struct NhSys {
  int nrow = 0;
  const int *kbas = nullptr;       // node -> basin
  const int *roff = nullptr;       // [NKN] first row of node k, -1 in hydrostatic basins
  const int *rnode = nullptr;      // [nrow] node of each row
  const int *rowptr = nullptr, *col = nullptr;
  double *val = nullptr, *rhs = nullptr;
  float *x = nullptr;              // the pressure per row (solver output)
  float *wnh = nullptr;            // [NKN*(NLV+1)] w of sp256wnh
};

// the device-wide CSR solver (k_nh_solve) over rows [r0, r1), whose columns
// lie in the same range; x holds the guess and receives the solution
struct CsrGrid {
  int r0 = 0, r1 = 0;
  const int *rowptr = nullptr, *col = nullptr;
  const double *val = nullptr, *rhs = nullptr;
  float *val32 = nullptr, *dinv = nullptr, *x = nullptr;
  double *x64 = nullptr;
  float *r = nullptr, *rh = nullptr, *p = nullptr, *v = nullptr, *s = nullptr, *t = nullptr, *z = nullptr,
        *q = nullptr, *e = nullptr;
  double *part = nullptr;          // [2][G][4] partial sums
  unsigned *ctr = nullptr;         // [4] barrier arrivals, release, abort
  BasinOut *out = nullptr;         // nh_* fields and status of the basin solved
  double rtol = 1e-8, atol = 1e-8;
  int maxit = 1000, max_outer = 12;
  float inner_rtol = 1e-4f;
  long long spin_limit = 1LL << 22;
};
// which: 0 k_nh_w (sp256wnh), 1 k_nh_sys (the 3D system), 2 k_nh_node, 3 k_nh_elem
void launch_nh(const Dev &d, const NhSys &s, int which, cudaStream_t st);
// G CTAs (cooperative; clears a.ctr first)
cudaError_t launch_nh_solve(const CsrGrid &a, int G, cudaStream_t st);
int nh_solve_capacity();           // CTAs of k_nh_solve that fit the device at once

// shape of the shared-memory zeta solver: CL CTAs of `threads` per basin,
// rows per CTA (capacity) and nonzeros per CTA (capacity), dynamic smem
struct ZetaShape {
  int CL = 0, threads = 0, chunk = 0, nnzcap = 0, halocap = 0;
  size_t smem = 0;
};

// maps of the shared-memory zeta solver for one cluster shape:
// loc[s]  -- local shared-memory column index of CSR slot s (own rows first,
//            then the CTA's halo slots)
// push    -- for each row (push_ptr[i]..push_ptr[i+1]) the halo slots of other
//            CTAs that hold a copy of it, packed (rank << 24) | slot
struct ZetaMaps {
  const int *loc = nullptr, *push_ptr = nullptr, *push = nullptr;
};

// the device-wide zeta solver (k_zeta_grid).  Each basin's rows are cut into
// tiles of a fixed row count (the last one shorter); tile t = {row0, row1,
// basin, slot} is worked by one CTA (cptr/clist), where `slot` indexes the CTA's table
// of basins: cslot[c*16 + slot] is the basin, bit slot of cowner[c] says the
// CTA holds the basin's first tile; basin b's tiles are btile[b].x .. .y-1
struct GridPlan {
  int ntile = 0;
  const int4 *tile = nullptr;
  const int2 *btile = nullptr;
  const int *cslot = nullptr, *cnslot = nullptr, *cowner = nullptr;
  const int *cptr = nullptr;       // CTA c works tiles clist[cptr[c]] .. clist[cptr[c+1]-1]
  const int *clist = nullptr;
  // the Jacobi-scaled system the FP32 iterations solve, S A S with S =
  // D^-1/2: its diagonal is one and is not stored.  Each row's first eight
  // off-diagonal entries sit in a fixed-width block of the row ([8*i + k]):
  // columns as 16-bit offsets j - i when every offset fits (ecol16), else
  // absolute (ecol32), padded with offset 0 / column i and value 0; rows
  // with more entries keep the rest in a CSR tail (xptr, xcol; nx entries
  // in all, 0: none).  The entries' slots in the full CSR (eslot, -1 on
  // padding, xslot), their FP32 values (eval, xval: written by the first
  // residual pass of each solve), S per row (sd) and the FP32 correction
  // per row (ecor).
  const short *ecol16 = nullptr;
  const int *ecol32 = nullptr;
  const int *eslot = nullptr;
  float *eval = nullptr;
  const int *xptr = nullptr, *xcol = nullptr, *xslot = nullptr;
  float *xval = nullptr;
  int nx = 0;
  float *sd = nullptr, *ecor = nullptr;
  double *partial = nullptr;       // [2][ntile][4] partial sums of the tiles
  unsigned *ctr = nullptr;         // [8]: barrier arrivals, 3 active counts, abort flag, release
  unsigned phantom = 0;            // arrivals the barrier waits for beyond its CTAs (0; 1 in the timeout test)
  long long spin_limit = 0;        // polls before a barrier wait gives up
};

// a group of basins solved by one launch with one cluster shape
struct ZetaClass {
  bool grid = false;               // device-wide cooperative variant (all basins, one launch)
  bool staged = false;             // its TMA-staged form
  int G = 0;                       // its CTAs
  size_t gsmem = 0;                // its dynamic shared memory
  GridPlan gp;
  bool sm = false;                 // shared-memory variant (else global memory)
  int CL = 1, threads = 512;
  ZetaShape zs;                    // capacities of the shared-memory variant
  std::vector<int> basins;
  int *d_blist = nullptr;          // device copy of basins
};

// nb clusters of CL CTAs; cluster c solves basin za.blist[c]
cudaError_t launch_zeta(const Dev &d, const ZetaArgs &za, int CL, int threads, int nb, cudaStream_t st);
cudaError_t launch_zeta_sm(const Dev &d, const ZetaArgs &za, const ZetaShape &zs, const ZetaMaps &zm,
                           int nb, cudaStream_t st);
// the device-wide variant: G CTAs, cooperative; clears gp.ctr first.  staged:
// the TMA-staged form with `smem` bytes of dynamic shared memory
cudaError_t launch_zeta_grid(const Dev &d, const ZetaArgs &za, const GridPlan &gp, int G, bool staged,
                             size_t smem, cudaStream_t st);
// CTAs of k_zeta_grid that fit the device at once (0 on error)
int zeta_grid_capacity(bool staged, size_t smem);
// dynamic shared memory of the staged form (16-bit or absolute columns)
size_t zeta_grid_stage_smem(bool c16);
int zeta_grid_max_slots();   // basins one CTA can hold
int zeta_grid_max_tiles();   // tiles one CTA can hold
int zeta_grid_tile_rows();   // rows per tile
long long zeta_grid_spin_limit();   // default barrier poll limit
// smem > 0 prepares the shared-memory variant for that many dynamic bytes
cudaError_t zeta_kernel_setup(int CL, size_t smem);
int zeta_max_active_clusters(int CL, int threads, size_t smem);

}  // namespace shy
