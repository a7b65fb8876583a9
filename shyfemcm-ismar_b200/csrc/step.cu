// step.cu -- the semi-implicit step on sm_100a (kernels in k_*.cuh).
//
// Per time step, for all basins of a model at once:
//   k_column  hydro_transports + hydro_intern + hydro_zeta element part
//             (hydrodynamic.f90:758-864, 868-1416, 488-733): one warp segment per
//             element column, vertical system by PCR across lanes, 3x3 element
//             system of the zeta equation written per element; k_column_t, the
//             same with one thread per column (Thomas sweep) for columns of at
//             most 16 layers.
//   k_zeta    system_init/assemble/add_rhs/solve/get (simsys_spkaux.f90:137-705,
//             sparskit_admin.f90:115-334): one thread-block cluster per basin;
//             atomic-free gather assembly into CSR in element order (FP64), then
//             FP32 preconditioned Krylov iterations inside FP64 residual
//             refinement, all in one persistent launch.  k_zeta_grid does the
//             same for basins too large for a cluster: one cooperative launch
//             over the whole device.
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

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "../../include/shygpu.h"
#include "common.cuh"
#include "launch.h"
#include "physics.cuh"
#include "k_column.cuh"
#include "k_column_t.cuh"
#include "k_final.cuh"
#include "k_node.cuh"
#include "k_conz.cuh"
#include "k_zeta.cuh"
#include "k_wetdry.cuh"
#include "k_zeta_global.cuh"
#include "k_zeta_grid.cuh"

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
    case 2:   // right-hand sides per PCR: scalars transported together
      if (d.nsc_max <= 1) k_conz<S, 1><<<blocks, threads, 0, st>>>(d, kbas, a);
      else if (d.nsc_max <= 2) k_conz<S, 2><<<blocks, threads, 0, st>>>(d, kbas, a);
      else if (d.nsc_max <= 4) k_conz<S, 4><<<blocks, threads, 0, st>>>(d, kbas, a);
      else k_conz<S, kMaxScal><<<blocks, threads, 0, st>>>(d, kbas, a);
      break;
    case 3: k_rhoset<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 4: k_rho<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 5: k_moment<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 6: k_tvdgrad<S><<<blocks, threads, 0, st>>>(d, kbas, a); break;
    case 7: k_conz<S, 1, true><<<blocks, threads, 0, st>>>(d, kbas, a); break;   // shygpu_conz3d's source terms
  }
}

template <int L>
static void launch_column_t(const Dev &d, cudaStream_t st, bool cor) {
  const int blocks = (d.NEL + 127) / 128;
  // the advective terms as a separate instance: the plain one keeps its registers
  if (d.mom) {
    if (cor) k_column_t<L, true, true><<<blocks, 128, 0, st>>>(d);
    else k_column_t<L, false, true><<<blocks, 128, 0, st>>>(d);
  } else if (cor) k_column_t<L, true, false><<<blocks, 128, 0, st>>>(d);
  else k_column_t<L, false, false><<<blocks, 128, 0, st>>>(d);
}

void launch_elem(const Dev &d, int which, int init_only, cudaStream_t st, bool cor) {
  const bool thr = (d.col_threads || d.any_wd) && d.NLV <= 16;
  if (which == 0 && thr) {
    if (d.NLV <= 8) launch_column_t<8>(d, st, cor);
    else if (d.NLV <= 12) launch_column_t<12>(d, st, cor);
    else launch_column_t<16>(d, st, cor);
    return;
  }
  if (which == 1 && thr) {
    if (cor || d.any_wd) {
      if (cor) k_final_t<true><<<(d.NEL + 255) / 256, 256, 0, st>>>(d, init_only);
      else k_final_t<false><<<(d.NEL + 255) / 256, 256, 0, st>>>(d, init_only);
    } else {
      const int blocks = (d.NEL + 127) / 128;            // 4 warps of 32 elements
      if (d.NLV <= 8) k_final_w<8><<<blocks, 128, 0, st>>>(d, init_only);
      else if (d.NLV <= 12) k_final_w<12><<<blocks, 128, 0, st>>>(d, init_only);
      else k_final_w<16><<<blocks, 128, 0, st>>>(d, init_only);
    }
    return;
  }
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
  if (which == 0 && (d.col_threads || d.any_wd) && d.NLV <= 16) {
    const int blocks = (d.NKN + 127) / 128;
    if (d.NLV <= 8) k_node_t<8><<<blocks, 128, 0, st>>>(d, kbas, a);
    else if (d.NLV <= 12) k_node_t<12><<<blocks, 128, 0, st>>>(d, kbas, a);
    else k_node_t<16><<<blocks, 128, 0, st>>>(d, kbas, a);
    return;
  }
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
  *d.nsub_launched += d.any_tvd ? 3 : 2;
  cudaGraphSetConditional(h, nj < *d.imax ? 1u : 0u);
}

void launch_wetdry(const Dev &d, const int *kbas, int which, int basin, cudaStream_t st) {
  if (which == 0) k_wd_set<<<(d.NEL + 255) / 256, 256, 0, st>>>(d);
  else if (which == 1) k_wd_init<<<(d.NEL + 255) / 256, 256, 0, st>>>(d, basin);
  else k_wd_znv<<<(d.NKN + 255) / 256, 256, 0, st>>>(d, kbas, basin);
}

void launch_subctl(const Dev &d, cudaGraphConditionalHandle h, cudaStream_t st) {
  k_subctl<<<1, 1, 0, st>>>(d, h);
}

void launch_reduce(const Dev &d, int nsub, int advance, cudaStream_t st) {
  k_reduce<<<d.nbasin, 1024, 0, st>>>(d, nsub, advance);
}

static cudaLaunchConfig_t zeta_config(int CL, int threads, int nclusters, size_t smem, cudaStream_t st,
                                      cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * CL, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

cudaError_t launch_zeta(const Dev &d, const ZetaArgs &za, int CL, int threads, int nb, cudaStream_t st) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = zeta_config(CL, threads, nb, 0, st, attr);
  return cudaLaunchKernelEx(&cfg, k_zeta, d, za, CL);
}

cudaError_t launch_zeta_sm(const Dev &d, const ZetaArgs &za, const ZetaShape &zs, const ZetaMaps &zm,
                           int nb, cudaStream_t st) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = zeta_config(zs.CL, zs.threads, nb, zs.smem, st, attr);
  return cudaLaunchKernelEx(&cfg, k_zeta_sm, d, za, zs, zm);
}

cudaError_t launch_zeta_grid(const Dev &d, const ZetaArgs &za, const GridPlan &gp, int G, bool staged,
                             size_t smem, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(gp.ctr, 0, 8 * sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.gridDim = dim3(G, 1, 1);
  cfg.blockDim = dim3(staged ? 1024 : 512, 1, 1);
  cfg.dynamicSmemBytes = staged ? smem : 0;
  cfg.stream = st;
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const bool c16 = gp.ocol16 != nullptr;
  if (staged) return c16 ? cudaLaunchKernelEx(&cfg, k_zeta_grid<1024, true, true>, d, za, gp)
                         : cudaLaunchKernelEx(&cfg, k_zeta_grid<1024, true, false>, d, za, gp);
  return c16 ? cudaLaunchKernelEx(&cfg, k_zeta_grid<512, false, true>, d, za, gp)
             : cudaLaunchKernelEx(&cfg, k_zeta_grid<512, false, false>, d, za, gp);
}

size_t zeta_grid_stage_smem(int nzcap, bool c16) {
  return 128 + 2 * (size_t)stage_layout(nzcap, c16 ? 2 : 4).bytes;
}

// resident CTAs of the device-wide solver; the fewer of its two column
// forms, so a plan holds whichever it launches
template <bool STAGED, bool C16>
static int grid_blocks(size_t smem) {
  constexpr int NT = STAGED ? 1024 : 512;
  int nb = 0;
  if (STAGED && cudaFuncSetAttribute(k_zeta_grid<NT, STAGED, C16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_zeta_grid<NT, STAGED, C16>, NT, STAGED ? smem : 0) !=
      cudaSuccess)
    return 0;
  return nb;
}

int zeta_grid_capacity(bool staged, size_t smem) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  const int nb = staged ? std::min(grid_blocks<true, true>(smem), grid_blocks<true, false>(smem))
                        : std::min(grid_blocks<false, true>(0), grid_blocks<false, false>(0));
  return nb * nsm;
}

int zeta_grid_max_slots() { return kGridMaxSlots; }
int zeta_grid_max_tiles() { return kGridMaxTiles; }
int zeta_grid_tile_rows() { return kGridTileRows; }
long long zeta_grid_spin_limit() { return kGridSpinLimit; }

cudaError_t zeta_kernel_setup(int CL, size_t smem) {
  cudaError_t e = cudaSuccess;
  if (CL > 8) {
    e = cudaFuncSetAttribute(k_zeta, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zeta_sm, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  }
  if (e == cudaSuccess && smem > 0)
    e = cudaFuncSetAttribute(k_zeta_sm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return e;
}

int zeta_max_active_clusters(int CL, int threads, size_t smem) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = zeta_config(CL, threads, 1, smem, nullptr, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, smem > 0 ? (const void *)k_zeta_sm : (const void *)k_zeta, &cfg) != cudaSuccess)
    return -1;
  return n;
}

}  // namespace shy
