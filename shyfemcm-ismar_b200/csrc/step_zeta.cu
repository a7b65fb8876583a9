// step_zeta.cu -- launch wrappers and set-up of the zeta solvers (k_zeta,
// k_zeta_sm, k_zeta_grid).  See step.cu.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "../../include/shygpu.h"
#include "common.cuh"
#include "launch.h"
#include "physics.cuh"
#include "k_wetdry.cuh"
#include "k_zeta.cuh"
#include "k_zeta_global.cuh"
#include "k_zeta_grid.cuh"

namespace shy {

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
  const bool c16 = gp.ecol16 != nullptr;
  if (staged) return c16 ? cudaLaunchKernelEx(&cfg, k_zeta_grid<1024, true, true>, d, za, gp)
                         : cudaLaunchKernelEx(&cfg, k_zeta_grid<1024, true, false>, d, za, gp);
  return c16 ? cudaLaunchKernelEx(&cfg, k_zeta_grid<512, false, true>, d, za, gp)
             : cudaLaunchKernelEx(&cfg, k_zeta_grid<512, false, false>, d, za, gp);
}

size_t zeta_grid_stage_smem(bool c16) { return 128 + 2 * (size_t)stage_layout(c16 ? 16 : 32).bytes; }

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
