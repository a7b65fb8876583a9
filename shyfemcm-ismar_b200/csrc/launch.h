// launch.h -- host-side launch interface of the kernels in kernels.cu.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace shy {

// arguments of the zeta assembly + solve kernel
struct ZetaArgs {
  const float *zguess;  // initial guess (the old water level, system_solve's z)
  const float *hia;     // element matrices: hia[c*cs + e*es], c = 3*i + j
  const float *hik;     // element right-hand sides: hik[i*cs + e*es]
  int cs, es;
  int explicit_mode;    // system_set_explicit: diagonal (lumped) solve
  float inner_rtol;     // FP32 inner iterations reduce the residual by this factor
  int max_outer;        // FP64 refinement sweeps
  int sym;              // 1: CG (symmetric system), 0: BiCGStab
};

// which: 0 k_column, 1 k_final
void launch_elem(const Dev &d, int which, int init_only, cudaStream_t st, bool cor);
// which: 0 k_node(init_only=a), 1 k_stab, 2 k_conz(j=a, nsub=b), 3 k_rhoset
void launch_node(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st);
void launch_reduce(const Dev &d, int nsub, int advance, cudaStream_t st);
void launch_subctl(const Dev &d, cudaGraphConditionalHandle h, cudaStream_t st);
cudaError_t launch_zeta(const Dev &d, const ZetaArgs &za, int CL, int threads, int b_first, int nb,
                        cudaStream_t st);
cudaError_t zeta_kernel_setup(int CL);
int zeta_max_active_clusters(int CL, int threads);

}  // namespace shy
