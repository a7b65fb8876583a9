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
#include "k_wetdry.cuh"

// ---------------------------------------------------------------------------
// launch wrappers (host side): the element-column kernels, wetting and
// drying, the sub-step loop's control; the node kernels are in
// step_node.cu, the zeta solvers in step_zeta.cu (separate translation
// units, compiled in parallel)
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

template <int L>
static void launch_column_t(const Dev &d, cudaStream_t st, bool cor) {
  const int blocks = (d.NEL + 127) / 128;
  // the advective terms as a separate instance: the plain one keeps its registers
  if (d.mom) {
    if (cor) k_column_t<L, true, true><<<blocks, 128, 0, st>>>(d);
    else if (d.col_staged) k_column_t<L, false, true, true><<<blocks, 128, 0, st>>>(d);
    else k_column_t<L, false, true><<<blocks, 128, 0, st>>>(d);
  } else if (cor) k_column_t<L, true, false><<<blocks, 128, 0, st>>>(d);
  else if (d.col_staged) {
    if (d.any_xt) k_column_t<L, false, false, true><<<blocks, 128, 0, st>>>(d);
    else k_column_t<L, false, false, true, false><<<blocks, 128, 0, st>>>(d);
  } else k_column_t<L, false, false><<<blocks, 128, 0, st>>>(d);
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
      if (d.any_zad) {
        if (d.NLV <= 8) k_final_w<8><<<blocks, 128, 0, st>>>(d, init_only);
        else if (d.NLV <= 12) k_final_w<12><<<blocks, 128, 0, st>>>(d, init_only);
        else k_final_w<16><<<blocks, 128, 0, st>>>(d, init_only);
      } else {
        if (d.NLV <= 8) k_final_w<8, false><<<blocks, 128, 0, st>>>(d, init_only);
        else if (d.NLV <= 12) k_final_w<12, false><<<blocks, 128, 0, st>>>(d, init_only);
        else k_final_w<16, false><<<blocks, 128, 0, st>>>(d, init_only);
      }
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

// control of the device-driven transport sub-step loop (body of a CUDA-graph
// WHILE node): advance the sub-step index and keep looping while any basin
// has sub-steps left (scal3sh's isact = 1..istot, concentration.f90:728).
__global__ void k_subctl(Dev d, cudaGraphConditionalHandle h) {
  const int nj = *d.subj + 1;
  *d.subj = nj;
  *d.nsub_launched += d.any_tvd ? 4 : 3;   // gradients, element part, node part, this
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

}  // namespace shy
