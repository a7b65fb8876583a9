// node_launch.cuh -- launches of the node-column kernels of one segment
// width S.  Its instances for the different S are compiled in separate
// translation units (step_node.cu: S <= 8, step_node16.cu, step_node32.cu).
#pragma once
#include "common.cuh"
#include "k_node.cuh"
#include "k_conz.cuh"

namespace shy {

// the transport's element part, its TVD instance only for models that use TVD
template <int S>
void launch_conz_el(const Dev &d, int a, cudaStream_t st) {
  const int threads = 256;
  const int blocks = (int)(((long long)d.NEL * S + threads - 1) / threads);
  if (d.any_tvd || d.tvdup) k_conz_el<S, true><<<blocks, threads, 0, st>>>(d, a);
  else k_conz_el<S, false><<<blocks, threads, 0, st>>>(d, a);
}

// the node part with as many right-hand sides per PCR as the model
// transports scalars together; TV: its vertical-TVD instance
template <int S, bool TV>
void launch_conz_node(const Dev &d, const int *kbas, int a, int blocks, int threads, cudaStream_t st) {
  if (d.nsc_max <= 1) k_conz<S, 1, false, TV><<<blocks, threads, 0, st>>>(d, kbas, a);
  else if (d.nsc_max <= 2) k_conz<S, 2, false, TV><<<blocks, threads, 0, st>>>(d, kbas, a);
  else if (d.nsc_max <= 3) k_conz<S, 3, false, TV><<<blocks, threads, 0, st>>>(d, kbas, a);
  else if (d.nsc_max <= 4) k_conz<S, 4, false, TV><<<blocks, threads, 0, st>>>(d, kbas, a);
  else k_conz<S, kMaxScal, false, TV><<<blocks, threads, 0, st>>>(d, kbas, a);
}

template <int S>
void launch_node_S(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st) {
  const int threads = 256;
  const long long nt = (long long)d.NKN * S;
  const int blocks = (int)((nt + threads - 1) / threads);
  switch (which) {
    case 0: k_node<S><<<blocks, threads, 0, st>>>(d, kbas, a); break;
    case 1: k_stab<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 2:   // the element part, then right-hand sides per PCR: scalars transported together
      launch_conz_el<S>(d, a, st);
      if (d.any_tvdv) launch_conz_node<S, true>(d, kbas, a, blocks, threads, st);
      else launch_conz_node<S, false>(d, kbas, a, blocks, threads, st);
      break;
    case 3: k_rhoset<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 4: k_rho<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 5: k_moment<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 6: k_tvdgrad<S><<<blocks, threads, 0, st>>>(d, kbas, a); break;
    case 7:   // shygpu_conz3d's source terms
      launch_conz_el<S>(d, a, st);
      if (d.any_tvdv) k_conz<S, 1, true, true><<<blocks, threads, 0, st>>>(d, kbas, a);
      else k_conz<S, 1, true, false><<<blocks, threads, 0, st>>>(d, kbas, a);
      break;
  }
}

}  // namespace shy
