// node_launch.cuh -- launches of the node-column kernels of one segment
// width S.  Its instances for the different S are compiled in separate
// translation units (step_node.cu: S <= 8, step_node16.cu, step_node32.cu).
#pragma once
#include "common.cuh"
#include "k_node.cuh"
#include "k_conz.cuh"

namespace shy {

template <int S>
void launch_node_S(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st) {
  const int threads = 256;
  const long long nt = (long long)d.NKN * S;
  const int blocks = (int)((nt + threads - 1) / threads);
  switch (which) {
    case 0: k_node<S><<<blocks, threads, 0, st>>>(d, kbas, a); break;
    case 1: k_stab<S><<<blocks, threads, 0, st>>>(d, kbas); break;
    case 2:   // right-hand sides per PCR: scalars transported together
      if (d.nsc_max <= 1) k_conz<S, 1><<<blocks, threads, 0, st>>>(d, kbas, a);
      else if (d.nsc_max <= 2) k_conz<S, 2><<<blocks, threads, 0, st>>>(d, kbas, a);
      else if (d.nsc_max <= 3) k_conz<S, 3><<<blocks, threads, 0, st>>>(d, kbas, a);
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

}  // namespace shy
