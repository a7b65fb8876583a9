// step_node.cu -- launch wrappers of the node-column kernels (k_node*,
// k_stab, k_conz, k_tvdgrad, k_moment, k_rho*, k_reduce); the instances of
// segment widths 16 and 32 are compiled in step_node16.cu and
// step_node32.cu.  See step.cu.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "../../include/shygpu.h"
#include "common.cuh"
#include "launch.h"
#include "physics.cuh"
#include "node_launch.cuh"

namespace shy {

extern template void launch_node_S<16>(const Dev &, const int *, int, int, int, cudaStream_t);
extern template void launch_node_S<32>(const Dev &, const int *, int, int, int, cudaStream_t);

void launch_node(const Dev &d, const int *kbas, int which, int a, int b, cudaStream_t st) {
  if (which == 0 && (d.col_threads || d.any_wd) && d.NLV <= 16) {
    const int blocks = (d.NKN + 127) / 128;
    if (d.node_prefetch) {
      if (d.NLV <= 8) k_node_t<8, true><<<blocks, 128, 0, st>>>(d, kbas, a);
      else if (d.NLV <= 12) k_node_t<12, true><<<blocks, 128, 0, st>>>(d, kbas, a);
      else k_node_t<16, true><<<blocks, 128, 0, st>>>(d, kbas, a);
    } else {
      if (d.any_zad) {
        if (d.NLV <= 8) k_node_t<8><<<blocks, 128, 0, st>>>(d, kbas, a);
        else if (d.NLV <= 12) k_node_t<12><<<blocks, 128, 0, st>>>(d, kbas, a);
        else k_node_t<16><<<blocks, 128, 0, st>>>(d, kbas, a);
      } else {
        if (d.NLV <= 8) k_node_t<8, false, false><<<blocks, 128, 0, st>>>(d, kbas, a);
        else if (d.NLV <= 12) k_node_t<12, false, false><<<blocks, 128, 0, st>>>(d, kbas, a);
        else k_node_t<16, false, false><<<blocks, 128, 0, st>>>(d, kbas, a);
      }
    }
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

void launch_reduce(const Dev &d, int nsub, int advance, cudaStream_t st) {
  k_reduce<<<d.nbasin, 1024, 0, st>>>(d, nsub, advance);
}

}  // namespace shy
