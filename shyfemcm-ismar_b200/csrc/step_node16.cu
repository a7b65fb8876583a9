// step_node16.cu -- the node-column kernels of segment width 16 (see
// node_launch.cuh), a translation unit of their own so the library's
// sources compile in parallel.
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
template void launch_node_S<16>(const Dev &, const int *, int, int, int, cudaStream_t);
}  // namespace shy
