// Device LBVH builder (rl_lbvh.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rl {

// Builds the binary traversal layout on the device from scene-space vertex
// positions (d_pos, [nverts][3]) and per-triangle vertex ids (d_vidx, a, b,
// c, mesh).  On success *d_nodes / *d_tris are cudaMalloc'd buffers owned by
// the caller; *depth is the tree depth.
bool build_lbvh_device(const float* d_pos, const int4* d_vidx, int n, cudaStream_t st, float4** d_nodes,
                       float4** d_tris, int64_t* nnodes, int* depth, const char** err);

}  // namespace rl
