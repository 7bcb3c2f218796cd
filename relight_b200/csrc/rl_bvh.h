// BVH construction for the B200 traversal kernels.
#pragma once

#include <cstdint>
#include <vector>

namespace rl {

struct BvhBuild {
    std::vector<float> nodes;  // 16 floats per node (four float4, see rl_device.cuh)
    std::vector<float> tris;   // 12 floats per triangle in leaf order (three float4)
    std::vector<float> nodes4; // 32 floats per 4-wide node (eight float4, see rl_device.cuh)
    int64_t nodes4_count = 0;
    std::vector<uint32_t> nodes8;  // 20 words per compressed 8-wide node (five uint4, see rl_device.cuh)
    std::vector<float> tris8;      // triangle records in 8-wide node order (12 floats each)
    int64_t nodes8_count = 0;
    int64_t leaves = 0;
    int depth = 0;
    double sah = 0.0;
};

// Binned-SAH build over `ntris` triangles given as three vertex ids into
// `pos` ([nverts][3]); triangle ids are the global ids (position in `tris`).
// wide8: also emit the compressed 8-wide tree (nodes8 / tris8).
bool build_bvh_sah(const float* pos, int nverts, const int32_t* tris, int ntris, BvhBuild& out, const char** err,
                   bool wide8 = false);

}  // namespace rl
