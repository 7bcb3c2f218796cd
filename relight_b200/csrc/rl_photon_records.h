// World-space photon records: each deposit of Photons::store
// (baker/Photons.cpp:119-126) kept as a point, for the k-nearest-neighbour
// irradiance estimate (rl_photonmap_gather_knn).  32 bytes.
#pragma once
#include <cstdint>

struct PhotonRecord {
    float x, y, z;       // hit point
    float r, g, b;       // deposited colour (the value added to the photonmap texel)
    uint32_t photon;     // global photon number
    uint16_t depth;      // bounce (0 = first hit)
    uint16_t slot;       // photonmap slot of the hit mesh
};
static_assert(sizeof(PhotonRecord) == 32, "PhotonRecord is 32 bytes");

// Unique, run-independent identity of a record: photon number and bounce.
inline __host__ __device__ uint64_t record_id(const PhotonRecord& r) {
    return ((uint64_t)r.photon << 4) | (uint64_t)(r.depth & 15);
}

struct rl_photons;  // record buffer + hash grid (rl_knn.cu)
struct PhotonSink {
    PhotonRecord* rec;
    unsigned long long* count;
    unsigned long long capacity;
};
// The sink of an rl_photons buffer (cleared count), for k_photons.
int rl_internal_photon_sink(rl_photons* p, PhotonSink* sink, void* stream);
