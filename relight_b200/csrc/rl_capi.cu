// C ABI and pass kernels of the B200 lightmap baker (include/relight_b200.h).
//
// Kernel map (reference function -> kernel):
//   rt::Embree::traceSegment           k_trace_segments
//   Lightmap::initializeLumels         k_raster_owner + k_raster_init
//   DirectLight::bakeLumel             k_direct
//   AmbientOcclusion::bakeLumel        k_ao
//   Photons::emit/trace/store          k_photons
//   Photonmap::gather                  k_gather
//   IndirectLight::bakeLumel           k_indirect
//   RadiosityBuilder form factors      k_ff_pairs (+ host CSR assembly)
//   hemisphere form factors            k_ff_hemi_rays + k_ff_hemi_rle + k_ff_hemi_compact
//   radiosity gather iterations        k_jacobi4 (k_jacobi_rows per row shard)
#include <cuda_runtime.h>

#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/relight_b200.h"
#include "rl_bvh.h"
#include "rl_device.cuh"
#include "rl_photon_records.h"
#include "rl_lbvh.h"

using namespace rl;

// ------------------------------------------------------------ errors

namespace {

thread_local std::string g_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(e_ == cudaErrorMemoryAllocation ? RL_OUT_OF_MEMORY : RL_CUDA_ERROR,        \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CK_LAUNCH(name)                                                                            \
    do {                                                                                           \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess)                                                                     \
            return fail(RL_CUDA_ERROR, "launch of %s failed: %s", name, cudaGetErrorString(e_));   \
    } while (0)

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Launch tuning (rl_tune_set): per ray-stream kernel, the number of lanes a
// warp waits for before refilling rays and the threads per block.  Defaults
// are the autotuner's picks on the terrain final-gather / room AO workloads.
// Then the BVH width, speculative traversal, the kNN grid's cell width in
// 64ths of the search radius (the fastest on the terrain kNN bench), the AO
// lane split, and the persistent lumel pool (off: see RL_TUNE_FG_POOL) and its chunk.
int g_tune[10] = {24, 256, 32, 128, 2, 0, 80, 0, 0, 32};

inline unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

template <typename T>
int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) return RL_OK;
    CK(cudaMalloc((void**)p, sizeof(T) * count));
    return RL_OK;
}

template <typename T>
int dupload(T** p, const T* host, size_t count, cudaStream_t st) {
    int rc = dalloc(p, count);
    if (rc) return rc;
    if (count && host) CK(cudaMemcpyAsync(*p, host, sizeof(T) * count, cudaMemcpyHostToDevice, st));
    return RL_OK;
}

// A stream-ordered scratch buffer freed when it goes out of scope, drawn from
// the library's memory pool (rl_internal_pool_alloc, below): freed blocks
// stay mapped for the next call.  The device's default pool returns them at
// every synchronisation, and a call that waits on the host in its middle
// (the form factors wait for their row counts) then maps ~100 MB afresh.
struct Scratch {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~Scratch() {
        if (p) cudaFreeAsync(p, st);
    }
};

}  // namespace
int rl_internal_pool_alloc(void** p, size_t bytes, cudaStream_t st);
namespace {

template <typename T>
int scratch(Scratch& s, T** out, size_t count, cudaStream_t st) {
    s.st = st;
    *out = nullptr;
    if (count == 0) return RL_OK;
    if (int rc = rl_internal_pool_alloc(&s.p, sizeof(T) * count, st)) return rc;
    *out = (T*)s.p;
    return RL_OK;
}

}  // namespace

// ------------------------------------------------------------- handles

struct rl_scene {
    DevScene dev{};
    std::vector<void*> owned;
    int* d_status = nullptr;  // bit 0: traversal stack overflow
    int64_t nnodes = 0, leaves = 0;
    int depth = 0;
    double sah = 0.0;
    int nmeshes = 0;
    std::vector<int> mesh_first_tri;
    std::vector<int> mesh_photonmap;
    ~rl_scene() {
        for (void* p : owned) cudaFree(p);
        if (d_status) cudaFree(d_status);
    }
};

struct rl_map {
    int kind = 0;
    DevMap dev{};
    int* d_owner = nullptr;  // rasterisation scratch: winning face per texel
    unsigned long long* d_work = nullptr;  // work-list counter of the persistent bake kernels
    char* block = nullptr;   // rl_map_create_async: every array carved from this block
    ~rl_map() {
        if (block) {
            cudaFree(block);
            return;
        }
        cudaFree(dev.flags); cudaFree(dev.face); cudaFree(dev.position); cudaFree(dev.normal);
        cudaFree(dev.color); cudaFree(dev.photons); cudaFree(dev.gathered); cudaFree(dev.mesh); cudaFree(d_owner);
        cudaFree(d_work);
    }
};

// Error entry for the host-only sources of the library (e.g. the OBJ loader).
int rl_internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }

// Device views of handles, for the library's other translation units.
const DevMap* rl_internal_map(const rl_map* m) { return m ? &m->dev : nullptr; }
const DevScene* rl_internal_scene(const rl_scene* s) { return s ? &s->dev : nullptr; }
int rl_internal_pool_alloc(void** p, size_t bytes, cudaStream_t st);

extern "C" int rl_last_error(char* buf, size_t len) {
    if (buf && len) {
        snprintf(buf, len, "%s", g_error.c_str());
    }
    return (int)g_error.size();
}

extern "C" const char* rl_version(void) { return "relight_b200 0.1 (sm_100a)"; }

extern "C" int rl_tune_set(int param, int value) {
    bool refill = param == RL_TUNE_FG_REFILL || param == RL_TUNE_AO_REFILL;
    bool block = param == RL_TUNE_FG_BLOCK || param == RL_TUNE_AO_BLOCK;
    bool width = param == RL_TUNE_BVH_WIDTH;
    bool spec = param == RL_TUNE_SPECULATIVE;
    bool cell = param == RL_TUNE_KNN_CELL;
    bool split = param == RL_TUNE_AO_SPLIT;
    bool pool = param == RL_TUNE_FG_POOL;
    bool chunk = param == RL_TUNE_FG_CHUNK;
    if ((refill && value >= 1 && value <= 32) || (block && (value == 64 || value == 128 || value == 256)) ||
        (width && (value == 2 || value == 4 || value == 8)) || (spec && (value == 0 || value == 1)) ||
        (cell && value >= 8 && value <= 256) ||
        (split && (value == 0 || value == 1 || value == 2 || value == 4 || value == 8)) ||
        (pool && (value == 0 || value == 1)) || (chunk && value >= 8 && value <= 256))
        g_tune[param] = value;
    else
        return fail(RL_INVALID_CALL, "rl_tune_set: bad parameter %d or value %d", param, value);
    return RL_OK;
}

extern "C" int rl_tune_get(int param, int* value) {
    if (!value || param < 0 || param > RL_TUNE_FG_CHUNK) return fail(RL_INVALID_CALL, "rl_tune_get: bad parameter");
    *value = g_tune[param];
    return RL_OK;
}

int rl_internal_tune(int param) { return g_tune[param]; }

// ------------------------------------------------------------- scene

extern "C" int rl_scene_create(const rl_scene_desc* d, int builder, void* stream, rl_scene** out) {
    if (!d || !out) return fail(RL_INVALID_CALL, "rl_scene_create: null argument");
    *out = nullptr;
    if (d->ntris < 0 || d->nverts < 0 || d->nmeshes < 0) return fail(RL_INVALID_CALL, "negative counts");
    if (d->ntris > 0 && (!d->pos || !d->tris || !d->mesh_first_tri))
        return fail(RL_INVALID_CALL, "rl_scene_create: missing geometry arrays");
    if (d->nmeshes > 0 && d->mesh_first_tri[d->nmeshes] != d->ntris)
        return fail(RL_INVALID_CALL, "mesh_first_tri[nmeshes] must equal ntris");
    if (builder != 0 && builder != 1) return fail(RL_INVALID_CALL, "builder must be 0 (SAH) or 1 (LBVH)");
    cudaStream_t st = S(stream);
    rl_scene* s = new (std::nothrow) rl_scene;
    if (!s) return fail(RL_OUT_OF_MEMORY, "host allocation failed");
    BvhBuild b;
    const char* err = "";
    for (int t = 0; t < 3 * d->ntris; t++)
        if (d->tris[t] < 0 || d->tris[t] >= d->nverts) {
            delete s;
            return fail(RL_INVALID_CALL, "triangle vertex index out of range");
        }
    // the compressed 8-wide tree is built only while width 8 is selected
    if (builder == 0 && !build_bvh_sah(d->pos, d->nverts, d->tris, d->ntris, b, &err, g_tune[RL_TUNE_BVH_WIDTH] == 8)) {
        delete s;
        return fail(RL_INVALID_CALL, "BVH build: %s", err);
    }
    s->nnodes = (int64_t)(b.nodes.size() / 16);
    s->leaves = b.leaves;
    s->depth = b.depth;
    s->sah = b.sah;
    if (b.depth >= kStackSize - 1) {
        delete s;
        return fail(RL_NOT_IMPLEMENTED, "BVH depth %d exceeds the traversal stack", b.depth);
    }
    // per-triangle vertex ids + mesh
    std::vector<int4> vidx(d->ntris);
    for (int m = 0; m < d->nmeshes; m++)
        for (int t = d->mesh_first_tri[m]; t < d->mesh_first_tri[m + 1]; t++)
            vidx[t] = make_int4(d->tris[3 * t], d->tris[3 * t + 1], d->tris[3 * t + 2], m);
    int has_alpha = 0;
    for (int m = 0; m < d->nmats; m++) {
        int t = d->mat_tex ? d->mat_tex[m] : -1;
        if (t >= 0 && d->tex_dims[3 * t + 2] == 4) has_alpha = 1;
    }
    std::vector<int> mat_tex(d->mat_tex ? d->mat_tex : nullptr, d->mat_tex ? d->mat_tex + d->nmats : nullptr);
    if (mat_tex.empty()) mat_tex.assign(d->nmats, -1);
    std::vector<int> vmat(d->vmat ? d->vmat : nullptr, d->vmat ? d->vmat + d->nverts : nullptr);
    if (vmat.empty()) vmat.assign(d->nverts, -1);
    std::vector<float> zeros2(2 * (size_t)d->nverts, 0.0f);
    std::vector<float> zeros3(d->nrm ? 0 : 3 * (size_t)d->nverts, 0.0f);
    std::vector<int> pmap(d->mesh_photonmap ? d->mesh_photonmap : nullptr,
                          d->mesh_photonmap ? d->mesh_photonmap + d->nmeshes : nullptr);
    if (pmap.empty()) pmap.assign(d->nmeshes, -1);
    s->mesh_first_tri.assign(d->mesh_first_tri, d->mesh_first_tri + d->nmeshes + 1);
    s->mesh_photonmap = pmap;
    s->nmeshes = d->nmeshes;
    // Per-triangle shading record for final-gather hits (64 B, one line):
    // the three vertex normals, each with its lightmap u, then the three
    // lightmap v and the mesh's photonmap slot (int bits).
    std::vector<float4> shade(4 * (size_t)d->ntris);
    {
        const float* vn = d->nrm ? d->nrm : zeros3.data();
        const float* vu = d->uv1 ? d->uv1 : zeros2.data();
        for (int t = 0; t < d->ntris; t++) {
            const int4 f = vidx[t];
            const int vs[3] = {f.x, f.y, f.z};
            for (int q = 0; q < 3; q++)
                shade[4 * (size_t)t + q] = make_float4(vn[3 * (size_t)vs[q]], vn[3 * (size_t)vs[q] + 1],
                                                       vn[3 * (size_t)vs[q] + 2], vu[2 * (size_t)vs[q]]);
            float slot;
            const int sl = pmap[f.w];
            std::memcpy(&slot, &sl, 4);
            shade[4 * (size_t)t + 3] = make_float4(vu[2 * (size_t)f.x + 1], vu[2 * (size_t)f.y + 1],
                                                   vu[2 * (size_t)f.z + 1], slot);
        }
    }

    int rc = RL_OK;
    auto up = [&](auto** dst, const auto* src, size_t count) {
        if (rc) return;
        rc = dupload(dst, src, count, st);
        if (!rc && *dst) s->owned.push_back((void*)*dst);
    };
    float4* nodes = nullptr; float4* tris = nullptr; int4* dvidx = nullptr;
    float *pos = nullptr, *nrm = nullptr, *uv0 = nullptr, *uv1 = nullptr, *mat_rgb = nullptr;
    int *dvmat = nullptr, *first = nullptr, *dpmap = nullptr, *dmat_tex = nullptr, *tex_dims = nullptr;
    long long* tex_off = nullptr;
    unsigned char* tex_px = nullptr;
    float4* nodes4 = nullptr;
    float4* dshade = nullptr;
    uint4* nodes8 = nullptr;
    float4* tris8 = nullptr;
    if (builder == 0) {
        up(&nodes, (const float4*)b.nodes.data(), b.nodes.size() / 4);
        up(&nodes4, (const float4*)b.nodes4.data(), b.nodes4.size() / 4);
        up(&tris, (const float4*)b.tris.data(), b.tris.size() / 4);
        if (!b.nodes8.empty()) {
            up(&nodes8, (const uint4*)b.nodes8.data(), b.nodes8.size() / 4);
            up(&tris8, (const float4*)b.tris8.data(), b.tris8.size() / 4);
        }
    }
    up(&dvidx, vidx.data(), vidx.size());
    up(&dshade, shade.data(), shade.size());
    up(&pos, d->pos, 3 * (size_t)d->nverts);
    up(&nrm, d->nrm ? d->nrm : zeros3.data(), 3 * (size_t)d->nverts);
    up(&uv0, d->uv0 ? d->uv0 : zeros2.data(), 2 * (size_t)d->nverts);
    up(&uv1, d->uv1 ? d->uv1 : zeros2.data(), 2 * (size_t)d->nverts);
    up(&dvmat, vmat.data(), vmat.size());
    up(&first, d->mesh_first_tri, (size_t)d->nmeshes + 1);
    up(&dpmap, pmap.data(), pmap.size());
    up(&mat_rgb, d->mat_rgb, 3 * (size_t)d->nmats);
    up(&dmat_tex, mat_tex.data(), mat_tex.size());
    if (d->ntex > 0) {
        up(&tex_dims, d->tex_dims, 3 * (size_t)d->ntex);
        up(&tex_off, (const long long*)d->tex_offset, (size_t)d->ntex);
        size_t bytes = 0;
        for (int t = 0; t < d->ntex; t++)
            bytes = std::max(bytes, (size_t)d->tex_offset[t] + (size_t)d->tex_dims[3 * t] * d->tex_dims[3 * t + 1] *
                                        d->tex_dims[3 * t + 2]);
        up(&tex_px, d->tex_pixels, bytes);
    }
    if (!rc && builder == 1 && d->ntris > 0) {
        int64_t nn = 0;
        int depth = 0;
        const char* lerr = "";
        if (!build_lbvh_device(pos, dvidx, d->ntris, st, &nodes, &tris, &nn, &depth, &lerr)) {
            rc = fail(RL_CUDA_ERROR, "LBVH build: %s", lerr);
        } else {
            s->owned.push_back(nodes);
            s->owned.push_back(tris);
            s->nnodes = nn;
            s->leaves = d->ntris;
            s->depth = depth;
            s->sah = 0.0;
            if (depth >= kStackSize - 1) rc = fail(RL_NOT_IMPLEMENTED, "LBVH depth %d exceeds the traversal stack", depth);
        }
    }
    if (!rc) {
        cudaError_t e = cudaMalloc(&s->d_status, sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_status, 0, sizeof(int), st);
        if (e != cudaSuccess) rc = fail(RL_CUDA_ERROR, "status word: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(st);  // host staging vectors die at return
        if (e != cudaSuccess) rc = fail(RL_CUDA_ERROR, "scene upload: %s", cudaGetErrorString(e));
    }
    if (rc) {
        delete s;
        return rc;
    }
    DevScene& v = s->dev;
    v.nodes = nodes; v.nodes4 = nodes4; v.tris = tris; v.tri_vidx = dvidx; v.shade = dshade;
    v.nodes8 = nodes8; v.tris8 = tris8;
    v.pos = pos; v.nrm = nrm; v.uv0 = uv0; v.uv1 = uv1; v.vmat = dvmat;
    v.mesh_first_tri = first; v.mesh_photonmap = dpmap;
    v.mat_rgb = mat_rgb; v.mat_tex = dmat_tex; v.tex_dims = tex_dims; v.tex_offset = tex_off; v.tex_pixels = tex_px;
    for (int k = 0; k < 3; k++) { v.bounds_lo[k] = d->bounds_lo[k]; v.bounds_hi[k] = d->bounds_hi[k]; }
    v.ntris = d->ntris;
    v.nmeshes = d->nmeshes;
    v.has_alpha = has_alpha;
    *out = s;
    return RL_OK;
}

extern "C" int rl_scene_destroy(rl_scene* s) {
    if (!s) return fail(RL_INVALID_CALL, "null scene");
    cudaDeviceSynchronize();
    delete s;
    return RL_OK;
}

extern "C" int rl_scene_bvh_stats(const rl_scene* s, int64_t* nodes, int64_t* leaves, int32_t* depth, double* sah) {
    if (!s) return fail(RL_INVALID_CALL, "null scene");
    if (nodes) *nodes = s->nnodes;
    if (leaves) *leaves = s->leaves;
    if (depth) *depth = s->depth;
    if (sah) *sah = s->sah;
    return RL_OK;
}

extern "C" int rl_scene_status(rl_scene* s, int clear, int32_t* flags, void* stream) {
    if (!s || !flags) return fail(RL_INVALID_CALL, "rl_scene_status: null argument");
    cudaStream_t st = S(stream);
    int h = 0;
    CK(cudaMemcpyAsync(&h, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (clear) CK(cudaMemsetAsync(s->d_status, 0, sizeof(int), st));
    CK(cudaStreamSynchronize(st));
    *flags = h;
    return RL_OK;
}

static int check_status(const rl_scene* s, cudaStream_t st) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h & 1) return fail(RL_CUDA_ERROR, "BVH traversal stack overflow (scene too deep)");
    return RL_OK;
}

// ------------------------------------------------------------- tracing

__global__ void k_trace_segments(DevScene s, long long n, const float* seg, int flags, int* hit, float* tuv,
                                 int* mesh_face, float* point, float* normal, float* rgba, float* uv, int* status) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    SegHit r;
    trace_segment(s, ld3(seg + 6 * i), ld3(seg + 6 * i + 3), flags, r, status);
    hit[i] = r.hit ? 1 : 0;
    if (tuv) { tuv[3 * i] = r.hit ? r.t : 0.f; tuv[3 * i + 1] = r.hit ? r.u : 0.f; tuv[3 * i + 2] = r.hit ? r.v : 0.f; }
    if (mesh_face) { mesh_face[2 * i] = r.hit ? r.mesh : -1; mesh_face[2 * i + 1] = r.hit ? r.face : -1; }
    if (point) st3(point + 3 * i, r.hit ? r.point : mk3(0.f, 0.f, 0.f));
    if (normal) st3(normal + 3 * i, r.hit && (flags & kHitNormal) ? r.normal : mk3(0.f, 0.f, 0.f));
    if (rgba) {
        float4 c = r.hit && (flags & kHitColor) ? r.rgba : make_float4(0.f, 0.f, 0.f, 0.f);
        rgba[4 * i] = c.x; rgba[4 * i + 1] = c.y; rgba[4 * i + 2] = c.z; rgba[4 * i + 3] = c.w;
    }
    if (uv) {
        uv[2 * i] = r.hit && (flags & kHitUv) ? r.uv.x : 0.f;
        uv[2 * i + 1] = r.hit && (flags & kHitUv) ? r.uv.y : 0.f;
    }
}

extern "C" int rl_trace_segments(const rl_scene* s, int64_t n, const float* d_seg, int flags, int32_t* d_hit,
                                 float* d_t_uv, int32_t* d_mesh_face, float* d_point, float* d_normal,
                                 float* d_rgba, float* d_uv, void* stream) {
    if (!s || (n > 0 && (!d_seg || !d_hit))) return fail(RL_INVALID_CALL, "rl_trace_segments: null argument");
    if (n <= 0) return RL_OK;
    k_trace_segments<<<blocks_for(n, 128), 128, 0, S(stream)>>>(s->dev, n, d_seg, flags, d_hit, d_t_uv,
                                                                d_mesh_face, d_point, d_normal, d_rgba, d_uv,
                                                                s->d_status);
    CK_LAUNCH("k_trace_segments");
    return RL_OK;
}

// rtcIntersect / rtcOccluded (embree2/rtcore_ray.h:24-51) for a batch of
// rays given as Embree takes them: closest hit (or, with any_hit, some hit)
// on the open interval (tnear, tfar) of org + t dir, ties to the smaller
// (geomID, primID).
__global__ void k_intersect_rays(DevScene s, long long n, const float4* rays, int any_hit, int* geom_prim,
                                 float* tuv, int* status) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = rays[2 * i], b = rays[2 * i + 1];
    const V3 o = mk3(a.x, a.y, a.z), d = mk3(b.x, b.y, b.z);
    RayHit h;
    const bool hit = any_hit ? traverse<true>(s, o, d, a.w, b.w, h, status)
                             : traverse<false>(s, o, d, a.w, b.w, h, status);
    int mesh = -1, prim = -1;
    if (hit) {
        mesh = __ldg(s.tri_vidx + h.gid).w;
        prim = h.gid - s.mesh_first_tri[mesh];
    }
    geom_prim[2 * i] = mesh;
    geom_prim[2 * i + 1] = prim;
    if (tuv) {
        tuv[3 * i] = hit ? h.t : 0.f;
        tuv[3 * i + 1] = hit ? h.u : 0.f;
        tuv[3 * i + 2] = hit ? h.v : 0.f;
    }
}

extern "C" int rl_intersect_rays(const rl_scene* s, int64_t n, const float* d_rays, int any_hit, int32_t* d_geom_prim,
                                 float* d_t_uv, void* stream) {
    if (!s || n < 0 || (n > 0 && (!d_rays || !d_geom_prim)))
        return fail(RL_INVALID_CALL, "rl_intersect_rays: bad arguments");
    if ((uintptr_t)d_rays % 16) return fail(RL_INVALID_CALL, "rl_intersect_rays: rays must be 16-byte aligned");
    if (n == 0) return RL_OK;
    k_intersect_rays<<<blocks_for(n, 128), 128, 0, S(stream)>>>(s->dev, n, reinterpret_cast<const float4*>(d_rays),
                                                                any_hit, d_geom_prim, d_t_uv, s->d_status);
    CK_LAUNCH("k_intersect_rays");
    return RL_OK;
}

namespace {
// Per-host-thread staging of rl_intersect_rays_host: its own stream and a
// device buffer that grows to the largest batch seen.
struct IntersectStaging {
    cudaStream_t stream = nullptr;
    char* dev = nullptr;
    size_t cap = 0;
    ~IntersectStaging() {
        if (dev) cudaFree(dev);
        if (stream) cudaStreamDestroy(stream);
    }
};
thread_local IntersectStaging t_staging;
}  // namespace

extern "C" int rl_intersect_rays_host(const rl_scene* s, int64_t n, const float* rays, int any_hit,
                                      int32_t* geom_prim, float* t_uv) {
    if (!s || n < 0 || (n > 0 && (!rays || !geom_prim)))
        return fail(RL_INVALID_CALL, "rl_intersect_rays_host: bad arguments");
    if (n == 0) return RL_OK;
    IntersectStaging& st = t_staging;
    if (!st.stream) CK(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
    const size_t in = 32 * (size_t)n, gp = 8 * (size_t)n, tu = 12 * (size_t)n, need = in + gp + tu;
    if (need > st.cap) {
        if (st.dev) cudaFree(st.dev);
        st.dev = nullptr;
        st.cap = 0;
        CK(cudaMalloc(&st.dev, need));
        st.cap = need;
    }
    float* d_rays = reinterpret_cast<float*>(st.dev);
    int32_t* d_gp = reinterpret_cast<int32_t*>(st.dev + in);
    float* d_tuv = reinterpret_cast<float*>(st.dev + in + gp);
    CK(cudaMemcpyAsync(d_rays, rays, in, cudaMemcpyHostToDevice, st.stream));
    int rc = rl_intersect_rays(s, n, d_rays, any_hit, d_gp, t_uv ? d_tuv : nullptr, st.stream);
    if (rc) return rc;
    CK(cudaMemcpyAsync(geom_prim, d_gp, gp, cudaMemcpyDeviceToHost, st.stream));
    if (t_uv) CK(cudaMemcpyAsync(t_uv, d_tuv, tu, cudaMemcpyDeviceToHost, st.stream));
    CK(cudaStreamSynchronize(st.stream));
    return RL_OK;
}


// ---------------------------------------------------------------- maps

extern "C" int rl_map_create(int kind, int width, int height, rl_map** out) {
    if (!out || width <= 0 || height <= 0 || kind < 0 || kind > 2)
        return fail(RL_INVALID_CALL, "rl_map_create: bad arguments");
    if ((long long)width * height > (1ll << 30)) return fail(RL_INVALID_CALL, "map too large");
    rl_map* m = new (std::nothrow) rl_map;
    if (!m) return fail(RL_OUT_OF_MEMORY, "host allocation failed");
    m->kind = kind;
    m->dev.width = width;
    m->dev.height = height;
    size_t n = (size_t)width * height;
    int rc = RL_OK;
    if (!rc) rc = dalloc(&m->dev.flags, n);
    if (!rc) rc = dalloc(&m->dev.face, n);
    if (!rc) rc = dalloc(&m->dev.position, 3 * n);
    if (!rc) rc = dalloc(&m->dev.normal, 3 * n);
    if (!rc) rc = dalloc(&m->dev.color, 3 * n);
    if (!rc) rc = dalloc(&m->dev.photons, n);
    if (!rc) rc = dalloc(&m->dev.gathered, 3 * n);
    if (!rc) rc = dalloc(&m->dev.mesh, n);
    if (!rc) rc = dalloc(&m->d_owner, n);
    if (!rc) rc = dalloc(&m->d_work, 2);
    if (rc) {
        delete m;
        return rc;
    }
    // Lumel::Lumel (Lightmap.h:52): faceIdx = (Index)-1, photons 0, flags 0, vectors 0
    cudaMemset(m->dev.flags, 0, 4 * n);
    cudaMemset(m->dev.face, 0, 4 * n);
    cudaMemset(m->dev.position, 0, 12 * n);
    cudaMemset(m->dev.normal, 0, 12 * n);
    cudaMemset(m->dev.color, 0, 12 * n);
    cudaMemset(m->dev.photons, 0, 4 * n);
    cudaMemset(m->dev.gathered, 0, 12 * n);
    cudaMemset(m->d_owner, 0xff, 4 * n);
    cudaMemset(m->dev.mesh, 0xff, 4 * n);
    std::vector<int> face(n, 0xffff);
    cudaMemcpy(m->dev.face, face.data(), 4 * n, cudaMemcpyHostToDevice);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        delete m;
        return fail(RL_CUDA_ERROR, "map init: %s", cudaGetErrorString(e));
    }
    *out = m;
    return RL_OK;
}

// The library's stream-ordered memory pool on the current device: lightmap
// blocks and batch tables come from it.  Freed blocks stay in the pool (no
// release at synchronisation points) until rl_pool_trim, so a serving loop
// that admits and retires lightmaps reuses memory without remapping it.
static std::mutex g_pool_mutex;
static cudaMemPool_t g_pool[64];

static int device_pool(cudaMemPool_t* out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(RL_INVALID_CALL, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_pool_mutex);
    if (!g_pool[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        CK(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = UINT64_MAX;
        cudaError_t e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return fail(RL_CUDA_ERROR, "memory pool: %s", cudaGetErrorString(e));
        }
        g_pool[dev] = pool;
    }
    *out = g_pool[dev];
    return RL_OK;
}

static int pool_alloc(void** p, size_t bytes, cudaStream_t st) {
    cudaMemPool_t pool = nullptr;
    if (int rc = device_pool(&pool)) return rc;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, st);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? RL_OUT_OF_MEMORY : RL_CUDA_ERROR, "pool allocation: %s",
                    cudaGetErrorString(e));
    return RL_OK;
}

int rl_internal_pool_alloc(void** p, size_t bytes, cudaStream_t st) { return pool_alloc(p, bytes, st); }

extern "C" int rl_pool_trim(int64_t keep_bytes) {
    cudaMemPool_t pool = nullptr;
    if (int rc = device_pool(&pool)) return rc;
    CK(cudaMemPoolTrimTo(pool, keep_bytes < 0 ? 0 : (size_t)keep_bytes));
    return RL_OK;
}

extern "C" int rl_pool_bytes(int64_t* reserved, int64_t* used) {
    cudaMemPool_t pool = nullptr;
    if (int rc = device_pool(&pool)) return rc;
    uint64_t r = 0, u = 0;
    CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
    CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
    if (reserved) *reserved = (int64_t)r;
    if (used) *used = (int64_t)u;
    return RL_OK;
}

// Lumel::Lumel (Lightmap.h:52) for a map carved from one block.
__global__ void k_map_init(DevMap m, int* owner, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        m.flags[i] = 0;
        m.face[i] = 0xffff;
        m.mesh[i] = -1;
        owner[i] = -1;
        m.photons[i] = 0;
        for (int c = 0; c < 3; c++) {
            m.position[3 * i + c] = 0.f;
            m.normal[3 * i + c] = 0.f;
            m.color[3 * i + c] = 0.f;
            m.gathered[3 * i + c] = 0.f;
        }
    }
}

static size_t map_block_bytes(size_t n, size_t offs[10]) {
    const size_t sz[10] = {4 * n, 4 * n, 4 * n, 12 * n, 12 * n, 12 * n, 4 * n, 12 * n, 4 * n, 16};
    size_t off = 0;
    for (int k = 0; k < 10; k++) {
        offs[k] = off;
        off = (off + sz[k] + 255) & ~(size_t)255;
    }
    return off;
}

extern "C" int rl_map_bytes(int width, int height, int64_t* bytes) {
    if (!bytes || width <= 0 || height <= 0) return fail(RL_INVALID_CALL, "rl_map_bytes: bad arguments");
    size_t offs[10];
    *bytes = (int64_t)map_block_bytes((size_t)width * height, offs);
    return RL_OK;
}

extern "C" int rl_map_create_async(int kind, int width, int height, void* stream, rl_map** out) {
    if (!out || width <= 0 || height <= 0 || kind < 0 || kind > 2)
        return fail(RL_INVALID_CALL, "rl_map_create_async: bad arguments");
    if ((long long)width * height > (1ll << 30)) return fail(RL_INVALID_CALL, "map too large");
    *out = nullptr;
    cudaStream_t st = S(stream);
    size_t n = (size_t)width * height, offs[10];
    size_t bytes = map_block_bytes(n, offs);
    char* blk = nullptr;
    if (int rc = pool_alloc((void**)&blk, bytes, st)) return rc;
    rl_map* m = new (std::nothrow) rl_map;
    if (!m) {
        cudaFreeAsync(blk, st);
        return fail(RL_OUT_OF_MEMORY, "host allocation failed");
    }
    m->kind = kind;
    m->block = blk;
    m->dev.width = width;
    m->dev.height = height;
    m->dev.flags = (int*)(blk + offs[0]);
    m->dev.face = (int*)(blk + offs[1]);
    m->dev.mesh = (int*)(blk + offs[2]);
    m->dev.position = (float*)(blk + offs[3]);
    m->dev.normal = (float*)(blk + offs[4]);
    m->dev.color = (float*)(blk + offs[5]);
    m->dev.photons = (int*)(blk + offs[6]);
    m->dev.gathered = (float*)(blk + offs[7]);
    m->d_owner = (int*)(blk + offs[8]);
    m->d_work = (unsigned long long*)(blk + offs[9]);
    int grid = (int)std::min<long long>(((long long)n + 255) / 256, 148 * 16);
    k_map_init<<<grid, 256, 0, st>>>(m->dev, m->d_owner, (long long)n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        m->block = nullptr;
        m->dev = DevMap{};
        m->d_owner = nullptr;
        m->d_work = nullptr;
        cudaFreeAsync(blk, st);
        delete m;
        return fail(RL_CUDA_ERROR, "k_map_init: %s", cudaGetErrorString(e));
    }
    *out = m;
    return RL_OK;
}

extern "C" int rl_map_destroy_async(rl_map* m, void* stream) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    if (!m->block) return fail(RL_INVALID_CALL, "rl_map_destroy_async: map was not made by rl_map_create_async");
    cudaError_t e = cudaFreeAsync(m->block, S(stream));
    m->block = nullptr;
    m->dev = DevMap{};
    m->d_owner = nullptr;
    m->d_work = nullptr;
    delete m;
    if (e != cudaSuccess) return fail(RL_CUDA_ERROR, "map free: %s", cudaGetErrorString(e));
    return RL_OK;
}

extern "C" int rl_map_destroy(rl_map* m) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    cudaDeviceSynchronize();
    delete m;
    return RL_OK;
}

// Face::isUvInside (scene/Mesh.cpp:415-438).
__device__ __forceinline__ bool uv_inside(float2 a, float2 b, float2 c, float2 uv, float& bu, float& bv) {
    float v0x = c.x - a.x, v0y = c.y - a.y;
    float v1x = b.x - a.x, v1y = b.y - a.y;
    float v2x = uv.x - a.x, v2y = uv.y - a.y;
    float dot00 = v0x * v0x + v0y * v0y;
    float dot01 = v0x * v1x + v0y * v1y;
    float dot02 = v0x * v2x + v0y * v2y;
    float dot11 = v1x * v1x + v1y * v1y;
    float dot12 = v1x * v2x + v1y * v2y;
    float invDenom = 1.0f / (dot00 * dot11 - dot01 * dot01);
    float u = (dot11 * dot02 - dot01 * dot12) * invDenom;
    float v = (dot00 * dot12 - dot01 * dot02) * invDenom;
    bu = u;
    bv = v;
    return (u >= 0.0f) && (v >= 0.0f) && (u + v < 1.0f);
}

__device__ __forceinline__ float2 ld2(const float* p) { return make_float2(p[0], p[1]); }

// Lightmap::initializeLumels(face) loop bounds (Lightmap.cpp:118-141): the
// face's uv rectangle scaled by the map size, clamped to the map.
__device__ __forceinline__ void face_rect(float2 a, float2 b, float2 c, int W, int H, int& u0, int& v0, int& u1,
                                          int& v1) {
    float minx = fminf(a.x, fminf(b.x, c.x)), maxx = fmaxf(a.x, fmaxf(b.x, c.x));
    float miny = fminf(a.y, fminf(b.y, c.y)), maxy = fmaxf(a.y, fmaxf(b.y, c.y));
    u0 = (int)(minx * W); u1 = (int)(maxx * W);
    v0 = (int)(miny * H); v1 = (int)(maxy * H);
    u1 = u1 < W - 1 ? u1 : W - 1;
    v1 = v1 < H - 1 ? v1 : H - 1;
    u0 = u0 < 0 ? 0 : u0;
    v0 = v0 < 0 ? 0 : v0;
}

// Pass 1: each face claims the texels whose centre it covers; the largest
// face index wins, as the reference's in-order loop lets the last face win.
__global__ void k_raster_owner(DevScene s, int t0, int t1, int W, int H, int* owner) {
    int t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= t1) return;
    int4 f = s.tri_vidx[t];
    float2 a = ld2(s.uv1 + 2 * f.x), b = ld2(s.uv1 + 2 * f.y), c = ld2(s.uv1 + 2 * f.z);
    int u0, v0, u1, v1;
    face_rect(a, b, c, W, H, u0, v0, u1, v1);
    for (int v = v0; v <= v1; v++)
        for (int u = u0; u <= u1; u++) {
            float2 uv = make_float2((u + 0.5f) / (float)W, (v + 0.5f) / (float)H);
            float bu, bv;
            if (uv_inside(a, b, c, uv, bu, bv)) atomicMax(&owner[v * W + u], t - t0);
        }
}

// Pass 2: Lightmap::initializeLumel (Lightmap.cpp:157-164) for the winner.
__global__ void k_raster_init(DevScene s, int mesh, int t0, DevMap m, int* owner) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int W = m.width, H = m.height;
    if (i >= W * H) return;
    int fl = owner[i];
    if (fl < 0) return;
    owner[i] = -1;
    int4 f = s.tri_vidx[t0 + fl];
    float2 a = ld2(s.uv1 + 2 * f.x), b = ld2(s.uv1 + 2 * f.y), c = ld2(s.uv1 + 2 * f.z);
    int u = i % W, v = i / W;
    float2 uv = make_float2((u + 0.5f) / (float)W, (v + 0.5f) / (float)H);
    float bu, bv;
    uv_inside(a, b, c, uv, bu, bv);
    m.face[i] = fl & 0xffff;
    m.mesh[i] = mesh;
    st3(m.position + 3 * (size_t)i, interp3(s.pos, f, bu, bv));
    st3(m.normal + 3 * (size_t)i, interp3(s.nrm, f, bu, bv));
    st3(m.color + 3 * (size_t)i, mk3(0.f, 0.f, 0.f));
    m.flags[i] |= 1;
}

extern "C" int rl_map_add_mesh(rl_map* m, const rl_scene* s, int mesh, void* stream) {
    if (!m || !s) return fail(RL_INVALID_CALL, "rl_map_add_mesh: null argument");
    if (mesh < 0 || mesh >= s->nmeshes) return fail(RL_INVALID_CALL, "rl_map_add_mesh: mesh %d out of range", mesh);
    int t0 = s->mesh_first_tri[mesh], t1 = s->mesh_first_tri[mesh + 1];
    if (t1 <= t0) return fail(RL_INVALID_CALL, "rl_map_add_mesh: mesh %d has no faces", mesh);
    cudaStream_t st = S(stream);
    k_raster_owner<<<blocks_for(t1 - t0, 128), 128, 0, st>>>(s->dev, t0, t1, m->dev.width, m->dev.height,
                                                            m->d_owner);
    CK_LAUNCH("k_raster_owner");
    long long n = (long long)m->dev.width * m->dev.height;
    k_raster_init<<<blocks_for(n, 256), 256, 0, st>>>(s->dev, mesh, t0, m->dev, m->d_owner);
    CK_LAUNCH("k_raster_init");
    return RL_OK;
}

extern "C" int rl_map_download(const rl_map* m, int32_t* flags, int32_t* face, float* position, float* normal,
                               float* color, int32_t* photons, float* gathered, void* stream) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    cudaStream_t st = S(stream);
    size_t n = (size_t)m->dev.width * m->dev.height;
    if (flags) CK(cudaMemcpyAsync(flags, m->dev.flags, 4 * n, cudaMemcpyDeviceToHost, st));
    if (face) CK(cudaMemcpyAsync(face, m->dev.face, 4 * n, cudaMemcpyDeviceToHost, st));
    if (position) CK(cudaMemcpyAsync(position, m->dev.position, 12 * n, cudaMemcpyDeviceToHost, st));
    if (normal) CK(cudaMemcpyAsync(normal, m->dev.normal, 12 * n, cudaMemcpyDeviceToHost, st));
    if (color) CK(cudaMemcpyAsync(color, m->dev.color, 12 * n, cudaMemcpyDeviceToHost, st));
    if (photons) CK(cudaMemcpyAsync(photons, m->dev.photons, 4 * n, cudaMemcpyDeviceToHost, st));
    if (gathered) CK(cudaMemcpyAsync(gathered, m->dev.gathered, 12 * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return RL_OK;
}

extern "C" int rl_map_download_async(const rl_map* m, float* color, void* stream) {
    if (!m || !color) return fail(RL_INVALID_CALL, "rl_map_download_async: null argument");
    size_t n = (size_t)m->dev.width * m->dev.height;
    CK(cudaMemcpyAsync(color, m->dev.color, 12 * n, cudaMemcpyDeviceToHost, S(stream)));
    return RL_OK;
}

extern "C" int rl_map_upload(rl_map* m, const int32_t* flags, const int32_t* face, const float* position,
                             const float* normal, const float* color, const int32_t* photons, const float* gathered,
                             void* stream) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    cudaStream_t st = S(stream);
    size_t n = (size_t)m->dev.width * m->dev.height;
    if (flags) CK(cudaMemcpyAsync(m->dev.flags, flags, 4 * n, cudaMemcpyHostToDevice, st));
    if (face) CK(cudaMemcpyAsync(m->dev.face, face, 4 * n, cudaMemcpyHostToDevice, st));
    if (position) CK(cudaMemcpyAsync(m->dev.position, position, 12 * n, cudaMemcpyHostToDevice, st));
    if (normal) CK(cudaMemcpyAsync(m->dev.normal, normal, 12 * n, cudaMemcpyHostToDevice, st));
    if (color) CK(cudaMemcpyAsync(m->dev.color, color, 12 * n, cudaMemcpyHostToDevice, st));
    if (photons) CK(cudaMemcpyAsync(m->dev.photons, photons, 4 * n, cudaMemcpyHostToDevice, st));
    if (gathered) CK(cudaMemcpyAsync(m->dev.gathered, gathered, 12 * n, cudaMemcpyHostToDevice, st));
    return RL_OK;
}

extern "C" int rl_map_clear(rl_map* m, int colors, int photons, void* stream) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    cudaStream_t st = S(stream);
    size_t n = (size_t)m->dev.width * m->dev.height;
    if (colors) CK(cudaMemsetAsync(m->dev.color, 0, 12 * n, st));
    if (photons) {
        CK(cudaMemsetAsync(m->dev.photons, 0, 4 * n, st));
        CK(cudaMemsetAsync(m->dev.gathered, 0, 12 * n, st));
        if (!colors) CK(cudaMemsetAsync(m->dev.color, 0, 12 * n, st));
    }
    return RL_OK;
}

extern "C" int rl_map_device_arrays(const rl_map* m, int32_t** flags, float** position, float** normal,
                                    float** color, int32_t** photons, float** gathered) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    if (flags) *flags = m->dev.flags;
    if (position) *position = m->dev.position;
    if (normal) *normal = m->dev.normal;
    if (color) *color = m->dev.color;
    if (photons) *photons = m->dev.photons;
    if (gathered) *gathered = m->dev.gathered;
    return RL_OK;
}

extern "C" int rl_map_valid_count(const rl_map* m, int64_t* count) {
    if (!m || !count) return fail(RL_INVALID_CALL, "null argument");
    size_t n = (size_t)m->dev.width * m->dev.height;
    std::vector<int> f(n);
    CK(cudaMemcpy(f.data(), m->dev.flags, 4 * n, cudaMemcpyDeviceToHost));
    int64_t c = 0;
    for (size_t i = 0; i < n; i++) c += f[i] & 1;
    *count = c;
    return RL_OK;
}

// ---------------------------------------------------------- light tables

constexpr int kMaxLights = 64;
constexpr int kMaxLightVerts = 1024;
constexpr int kMaxPhotonmaps = 64;

// Lights and area-light sample points, passed to kernels by value
// (__grid_constant__), so a bake call needs no device copy of host tables.
struct LightTable {
    int n;
    int nverts;
    rl_light l[kMaxLights];
    float verts[3 * kMaxLightVerts];
};

static int make_light_table(const rl_light* lights, int nlights, const float* lverts, int nverts, LightTable& T,
                            bool use_vertices = true) {
    if (nlights < 0 || nlights > kMaxLights) return fail(RL_INVALID_CALL, "at most %d lights per call", kMaxLights);
    if (nverts < 0 || nverts > kMaxLightVerts)
        return fail(RL_INVALID_CALL, "at most %d light vertices per call", kMaxLightVerts);
    if (nlights > 0 && !lights) return fail(RL_INVALID_CALL, "null light array");
    if (nverts > 0 && !lverts) return fail(RL_INVALID_CALL, "null light-vertex array");
    memset(&T, 0, sizeof T);
    T.n = nlights;
    T.nverts = nverts;
    for (int l = 0; l < nlights; l++) {
        T.l[l] = lights[l];
        if (!use_vertices) {
            // photon emission starts at the light's position only
            // (PhotonEmitter::emit, scene/Light.cpp:340-344)
            T.l[l].vertex_first = T.l[l].vertex_count = 0;
            continue;
        }
        if (lights[l].vertex_count > 0 &&
            (lights[l].vertex_first < 0 || lights[l].vertex_first + lights[l].vertex_count > nverts))
            return fail(RL_INVALID_CALL, "light %d: vertex range outside the light-vertex pool", l);
    }
    if (nverts) memcpy(T.verts, lverts, 12 * (size_t)nverts);
    return RL_OK;
}

// ---------------------------------------------------------- direct light

// LightSpotCutoff::cutoffForDirection (scene/Light.cpp:461-476).
__device__ __forceinline__ float spot_cutoff(const rl_light& L, V3 direction) {
    float value = dot3(direction, ld3(L.spot_direction));
    if (value <= L.spot_cutoff) return 0.0f;
    value = (1.0f - (1.0f - value) * 1.0f / (1.0f - L.spot_cutoff));
    if (fabsf(1.0f - L.spot_exponent) > 0.01f) value = powf(value, L.spot_exponent);
    return value;
}

__device__ __forceinline__ float lambert(V3 dir, V3 n) {
    float dp = dot3(dir, n);
    return dp < 0.0f ? 0.0f : dp;
}

// DirectLight::influenceFromPoint (baker/DirectLight.cpp:101-125) with the
// light's influence, cutoff and attenuation models (scene/Light.cpp:372-500).
__device__ float influence_from_point(const DevScene& s, V3 lpos, V3 lnrm, V3 point, const rl_light& L,
                                      int* status) {
    float inf = 0.0f, att = 1.0f, cut = 1.0f, distance = 0.0f;
    if (L.influence == 1) {
        V3 direction = sub3(point, lpos);
        distance = normalize3(direction);
        float intensity = lambert(direction, lnrm);
        if (intensity <= 0.001f) {
            inf = 0.0f;
        } else {
            if (L.casts_shadow) intensity *= segment_blocked(s, lpos, point, kHitUseAlpha, status) ? 0.0f : 1.0f;
            inf = intensity;
        }
    } else if (L.influence == 2) {
        V3 ldir = ld3(L.direction);
        float intensity = lambert(neg3(ldir), lnrm);
        if (intensity <= 0.001f) {
            inf = 0.0f;
        } else {
            if (L.casts_shadow)
                intensity *= segment_blocked(s, lpos, sub3(lpos, mul3(ldir, 1000.0f)), kHitUseAlpha, status) ? 0.0f
                                                                                                           : 1.0f;
            inf = intensity;
        }
    }
    if (L.cutoff == 2) {
        V3 dir = sub3(lpos, ld3(L.position));
        normalize3(dir);
        cut = spot_cutoff(L, dir);
    }
    if (L.attenuation) {
        float r = distance / L.att_radius;
        float a = 1.0f / (1.0f + L.att_const + L.att_linear * r + L.att_quadratic * r * r);
        att = a > 0.0f ? a : 0.0f;
    }
    return inf * att * cut;
}

// DirectLight::bakeLumel (baker/DirectLight.cpp:46-98) for lumel i.
__device__ void direct_lumel(const DevScene& s, const DevMap& m, const LightTable& T, long long i, int* status) {
    V3 pos = ld3(m.position + 3 * i), nrm = ld3(m.normal + 3 * i);
    float* col = m.color + 3 * i;
    float cr = col[0], cg = col[1], cb = col[2];
    for (int l = 0; l < T.n; l++) {
        const rl_light& L = T.l[l];
        V3 lc = ld3(L.color);
        V3 infl = mk3(0.f, 0.f, 0.f);
        if (L.vertex_count > 0) {
            V3 acc = mk3(0.f, 0.f, 0.f);
            for (int v = 0; v < L.vertex_count; v++) {
                V3 vp = ld3(T.verts + 3 * (L.vertex_first + v));
                float inf = influence_from_point(s, pos, nrm, add3(vp, ld3(L.position)), L, status);
                if (inf > 0.0f) acc = add3(acc, mul3(mul3(lc, L.intensity), inf));
            }
            float n = (float)L.vertex_count;
            infl = mk3(acc.x / n, acc.y / n, acc.z / n);
        } else {
            float inf = influence_from_point(s, pos, nrm, ld3(L.position), L, status);
            if (inf > 0.0f) infl = mul3(mul3(lc, L.intensity), inf);
        }
        cr = cr + infl.x; cg = cg + infl.y; cb = cb + infl.z;
    }
    col[0] = cr; col[1] = cg; col[2] = cb;
}

// One thread per visited lumel.
__global__ void k_direct(DevScene s, DevMap m, const __grid_constant__ LightTable T, Iter it, long long count,
                         int* status) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= count) return;
    long long i;
    if (!iter_lumel(m, it, k, i)) return;
    direct_lumel(s, m, T, i, status);
}

// Validate an rl_iterator (NULL = LumelBakeIterator(0, 1)) and size the
// launch: one thread per visited lumel (kind 0) or per lumel (kind 1).
static int make_iter(const rl_iterator* it, const rl_scene* s, long long n, Iter& out, long long& count) {
    Iter d{0, 0, 1, -1};
    if (it) d = Iter{it->kind, it->first, it->step, it->mesh};
    if (d.kind < 0 || d.kind > 1 || d.first < 0 || d.step <= 0)
        return fail(RL_INVALID_CALL, "bad iterator (kind %d first %d step %d)", d.kind, d.first, d.step);
    if (d.kind == 1 && (d.mesh < 0 || d.mesh >= s->nmeshes))
        return fail(RL_INVALID_CALL, "face iterator: mesh %d out of range", d.mesh);
    out = d;
    if (d.kind == 1) count = n;
    else count = d.first >= n ? 0 : (n - d.first + d.step - 1) / d.step;
    return RL_OK;
}

// A whole-map lumel iteration (LumelBakeIterator(0, 1)) runs in 8x8 lumel
// tiles (iterator kind 2): the same lumels, each baked by one thread, with
// neighbouring lumels in one warp.  The final gather measured 51.0 -> 48.8 ms
// on the terrain bench (its rays start closer together).  Other iterators
// keep their order.
static void tile_whole_map(Iter& it, long long& count, const DevMap& m) {
    if (it.kind != 0 || it.first != 0 || it.step != 1 || count != (long long)m.width * m.height) return;
    const long long tx = (m.width + 7) / 8, ty = (m.height + 7) / 8;
    it.kind = 2;
    it.first = (int)tx;
    count = tx * ty * 64;
}

extern "C" int rl_bake_direct(const rl_scene* s, rl_map* lm, const rl_light* lights, int nlights,
                              const float* light_vertices, int nlight_vertices, const rl_iterator* iterator,
                              void* stream) {
    if (!s || !lm) return fail(RL_INVALID_CALL, "rl_bake_direct: null argument");
    static thread_local LightTable T;
    int rc = make_light_table(lights, nlights, light_vertices, nlight_vertices, T);
    if (rc) return rc;
    long long n = (long long)lm->dev.width * lm->dev.height, count = 0;
    Iter it;
    rc = make_iter(iterator, s, n, it, count);
    if (rc) return rc;
    if (count == 0 || nlights == 0) return RL_OK;
    tile_whole_map(it, count, lm->dev);
    k_direct<<<blocks_for(count, 128), 128, 0, S(stream)>>>(s->dev, lm->dev, T, it, count, s->d_status);
    CK_LAUNCH("k_direct");
    return RL_OK;
}

// Blocks of `threads` that fit on the device at once for `kernel`
// (persistent grids), cached per kernel and block size.
template <typename K>
static int resident_blocks(K kernel, int threads) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> cache;
    std::lock_guard<std::mutex> g(mu);
    const auto key = std::make_pair((const void*)kernel, threads);
    auto f = cache.find(key);
    if (f != cache.end()) return f->second;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm <= 0)
        return 0;
    return cache[key] = sms * per_sm;
}

// ------------------------------------------------------------------ AO

// AmbientOcclusion::bakeLumel (baker/AmbientOcclusion.cpp:46-66): the
// lumel's samples as one lane's ray stream (first-hit rays).
struct AoGen {
    V3 pos, nrm;
    uint2 key;
    uint32_t item;
    int j, stride, samples, occluded;
    float maxd;
    __device__ bool next(V3& o, V3& d, float& tnear, float& tfar) {
        if (j >= samples) return false;
        V3 dir = random_hemisphere(nrm, key, item, (uint32_t)j, kTagAO);
        segment_ray(pos, dir, maxd, o, d, tnear, tfar);
        j += stride;
        return true;
    }
    __device__ void finish(const RayHit& h) {
        if (h.gid >= 0) occluded++;
    }
};

// `split` (a power of two, at most 8) adjacent lanes share one lumel: lane
// part takes samples part, part + split, ...  The occlusion count is an
// integer, so adding the lanes' counts gives the same value as one lane's
// loop.  `count` is lumels x split, so lanes past it leave in whole groups.
template <int kWidth>
__global__ void __launch_bounds__(256) k_ao(DevScene s, DevMap m, int samples, float fraction, float maxd,
                                            float exponent, uint2 key, Iter it, long long count, int split,
                                            int refill, int* status) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const unsigned live = __ballot_sync(0xffffffffu, k < count);  // whole groups of `split` lanes
    if (k >= count) return;
    const int part = (int)(k & (split - 1));
    long long i;
    bool valid = iter_lumel(m, it, k / split, i);
    AoGen g;
    g.pos = ld3(m.position + 3 * i);
    g.nrm = ld3(m.normal + 3 * i);
    g.key = key;
    g.item = (uint32_t)i;
    g.j = part;
    g.stride = split;
    g.samples = valid ? samples : 0;
    g.occluded = 0;
    g.maxd = maxd;
    if (kWidth == 8) ray_loop8<true>(s, g, refill, status);
    else if (kWidth == 4) ray_loop4<true>(s, g, refill, status);
    else if (kWidth == 3) ray_loop_spec<true>(s, g, refill, status);
    else ray_loop<true>(s, g, refill, status);
    if (split > 1)
        for (int o = 1; o < split; o <<= 1) g.occluded += __shfl_xor_sync(live, g.occluded, o);
    if (!valid || part != 0) return;
    float value = 1.0f - g.occluded / (samples * fraction);
    if (fabsf(1.0f - exponent) > 0.01f) value = powf(value, exponent);
    float* col = m.color + 3 * i;
    col[0] = col[0] * value; col[1] = col[1] * value; col[2] = col[2] * value;
}

// AoGen over a work list of lumels (ray_loop_pool): lumel item k of the
// iteration (items k_begin + k, k < limit), its samples in order, its colour
// scaled when its last sample is counted — the same arithmetic as k_ao.
struct AoPoolGen : AoGen {
    const DevMap* map;
    const Iter* it;
    int nsamples;
    float fraction, exponent;
    long long li, k_begin, limit;
    __device__ bool has_more() const { return j < samples; }
    __device__ void end_item() {
        if (samples == 0) return;
        float value = 1.0f - occluded / (samples * fraction);
        if (fabsf(1.0f - exponent) > 0.01f) value = powf(value, exponent);
        float* col = map->color + 3 * li;
        col[0] = col[0] * value; col[1] = col[1] * value; col[2] = col[2] * value;
        samples = 0;
    }
    __device__ bool start_item(long long k) {
        long long i;
        if (k >= limit || !iter_lumel(*map, *it, k_begin + k, i)) return false;
        li = i;
        pos = ld3(map->position + 3 * i);
        nrm = ld3(map->normal + 3 * i);
        item = (uint32_t)i;
        j = 0;
        samples = nsamples;
        occluded = 0;
        return true;
    }
};

// Persistent AO over a whole-lumel work list (one lane per lumel at a time,
// lanes refilled from their warp's pool), for maps that need no lane split.
__global__ void __launch_bounds__(256, 4) k_ao_pool(DevScene s, const __grid_constant__ DevMap m, int samples,
                                                    float fraction, float maxd, float exponent, uint2 key,
                                                    const __grid_constant__ Iter it, long long count, int refill,
                                                    int* status, unsigned long long* counter, int chunk) {
    AoPoolGen g;
    g.map = &m;
    g.it = &it;
    g.nsamples = samples;
    g.fraction = fraction;
    g.exponent = exponent;
    g.li = 0;
    g.k_begin = 0;
    g.limit = count;
    g.pos = g.nrm = mk3(0.f, 0.f, 0.f);
    g.key = key;
    g.item = 0;
    g.j = 0;
    g.stride = 1;
    g.samples = 0;
    g.occluded = 0;
    g.maxd = maxd;
    CounterSource src{counter, count, chunk};
    ray_loop_pool<true>(s, g, refill, status, src);
}

extern "C" int rl_bake_ao(const rl_scene* s, rl_map* lm, int samples, float fraction, float maxd, float exponent,
                          uint64_t seed, const rl_iterator* iterator, void* stream) {
    if (!s || !lm) return fail(RL_INVALID_CALL, "rl_bake_ao: null argument");
    if (samples <= 0) return fail(RL_INVALID_CALL, "rl_bake_ao: samples must be positive");
    long long n = (long long)lm->dev.width * lm->dev.height, count = 0;
    Iter it;
    int rc = make_iter(iterator, s, n, it, count);
    if (rc) return rc;
    if (count == 0) return RL_OK;
    tile_whole_map(it, count, lm->dev);
    // Small maps leave most of the GPU idle with one lane per lumel: share
    // each lumel's samples between up to 8 lanes while the launch stays
    // within about two waves of resident threads (RL_TUNE_AO_SPLIT forces it).
    int split = g_tune[RL_TUNE_AO_SPLIT];
    if (split == 0) {
        static int sms = 0;
        if (sms == 0) {
            int dev = 0;
            CK(cudaGetDevice(&dev));
            CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        }
        split = 1;
        while (split < 8 && split * 2 <= samples && count * split * 2 <= 2LL * sms * 2048) split *= 2;
    }
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    int bs = g_tune[RL_TUNE_AO_BLOCK];
    bool wide = g_tune[RL_TUNE_BVH_WIDTH] == 4 && s->dev.nodes4 != nullptr;
    bool wide8 = g_tune[RL_TUNE_BVH_WIDTH] == 8 && s->dev.nodes8 != nullptr;
    if (split == 1 && g_tune[RL_TUNE_FG_POOL] && !wide && !wide8 && !g_tune[RL_TUNE_SPECULATIVE]) {
        const int resident = resident_blocks(k_ao_pool, bs);
        if (resident <= 0) return fail(RL_CUDA_ERROR, "k_ao_pool: occupancy query failed");
        const long long want = ((long long)count + bs - 1) / bs;
        const unsigned grid = (unsigned)(want < resident ? want : resident);
        CK(cudaMemsetAsync(lm->d_work, 0, sizeof(unsigned long long), S(stream)));
        k_ao_pool<<<grid, bs, 0, S(stream)>>>(s->dev, lm->dev, samples, fraction, maxd, exponent, key, it, count,
                                              g_tune[RL_TUNE_AO_REFILL], s->d_status, lm->d_work,
                                              g_tune[RL_TUNE_FG_CHUNK]);
        CK_LAUNCH("k_ao_pool");
        return RL_OK;
    }
    auto kern = wide8 ? k_ao<8> : wide ? k_ao<4> : (g_tune[RL_TUNE_SPECULATIVE] ? k_ao<3> : k_ao<2>);
    kern<<<blocks_for(count * split, bs), bs, 0, S(stream)>>>(s->dev, lm->dev, samples, fraction, maxd, exponent,
                                                              key, it, count * split, split,
                                                              g_tune[RL_TUNE_AO_REFILL], s->d_status);
    CK_LAUNCH("k_ao");
    return RL_OK;
}

// -------------------------------------------------------------- photons

struct PhotonTables {
    int nl;                       // lights with an emitter, in scene order
    int light[kMaxLights];        // light index of emitter slot e
    unsigned prefix[kMaxLights + 1];  // photon offsets within one pass
    unsigned per_pass;
    int nmaps;
    DevMap maps[kMaxPhotonmaps];
};

// Photons::emit -> emitPhotons -> trace -> store (baker/Photons.cpp:50-144),
// one thread per photon; photon p is the p-th iteration of the reference's
// pass / light / photon loops.
__global__ void k_photons(DevScene s, const __grid_constant__ LightTable LT, const __grid_constant__ PhotonTables T,
                          unsigned first, unsigned total, int max_depth, float threshold, float maxd, uint2 key,
                          unsigned long long* stored, PhotonSink sink, int* status) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    unsigned p = first + t;
    unsigned r = p % T.per_pass;
    int e = 0;
    while (e + 1 < T.nl && T.prefix[e + 1] <= r) e++;
    const rl_light& L = LT.l[T.light[e]];
    V3 pos, dir;
    if (L.emitter == 1) {
        // PhotonEmitter::emit (scene/Light.cpp:340-344)
        pos = ld3(L.position);
        dir = random_direction(key, p, 0, kTagEmit);
    } else {
        // DirectionalPhotonEmitter::emit (scene/Light.cpp:355-361)
        uint4 q = philox(make_uint4(p, 0, 0, kTagEmitPoint), key);
        float s0 = u01(q.x), s1 = u01(q.y), s2 = u01(q.z);
        V3 pt = mk3(s.bounds_lo[0] * (1.0f - s0) + s.bounds_hi[0] * s0, s.bounds_lo[1] * (1.0f - s1) + s.bounds_hi[1] * s1,
                    s.bounds_lo[2] * (1.0f - s2) + s.bounds_hi[2] * s2);
        V3 pn = ld3(L.emitter_plane);
        float dist = dot3(pn, pt) + L.emitter_plane[3];
        V3 onplane = sub3(pt, mul3(pn, dist));
        dir = ld3(L.direction);
        pos = sub3(onplane, mul3(dir, 5.0f));
    }
    float cut = 1.0f;
    if (L.cutoff == 2) cut = spot_cutoff(L, dir);
    if (cut <= 0.0f) return;
    V3 col = mul3(mul3(ld3(L.color), L.intensity), cut);
    for (int depth = 0;; depth++) {
        if (depth > max_depth || (0.2126f * col.x + 0.7152f * col.y + 0.0722f * col.z) < threshold) break;
        SegHit h;
        trace_segment(s, pos, add3(pos, mul3(dir, maxd)), kHitPoint | kHitUv | kHitColor | kHitNormal, h, status);
        if (!h.hit) break;
        float influence = lambert(neg3(dir), h.normal) * 1.0f;
        V3 hc = mul3(mk3(col.x * h.rgba.x, col.y * h.rgba.y, col.z * h.rgba.z), influence);
        int slot = s.mesh_photonmap[h.mesh];
        if (slot >= 0 && slot < T.nmaps) {
            const DevMap& P = T.maps[slot];
            int ti = lumel_at_uv(P.width, P.height, h.uv);
            if (P.flags[ti] & 1) {
                atomicAdd(P.color + 3 * ti, hc.x);
                atomicAdd(P.color + 3 * ti + 1, hc.y);
                atomicAdd(P.color + 3 * ti + 2, hc.z);
                atomicAdd(P.photons + ti, 1);
                if (stored) atomicAdd(stored, 1ull);
                if (sink.rec) {  // the same deposit as a world-space record
                    unsigned long long q = atomicAdd(sink.count, 1ull);
                    if (q < sink.capacity)
                        sink.rec[q] = PhotonRecord{h.point.x, h.point.y, h.point.z, hc.x, hc.y, hc.z, p,
                                                   (uint16_t)depth, (uint16_t)slot};
                }
            }
        }
        dir = random_hemisphere(h.normal, key, p, (uint32_t)(depth + 1), kTagBounce);
        pos = h.point;
        col = hc;
    }
}

static int emit_photons(const rl_scene* s, rl_map* const* maps, int nmaps, const rl_light* lights, int nlights,
                        int pass_count, int max_depth, float threshold, float maxd, uint64_t seed, int64_t first_photon,
                        int64_t photon_count, int64_t* stored, void* stream, rl_photons* records = nullptr) {
    if (!s || (nmaps > 0 && !maps)) return fail(RL_INVALID_CALL, "rl_emit_photons: null argument");
    if (nmaps > kMaxPhotonmaps) return fail(RL_INVALID_CALL, "rl_emit_photons: at most %d photonmaps", kMaxPhotonmaps);
    cudaStream_t st = S(stream);
    static thread_local LightTable LT;
    int rc = make_light_table(lights, nlights, nullptr, 0, LT, false);
    if (rc) return rc;
    static thread_local PhotonTables T;
    memset(&T, 0, sizeof T);
    unsigned long long per_pass = 0;
    for (int l = 0; l < nlights; l++) {
        if (!lights[l].emitter) continue;
        // PhotonEmitter::photonCount (scene/Light.cpp:334-337)
        int cnt = (int)(lights[l].intensity * 25000);
        T.light[T.nl] = l;
        T.prefix[T.nl] = (unsigned)per_pass;
        per_pass += (unsigned long long)std::max(cnt, 0);
        T.nl++;
    }
    T.prefix[T.nl] = (unsigned)per_pass;
    T.per_pass = (unsigned)per_pass;
    T.nmaps = nmaps;
    for (int k = 0; k < nmaps; k++) {
        if (!maps[k]) return fail(RL_INVALID_CALL, "photonmap %d is null", k);
        T.maps[k] = maps[k]->dev;
    }
    unsigned long long all = per_pass * (unsigned long long)std::max(pass_count, 0);
    if (all >= (1ull << 32)) return fail(RL_INVALID_CALL, "too many photons (%llu)", all);
    if (stored) *stored = 0;
    unsigned long long first = first_photon < 0 ? 0 : (unsigned long long)first_photon;
    unsigned long long total = photon_count < 0 ? all : (unsigned long long)photon_count;
    if (first > all) first = all;
    if (first + total > all) total = all - first;
    if (total == 0) return RL_OK;
    Scratch sc;
    unsigned long long* dc = nullptr;
    if (stored) {
        rc = scratch(sc, &dc, 1, st);
        if (rc) return rc;
        CK(cudaMemsetAsync(dc, 0, 8, st));
    }
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    PhotonSink sink{nullptr, nullptr, 0};
    if (records) {
        rc = rl_internal_photon_sink(records, &sink, st);
        if (rc) return rc;
    }
    k_photons<<<blocks_for((long long)total, 128), 128, 0, st>>>(s->dev, LT, T, (unsigned)first, (unsigned)total,
                                                                max_depth, threshold, maxd, key, dc, sink,
                                                                s->d_status);
    CK_LAUNCH("k_photons");
    if (stored) {
        unsigned long long h = 0;
        CK(cudaMemcpyAsync(&h, dc, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        *stored = (int64_t)h;
    }
    return RL_OK;
}

extern "C" int rl_emit_photons(const rl_scene* s, rl_map* const* maps, int nmaps, const rl_light* lights,
                               int nlights, int pass_count, int max_depth, float threshold, float maxd, uint64_t seed,
                               int64_t* stored, void* stream) {
    return emit_photons(s, maps, nmaps, lights, nlights, pass_count, max_depth, threshold, maxd, seed, 0, -1, stored,
                        stream);
}

extern "C" int rl_emit_photons_records(const rl_scene* s, rl_map* const* maps, int nmaps, const rl_light* lights,
                                       int nlights, int pass_count, int max_depth, float threshold, float maxd,
                                       uint64_t seed, rl_photons* records, int64_t* stored, void* stream) {
    if (!records) return fail(RL_INVALID_CALL, "rl_emit_photons_records: null record buffer");
    return emit_photons(s, maps, nmaps, lights, nlights, pass_count, max_depth, threshold, maxd, seed, 0, -1, stored,
                        stream, records);
}

extern "C" int rl_emit_photons_range(const rl_scene* s, rl_map* const* maps, int nmaps, const rl_light* lights,
                                     int nlights, int pass_count, int max_depth, float threshold, float maxd,
                                     uint64_t seed, int64_t first_photon, int64_t photon_count, int64_t* stored,
                                     void* stream) {
    if (first_photon < 0 || photon_count < 0) return fail(RL_INVALID_CALL, "rl_emit_photons_range: negative range");
    return emit_photons(s, maps, nmaps, lights, nlights, pass_count, max_depth, threshold, maxd, seed, first_photon,
                        photon_count, stored, stream);
}

extern "C" int rl_photon_count(const rl_light* lights, int nlights, int pass_count, int64_t* total) {
    if (!total || (nlights > 0 && !lights)) return fail(RL_INVALID_CALL, "rl_photon_count: null argument");
    long long per_pass = 0;
    for (int l = 0; l < nlights; l++)
        if (lights[l].emitter) per_pass += std::max((int)(lights[l].intensity * 25000), 0);
    *total = per_pass * (long long)std::max(pass_count, 0);
    return RL_OK;
}

// Photonmap::gather (Lightmap.cpp:376-413): mean photon colour over the disc
// of `radius` texels, for y < height and x < height (the loop bound of :379).
__global__ void k_gather(DevMap m, int radius) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    int W = m.width, H = m.height;
    if (x >= H || y >= H) return;
    long long o = (long long)y * W + x;
    if (o >= (long long)W * H) return;
    float cr = 0.f, cg = 0.f, cb = 0.f;
    int photons = 0;
    for (int j = y - radius; j <= y + radius; j++) {
        for (int i = x - radius; i <= x + radius; i++) {
            if (i < 0 || j < 0 || i >= W || j >= H) continue;
            float distance = sqrtf((float)((x - i) * (x - i) + (y - j) * (y - j)));
            if (distance > radius) continue;
            long long li = (long long)j * W + i;
            cr = cr + m.color[3 * li]; cg = cg + m.color[3 * li + 1]; cb = cb + m.color[3 * li + 2];
            photons += m.photons[li];
        }
    }
    float* g = m.gathered + 3 * o;
    if (photons == 0) {
        g[0] = 0.f; g[1] = 0.f; g[2] = 0.f;
    } else {
        float p = (float)photons;
        g[0] = cr / p; g[1] = cg / p; g[2] = cb / p;
    }
}

extern "C" int rl_photonmap_gather(rl_map* pm, int radius, void* stream) {
    if (!pm) return fail(RL_INVALID_CALL, "null photonmap");
    if (radius < 0) return fail(RL_INVALID_CALL, "negative radius");
    dim3 b(32, 8);
    int H = pm->dev.height;
    dim3 g((unsigned)((H + 31) / 32), (unsigned)((H + 7) / 8));
    k_gather<<<g, b, 0, S(stream)>>>(pm->dev, radius);
    CK_LAUNCH("k_gather");
    return RL_OK;
}

// -------------------------------------------------------- final gather

struct GatherMaps {
    int nmaps;
    DevMap maps[kMaxPhotonmaps];
};

// IndirectLight::bakeLumel (baker/IndirectLight.cpp:47-75): the lumel's
// final-gather samples as one lane's ray stream; each closest hit is shaded
// (hit normal and lightmap uv by Barycentric(u, v), photonmap lookup) as soon
// as its ray ends, in sample order.
struct FgGen {
    const DevScene* s;
    const GatherMaps* G;
    V3 pos, nrm, dir, sky, amb;
    uint2 key;
    uint32_t item;
    int j, samples;
    float maxd, influence, gr, gg, gb;
    __device__ bool next(V3& o, V3& d, float& tnear, float& tfar) {
        if (j >= samples) return false;
        dir = random_hemisphere(nrm, key, item, (uint32_t)j, kTagFG);
        float dp = dot3(nrm, dir);
        influence = dp > 0.0f ? dp : 0.0f;
        segment_ray(pos, dir, maxd, o, d, tnear, tfar);
        j++;
        return true;
    }
    __device__ void finish(const RayHit& h) {
        if (h.gid < 0) {
            gr = gr + (sky.x * influence + amb.x);
            gg = gg + (sky.y * influence + amb.y);
            gb = gb + (sky.z * influence + amb.z);
            return;
        }
        // the hit's shading record: interp3 / interp2 on the same values
        const float4* rec = s->shade + 4 * (size_t)h.gid;
        const float4 ra = __ldg(rec), rb = __ldg(rec + 1), rc = __ldg(rec + 2);
        const float bx = h.u, by = h.v;
        V3 hn = mk3(ra.x + (rb.x - ra.x) * by + (rc.x - ra.x) * bx, ra.y + (rb.y - ra.y) * by + (rc.y - ra.y) * bx,
                    ra.z + (rb.z - ra.z) * by + (rc.z - ra.z) * bx);
        if (dot3(dir, hn) >= 0.0f) return;
        const float4 rv = __ldg(rec + 3);
        int slot = __float_as_int(rv.w);
        if (slot >= 0 && slot < G->nmaps) {
            const DevMap& P = G->maps[slot];
            float2 uv = make_float2(ra.w + (rb.w - ra.w) * by + (rc.w - ra.w) * bx,
                                    rv.x + (rv.y - rv.x) * by + (rv.z - rv.x) * bx);
            int ti = lumel_at_uv(P.width, P.height, uv);
            const float* g = P.gathered + 3 * (size_t)ti;
            gr = gr + (g[0] * influence + amb.x);
            gg = gg + (g[1] * influence + amb.y);
            gb = gb + (g[2] * influence + amb.z);
        }
    }
};

// At most 64 registers (four 256-thread blocks' worth per SM): the ray loop
// is latency-bound and gains more from resident warps than it loses to the
// few spills (measured 52.3 -> 50.9 ms on the terrain final gather).
template <int kWidth>
__global__ void __launch_bounds__(256, 4) k_indirect(DevScene s, DevMap m, const __grid_constant__ GatherMaps G,
                                                  int samples, float maxd, V3 sky, V3 amb, uint2 key, Iter it,
                                                  long long count, int refill, int* status) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= count) return;
    long long i;
    bool valid = iter_lumel(m, it, k, i);
    FgGen g;
    g.s = &s;
    g.G = &G;
    g.pos = ld3(m.position + 3 * i);
    g.nrm = ld3(m.normal + 3 * i);
    g.sky = sky;
    g.amb = amb;
    g.key = key;
    g.item = (uint32_t)i;
    g.j = 0;
    g.samples = valid ? samples : 0;
    g.maxd = maxd;
    g.gr = g.gg = g.gb = 0.f;
    g.influence = 0.f;
    g.dir = mk3(0.f, 0.f, 0.f);
    if (kWidth == 8) ray_loop8<false>(s, g, refill, status);
    else if (kWidth == 4) ray_loop4<false>(s, g, refill, status);
    else if (kWidth == 3) ray_loop_spec<false>(s, g, refill, status);
    else ray_loop<false>(s, g, refill, status);
    if (!valid) return;
    float ns = (float)samples;
    float* col = m.color + 3 * i;
    col[0] = col[0] + g.gr / ns; col[1] = col[1] + g.gg / ns; col[2] = col[2] + g.gb / ns;
}

// FgGen over a work list of lumels (ray_loop_pool): lumel item k of the
// iteration `it` (iter_lumel), its samples in order, its colour written when
// its last sample is shaded — the same arithmetic as k_indirect.
struct FgPoolGen : FgGen {
    const DevMap* map;
    const Iter* it;
    int nsamples;
    long long li;
    long long k_begin, limit;  // item k is iteration item k_begin + k, for k < limit
    __device__ bool has_more() const { return j < samples; }
    __device__ void end_item() {
        if (samples == 0) return;
        const float ns = (float)samples;
        float* col = map->color + 3 * li;
        col[0] = col[0] + gr / ns; col[1] = col[1] + gg / ns; col[2] = col[2] + gb / ns;
        samples = 0;
    }
    __device__ bool start_item(long long k) {
        long long i;
        if (k >= limit || !iter_lumel(*map, *it, k_begin + k, i)) return false;
        li = i;
        pos = ld3(map->position + 3 * i);
        nrm = ld3(map->normal + 3 * i);
        item = (uint32_t)i;
        j = 0;
        samples = nsamples;
        gr = gg = gb = 0.f;
        return true;
    }
};

// Persistent final gather: a grid the size of the resident blocks, lanes
// taking lumels from their warp's pool (ray_loop_pool).
__global__ void __launch_bounds__(256, 4) k_indirect_pool(DevScene s, const __grid_constant__ DevMap m,
                                                          const __grid_constant__ GatherMaps G, int samples,
                                                          float maxd, V3 sky, V3 amb, uint2 key,
                                                          const __grid_constant__ Iter it, long long count,
                                                          int refill, int* status, unsigned long long* counter,
                                                          int chunk) {
    FgPoolGen g;
    g.s = &s;
    g.G = &G;
    g.map = &m;
    g.it = &it;
    g.nsamples = samples;
    g.samples = 0;
    g.j = 0;
    g.li = 0;
    g.k_begin = 0;
    g.limit = count;
    g.sky = sky;
    g.amb = amb;
    g.key = key;
    g.item = 0;
    g.maxd = maxd;
    g.gr = g.gg = g.gb = 0.f;
    g.influence = 0.f;
    g.pos = g.nrm = g.dir = mk3(0.f, 0.f, 0.f);
    CounterSource src{counter, count, chunk};
    ray_loop_pool<false>(s, g, refill, status, src);
}

extern "C" int rl_bake_indirect(const rl_scene* s, rl_map* lm, rl_map* const* maps, int nmaps, int samples,
                                float maxd, const float sky[3], const float ambient[3], uint64_t seed,
                                const rl_iterator* iterator, void* stream) {
    if (!s || !lm || (nmaps > 0 && !maps)) return fail(RL_INVALID_CALL, "rl_bake_indirect: null argument");
    if (samples <= 0 || nmaps > kMaxPhotonmaps) return fail(RL_INVALID_CALL, "rl_bake_indirect: bad arguments");
    cudaStream_t st = S(stream);
    long long n = (long long)lm->dev.width * lm->dev.height, count = 0;
    Iter it;
    int rc = make_iter(iterator, s, n, it, count);
    if (rc) return rc;
    if (count == 0) return RL_OK;
    tile_whole_map(it, count, lm->dev);
    static thread_local GatherMaps G;
    memset(&G, 0, sizeof G);
    G.nmaps = nmaps;
    for (int k = 0; k < nmaps; k++) {
        if (!maps[k]) return fail(RL_INVALID_CALL, "photonmap %d is null", k);
        G.maps[k] = maps[k]->dev;
    }
    V3 skyv = {sky ? sky[0] : 0.f, sky ? sky[1] : 0.f, sky ? sky[2] : 0.f};
    V3 ambv = {ambient ? ambient[0] : 0.f, ambient ? ambient[1] : 0.f, ambient ? ambient[2] : 0.f};
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    int bs = g_tune[RL_TUNE_FG_BLOCK];
    bool wide = g_tune[RL_TUNE_BVH_WIDTH] == 4 && s->dev.nodes4 != nullptr;
    bool wide8 = g_tune[RL_TUNE_BVH_WIDTH] == 8 && s->dev.nodes8 != nullptr;
    if (g_tune[RL_TUNE_FG_POOL] && !wide && !wide8 && !g_tune[RL_TUNE_SPECULATIVE]) {
        const int resident = resident_blocks(k_indirect_pool, bs);
        if (resident <= 0) return fail(RL_CUDA_ERROR, "k_indirect_pool: occupancy query failed");
        const long long want = ((long long)count + bs - 1) / bs;
        const unsigned grid = (unsigned)(want < resident ? want : resident);
        CK(cudaMemsetAsync(lm->d_work, 0, sizeof(unsigned long long), st));
        k_indirect_pool<<<grid, bs, 0, st>>>(s->dev, lm->dev, G, samples, maxd, skyv, ambv, key, it, count,
                                             g_tune[RL_TUNE_FG_REFILL], s->d_status, lm->d_work,
                                             g_tune[RL_TUNE_FG_CHUNK]);
        CK_LAUNCH("k_indirect_pool");
        return RL_OK;
    }
    auto kern = wide8 ? k_indirect<8> : wide ? k_indirect<4> : (g_tune[RL_TUNE_SPECULATIVE] ? k_indirect<3> : k_indirect<2>);
    kern<<<blocks_for(count, bs), bs, 0, st>>>(s->dev, lm->dev, G, samples, maxd, skyv, ambv, key, it, count,
                                              g_tune[RL_TUNE_FG_REFILL], s->d_status);
    CK_LAUNCH("k_indirect");
    return RL_OK;
}

// ------------------------------------------------------------- radiosity

struct FFPair {
    int i, j;
    float w;
};

// RadiosityBuilder::distanceFormFactor (radiosity/RadiosityBuilder.cpp:142-176)
// for the pair i < j.
__device__ __forceinline__ void ff_pair(const DevScene& s, int n, const float* pos, const float* nrm, float threshold,
                                        FFPair* out, unsigned long long cap, unsigned long long* counter, int* status,
                                        int i, int j) {
    const float Pi = 3.1415926535897932f;
    V3 rPos = ld3(pos + 3 * (size_t)i), rN = ld3(nrm + 3 * (size_t)i);
    V3 sPos = ld3(pos + 3 * (size_t)j), sN = ld3(nrm + 3 * (size_t)j);
    V3 dir = sub3(sPos, rPos);
    float r = normalize3(dir);
    float cosBA = dot3(dir, rN);
    float cosAB = -(dot3(dir, sN));
    if (r == 0.0f || cosAB < 0.0f || cosBA < 0.0f) return;
    float wBA = ((cosBA * cosAB) / (Pi * r * r));
    if (wBA < threshold) return;
    if (segment_blocked(s, rPos, sPos, kHitPoint | kHitUv | kHitColor | kHitNormal, status)) return;
    unsigned long long slot = atomicAdd(counter, 1ull);
    if (slot < cap) out[slot] = FFPair{i, j, wBA};
}

// Every pair i < j: rows over blockIdx.y (grid-strided), j over threads.
__global__ void k_ff_pairs(DevScene s, int n, const float* pos, const float* nrm, float threshold, FFPair* out,
                           unsigned long long cap, unsigned long long* counter, int* status) {
    for (int i = blockIdx.y; i < n; i += gridDim.y) {
        int j = i + 1 + blockIdx.x * blockDim.x + threadIdx.x;
        if (j < n) ff_pair(s, n, pos, nrm, threshold, out, cap, counter, status, i, j);
    }
}

static int assemble_csr(int n, std::vector<FFPair>& pairs, int64_t* row_ptr, int32_t* cols, float* vals,
                        int64_t capacity, int64_t* nnz_out) {
    int64_t nnz = 2 * (int64_t)pairs.size();
    if (nnz_out) *nnz_out = nnz;
    if (!cols) return RL_OK;
    if (!row_ptr || !vals) return fail(RL_INVALID_CALL, "form factors: row_ptr/vals missing");
    if (capacity < nnz) return fail(RL_CAPACITY, "form factors: capacity %lld < nnz %lld", (long long)capacity, (long long)nnz);
    std::sort(pairs.begin(), pairs.end(), [](const FFPair& a, const FFPair& b) {
        return a.i != b.i ? a.i < b.i : a.j < b.j;
    });
    std::vector<int64_t> fill((size_t)n + 1, 0);
    for (const FFPair& p : pairs) { fill[p.i + 1]++; fill[p.j + 1]++; }
    for (int i = 0; i < n; i++) fill[i + 1] += fill[i];
    std::memcpy(row_ptr, fill.data(), sizeof(int64_t) * ((size_t)n + 1));
    // pairs in (i, j) order: appending both directions lists each row in
    // ascending column order, the reference's push_back order
    for (const FFPair& p : pairs) {
        int64_t a = fill[p.i]++;
        cols[a] = p.j; vals[a] = p.w;
        int64_t b = fill[p.j]++;
        cols[b] = p.i; vals[b] = p.w;
    }
    // RadiosityBuilder::refineFormFactors (:111-120): normalise each row
    for (int i = 0; i < n; i++) {
        float sum = 0.0f;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) sum += vals[k];
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) vals[k] /= sum;
    }
    return RL_OK;
}

extern "C" int rl_ff_pairwise(const rl_scene* s, int n, const float* d_pos, const float* d_nrm, float threshold,
                              int64_t* row_ptr, int32_t* cols, float* vals, int64_t capacity, int64_t* nnz,
                              void* stream) {
    if (!s || n < 0 || (n > 0 && (!d_pos || !d_nrm))) return fail(RL_INVALID_CALL, "rl_ff_pairwise: bad arguments");
    cudaStream_t st = S(stream);
    std::vector<FFPair> pairs;
    if (n > 1) {
        unsigned long long cap = 1ull << 20;
        for (int attempt = 0; attempt < 2; attempt++) {
            Scratch sp, sc;
            FFPair* dp = nullptr;
            unsigned long long* dc = nullptr;
            int rc = scratch(sp, &dp, (size_t)cap, st);
            if (!rc) rc = scratch(sc, &dc, 1, st);
            if (rc) return rc;
            CK(cudaMemsetAsync(dc, 0, 8, st));
            dim3 grid((unsigned)((n + 255) / 256), (unsigned)std::min(n, 65535));
            k_ff_pairs<<<grid, 256, 0, st>>>(s->dev, n, d_pos, d_nrm, threshold, dp, cap, dc, s->d_status);
            CK_LAUNCH("k_ff_pairs");
            unsigned long long count = 0;
            CK(cudaMemcpyAsync(&count, dc, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (count <= cap) {
                pairs.resize(count);
                if (count) CK(cudaMemcpyAsync(pairs.data(), dp, sizeof(FFPair) * count, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                break;
            }
            cap = count;
        }
    }
    int rc = check_status(s, st);
    if (rc) return rc;
    return assemble_csr(n, pairs, row_ptr, cols, vals, capacity, nnz);
}

// Orthonormal basis (Duff et al., JCGT 6(1) 2017) and Malley's cosine
// direction by disc rejection, matching the oracle's sequence.
__device__ __forceinline__ V3 cosine_direction(V3 n, uint2 key, uint32_t item, uint32_t sample) {
    float x = 0.f, y = 0.f;
    for (uint32_t a = 0; a < kMaxAttempts; a++) {
        uint4 r = philox(make_uint4(item, sample, a, kTagHemiFF), key);
        x = u01(r.x) * 2.0f - 1.0f;
        y = u01(r.y) * 2.0f - 1.0f;
        if (x * x + y * y <= 1.0f) break;
    }
    float zz = 1.0f - x * x - y * y;
    float z = sqrtf(zz > 0.0f ? zz : 0.0f);
    float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    V3 b1 = mk3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    V3 b2 = mk3(b, sign + n.y * n.y * a, -n.y);
    return mk3(b1.x * x + b2.x * y + n.x * z, b1.y * x + b2.y * y + n.y * z, b1.z * x + b2.z * y + n.z * z);
}

struct HemiMaps {
    const int* mesh_map;
    const int* map_dims;
    const long long* map_base;
    const int* patch_of_texel;
    int nmaps;
};

__global__ void k_ff_hemi_rays(DevScene s, int n, const float* pos, const float* nrm, int rays, float maxd, uint2 key,
                               HemiMaps hm, int* hits, int* status) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= (long long)n * rays) return;
    int i = (int)(k / rays), r = (int)(k % rays);
    V3 p = ld3(pos + 3 * (size_t)i), nn = ld3(nrm + 3 * (size_t)i);
    V3 dir = cosine_direction(nn, key, (uint32_t)i, (uint32_t)r);
    SegHit h;
    trace_segment(s, p, add3(p, mul3(dir, maxd)), kHitUv, h, status);
    int out = -1;
    if (h.hit) {
        int map = hm.mesh_map[h.mesh];
        if (map >= 0 && map < hm.nmaps) {
            int ti = lumel_at_uv(hm.map_dims[2 * map], hm.map_dims[2 * map + 1], h.uv);
            out = hm.patch_of_texel[hm.map_base[map] + ti];
        }
    }
    hits[k] = out;
}

// Per patch: sort its hit patch ids in shared memory (bitonic), then
// run-length encode them into (patch, count) pairs.
__global__ void k_ff_hemi_rle(int rays, int pow2, const int* hits, int2* runs, int* run_count) {
    extern __shared__ int sh[];
    int* key = sh;
    int* start = sh + pow2;
    int i = blockIdx.x;
    __shared__ int s_end;  // first empty sorted key (pow2 when every ray hit a patch)
    if (threadIdx.x == 0) s_end = pow2;
    for (int t = threadIdx.x; t < pow2; t += blockDim.x)
        key[t] = t < rays ? (hits[(size_t)i * rays + t] < 0 ? 0x7fffffff : hits[(size_t)i * rays + t]) : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= pow2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < pow2; t += blockDim.x) {
                int ixj = t ^ j;
                if (ixj > t) {
                    bool up = (t & k) == 0;
                    int a = key[t], b = key[ixj];
                    if ((a > b) == up) { key[t] = b; key[ixj] = a; }
                }
            }
            __syncthreads();
        }
    // Run starts (a key that differs from its predecessor), ranked by a block
    // scan over contiguous chunks, so they land in key order; the first empty
    // key ends the last run.
    constexpr int kThreads = 256;  // the launch's block size
    typedef cub::BlockScan<int, kThreads> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;
    const int per = (pow2 + kThreads - 1) / kThreads;
    const int t0 = threadIdx.x * per, t1 = min(t0 + per, pow2);
    int c = 0;
    for (int t = t0; t < t1; t++) {
        const int v = key[t];
        if (v != 0x7fffffff && (t == 0 || key[t - 1] != v)) c++;
        if (v == 0x7fffffff && (t == 0 || key[t - 1] != 0x7fffffff)) s_end = t;
    }
    int at, nr;
    Scan(scan_tmp).ExclusiveSum(c, at, nr);
    for (int t = t0; t < t1; t++) {
        const int v = key[t];
        if (v != 0x7fffffff && (t == 0 || key[t - 1] != v)) start[at++] = t;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr; q += kThreads) {
        const int b = start[q], e = q + 1 < nr ? start[q + 1] : s_end;
        runs[(size_t)i * rays + q] = make_int2(key[b], e - b);
    }
    if (threadIdx.x == 0) run_count[i] = nr;
}

__global__ void k_ff_hemi_compact(int n, int rays, const int2* runs, const long long* row_ptr, int* cols, float* vals) {
    int i = blockIdx.x;
    long long b = row_ptr[i], e = row_ptr[i + 1];
    for (long long q = threadIdx.x; q < e - b; q += blockDim.x) {
        int2 r = runs[(size_t)i * rays + q];
        cols[b + q] = r.x;
        vals[b + q] = (float)r.y / (float)rays;
    }
}

// Hemisphere form factors; the CSR goes to host arrays (device_out false,
// stream synchronised on return) or to the caller's device arrays
// (device_out true, stream-ordered; only the per-row counts come back for
// the row offsets and the capacity check).
static int ff_hemisphere(const rl_scene* s, int n, const float* d_pos, const float* d_nrm, int rays, float maxd,
                         uint64_t seed, const int32_t* mesh_map, int nmaps, const int32_t* map_dims,
                         const int64_t* map_base, const int32_t* patch_of_texel, int64_t ntexels, int64_t* row_ptr,
                         int32_t* cols, float* vals, int64_t capacity, int64_t* nnz, void* stream, bool device_out) {
    if (!s || n < 0 || rays <= 0 || rays > 1024 || !mesh_map || !map_dims || !map_base || !patch_of_texel)
        return fail(RL_INVALID_CALL, "rl_ff_hemisphere: bad arguments (rays must be 1..1024)");
    cudaStream_t st = S(stream);
    if (n == 0) {
        if (nnz) *nnz = 0;
        if (row_ptr) {
            if (device_out) {
                const int64_t zero = 0;
                CK(cudaMemcpyAsync(row_ptr, &zero, sizeof zero, cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
            } else {
                row_ptr[0] = 0;
            }
        }
        return RL_OK;
    }
    for (int m = 0; m < nmaps; m++)
        if (map_base[m] < 0 || map_base[m] + (int64_t)map_dims[2 * m] * map_dims[2 * m + 1] > ntexels)
            return fail(RL_INVALID_CALL, "rl_ff_hemisphere: map %d outside patch_of_texel", m);
    Scratch s1, s2, s3, s4, s5, s6, s7, s8;
    int *dmm = nullptr, *ddims = nullptr, *dpot = nullptr, *dhits = nullptr, *dcnt = nullptr, *dcols = nullptr;
    long long *dbase = nullptr, *drow = nullptr;
    int2* druns = nullptr;
    float* dvals = nullptr;
    int rc = scratch(s1, &dmm, (size_t)s->nmeshes, st);
    if (!rc) rc = scratch(s2, &ddims, 2 * (size_t)std::max(nmaps, 1), st);
    if (!rc) rc = scratch(s3, &dbase, (size_t)std::max(nmaps, 1), st);
    if (!rc) rc = scratch(s4, &dpot, (size_t)std::max<int64_t>(ntexels, 1), st);
    if (!rc) rc = scratch(s5, &dhits, (size_t)n * rays, st);
    if (!rc) rc = scratch(s6, &druns, (size_t)n * rays, st);
    if (!rc) rc = scratch(s7, &dcnt, (size_t)n, st);
    if (rc) return rc;
    CK(cudaMemcpyAsync(dmm, mesh_map, 4 * (size_t)s->nmeshes, cudaMemcpyHostToDevice, st));
    if (nmaps) {
        CK(cudaMemcpyAsync(ddims, map_dims, 8 * (size_t)nmaps, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(dbase, map_base, 8 * (size_t)nmaps, cudaMemcpyHostToDevice, st));
    }
    if (ntexels) CK(cudaMemcpyAsync(dpot, patch_of_texel, 4 * (size_t)ntexels, cudaMemcpyHostToDevice, st));
    HemiMaps hm{dmm, ddims, dbase, dpot, nmaps};
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    long long total = (long long)n * rays;
    k_ff_hemi_rays<<<blocks_for(total, 128), 128, 0, st>>>(s->dev, n, d_pos, d_nrm, rays, maxd, key, hm, dhits,
                                                          s->d_status);
    CK_LAUNCH("k_ff_hemi_rays");
    int pow2 = 1;
    while (pow2 < rays) pow2 <<= 1;
    k_ff_hemi_rle<<<n, 256, 2 * pow2 * sizeof(int), st>>>(rays, pow2, dhits, druns, dcnt);
    CK_LAUNCH("k_ff_hemi_rle");
    std::vector<int> cnt(n);
    CK(cudaMemcpyAsync(cnt.data(), dcnt, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<long long> rp((size_t)n + 1, 0);
    for (int i = 0; i < n; i++) rp[i + 1] = rp[i] + cnt[i];
    int64_t total_nnz = rp[n];
    if (nnz) *nnz = total_nnz;
    rc = check_status(s, st);
    if (rc) return rc;
    if (!cols) return RL_OK;
    if (!row_ptr || !vals) return fail(RL_INVALID_CALL, "rl_ff_hemisphere: row_ptr/vals missing");
    if (capacity < total_nnz) return fail(RL_CAPACITY, "rl_ff_hemisphere: capacity %lld < nnz %lld",
                                          (long long)capacity, (long long)total_nnz);
    if (device_out) {
        CK(cudaMemcpyAsync(row_ptr, rp.data(), 8 * ((size_t)n + 1), cudaMemcpyHostToDevice, st));
        k_ff_hemi_compact<<<n, 128, 0, st>>>(n, rays, druns, (const long long*)row_ptr, cols, vals);
        CK_LAUNCH("k_ff_hemi_compact");
        return RL_OK;
    }
    std::memcpy(row_ptr, rp.data(), sizeof(int64_t) * ((size_t)n + 1));
    rc = scratch(s8, &drow, (size_t)n + 1, st);
    if (rc) return rc;
    Scratch s9, s10;
    rc = scratch(s9, &dcols, (size_t)std::max<int64_t>(total_nnz, 1), st);
    if (!rc) rc = scratch(s10, &dvals, (size_t)std::max<int64_t>(total_nnz, 1), st);
    if (rc) return rc;
    CK(cudaMemcpyAsync(drow, rp.data(), 8 * ((size_t)n + 1), cudaMemcpyHostToDevice, st));
    k_ff_hemi_compact<<<n, 128, 0, st>>>(n, rays, druns, drow, dcols, dvals);
    CK_LAUNCH("k_ff_hemi_compact");
    if (total_nnz) {
        CK(cudaMemcpyAsync(cols, dcols, 4 * (size_t)total_nnz, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(vals, dvals, 4 * (size_t)total_nnz, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return RL_OK;
}

extern "C" int rl_ff_hemisphere(const rl_scene* s, int n, const float* d_pos, const float* d_nrm, int rays,
                                float maxd, uint64_t seed, const int32_t* mesh_map, int nmaps, const int32_t* map_dims,
                                const int64_t* map_base, const int32_t* patch_of_texel, int64_t ntexels,
                                int64_t* row_ptr, int32_t* cols, float* vals, int64_t capacity, int64_t* nnz,
                                void* stream) {
    return ff_hemisphere(s, n, d_pos, d_nrm, rays, maxd, seed, mesh_map, nmaps, map_dims, map_base, patch_of_texel,
                         ntexels, row_ptr, cols, vals, capacity, nnz, stream, false);
}

extern "C" int rl_ff_hemisphere_device(const rl_scene* s, int n, const float* d_pos, const float* d_nrm, int rays,
                                       float maxd, uint64_t seed, const int32_t* mesh_map, int nmaps,
                                       const int32_t* map_dims, const int64_t* map_base, const int32_t* patch_of_texel,
                                       int64_t ntexels, int64_t* d_row_ptr, int32_t* d_cols, float* d_vals,
                                       int64_t capacity, int64_t* nnz, void* stream) {
    return ff_hemisphere(s, n, d_pos, d_nrm, rays, maxd, seed, mesh_map, nmaps, map_dims, map_base, patch_of_texel,
                         ntexels, d_row_ptr, d_cols, d_vals, capacity, nnz, stream, true);
}

// B_k of one patch: three floats ([n][3], kB = 0) or a float4 whose w is
// unused ([n][4], one 16-byte gather, kB = 1).
template <int kB>
__device__ __forceinline__ float3 patch_b(const float* __restrict__ B, int c) {
    if (kB == 2) {  // [n][3] staged in shared memory
        const float* x = B + 3 * (size_t)c;
        return make_float3(x[0], x[1], x[2]);
    }
    if (kB == 1) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(B) + c);
        return make_float3(v.x, v.y, v.z);
    }
    const float* x = B + 3 * (size_t)c;
    return make_float3(__ldg(x), __ldg(x + 1), __ldg(x + 2));
}

// sum_k F_ik B_k (RGB) over row i's nonzeros [b, e), by one warp: four
// 32-wide chunks in flight (their columns, then their B gathers), each into
// its own partial sums, so a row costs two memory latencies per four chunks
// rather than per chunk.  The result is reduced across the warp.  Both B
// layouts load the same values, so they give the same bits.
template <int kB>
__device__ __forceinline__ void row_dot3(int64_t b, int64_t e, int lane, const int32_t* __restrict__ cols,
                                         const float* __restrict__ vals, const float* __restrict__ B, float& r0,
                                         float& r1, float& r2) {
    float s[4][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    int64_t k = b + lane;
    for (; k + 96 < e; k += 128) {
        int c[4];
        float w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            c[u] = __ldg(cols + k + 32 * u);
            w[u] = __ldg(vals + k + 32 * u);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const float3 x = patch_b<kB>(B, c[u]);
            s[u][0] = __fmaf_rn(w[u], x.x, s[u][0]);
            s[u][1] = __fmaf_rn(w[u], x.y, s[u][1]);
            s[u][2] = __fmaf_rn(w[u], x.z, s[u][2]);
        }
    }
    for (; k < e; k += 32) {
        const float w = __ldg(vals + k);
        const float3 x = patch_b<kB>(B, __ldg(cols + k));
        s[0][0] = __fmaf_rn(w, x.x, s[0][0]);
        s[0][1] = __fmaf_rn(w, x.y, s[0][1]);
        s[0][2] = __fmaf_rn(w, x.z, s[0][2]);
    }
    r0 = (s[0][0] + s[1][0]) + (s[2][0] + s[3][0]);
    r1 = (s[0][1] + s[1][1]) + (s[2][1] + s[3][1]);
    r2 = (s[0][2] + s[1][2]) + (s[2][2] + s[3][2]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r0 += __shfl_xor_sync(0xffffffffu, r0, o);
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    }
}

// Row dot with 16-byte column and weight loads: lane l takes the aligned
// quads base + 4 l and base + 128 + 4 l, two per step (256 nonzeros per warp
// step, about 6 KB in flight with their gathers); elements outside [b, e)
// are loaded one by one or skipped, so no load leaves the row.  cols and
// vals must be 16-byte aligned.  Both B layouts (kB as in row_dot3) load the
// same values, so they give the same bits.
template <int kB>
__device__ __forceinline__ void row_dot3_quads(int64_t b, int64_t e, int lane, const int32_t* __restrict__ cols,
                                               const float* __restrict__ vals, const float* __restrict__ B,
                                               float& r0, float& r1, float& r2) {
    float s[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (int64_t base = b & ~(int64_t)3; base < e; base += 256) {
        int c[2][4];
        float w[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int64_t q = base + 128 * u + 4 * lane;
            if (q >= b && q + 4 <= e) {
                const int4 cc = __ldg(reinterpret_cast<const int4*>(cols + q));
                const float4 ww = __ldg(reinterpret_cast<const float4*>(vals + q));
                c[u][0] = cc.x; c[u][1] = cc.y; c[u][2] = cc.z; c[u][3] = cc.w;
                w[u][0] = ww.x; w[u][1] = ww.y; w[u][2] = ww.z; w[u][3] = ww.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int64_t k = q + j;
                    c[u][j] = -1;
                    w[u][j] = 0.f;
                    if (k >= b && k < e) {
                        c[u][j] = __ldg(cols + k);
                        w[u][j] = __ldg(vals + k);
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (c[u][j] >= 0) {
                    const float3 x = patch_b<kB>(B, c[u][j]);
                    s[u][0] = __fmaf_rn(w[u][j], x.x, s[u][0]);
                    s[u][1] = __fmaf_rn(w[u][j], x.y, s[u][1]);
                    s[u][2] = __fmaf_rn(w[u][j], x.z, s[u][2]);
                }
    }
    r0 = s[0][0] + s[1][0];
    r1 = s[0][1] + s[1][1];
    r2 = s[0][2] + s[1][2];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r0 += __shfl_xor_sync(0xffffffffu, r0, o);
        r1 += __shfl_xor_sync(0xffffffffu, r1, o);
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    }
}

// One warp per patch row on [n][4] iterates (w unused), one 16-byte gather
// per nonzero: B'_i = E_i + rho_i * sum_k F_ik B_k (RGB).  With kQuads,
// 16-byte column and weight loads as well (a different accumulation order
// from row_dot3, within the fp32 tolerance).
template <bool kQuads>
__global__ void k_jacobi4(int n, const int64_t* row_ptr, const int32_t* cols, const float* vals, const float* E,
                          const float* rho, const float4* B, float4* Bn) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n) return;
    float s0, s1, s2;
    if (kQuads)
        row_dot3_quads<1>(row_ptr[warp], row_ptr[warp + 1], lane, cols, vals, reinterpret_cast<const float*>(B), s0,
                          s1, s2);
    else
        row_dot3<1>(row_ptr[warp], row_ptr[warp + 1], lane, cols, vals, reinterpret_cast<const float*>(B), s0, s1,
                    s2);
    if (lane == 0) {
        size_t i = 3 * (size_t)warp;
        Bn[warp] = make_float4(__fmaf_rn(rho[i], s0, E[i]), __fmaf_rn(rho[i + 1], s1, E[i + 1]),
                               __fmaf_rn(rho[i + 2], s2, E[i + 2]), 0.f);
    }
}

// k_jacobi4 with the whole iterate staged in shared memory as [n][3] floats
// (12 n bytes: up to kJacobiSmemPatches patches) by every block, the blocks
// then taking rows blockIdx.x * warps + warp, + gridDim.x * warps, ...  The
// column gathers (one per nonzero, scattered over the iterate) then read
// shared memory instead of 32-byte L2 sectors; the row arithmetic is
// k_jacobi4's, so the bits are the same.
constexpr int kJacobiSmemPatches = (224 * 1024) / 12;
template <bool kQuads>
__global__ void __launch_bounds__(1024, 1) k_jacobi4_smem(int n, const int64_t* row_ptr, const int32_t* cols,
                                                          const float* vals, const float* E, const float* rho,
                                                          const float4* B, float4* Bn) {
    extern __shared__ float sb[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 v = __ldg(B + i);
        sb[3 * i] = v.x;
        sb[3 * i + 1] = v.y;
        sb[3 * i + 2] = v.z;
    }
    __syncthreads();
    const int warps = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < n; row += gridDim.x * warps) {
        float s0, s1, s2;
        if (kQuads)
            row_dot3_quads<2>(row_ptr[row], row_ptr[row + 1], lane, cols, vals, sb, s0, s1, s2);
        else
            row_dot3<2>(row_ptr[row], row_ptr[row + 1], lane, cols, vals, sb, s0, s1, s2);
        if (lane == 0) {
            size_t i = 3 * (size_t)row;
            Bn[row] = make_float4(__fmaf_rn(rho[i], s0, E[i]), __fmaf_rn(rho[i + 1], s1, E[i + 1]),
                                  __fmaf_rn(rho[i + 2], s2, E[i + 2]), 0.f);
        }
    }
}

// One Jacobi step of rl_radiosity_solve (and its no-allocation form): the
// shared-memory kernel when the iterate fits, else k_jacobi4.
static int jacobi4_step(int n, const int64_t* row_ptr, const int32_t* cols, const float* vals, const float* E,
                 const float* rho, const float4* B, float4* Bn, cudaStream_t st) {
    const bool quads = ((uintptr_t)cols % 16) == 0 && ((uintptr_t)vals % 16) == 0;
    if (n <= kJacobiSmemPatches) {
        static int sms = 0;
        static std::once_flag once;
        cudaError_t ae = cudaSuccess;
        std::call_once(once, [&] {
            ae = cudaFuncSetAttribute(k_jacobi4_smem<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            if (ae == cudaSuccess)
                ae = cudaFuncSetAttribute(k_jacobi4_smem<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          227 * 1024);
            int dev = 0;
            if (ae == cudaSuccess) ae = cudaGetDevice(&dev);
            if (ae == cudaSuccess) ae = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        });
        if (ae != cudaSuccess) return fail(RL_CUDA_ERROR, "jacobi set-up: %s", cudaGetErrorString(ae));
        const int grid = std::max(1, std::min(sms, (n + 31) / 32));
        const size_t smem = 12 * (size_t)n;
        if (quads)
            k_jacobi4_smem<true><<<grid, 1024, smem, st>>>(n, row_ptr, cols, vals, E, rho, B, Bn);
        else
            k_jacobi4_smem<false><<<grid, 1024, smem, st>>>(n, row_ptr, cols, vals, E, rho, B, Bn);
        CK_LAUNCH("k_jacobi4_smem");
        return RL_OK;
    }
    const unsigned grid = blocks_for((long long)n * 32, 256);
    if (quads)
        k_jacobi4<true><<<grid, 256, 0, st>>>(n, row_ptr, cols, vals, E, rho, B, Bn);
    else
        k_jacobi4<false><<<grid, 256, 0, st>>>(n, row_ptr, cols, vals, E, rho, B, Bn);
    CK_LAUNCH("k_jacobi4");
    return RL_OK;
}

// [n][3] <-> [n][4] (w = 0).
__global__ void k_pack4(int n, const float* src, float4* dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.f);
}
__global__ void k_unpack4(int n, const float4* src, float* dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float4 v = src[i];
        dst[3 * i] = v.x;
        dst[3 * i + 1] = v.y;
        dst[3 * i + 2] = v.z;
    }
}

// One Jacobi step over rows [row_begin, row_end): Bn[row] from the full B,
// [n][3] iterates, with k_jacobi4's row arithmetic (16-byte column and
// weight loads under the same alignment rule), so a row-sharded solve gives
// rl_radiosity_solve's bits.
template <bool kQuads>
__global__ void k_jacobi_rows(int row_begin, int row_end, const int64_t* row_ptr, const int32_t* cols,
                              const float* vals, const float* E, const float* rho, const float* B, float* Bn) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int row = row_begin + warp;
    if (row >= row_end) return;
    float s0, s1, s2;
    if (kQuads)
        row_dot3_quads<0>(row_ptr[row], row_ptr[row + 1], lane, cols, vals, B, s0, s1, s2);
    else
        row_dot3<0>(row_ptr[row], row_ptr[row + 1], lane, cols, vals, B, s0, s1, s2);
    if (lane == 0) {
        size_t i = 3 * (size_t)row;
        Bn[i] = __fmaf_rn(rho[i], s0, E[i]);
        Bn[i + 1] = __fmaf_rn(rho[i + 1], s1, E[i + 1]);
        Bn[i + 2] = __fmaf_rn(rho[i + 2], s2, E[i + 2]);
    }
}

extern "C" int rl_radiosity_step(int row_begin, int row_end, const int64_t* d_row_ptr, const int32_t* d_cols,
                                 const float* d_vals, const float* d_E, const float* d_rho, const float* d_B,
                                 float* d_B_next, void* stream) {
    if (row_begin < 0 || row_end < row_begin || !d_row_ptr || !d_E || !d_rho || !d_B || !d_B_next)
        return fail(RL_INVALID_CALL, "rl_radiosity_step: bad arguments");
    if (row_end == row_begin) return RL_OK;
    const unsigned grid = blocks_for((long long)(row_end - row_begin) * 32, 256);
    if (((uintptr_t)d_cols % 16) == 0 && ((uintptr_t)d_vals % 16) == 0)
        k_jacobi_rows<true><<<grid, 256, 0, S(stream)>>>(row_begin, row_end, d_row_ptr, d_cols, d_vals, d_E, d_rho,
                                                         d_B, d_B_next);
    else
        k_jacobi_rows<false><<<grid, 256, 0, S(stream)>>>(row_begin, row_end, d_row_ptr, d_cols, d_vals, d_E, d_rho,
                                                          d_B, d_B_next);
    CK_LAUNCH("k_jacobi_rows");
    return RL_OK;
}

extern "C" int rl_radiosity_solve(int n, const int64_t* d_row_ptr, const int32_t* d_cols, const float* d_vals,
                                  const float* d_E, const float* d_rho, int iters, float* d_B, void* stream) {
    if (n < 0 || iters < 0 || (n > 0 && (!d_row_ptr || !d_E || !d_rho || !d_B)))
        return fail(RL_INVALID_CALL, "rl_radiosity_solve: bad arguments");
    cudaStream_t st = S(stream);
    if (n == 0) return RL_OK;
    if (iters == 0) {
        CK(cudaMemcpyAsync(d_B, d_E, 12 * (size_t)n, cudaMemcpyDeviceToDevice, st));
        return RL_OK;
    }
    // iterates in [n][4] ping-pong buffers, B0 = E
    Scratch sa, sb;
    float4 *src = nullptr, *dst = nullptr;
    int rc = scratch(sa, &src, (size_t)n, st);
    if (!rc) rc = scratch(sb, &dst, (size_t)n, st);
    if (rc) return rc;
    k_pack4<<<blocks_for(n, 256), 256, 0, st>>>(n, d_E, src);
    CK_LAUNCH("k_pack4");
    for (int it = 0; it < iters; it++) {
        if (int rc2 = jacobi4_step(n, d_row_ptr, d_cols, d_vals, d_E, d_rho, src, dst, st)) return rc2;
        std::swap(src, dst);
    }
    k_unpack4<<<blocks_for(n, 256), 256, 0, st>>>(n, src, d_B);
    CK_LAUNCH("k_unpack4");
    return RL_OK;
}

// ---------------------------------------------------------- post-process

// Lightmap::expand (Lightmap.cpp:167-193).  The reference walks the interior
// in scan order and every valid lumel copies its colour into its invalid
// diagonal neighbours; only invalid texels change, so each invalid texel
// ends with the colour of the LAST valid interior writer in scan order:
// (x+1, y+1), else (x-1, y+1), else (x+1, y-1), else (x-1, y-1).
__global__ void k_expand(DevMap m) {
    const int W = m.width, H = m.height;
    const long long n = (long long)W * H;
    const int dx[4] = {1, -1, 1, -1}, dy[4] = {1, 1, -1, -1};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        if (m.flags[t] & 1) continue;
        int x = (int)(t % W), y = (int)(t / W);
        for (int k = 0; k < 4; k++) {
            int cx = x + dx[k], cy = y + dy[k];
            if (cx < 1 || cx > W - 2 || cy < 1 || cy > H - 2) continue;
            long long c = (long long)cy * W + cx;
            if (!(m.flags[c] & 1)) continue;
            m.color[3 * t] = m.color[3 * c];
            m.color[3 * t + 1] = m.color[3 * c + 1];
            m.color[3 * t + 2] = m.color[3 * c + 2];
            break;
        }
    }
}

// Lightmap::blur (Lightmap.cpp:196-220).  The reference blurs in place in
// scan order, so texel (x, y) reads the already-blurred (x-1..x+1, y-1) and
// (x-1, y) and the original rest of its window.  Every such input has a
// smaller t = (x-1) + 2(y-1), and texels of one t never share a window, so
// one block walks t = 0, 1, ... with a barrier per step (a wavefront), each
// thread owning rows y = 1 + tid, 1 + tid + blockDim, ...  Sums run in the
// reference's window order, so the result is bit-identical.
__global__ void __launch_bounds__(1024) k_blur(DevMap m) {
    const int W = m.width, H = m.height;
    if (W < 3 || H < 3) return;
    const long long T = (long long)(W - 3) + 2LL * (H - 3);
    for (long long t = 0; t <= T; t++) {
        for (int y = 1 + threadIdx.x; y <= H - 2; y += blockDim.x) {
            long long x = t - 2LL * (y - 1) + 1;
            if (x < 1 || x > W - 2) continue;
            float r = 0.0f, g = 0.0f, b = 0.0f;
            int count = 0;
            for (int j = y - 1; j <= y + 1; j++) {
                for (long long i = x - 1; i <= x + 1; i++) {
                    long long l = (long long)j * W + i;
                    if (m.flags[l] & 1) {
                        r += m.color[3 * l]; g += m.color[3 * l + 1]; b += m.color[3 * l + 2];
                        count++;
                    }
                }
            }
            if (count) {
                float inv = 1.0f / (float)count;
                long long o = (long long)y * W + x;
                m.color[3 * o] = r * inv; m.color[3 * o + 1] = g * inv; m.color[3 * o + 2] = b * inv;
            }
        }
        __syncthreads();
    }
}

// static_cast<unsigned char>(float) as x86-64 code performs it: truncation
// to a 32-bit integer (0x80000000 when out of range or NaN), low byte kept.
__device__ __forceinline__ uint8_t f2u8(float v) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return (uint8_t)(uint32_t)__float2int_rz(v);
}
__device__ __forceinline__ float min2f(float a, float b) { return a < b ? a : b; }  // Types.h:87-89
__device__ __forceinline__ float max2f(float a, float b) { return a > b ? a : b; }  // Types.h:99-101

// Lightmap::toDoubleLdr / toRgbmLdr (Lightmap.cpp:288-330) with
// Rgb::doubleLdr / Rgb::rgbm (Types.h:215-235), into the reference's pixel
// buffer layout.  RGBM keeps the reference's pixel offset x*3 inside a row
// of stride w*4: pixel x writes bytes 3x..3x+2 and, being overwritten there
// by pixel x+1's r, its m byte survives only for the last pixel of a row.
__global__ void k_encode(DevMap m, int format, uint8_t* out) {
    const int W = m.width;
    const long long n = (long long)W * m.height;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float* c = m.color + 3 * i;
        if (format == 1) {
            for (int k = 0; k < 3; k++) out[3 * i + k] = f2u8(min2f(255.0f, c[k] * 0.5f * 255.0f));
        } else {
            long long x = i % W, y = i / W;
            float mm = 255.0f / max2f(c[0], max2f(c[1], c[2]));
            uint8_t* px = out + y * (4LL * W) + 3 * x;
            px[0] = f2u8(min2f(255.0f, c[0] / mm * 255.0f));
            px[1] = f2u8(min2f(255.0f, c[1] / mm * 255.0f));
            px[2] = f2u8(min2f(255.0f, c[2] / mm * 255.0f));
            if (x == W - 1) px[3] = f2u8(min2f(255.0f, mm * 255.0f));
        }
    }
}

static int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 32));
}

extern "C" int rl_map_expand(rl_map* m, void* stream) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    long long n = (long long)m->dev.width * m->dev.height;
    k_expand<<<grid_for(n, 256), 256, 0, S(stream)>>>(m->dev);
    CK_LAUNCH("k_expand");
    return RL_OK;
}

extern "C" int rl_map_blur(rl_map* m, void* stream) {
    if (!m) return fail(RL_INVALID_CALL, "null map");
    k_blur<<<1, 1024, 0, S(stream)>>>(m->dev);
    CK_LAUNCH("k_blur");
    return RL_OK;
}

static long long encoded_bytes(const rl_map* m, int format) {
    long long n = (long long)m->dev.width * m->dev.height;
    return format == 0 ? 12 * n : format == 1 ? 3 * n : 4 * n;
}

extern "C" int rl_map_encode(const rl_map* m, int format, uint8_t* out, void* stream) {
    if (!m || !out || format < 0 || format > 2) return fail(RL_INVALID_CALL, "rl_map_encode: bad arguments");
    cudaStream_t st = S(stream);
    long long bytes = encoded_bytes(m, format), n = (long long)m->dev.width * m->dev.height;
    if (format == 0) {
        CK(cudaMemcpyAsync(out, m->dev.color, bytes, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return RL_OK;
    }
    uint8_t* d = nullptr;
    if (int rc = pool_alloc((void**)&d, (size_t)bytes, st)) return rc;
    int rc = RL_OK;
    cudaError_t e = cudaMemsetAsync(d, 0, bytes, st);
    if (e == cudaSuccess) {
        k_encode<<<grid_for(n, 256), 256, 0, st>>>(m->dev, format, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(RL_CUDA_ERROR, "rl_map_encode: %s", cudaGetErrorString(e));
    return rc;
}

// Lightmap::save (Lightmap.cpp:223-283): RawHdr = width, height (int32)
// and the colours; TGA = the 18-byte uncompressed true-colour header and
// each pixel's bytes 2, 1, 0 (and 3 for RGBM) of the encoded buffer.
extern "C" int rl_map_save(const rl_map* m, const char* path, int format, void* stream) {
    if (!m || !path || format < 0 || format > 2) return fail(RL_INVALID_CALL, "rl_map_save: bad arguments");
    std::vector<uint8_t> buf((size_t)encoded_bytes(m, format));
    if (int rc = rl_map_encode(m, format, buf.data(), stream)) return rc;
    FILE* f = fopen(path, "wb");
    if (!f) return fail(RL_INVALID_CALL, "rl_map_save: cannot open %s", path);
    int W = m->dev.width, H = m->dev.height;
    bool ok = true;
    if (format == 0) {
        ok = fwrite(&W, sizeof(int), 1, f) == 1 && fwrite(&H, sizeof(int), 1, f) == 1 &&
             fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    } else {
        int ch = format == 1 ? 3 : 4;
        uint8_t head[18] = {0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, (uint8_t)(W % 256), (uint8_t)(W / 256),
                            (uint8_t)(H % 256), (uint8_t)(H / 256), (uint8_t)(ch * 8), 0};
        std::vector<uint8_t> px(buf.size());
        size_t n = (size_t)W * H;
        for (size_t i = 0; i < n; i++) {
            const uint8_t* s = &buf[i * ch];
            uint8_t* d = &px[i * ch];
            d[0] = s[2]; d[1] = s[1]; d[2] = s[0];
            if (ch == 4) d[3] = s[3];
        }
        ok = fwrite(head, 1, 18, f) == 18 && fwrite(px.data(), 1, px.size(), f) == px.size();
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) return fail(RL_INVALID_CALL, "rl_map_save: write to %s failed", path);
    return RL_OK;
}

// --------------------------------------------------------------- batches

// One job of a batch on the device: its scene and lightmap views, pass and
// parameters, and the slice [k_begin, k_begin + count) of its iterator.
struct DevJob {
    DevScene s;
    DevMap m;
    const LightTable* lights;
    const GatherMaps* maps;
    int* status;
    Iter it;
    long long k_begin, count;
    int kind, samples;
    float fraction, maxd, exponent;
    V3 sky, amb;
    uint2 key;
};

// Where the batch kernel of one pass kind finds its jobs.  The headers sit
// at a fixed device address and the kernels read them at run time, so a
// captured launch stays valid when rl_batch_update rewrites the tables.
struct BatchHeader {
    const DevJob* jobs;
    const long long* prefix;  // work-item offset of each job (multiples of 32)
    long long total;          // work items incl. padding
    int njobs, pad;
};

// The job table is split by pass: one persistent kernel per pass kind takes
// the items of every job of that kind, so each kernel keeps only its own ray
// loop's registers.  Tables live in one device buffer, written from pinned
// staging that alternates between two slots so the host can fill the next
// table while the previous copy is in flight.
struct rl_batch {
    BatchHeader* d_hdr = nullptr;             // 3 headers
    unsigned long long* d_counter = nullptr;  // 3 work counters
    char* d_buf = nullptr;
    size_t d_cap = 0;
    char* h_stage[2] = {nullptr, nullptr};
    size_t h_cap[2] = {0, 0};
    cudaEvent_t staged[2] = {nullptr, nullptr};
    int slot = 0;
    long long items = 0, total[3] = {0, 0, 0};
    int grid[3] = {0, 0, 0}, block[3] = {128, 128, 128}, refill[3] = {0, 0, 0};
    bool pool = false;  // AO / final gather through k_batch_pool (RL_TUNE_FG_POOL at creation)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~rl_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (int k = 0; k < 2; k++) {
            if (staged[k]) cudaEventDestroy(staged[k]);
            if (h_stage[k]) cudaFreeHost(h_stage[k]);
        }
        cudaFree(d_buf);
        cudaFree(d_hdr);
        cudaFree(d_counter);
    }
};

// Largest j with prefix[j] <= w.
__device__ __forceinline__ int find_job(const long long* prefix, int njobs, long long w) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Persistent batch kernel for one pass kind (0 direct, 1 AO, 2 final
// gather).  Warps take 32 work items at a time from one counter across all
// the batch's jobs of that kind; every job's items are padded to a multiple
// of 32, so a warp's chunk lies in one job and the scene and the ray loop's
// warp votes are warp-uniform.  Each lane bakes one lumel with the same code
// and Philox keys as the single-job calls, so the lumels come out
// bit-identical to rl_bake_direct / rl_bake_ao / rl_bake_indirect.
template <int kKind>
__global__ void __launch_bounds__(kKind == 0 ? 128 : 256, kKind == 0 ? 1 : 4) k_batch(const BatchHeader* __restrict__ hdrs,
                                                                  unsigned long long* counter, int refill) {
    if (hdrs[kKind].total <= 0) return;
    const int lane = threadIdx.x & 31;
    for (;;) {
        // lane 0 takes the next chunk and finds its job; the header is
        // re-read per chunk (L1-resident) so no table state stays live in
        // registers across the ray loop
        unsigned long long jp = 0;
        long long off = -1;
        if (lane == 0) {
            const BatchHeader* H = hdrs + kKind;
            unsigned long long base = atomicAdd(counter + kKind, 32ull);
            long long total = H->total;
            if (base < (unsigned long long)total) {
                int j = find_job(H->prefix, H->njobs, (long long)base);
                jp = (unsigned long long)(H->jobs + j);
                off = (long long)base - H->prefix[j];
            }
        }
        off = __shfl_sync(0xffffffffu, off, 0);
        if (off < 0) break;
        jp = __shfl_sync(0xffffffffu, jp, 0);
        const DevJob& J = *(const DevJob*)jp;
        const long long r = off + lane;
        long long i = 0;
        const bool valid = r < J.count && iter_lumel(J.m, J.it, J.k_begin + r, i);
        if (kKind == 0) {
            if (valid) direct_lumel(J.s, J.m, *J.lights, i, J.status);
        } else if (kKind == 1) {
            const DevScene s = J.s;
            AoGen g;
            g.pos = valid ? ld3(J.m.position + 3 * i) : mk3(0.f, 0.f, 0.f);
            g.nrm = valid ? ld3(J.m.normal + 3 * i) : mk3(0.f, 0.f, 1.f);
            g.key = J.key;
            g.item = (uint32_t)i;
            g.j = 0;
            g.stride = 1;
            g.samples = valid ? J.samples : 0;
            g.occluded = 0;
            g.maxd = J.maxd;
            __syncwarp();
            ray_loop<true>(s, g, refill, J.status);
            if (valid) {
                float value = 1.0f - g.occluded / (J.samples * J.fraction);
                if (fabsf(1.0f - J.exponent) > 0.01f) value = powf(value, J.exponent);
                float* col = J.m.color + 3 * i;
                col[0] = col[0] * value; col[1] = col[1] * value; col[2] = col[2] * value;
            }
        } else {
            const DevScene s = J.s;
            FgGen g;
            g.s = &J.s;
            g.G = J.maps;
            g.pos = valid ? ld3(J.m.position + 3 * i) : mk3(0.f, 0.f, 0.f);
            g.nrm = valid ? ld3(J.m.normal + 3 * i) : mk3(0.f, 0.f, 1.f);
            g.sky = J.sky;
            g.amb = J.amb;
            g.key = J.key;
            g.item = (uint32_t)i;
            g.j = 0;
            g.samples = valid ? J.samples : 0;
            g.maxd = J.maxd;
            g.gr = g.gg = g.gb = 0.f;
            g.influence = 0.f;
            g.dir = mk3(0.f, 0.f, 0.f);
            __syncwarp();
            ray_loop<false>(s, g, refill, J.status);
            if (valid) {
                float ns = (float)J.samples;
                float* col = J.m.color + 3 * i;
                col[0] = col[0] + g.gr / ns; col[1] = col[1] + g.gg / ns; col[2] = col[2] + g.gb / ns;
            }
        }
        __syncwarp();
    }
}

// Work source of the pooled batch kernel: the kind's 32-item chunks in
// counter order, restricted to one job ([job_lo, job_hi) of the kind's item
// space).  A chunk of a later job ends this job's pass and is kept in `next`
// for the warp's next job; `first` is the chunk the pass starts with.
struct BatchSource {
    unsigned long long* counter;
    long long total, job_lo, job_hi, first, next;
    __device__ __forceinline__ bool claim(long long& lo, long long& hi) {
        long long base = first;
        first = -1;
        if (base < 0) {
            unsigned long long b = 0;
            if ((threadIdx.x & 31) == 0) b = atomicAdd(counter, 32ull);
            base = (long long)__shfl_sync(0xffffffffu, b, 0);
        }
        if (base >= total) return false;
        if (base >= job_hi) {
            next = base;
            return false;
        }
        lo = base - job_lo;
        hi = lo + 32;
        return true;
    }
};

// The AO / final-gather batch kernels with ray_loop_pool: a warp keeps its
// lanes on the lumels of one job, taking the job's next chunk as lanes
// finish instead of waiting for the chunk's slowest lumel, and moves to the
// next job when the chunks run past its own.  Same lumels, keys and
// arithmetic as k_batch.
template <int kKind>
__global__ void __launch_bounds__(256, 4) k_batch_pool(const BatchHeader* __restrict__ hdrs,
                                                       unsigned long long* counter, int refill) {
    const BatchHeader* H = hdrs + kKind;
    const long long total = H->total;
    if (total <= 0) return;
    long long next;
    {
        unsigned long long b = 0;
        if ((threadIdx.x & 31) == 0) b = atomicAdd(counter + kKind, 32ull);
        next = (long long)__shfl_sync(0xffffffffu, b, 0);
    }
    while (next >= 0 && next < total) {
        const int jx = find_job(H->prefix, H->njobs, next);
        const DevJob& J = H->jobs[jx];
        BatchSource src{counter + kKind, total, H->prefix[jx], jx + 1 < H->njobs ? H->prefix[jx + 1] : total, next,
                        -1};
        const DevScene s = J.s;
        if (kKind == 1) {
            AoPoolGen g;
            g.map = &J.m;
            g.it = &J.it;
            g.nsamples = J.samples;
            g.fraction = J.fraction;
            g.exponent = J.exponent;
            g.li = 0;
            g.k_begin = J.k_begin;
            g.limit = J.count;
            g.pos = g.nrm = mk3(0.f, 0.f, 0.f);
            g.key = J.key;
            g.item = 0;
            g.j = 0;
            g.stride = 1;
            g.samples = 0;
            g.occluded = 0;
            g.maxd = J.maxd;
            ray_loop_pool<true>(s, g, refill, J.status, src);
        } else {
            FgPoolGen g;
            g.s = &J.s;
            g.G = J.maps;
            g.map = &J.m;
            g.it = &J.it;
            g.nsamples = J.samples;
            g.samples = 0;
            g.j = 0;
            g.li = 0;
            g.k_begin = J.k_begin;
            g.limit = J.count;
            g.sky = J.sky;
            g.amb = J.amb;
            g.key = J.key;
            g.item = 0;
            g.maxd = J.maxd;
            g.gr = g.gg = g.gb = 0.f;
            g.influence = 0.f;
            g.pos = g.nrm = g.dir = mk3(0.f, 0.f, 0.f);
            ray_loop_pool<false>(s, g, refill, J.status, src);
        }
        next = src.next;
        __syncwarp();
    }
}

// Whether two jobs of one pass kind may visit a common lumel (a race: both
// read-modify-write its colour).  Disjoint for sure: different lightmaps;
// face iterators over different meshes; lumel iterators of one step with
// different residues; or one iterator with disjoint [begin, end) slices.
static bool jobs_may_overlap(const rl_batch_job& a, const rl_batch_job& b) {
    if (a.lightmap != b.lightmap) return false;
    const rl_iterator &x = a.iterator, &y = b.iterator;
    if (x.kind == 1 && y.kind == 1 && x.mesh != y.mesh) return false;
    if (x.kind == 0 && y.kind == 0 && x.step == y.step && x.step > 0 && x.first % x.step != y.first % y.step)
        return false;
    if (x.kind == y.kind && x.first == y.first && x.step == y.step && (x.kind == 0 || x.mesh == y.mesh)) {
        long long ab = a.begin < 0 ? 0 : a.begin, bb = b.begin < 0 ? 0 : b.begin;
        long long ae = a.end < 0 ? LLONG_MAX : a.end, be = b.end < 0 ? LLONG_MAX : b.end;
        return ab < be && bb < ae;
    }
    return true;
}

// Relative cost of one work item, for ordering the job table: the most
// expensive items are handed out first so the launch ends on cheap ones.
static double job_item_cost(const rl_batch_job& J) {
    if (J.kind == 2) return 2.0 * J.samples;
    if (J.kind == 1) return (double)J.samples;
    double c = 0;
    for (int l = 0; l < J.nlights; l++) c += J.lights[l].vertex_count > 0 ? J.lights[l].vertex_count : 1;
    return c;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static int batch_init(rl_batch* b) {
    CK(cudaMalloc(&b->d_hdr, 3 * sizeof(BatchHeader)));
    CK(cudaMemset(b->d_hdr, 0, 3 * sizeof(BatchHeader)));
    CK(cudaMalloc(&b->d_counter, 3 * sizeof(unsigned long long)));
    for (int k = 0; k < 2; k++) CK(cudaEventCreateWithFlags(&b->staged[k], cudaEventDisableTiming));
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    b->pool = g_tune[RL_TUNE_FG_POOL] != 0;
    const void* kern[3] = {(const void*)k_batch<0>,
                           b->pool ? (const void*)k_batch_pool<1> : (const void*)k_batch<1>,
                           b->pool ? (const void*)k_batch_pool<2> : (const void*)k_batch<2>};
    b->block[0] = 128;
    b->block[1] = g_tune[RL_TUNE_AO_BLOCK];
    b->block[2] = g_tune[RL_TUNE_FG_BLOCK];
    b->refill[1] = g_tune[RL_TUNE_AO_REFILL];
    b->refill[2] = g_tune[RL_TUNE_FG_REFILL];
    for (int k = 0; k < 3; k++) {
        int per = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern[k], b->block[k], 0));
        b->grid[k] = sms * std::max(per, 1);
    }
    return RL_OK;
}

// Validate `jobs`, lay out the tables (jobs sorted by kind, then by item
// cost), fill the pinned staging slot with device addresses, and enqueue
// the copies on `st`.  On error the batch keeps its previous tables.
// Host-side checks of a job table (no device access).
static int batch_validate(const rl_batch_job* jobs, int njobs) {
    if (njobs < 0 || (njobs > 0 && !jobs)) return fail(RL_INVALID_CALL, "batch: bad job array");
    for (int q = 0; q < njobs; q++) {
        const rl_batch_job& J = jobs[q];
        if (!J.scene || !J.lightmap || J.kind < 0 || J.kind > 2)
            return fail(RL_INVALID_CALL, "batch job %d: bad scene, lightmap or kind", q);
        if (J.kind == 0 && J.nlights > 0 && !J.lights) return fail(RL_INVALID_CALL, "batch job %d: null light array", q);
        if ((J.kind == 1 || J.kind == 2) && J.samples <= 0)
            return fail(RL_INVALID_CALL, "batch job %d: samples must be positive", q);
        if (J.kind == 2 && (J.nmaps < 0 || J.nmaps > kMaxPhotonmaps || (J.nmaps > 0 && !J.photonmaps)))
            return fail(RL_INVALID_CALL, "batch job %d: bad photonmaps", q);
        for (int k = 0; J.kind == 2 && k < J.nmaps; k++)
            if (!J.photonmaps[k]) return fail(RL_INVALID_CALL, "batch job %d: null photonmap", q);
    }
    {
        std::map<std::pair<int, const rl_map*>, std::vector<int>> by_map;
        for (int q = 0; q < njobs; q++) by_map[{jobs[q].kind, jobs[q].lightmap}].push_back(q);
        for (auto& kv : by_map)
            for (size_t x = 0; x < kv.second.size(); x++)
                for (size_t y = x + 1; y < kv.second.size(); y++)
                    if (jobs_may_overlap(jobs[kv.second[x]], jobs[kv.second[y]]))
                        return fail(RL_INVALID_CALL, "batch jobs %d and %d: one pass over shared lumels of one lightmap",
                                    kv.second[x], kv.second[y]);
    }
    return RL_OK;
}

static int batch_update(rl_batch* b, const rl_batch_job* jobs, int njobs, cudaStream_t st) {
    if (int rc = batch_validate(jobs, njobs)) return rc;
    std::vector<int> order(njobs);
    for (int q = 0; q < njobs; q++) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        if (jobs[x].kind != jobs[y].kind) return jobs[x].kind < jobs[y].kind;
        return job_item_cost(jobs[x]) > job_item_cost(jobs[y]);
    });
    // pass 1: slices, counts and the distinct light tables / photonmap sets
    struct Slot { int q; long long b0, count; Iter it; };
    std::vector<Slot> live[3];
    std::map<const rl_light*, int> light_idx;
    std::map<std::vector<const rl_map*>, int> maps_idx;
    std::vector<const rl_batch_job*> light_src, maps_src;
    for (int q : order) {
        const rl_batch_job& J = jobs[q];
        long long n = (long long)J.lightmap->dev.width * J.lightmap->dev.height, count = 0;
        Iter it;
        int rc = make_iter(&J.iterator, J.scene, n, it, count);
        if (rc) return rc;
        long long b0 = J.begin < 0 ? 0 : (J.begin < count ? J.begin : count);
        long long e0 = J.end < 0 || J.end > count ? count : J.end;
        if (e0 < b0) e0 = b0;
        if (J.kind == 0 && J.nlights == 0) e0 = b0;  // rl_bake_direct with no lights bakes nothing
        if (e0 == b0) continue;
        if (J.kind == 0) {
            if (J.nlights > kMaxLights || J.nlight_vertices < 0 || J.nlight_vertices > kMaxLightVerts)
                return fail(RL_INVALID_CALL, "batch job %d: too many lights or light vertices", q);
            if (!light_idx.count(J.lights)) {
                light_idx[J.lights] = (int)light_src.size();
                light_src.push_back(&J);
            }
        }
        if (J.kind == 2) {
            std::vector<const rl_map*> key(J.photonmaps, J.photonmaps + J.nmaps);
            if (!maps_idx.count(key)) {
                maps_idx[key] = (int)maps_src.size();
                maps_src.push_back(&J);
            }
        }
        live[J.kind].push_back(Slot{q, b0, e0 - b0, it});
    }
    // layout
    size_t off_jobs[3], off_prefix[3], off = 0;
    for (int k = 0; k < 3; k++) {
        off_jobs[k] = off;
        off = align256(off + live[k].size() * sizeof(DevJob));
        off_prefix[k] = off;
        off = align256(off + live[k].size() * sizeof(long long));
    }
    size_t off_lights = off;
    off = align256(off + light_src.size() * sizeof(LightTable));
    size_t off_maps = off;
    off = align256(off + maps_src.size() * sizeof(GatherMaps));
    size_t off_hdr = off;
    size_t bytes = off + 3 * sizeof(BatchHeader);
    // device buffer (stream-ordered, so growing it does not stall the device)
    if (bytes > b->d_cap) {
        size_t cap = std::max(bytes, b->d_cap * 2);
        char* nb = nullptr;
        if (int rc = pool_alloc((void**)&nb, cap, st)) return rc;
        if (b->d_buf) CK(cudaFreeAsync(b->d_buf, st));
        b->d_buf = nb;
        b->d_cap = cap;
    }
    // staging slot: wait for the copy that used it last
    int sl = b->slot;
    CK(cudaEventSynchronize(b->staged[sl]));
    if (bytes > b->h_cap[sl]) {
        if (b->h_stage[sl]) CK(cudaFreeHost(b->h_stage[sl]));
        b->h_stage[sl] = nullptr;
        b->h_cap[sl] = 0;
        size_t cap = std::max(bytes, (size_t)1 << 16);
        CK(cudaHostAlloc((void**)&b->h_stage[sl], cap, cudaHostAllocDefault));
        b->h_cap[sl] = cap;
    }
    char* h = b->h_stage[sl];
    char* d = b->d_buf;
    for (size_t t = 0; t < light_src.size(); t++) {
        const rl_batch_job& J = *light_src[t];
        LightTable* T = (LightTable*)(h + off_lights + t * sizeof(LightTable));
        int rc = make_light_table(J.lights, J.nlights, J.light_vertices, J.nlight_vertices, *T);
        if (rc) return rc;
    }
    for (size_t t = 0; t < maps_src.size(); t++) {
        const rl_batch_job& J = *maps_src[t];
        GatherMaps* G = (GatherMaps*)(h + off_maps + t * sizeof(GatherMaps));
        memset(G, 0, sizeof(GatherMaps));
        G->nmaps = J.nmaps;
        for (int k = 0; k < J.nmaps; k++) G->maps[k] = J.photonmaps[k]->dev;
    }
    BatchHeader hdr[3];
    long long items = 0;
    for (int k = 0; k < 3; k++) {
        DevJob* tab = (DevJob*)(h + off_jobs[k]);
        long long* pre = (long long*)(h + off_prefix[k]);
        long long total = 0;
        for (size_t t = 0; t < live[k].size(); t++) {
            const Slot& L = live[k][t];
            const rl_batch_job& J = jobs[L.q];
            DevJob dj;
            memset(&dj, 0, sizeof dj);
            dj.s = J.scene->dev;
            dj.m = J.lightmap->dev;
            dj.status = J.scene->d_status;
            dj.it = L.it;
            dj.k_begin = L.b0;
            dj.count = L.count;
            dj.kind = J.kind;
            dj.samples = J.samples;
            dj.fraction = J.occluded_fraction;
            dj.maxd = J.max_distance;
            dj.exponent = J.exponent;
            dj.sky = V3{J.sky[0], J.sky[1], J.sky[2]};
            dj.amb = V3{J.ambient[0], J.ambient[1], J.ambient[2]};
            dj.key = make_uint2((uint32_t)J.seed, (uint32_t)(J.seed >> 32));
            if (k == 0)
                dj.lights = (const LightTable*)(d + off_lights + light_idx[J.lights] * sizeof(LightTable));
            if (k == 2) {
                std::vector<const rl_map*> key(J.photonmaps, J.photonmaps + J.nmaps);
                dj.maps = (const GatherMaps*)(d + off_maps + maps_idx[key] * sizeof(GatherMaps));
            }
            tab[t] = dj;
            pre[t] = total;
            items += L.count;
            total += (L.count + 31) / 32 * 32;
        }
        hdr[k].jobs = (const DevJob*)(d + off_jobs[k]);
        hdr[k].prefix = (const long long*)(d + off_prefix[k]);
        hdr[k].total = total;
        hdr[k].njobs = (int)live[k].size();
        hdr[k].pad = 0;
        b->total[k] = total;
    }
    memcpy(h + off_hdr, hdr, sizeof hdr);
    b->items = items;
    if (off_hdr > 0) CK(cudaMemcpyAsync(d, h, off_hdr, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(b->d_hdr, h + off_hdr, sizeof hdr, cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(b->staged[sl], st));
    b->slot ^= 1;
    return RL_OK;
}

extern "C" int rl_batch_create(const rl_batch_job* jobs, int njobs, rl_batch** out) {
    if (!out || njobs < 0 || (njobs > 0 && !jobs)) return fail(RL_INVALID_CALL, "rl_batch_create: bad arguments");
    *out = nullptr;
    if (int rc = batch_validate(jobs, njobs)) return rc;
    rl_batch* b = new (std::nothrow) rl_batch;
    if (!b) return fail(RL_OUT_OF_MEMORY, "host allocation failed");
    int rc = batch_init(b);
    if (!rc) rc = batch_update(b, jobs, njobs, 0);
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) rc = fail(RL_CUDA_ERROR, "batch upload: %s", cudaGetErrorString(e));
    }
    if (rc) {
        cudaDeviceSynchronize();
        delete b;
        return rc;
    }
    *out = b;
    return RL_OK;
}

extern "C" int rl_batch_update(rl_batch* b, const rl_batch_job* jobs, int njobs, void* stream) {
    if (!b) return fail(RL_INVALID_CALL, "null batch");
    return batch_update(b, jobs, njobs, S(stream));
}

// The kinds run in sequence on the stream in the order a bake applies them
// to one lightmap (direct light adds, AO scales, final gather adds: the
// demo's Bake job, src/demo/Lightmapping.cpp:270-279, plus AO between), so a
// lightmap baked by several passes of one batch gets the sequential result.
// Every kind is launched (an empty one returns at once), so the launch
// sequence is the same for any table.
static int batch_enqueue(rl_batch* b, cudaStream_t st) {
    CK(cudaMemsetAsync(b->d_counter, 0, 3 * sizeof(unsigned long long), st));
    for (int k = 0; k < 3; k++) {
        auto kern = k == 0 ? k_batch<0>
                    : k == 1 ? (b->pool ? k_batch_pool<1> : k_batch<1>)
                             : (b->pool ? k_batch_pool<2> : k_batch<2>);
        kern<<<b->grid[k], b->block[k], 0, st>>>(b->d_hdr, b->d_counter, b->refill[k]);
        CK_LAUNCH("k_batch");
    }
    return RL_OK;
}

extern "C" int rl_batch_launch(rl_batch* b, void* stream) {
    if (!b) return fail(RL_INVALID_CALL, "null batch");
    if (b->items == 0) return RL_OK;
    return batch_enqueue(b, S(stream));
}

extern "C" int rl_batch_capture(rl_batch* b, void* stream) {
    if (!b) return fail(RL_INVALID_CALL, "null batch");
    if (!stream) return fail(RL_INVALID_CALL, "rl_batch_capture needs a non-default stream");
    cudaStream_t st = S(stream);
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = batch_enqueue(b, st);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(RL_CUDA_ERROR, "stream capture: %s", cudaGetErrorString(e));
    b->graph = g;
    CK(cudaGraphInstantiate(&b->exec, g, 0));
    return RL_OK;
}

extern "C" int rl_batch_replay(rl_batch* b, void* stream) {
    if (!b || !b->exec) return fail(RL_INVALID_CALL, "rl_batch_replay: batch has no captured graph");
    CK(cudaGraphLaunch(b->exec, S(stream)));
    return RL_OK;
}

extern "C" int rl_batch_work_items(const rl_batch* b, int64_t* items) {
    if (!b || !items) return fail(RL_INVALID_CALL, "null argument");
    *items = b->items;
    return RL_OK;
}

extern "C" int rl_batch_destroy(rl_batch* b) {
    if (!b) return fail(RL_INVALID_CALL, "null batch");
    cudaDeviceSynchronize();
    delete b;
    return RL_OK;
}

// ------------------------------------------------- solve without allocation

// The two [n][4] ping-pong iterates of rl_radiosity_solve_noalloc: a fixed
// array in device memory (2 x RL_SOLVE_NOALLOC_MAX_PATCHES float4, 2 MiB).
// It is committed on a device when this file's module first loads there:
// with CUDA's lazy module loading, at the first launch of any kernel of this
// file or at the first rl_radiosity_solve_noalloc call (an n = 0 call is
// enough), and it stays until the process exits.
static __device__ __align__(256) float4 g_solve_scratch[2 * RL_SOLVE_NOALLOC_MAX_PATCHES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
float4* g_scratch_ptr[kMaxDevices] = {};  // device address of g_solve_scratch, per device
}  // namespace

// Host code only sees a host-side stand-in for g_solve_scratch; the device
// address comes from cudaGetSymbolAddress, looked up once per device with
// that device current.
static int solve_scratch(float4** out) {
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(RL_INVALID_CALL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);
        if (e != cudaSuccess || !p)
            return fail(RL_CUDA_ERROR, "cudaGetSymbolAddress(g_solve_scratch) failed on device %d: %s", dev,
                        cudaGetErrorString(e));
        g_scratch_ptr[dev] = (float4*)p;
    }
    *out = g_scratch_ptr[dev];
    return RL_OK;
}

// The kernels and launch sequence of rl_radiosity_solve (k_pack4, k_jacobi4
// with the same 16-byte-load choice, k_unpack4), so the two give the same
// bits.  d_B is written only by the final k_unpack4, after every read of
// d_E and d_rho, so d_B may alias either input.
extern "C" int rl_radiosity_solve_noalloc(int n, const int64_t* d_row_ptr, const int32_t* d_cols,
                                          const float* d_vals, const float* d_E, const float* d_rho, int iters,
                                          float* d_B, void* stream) {
    if (n < 0 || iters < 0 || (n > 0 && (!d_row_ptr || !d_E || !d_rho || !d_B)))
        return fail(RL_INVALID_CALL, "rl_radiosity_solve_noalloc: bad arguments");
    if (n > RL_SOLVE_NOALLOC_MAX_PATCHES)
        return fail(RL_INVALID_CALL, "rl_radiosity_solve_noalloc: %d patches exceed the fixed maximum of %d "
                                     "(use rl_radiosity_solve)", n, RL_SOLVE_NOALLOC_MAX_PATCHES);
    float4* scratch_base = nullptr;
    int rc = solve_scratch(&scratch_base);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    if (n == 0) return RL_OK;
    if (iters == 0) {
        if (d_B != d_E) CK(cudaMemcpyAsync(d_B, d_E, 12 * (size_t)n, cudaMemcpyDeviceToDevice, st));
        return RL_OK;
    }
    // B0 = E; every iteration writes all n entries of its destination before
    // the next one reads them, so what earlier calls left in the array is
    // never read.
    float4* src = scratch_base;
    float4* dst = scratch_base + RL_SOLVE_NOALLOC_MAX_PATCHES;
    k_pack4<<<blocks_for(n, 256), 256, 0, st>>>(n, d_E, src);
    CK_LAUNCH("k_pack4");
    for (int it = 0; it < iters; it++) {
        if (int rc2 = jacobi4_step(n, d_row_ptr, d_cols, d_vals, d_E, d_rho, src, dst, st)) return rc2;
        std::swap(src, dst);
    }
    k_unpack4<<<blocks_for(n, 256), 256, 0, st>>>(n, src, d_B);
    CK_LAUNCH("k_unpack4");
    return RL_OK;
}

// ------------------------------------------------------------ bandwidth probe

// Streams `bytes` of device memory `iters` times with 16-byte loads (a
// grid of 4 x 148 x 8 blocks of 256 threads); with bytes well under the
// 126 MB L2 the loads are served from L2 after the first pass.
__global__ void k_read_probe(const float4* __restrict__ buf, size_t n4, int iters, float* sink) {
    float acc = 0.f;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (int it = 0; it < iters; it++)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
            float4 v = __ldcg(buf + i);
            acc += v.x + v.y + v.z + v.w;
        }
    if (acc == 1234.5f) *sink = acc;
}

extern "C" int rl_measure_read_bandwidth(size_t bytes, int iters, double* gbs) {
    if (!gbs || bytes < 4096 || iters <= 0) return fail(RL_INVALID_CALL, "rl_measure_read_bandwidth: bad arguments");
    float4* buf = nullptr;
    float* sink = nullptr;
    CK(cudaMalloc(&buf, bytes));
    CK(cudaMalloc(&sink, sizeof(float)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaMemset(buf, 0, bytes));
    size_t n4 = bytes / 16;
    k_read_probe<<<4 * 148 * 8, 256>>>(buf, n4, 1, sink);  // warm
    CK(cudaEventRecord(e0));
    k_read_probe<<<4 * 148 * 8, 256>>>(buf, n4, iters, sink);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *gbs = (double)bytes * iters / (ms * 1e-3) / 1e9;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(sink);
    return RL_OK;
}

// Each block walks the same `n4` float4s (a multiple of 1024) `iters` times
// with ld.global.nc (L1-cached) loads, four independent loads in flight per
// thread: 148 x 4 blocks of 256 threads; after the first pass every load is
// an L1 hit.
__global__ void __launch_bounds__(256) k_read_probe_l1(const float4* __restrict__ buf, size_t n4, int iters,
                                                       float* sink) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    for (int it = 0; it < iters; it++)
        for (size_t i = threadIdx.x; i + 3 * 256 < n4; i += 4 * 256) {
            const float4 v0 = __ldg(buf + i), v1 = __ldg(buf + i + 256), v2 = __ldg(buf + i + 512),
                         v3 = __ldg(buf + i + 768);
            a0 += v0.x + v0.w;
            a1 += v1.x + v1.w;
            a2 += v2.x + v2.w;
            a3 += v3.x + v3.w;
        }
    if (a0 + a1 + a2 + a3 == 1234.5f) *sink = a0;
}

extern "C" int rl_measure_l1_read_bandwidth(size_t bytes_per_block, int iters, double* gbs) {
    if (!gbs || bytes_per_block < 16384 || bytes_per_block > (128u << 10) || bytes_per_block % 16384 || iters <= 0)
        return fail(RL_INVALID_CALL, "rl_measure_l1_read_bandwidth: bad arguments (16 KiB multiple, at most 128 KiB)");
    float4* buf = nullptr;
    float* sink = nullptr;
    CK(cudaMalloc(&buf, bytes_per_block));
    CK(cudaMalloc(&sink, sizeof(float)));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaMemset(buf, 0, bytes_per_block));
    const size_t n4 = bytes_per_block / 16;
    const int blocks = 4 * 148;
    k_read_probe_l1<<<blocks, 256>>>(buf, n4, 1, sink);  // warm
    CK(cudaEventRecord(e0));
    k_read_probe_l1<<<blocks, 256>>>(buf, n4, iters, sink);
    CK(cudaEventRecord(e1));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *gbs = (double)bytes_per_block * blocks * iters / (ms * 1e-3) / 1e9;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(sink);
    return RL_OK;
}
