/*
 * The eleven Embree 2 C-API entry points that the reference's rt/Embree.cpp
 * calls (rtcInit :39, rtcExit :45, rtcNewScene :51, rtcCommit :57,
 * rtcIntersect4 :88, rtcOccluded :139, rtcIntersect :151, rtcNewTriangleMesh
 * :183, rtcMapBuffer :186/:201, rtcUnmapBuffer :198/:213, rtcDeleteScene
 * :44), served by the B200 library: rtcCommit builds an rl_scene (the
 * library's BVH on the GPU) from the mapped vertex and index buffers, and
 * every rtcIntersect / rtcIntersect4 / rtcOccluded is one batch of
 * rl_intersect_rays_host.
 *
 * Linked with the reference's own sources (oracle/Makefile:
 * _ref/librelight_ref_gpu.so) in place of oracle/embree2_cpu.cpp, it runs the
 * reference's rt::Embree — its rt::ITracer, hit post-processing and
 * HitUseAlpha loop included — and every baker above it unchanged, with only
 * the ray queries on the GPU.  The bakers ask for one ray at a time, so this
 * backend is for parity (the same hits as the CPU backend, bit for bit), not
 * speed: the library's bake passes keep whole lightmaps of rays on the device.
 *
 * Contract as embree2_cpu.cpp: a hit sets tfar = t, u, v, Ng, geomID,
 * primID; a miss leaves the ray as it was; rtcOccluded sets geomID = 0 on an
 * occluded ray.
 */
#include <embree2/rtcore.h>
#include <embree2/rtcore_ray.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../include/relight_b200.h"

namespace {

struct Geometry {
    std::vector<float> verts;  // 4 floats per vertex (x, y, z, a), as Embree maps them
    std::vector<int> tris;     // 3 ints per triangle
};

struct Scene {
    std::vector<Geometry*> geoms;
    rl_scene* gpu = nullptr;
};

inline Scene* S(RTCScene s) { return reinterpret_cast<Scene*>(s); }

void die(const char* what) {
    char buf[512];
    rl_last_error(buf, sizeof buf);
    fprintf(stderr, "embree2_gpu: %s failed: %s\n", what, buf);
    abort();
}

// Geometric normal, as embree2_cpu.cpp computes it.
void normal_of(const Scene* sc, int geom, int prim, float* Ng) {
    const Geometry* g = sc->geoms[geom];
    const int* tri = &g->tris[3 * prim];
    const float* p0 = &g->verts[4 * tri[0]];
    const float* p1 = &g->verts[4 * tri[1]];
    const float* p2 = &g->verts[4 * tri[2]];
    float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    Ng[0] = e1[1] * e2[2] - e1[2] * e2[1];
    Ng[1] = e1[2] * e2[0] - e1[0] * e2[2];
    Ng[2] = e1[0] * e2[1] - e1[1] * e2[0];
}

// The rays of one call, 8 floats each: org xyz, tnear, dir xyz, tfar.
struct alignas(16) Ray8 {
    float v[8];
};

void query(Scene* s, std::vector<Ray8>& rays, int any_hit, std::vector<int>& gp, std::vector<float>& tuv) {
    gp.assign(2 * rays.size(), -1);
    tuv.assign(3 * rays.size(), 0.0f);
    if (!s->gpu) return;  // empty scene: every ray misses
    if (rl_intersect_rays_host(s->gpu, (int64_t)rays.size(), &rays[0].v[0], any_hit, gp.data(), tuv.data()) != RL_OK)
        die("rl_intersect_rays_host");
}

}  // namespace

RTCORE_API void rtcInit(const char*) {}
RTCORE_API void rtcExit() {}

RTCORE_API RTCScene rtcNewScene(RTCSceneFlags, RTCAlgorithmFlags) { return reinterpret_cast<RTCScene>(new Scene); }

RTCORE_API void rtcDeleteScene(RTCScene scene) {
    Scene* s = S(scene);
    if (!s) return;
    for (Geometry* g : s->geoms) delete g;
    if (s->gpu) rl_scene_destroy(s->gpu);
    delete s;
}

RTCORE_API unsigned rtcNewTriangleMesh(RTCScene scene, RTCGeometryFlags, size_t numTriangles, size_t numVertices,
                                       size_t) {
    Scene* s = S(scene);
    Geometry* g = new Geometry;
    g->verts.assign(4 * numVertices, 0.0f);
    g->tris.assign(3 * numTriangles, 0);
    s->geoms.push_back(g);
    return static_cast<unsigned>(s->geoms.size() - 1);
}

RTCORE_API void* rtcMapBuffer(RTCScene scene, unsigned geomID, RTCBufferType type) {
    Geometry* g = S(scene)->geoms[geomID];
    if (type == RTC_INDEX_BUFFER) return g->tris.data();
    return g->verts.data();
}

RTCORE_API void rtcUnmapBuffer(RTCScene, unsigned, RTCBufferType) {}

// One rl_scene over all geometries: geometry k is scene mesh k, its faces in
// order, so (geomID, primID) come back as Embree numbers them.  Only
// positions matter for intersection; the other attributes stay zero.
RTCORE_API void rtcCommit(RTCScene scene) {
    Scene* s = S(scene);
    if (s->gpu) rl_scene_destroy(s->gpu);
    s->gpu = nullptr;
    std::vector<float> pos, zero3, zero2;
    std::vector<int32_t> tris, first, none, vmat;
    float lo[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float hi[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    int base = 0, ntris = 0;
    for (Geometry* g : s->geoms) {
        const int nv = (int)(g->verts.size() / 4);
        for (int v = 0; v < nv; v++)
            for (int k = 0; k < 3; k++) {
                const float x = g->verts[4 * v + k];
                pos.push_back(x);
                lo[k] = x < lo[k] ? x : lo[k];
                hi[k] = x > hi[k] ? x : hi[k];
            }
        first.push_back(ntris);
        for (int t : g->tris) tris.push_back(base + t);
        ntris += (int)(g->tris.size() / 3);
        base += nv;
    }
    first.push_back(ntris);
    if (ntris == 0) return;
    zero3.assign(pos.size(), 0.0f);
    zero2.assign(2 * (size_t)base, 0.0f);
    vmat.assign(base, -1);
    none.assign(s->geoms.size(), -1);
    rl_scene_desc d;
    d.nverts = base;
    d.pos = pos.data();
    d.nrm = zero3.data();
    d.uv0 = zero2.data();
    d.uv1 = zero2.data();
    d.vmat = vmat.data();
    d.ntris = ntris;
    d.tris = tris.data();
    d.nmeshes = (int32_t)s->geoms.size();
    d.mesh_first_tri = first.data();
    d.mesh_lightmap = none.data();
    d.mesh_photonmap = none.data();
    d.nmats = 0;
    d.mat_rgb = nullptr;
    d.mat_tex = nullptr;
    d.ntex = 0;
    d.tex_dims = nullptr;
    d.tex_offset = nullptr;
    d.tex_pixels = nullptr;
    for (int k = 0; k < 3; k++) {
        d.bounds_lo[k] = lo[k];
        d.bounds_hi[k] = hi[k];
    }
    if (rl_scene_create(&d, 0, nullptr, &s->gpu) != RL_OK) die("rl_scene_create");
}

RTCORE_API void rtcIntersect(RTCScene scene, RTCRay& ray) {
    Scene* s = S(scene);
    std::vector<Ray8> rays(1);
    rays[0] = Ray8{{ray.org[0], ray.org[1], ray.org[2], ray.tnear, ray.dir[0], ray.dir[1], ray.dir[2], ray.tfar}};
    std::vector<int> gp;
    std::vector<float> tuv;
    query(s, rays, 0, gp, tuv);
    if (gp[0] < 0) return;
    ray.tfar = tuv[0];
    ray.u = tuv[1];
    ray.v = tuv[2];
    ray.geomID = gp[0];
    ray.primID = gp[1];
    normal_of(s, gp[0], gp[1], ray.Ng);
}

RTCORE_API void rtcOccluded(RTCScene scene, RTCRay& ray) {
    Scene* s = S(scene);
    std::vector<Ray8> rays(1);
    rays[0] = Ray8{{ray.org[0], ray.org[1], ray.org[2], ray.tnear, ray.dir[0], ray.dir[1], ray.dir[2], ray.tfar}};
    std::vector<int> gp;
    std::vector<float> tuv;
    query(s, rays, 1, gp, tuv);
    if (gp[0] >= 0) ray.geomID = 0;
}

RTCORE_API void rtcIntersect4(const void* valid, RTCScene scene, RTCRay4& r) {
    Scene* s = S(scene);
    const int* vmask = static_cast<const int*>(valid);
    std::vector<Ray8> rays;
    std::vector<int> lane;
    for (int i = 0; i < 4; i++) {
        if (vmask && vmask[i] == 0) continue;
        rays.push_back(Ray8{{r.orgx[i], r.orgy[i], r.orgz[i], r.tnear[i], r.dirx[i], r.diry[i], r.dirz[i], r.tfar[i]}});
        lane.push_back(i);
    }
    if (rays.empty()) return;
    std::vector<int> gp;
    std::vector<float> tuv;
    query(s, rays, 0, gp, tuv);
    for (size_t k = 0; k < lane.size(); k++) {
        if (gp[2 * k] < 0) continue;
        const int i = lane[k];
        r.tfar[i] = tuv[3 * k];
        r.u[i] = tuv[3 * k + 1];
        r.v[i] = tuv[3 * k + 2];
        r.geomID[i] = gp[2 * k];
        r.primID[i] = gp[2 * k + 1];
        float Ng[3];
        normal_of(s, gp[2 * k], gp[2 * k + 1], Ng);
        r.Ngx[i] = Ng[0];
        r.Ngy[i] = Ng[1];
        r.Ngz[i] = Ng[2];
    }
}
