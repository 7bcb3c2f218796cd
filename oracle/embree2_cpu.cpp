/*
 * A project-written implementation of the eleven Embree 2 C-API entry points
 * that the reference's rt/Embree.cpp calls (rtcInit :39, rtcExit :45,
 * rtcNewScene :51, rtcCommit :57, rtcIntersect4 :88, rtcOccluded :139,
 * rtcIntersect :151, rtcNewTriangleMesh :183, rtcMapBuffer :186/:201,
 * rtcUnmapBuffer :198/:213, rtcDeleteScene :44), over the oracle's CPU BVH
 * (ort.c).  Intel ships Embree 2 only as macOS/Windows binaries, so this
 * stands in for it and lets the reference's own rt/Embree.cpp — hit
 * post-processing, HitUseAlpha loop and all — compile and run unchanged.
 *
 * TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/librelight_ref.so, never
 * into the product.  The contract follows embree2/rtcore_ray.h:24-51 (hit
 * sets tfar = t, u, v, Ng, geomID, primID; a miss leaves geomID/primID at
 * RTC_INVALID_GEOMETRY_ID) and rtcore_scene.h (rtcOccluded sets geomID = 0 on
 * an occluded ray).
 */
#include <embree2/rtcore.h>
#include <embree2/rtcore_ray.h>

#include <cstdlib>
#include <vector>

#include "ort.h"

namespace {

struct Geometry {
    std::vector<float> verts;  // 4 floats per vertex (x, y, z, a)
    std::vector<int>   tris;   // 3 ints per triangle
};

struct Scene {
    std::vector<Geometry*> geoms;
    ort_scene* bvh = nullptr;
};

inline Scene* S(RTCScene s) { return reinterpret_cast<Scene*>(s); }

void fill_hit(const ort_hit& h, float& tfar, float* Ng, float& u, float& v, int& geomID, int& primID,
              const Scene* sc) {
    tfar = h.t; u = h.u; v = h.v; geomID = h.geom; primID = h.prim;
    const Geometry* g = sc->geoms[h.geom];
    const int* tri = &g->tris[3 * h.prim];
    const float* p0 = &g->verts[4 * tri[0]];
    const float* p1 = &g->verts[4 * tri[1]];
    const float* p2 = &g->verts[4 * tri[2]];
    float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    float e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    Ng[0] = e1[1] * e2[2] - e1[2] * e2[1];
    Ng[1] = e1[2] * e2[0] - e1[0] * e2[2];
    Ng[2] = e1[0] * e2[1] - e1[1] * e2[0];
}

}  // namespace

RTCORE_API void rtcInit(const char*) {}
RTCORE_API void rtcExit() {}

RTCORE_API RTCScene rtcNewScene(RTCSceneFlags, RTCAlgorithmFlags) {
    return reinterpret_cast<RTCScene>(new Scene);
}

RTCORE_API void rtcDeleteScene(RTCScene scene) {
    Scene* s = S(scene);
    if (!s) return;
    for (Geometry* g : s->geoms) delete g;
    if (s->bvh) ort_destroy(s->bvh);
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

RTCORE_API void rtcCommit(RTCScene scene) {
    Scene* s = S(scene);
    if (s->bvh) ort_destroy(s->bvh);
    s->bvh = ort_create();
    for (Geometry* g : s->geoms)
        ort_add_mesh(s->bvh, g->verts.data(), 4, static_cast<int>(g->verts.size() / 4), g->tris.data(),
                     static_cast<int>(g->tris.size() / 3));
    ort_commit(s->bvh);
}

RTCORE_API void rtcIntersect(RTCScene scene, RTCRay& ray) {
    Scene* s = S(scene);
    ort_hit h;
    if (ort_intersect(s->bvh, ray.org, ray.dir, ray.tnear, ray.tfar, &h, nullptr))
        fill_hit(h, ray.tfar, ray.Ng, ray.u, ray.v, ray.geomID, ray.primID, s);
}

RTCORE_API void rtcOccluded(RTCScene scene, RTCRay& ray) {
    Scene* s = S(scene);
    if (ort_occluded(s->bvh, ray.org, ray.dir, ray.tnear, ray.tfar, nullptr)) ray.geomID = 0;
}

RTCORE_API void rtcIntersect4(const void* valid, RTCScene scene, RTCRay4& r) {
    Scene* s = S(scene);
    const int* vmask = static_cast<const int*>(valid);
    for (int i = 0; i < 4; i++) {
        if (vmask && vmask[i] == 0) continue;
        float o[3] = {r.orgx[i], r.orgy[i], r.orgz[i]};
        float d[3] = {r.dirx[i], r.diry[i], r.dirz[i]};
        ort_hit h;
        if (ort_intersect(s->bvh, o, d, r.tnear[i], r.tfar[i], &h, nullptr)) {
            float Ng[3];
            fill_hit(h, r.tfar[i], Ng, r.u[i], r.v[i], r.geomID[i], r.primID[i], s);
            r.Ngx[i] = Ng[0]; r.Ngy[i] = Ng[1]; r.Ngz[i] = Ng[2];
        }
    }
}
