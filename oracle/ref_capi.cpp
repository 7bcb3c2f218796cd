/*
 * C-ABI driver over the reference baker compiled from its own sources
 * (Relight.cpp, Lightmap.cpp, Worker.cpp, baker/*.cpp, scene/*.cpp,
 * radiosity/*.cpp, rt/Embree.cpp) — the "reference" arm of the oracle.
 * TEST INFRASTRUCTURE ONLY: tests/ and bench.py's reference / cpu_baseline
 * legs load oracle/_ref/librelight_ref.so through ctypes; the product never
 * does.
 *
 * Everything here drives the reference through its public API
 * (Relight.h:155-189, scene/Scene.h:49-84, scene/Light.h:292-301,
 * Lightmap.h:63-121) and its own thread fan-out (Relight::bake ->
 * FullBakeJob::execute, Worker.cpp:43-83).  Three things the public API
 * cannot reach are opened with the access hack below:
 *   - Radiancemap's private constructor (Lightmap.h:180-183; no factory
 *     exists, so the radiosity builder is otherwise unreachable),
 *   - Radiosity::patchCount/patch, declared at radiosity/Radiosity.h:75-81
 *     but never defined in the reference; defined here,
 *   - Mesh vertex/index buffers, filled exactly as Mesh::addFaces does
 *     (scene/Mesh.cpp:146-165) but with a per-vertex material.
 * It also supplies Rgb::Rgb(const Rgba&), declared at Types.h:161 but never
 * defined, without which the reference does not link.
 *
 * rand(): the reference draws every random number from the C library's
 * global rand() (Types.h:110-113).  This file interposes rand/srand with a
 * per-thread generator (the .so is linked -Bsymbolic so the reference's calls
 * bind here) so that threads do not serialise on glibc's lock; mode 1 calls
 * through to glibc's own rand() instead.
 */
#include <atomic>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <dlfcn.h>
#include <thread>
#include <vector>

#define private public
#define protected public
#include "Relight.h"
#include "Lightmap.h"
#include "Worker.h"
#include "scene/Scene.h"
#include "scene/Mesh.h"
#include "scene/Light.h"
#include "scene/Material.h"
#include "baker/Baker.h"
#include "radiosity/Radiosity.h"
#include "radiosity/RadiosityBuilder.h"
#include "rt/Tracer.h"
#undef private
#undef protected

using namespace relight;

/* ------------------------------------------------------------- rand() */

static std::atomic<int> g_rand_mode{0};
static std::atomic<uint64_t> g_rand_seed{12345};
static std::atomic<int> g_thread_ordinal{0};
static std::atomic<uint64_t> g_rand_epoch{0};

struct TlsRand {
    uint64_t state = 0;
    uint64_t epoch = ~0ull;
    int ordinal = -1;
};
static thread_local TlsRand t_rand;

static inline uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

extern "C" int rand(void) {
    if (g_rand_mode.load(std::memory_order_relaxed) == 1) {
        static int (*real_rand)(void) = (int (*)(void))dlsym(RTLD_NEXT, "rand");
        return real_rand();
    }
    TlsRand& r = t_rand;
    uint64_t ep = g_rand_epoch.load(std::memory_order_relaxed);
    if (r.epoch != ep) {
        if (r.ordinal < 0) r.ordinal = g_thread_ordinal.fetch_add(1);
        r.epoch = ep;
        r.state = g_rand_seed.load() * 0x100000001B3ull + (uint64_t)r.ordinal * 0x9E3779B97F4A7C15ull;
    }
    return (int)(splitmix64(r.state) >> 33);  /* [0, 2^31-1] = [0, RAND_MAX] */
}

extern "C" void srand(unsigned seed) {
    if (g_rand_mode.load() == 1) {
        static void (*real_srand)(unsigned) = (void (*)(unsigned))dlsym(RTLD_NEXT, "srand");
        real_srand(seed);
        return;
    }
    g_rand_seed.store(seed);
    g_rand_epoch.fetch_add(1);
}

/* Radiosity::patchCount / patch are declared (radiosity/Radiosity.h:75-81)
   but have no definition anywhere in the reference; neither has
   Rgb::Rgb(const Rgba&) (Types.h:161), which Photons::trace calls
   (baker/Photons.cpp:119).  Defined here with their evident meaning. */
namespace relight {
Rgb::Rgb(const Rgba& other) : r(other.r), g(other.g), b(other.b) {}
s32 Radiosity::patchCount(void) const { return (s32)m_patches.size(); }
Radiosity::Patch& Radiosity::patch(s32 index) { return m_patches[index]; }
const Radiosity::Patch& Radiosity::patch(s32 index) const { return m_patches[index]; }
}  // namespace relight

/* ------------------------------------------------------------- handles */

struct RefCtx {
    Relight* relight = nullptr;
    Scene* scene = nullptr;
    std::vector<Material*> materials;
    std::vector<Texture*> textures;
    std::vector<Mesh*> meshes;        /* scene instances (Scene::addMesh copies) */
    std::vector<Mesh*> light_meshes;  /* source meshes of area lights */
    std::vector<Light*> lights;
    std::vector<Lightmap*> maps;      /* lightmaps, photonmaps and radiancemaps */
    std::vector<int> map_kind;        /* 0 lightmap, 1 photonmap, 2 radiancemap */
    Radiosity radiosity;
};

static Mesh* build_mesh(RefCtx* c, int nverts, const float* pos, const float* nrm, const float* uv0,
                        const float* uv1, const int* vmat, int nidx, const int* idx) {
    Mesh* m = Mesh::create();
    for (int i = 0; i < nidx; i++) m->m_indices.push_back((Index)idx[i]);
    for (int i = 0; i < nverts; i++) {
        Vertex v;
        v.position = Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        v.normal = nrm ? Vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]) : Vec3(0, 0, 0);
        v.uv[0] = uv0 ? Vec2(uv0[2 * i], uv0[2 * i + 1]) : Vec2();
        v.uv[1] = uv1 ? Vec2(uv1[2 * i], uv1[2 * i + 1]) : Vec2();
        v.material = (vmat && vmat[i] >= 0) ? c->materials[vmat[i]] : NULL;
        m->m_vertices.push_back(v);
    }
    m->buildFaces();
    return m;
}

extern "C" {

void* ref_create(void) {
    RefCtx* c = new RefCtx;
    c->relight = Relight::create();
    c->scene = c->relight->createScene();
    c->scene->begin();
    return c;
}

void ref_destroy(void* h) {
    RefCtx* c = (RefCtx*)h;
    /* Objects are leaked on purpose where the reference's destructors are
       unsafe (Progress::~Progress asserts); the process is a test runner. */
    delete c;
}

void ref_set_rand(int mode, unsigned seed) {
    g_rand_mode.store(mode);
    srand(seed);
}

int ref_add_material(void* h, float r, float g, float b, int tex_w, int tex_h, int tex_c, const unsigned char* px) {
    RefCtx* c = (RefCtx*)h;
    Material* m;
    if (px) {
        Texture* t = Texture::create(tex_w, tex_h, tex_c, px);
        c->textures.push_back(t);
        m = new TexturedMaterial(t, Rgb(r, g, b));
    } else {
        m = new Material(Rgb(r, g, b));
    }
    c->materials.push_back(m);
    return (int)c->materials.size() - 1;
}

/* Scene::addMesh(mesh, identity, NULL) (scene/Scene.cpp:98-107). */
int ref_add_mesh(void* h, int nverts, const float* pos, const float* nrm, const float* uv0, const float* uv1,
                 const int* vmat, int nidx, const int* idx) {
    RefCtx* c = (RefCtx*)h;
    Mesh* src = build_mesh(c, nverts, pos, nrm, uv0, uv1, vmat, nidx, idx);
    Mesh* inst = c->scene->addMesh(src, Matrix4(), NULL);
    c->meshes.push_back(inst);
    return (int)c->meshes.size() - 1;
}

/* Scene::addMesh(mesh, M, NULL) with a caller-supplied Matrix4 (16 floats,
   Types.h:1177-1185 member order). */
int ref_add_mesh_transformed(void* h, int nverts, const float* pos, const float* nrm, const float* uv0,
                             const float* uv1, const int* vmat, int nidx, const int* idx, const float* m) {
    RefCtx* c = (RefCtx*)h;
    Mesh* src = build_mesh(c, nverts, pos, nrm, uv0, uv1, vmat, nidx, idx);
    Matrix4 M(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8], m[9], m[10], m[11], m[12], m[13], m[14], m[15]);
    Mesh* inst = c->scene->addMesh(src, M, NULL);
    c->meshes.push_back(inst);
    return (int)c->meshes.size() - 1;
}

/* Read back a scene mesh's (transformed) vertex positions and normals. */
void ref_mesh_vertices(void* h, int mesh, float* pos, float* nrm) {
    RefCtx* c = (RefCtx*)h;
    Mesh* m = c->meshes[mesh];
    for (int i = 0; i < m->vertexCount(); i++) {
        const Vertex& v = m->vertex(i);
        pos[3 * i] = v.position.x; pos[3 * i + 1] = v.position.y; pos[3 * i + 2] = v.position.z;
        nrm[3 * i] = v.normal.x; nrm[3 * i + 1] = v.normal.y; nrm[3 * i + 2] = v.normal.z;
    }
}

int ref_add_point_light(void* h, const float* p, float radius, const float* rgb, float intensity, int shadow) {
    RefCtx* c = (RefCtx*)h;
    Light* l = Light::createPointLight(Vec3(p[0], p[1], p[2]), radius, Rgb(rgb[0], rgb[1], rgb[2]), intensity,
                                       shadow != 0);
    c->lights.push_back(l); c->scene->addLight(l);
    return (int)c->lights.size() - 1;
}

int ref_add_spot_light(void* h, const float* p, const float* dir, float cutoff, float radius, const float* rgb,
                       float intensity, int shadow) {
    RefCtx* c = (RefCtx*)h;
    Light* l = Light::createSpotLight(Vec3(p[0], p[1], p[2]), Vec3(dir[0], dir[1], dir[2]), cutoff, radius,
                                      Rgb(rgb[0], rgb[1], rgb[2]), intensity, shadow != 0);
    c->lights.push_back(l); c->scene->addLight(l);
    return (int)c->lights.size() - 1;
}

int ref_add_directional_light(void* h, const float* dir, const float* rgb, float intensity, int shadow) {
    RefCtx* c = (RefCtx*)h;
    Light* l = Light::createDirectionalLight(Vec3(dir[0], dir[1], dir[2]), Rgb(rgb[0], rgb[1], rgb[2]),
                                             intensity, shadow != 0);
    c->lights.push_back(l); c->scene->addLight(l);
    return (int)c->lights.size() - 1;
}

/* Light::createAreaLight over a light mesh given as arrays (not added to the scene). */
int ref_add_area_light(void* h, int nverts, const float* pos, const float* nrm, int nidx, const int* idx,
                       const float* p, const float* rgb, float intensity, int shadow) {
    RefCtx* c = (RefCtx*)h;
    Mesh* m = build_mesh(c, nverts, pos, nrm, nullptr, nullptr, nullptr, nidx, idx);
    c->light_meshes.push_back(m);
    Light* l = Light::createAreaLight(m, Vec3(p[0], p[1], p[2]), Rgb(rgb[0], rgb[1], rgb[2]), intensity,
                                      shadow != 0);
    c->lights.push_back(l); c->scene->addLight(l);
    return (int)c->lights.size() - 1;
}

void ref_light_set_attenuation(void* h, int light, float radius, float k_const, float k_lin, float k_quad) {
    RefCtx* c = (RefCtx*)h;
    Light* l = c->lights[light];
    l->setAttenuation(new LinearLightAttenuation(l, radius, k_const, k_lin, k_quad));
}

void ref_light_clear_emitter(void* h, int light) {
    RefCtx* c = (RefCtx*)h;
    c->lights[light]->setPhotonEmitter(NULL);
}

/* Area light sample points (FaceLightVertexGenerator output, light-local). */
int ref_light_vertices(void* h, int light, float* out) {
    RefCtx* c = (RefCtx*)h;
    LightVertexGenerator* g = c->lights[light]->vertexGenerator();
    if (!g) return 0;
    const LightVertexBuffer& v = g->vertices();
    if (out)
        for (int i = 0; i < (int)v.size(); i++) {
            out[3 * i] = v[i].m_position.x; out[3 * i + 1] = v[i].m_position.y; out[3 * i + 2] = v[i].m_position.z;
        }
    return (int)v.size();
}

/* kind: 0 Lightmap, 1 Photonmap, 2 Radiancemap. */
int ref_create_map(void* h, int kind, int w, int hgt) {
    RefCtx* c = (RefCtx*)h;
    Lightmap* m;
    if (kind == 0) m = c->relight->createLightmap(w, hgt);
    else if (kind == 1) m = c->relight->createPhotonmap(w, hgt);
    else m = new Radiancemap(w, hgt);
    c->maps.push_back(m); c->map_kind.push_back(kind);
    return (int)c->maps.size() - 1;
}

int ref_map_add_mesh(void* h, int map, int mesh) {
    RefCtx* c = (RefCtx*)h;
    Lightmap* m = c->maps[map];
    switch (c->map_kind[map]) {
    case 1: return ((Photonmap*)m)->addMesh(c->meshes[mesh]);
    case 2: return ((Radiancemap*)m)->addMesh(c->meshes[mesh]);
    default: return m->addMesh(c->meshes[mesh]);
    }
}

int ref_scene_end(void* h) {
    RefCtx* c = (RefCtx*)h;
    return c->scene->end();
}

void ref_scene_bounds(void* h, float* lo, float* hi) {
    RefCtx* c = (RefCtx*)h;
    const Bounds& b = c->scene->bounds();
    lo[0] = b.min().x; lo[1] = b.min().y; lo[2] = b.min().z;
    hi[0] = b.max().x; hi[1] = b.max().y; hi[2] = b.max().z;
}

/* Lumel read-back: any output may be NULL. */
void ref_map_lumels(void* h, int map, int* flags, int* face, float* pos, float* nrm, float* color, int* photons,
                    float* gathered) {
    RefCtx* c = (RefCtx*)h;
    Lightmap* m = c->maps[map];
    int n = m->width() * m->height();
    Lumel* L = m->lumels();
    for (int i = 0; i < n; i++) {
        if (flags) flags[i] = L[i].m_flags;
        if (face) face[i] = L[i].m_faceIdx;
        if (pos) { pos[3 * i] = L[i].m_position.x; pos[3 * i + 1] = L[i].m_position.y; pos[3 * i + 2] = L[i].m_position.z; }
        if (nrm) { nrm[3 * i] = L[i].m_normal.x; nrm[3 * i + 1] = L[i].m_normal.y; nrm[3 * i + 2] = L[i].m_normal.z; }
        if (color) { color[3 * i] = L[i].m_color.r; color[3 * i + 1] = L[i].m_color.g; color[3 * i + 2] = L[i].m_color.b; }
        if (photons) photons[i] = L[i].m_photons;
        if (gathered) { gathered[3 * i] = L[i].m_gathered.r; gathered[3 * i + 1] = L[i].m_gathered.g; gathered[3 * i + 2] = L[i].m_gathered.b; }
    }
}

void ref_map_set_colors(void* h, int map, const float* color) {
    RefCtx* c = (RefCtx*)h;
    Lightmap* m = c->maps[map];
    int n = m->width() * m->height();
    Lumel* L = m->lumels();
    for (int i = 0; i < n; i++) L[i].m_color = Rgb(color[3 * i], color[3 * i + 1], color[3 * i + 2]);
}

/* Mesh::createFromFile -> MeshLoader::load (scene/Mesh.cpp:111-122,
   scene/MeshLoader.cpp:44-226), run by the reference itself.  Returns the
   vertex count (-1 if the file cannot be opened); the arrays (any may be
   NULL) receive position, normal, uv[Diffuse], uv[Lightmap] per vertex and
   the 16-bit indices. */
static Mesh* g_obj_mesh = nullptr;
int ref_load_obj(const char* path, int* nindices) {
    delete g_obj_mesh;
    g_obj_mesh = Mesh::createFromFile(path);
    if (!g_obj_mesh) return -1;
    if (nindices) *nindices = g_obj_mesh->indexCount();
    return g_obj_mesh->vertexCount();
}
void ref_obj_arrays(float* pos, float* nrm, float* uv0, float* uv1, int* idx) {
    Mesh* m = g_obj_mesh;
    if (!m) return;
    for (int i = 0; i < m->vertexCount(); i++) {
        const Vertex& v = m->vertex(i);
        if (pos) { pos[3 * i] = v.position.x; pos[3 * i + 1] = v.position.y; pos[3 * i + 2] = v.position.z; }
        if (nrm) { nrm[3 * i] = v.normal.x; nrm[3 * i + 1] = v.normal.y; nrm[3 * i + 2] = v.normal.z; }
        if (uv0) { uv0[2 * i] = v.uv[0].x; uv0[2 * i + 1] = v.uv[0].y; }
        if (uv1) { uv1[2 * i] = v.uv[1].x; uv1[2 * i + 1] = v.uv[1].y; }
    }
    if (idx)
        for (int i = 0; i < m->indexCount(); i++) idx[i] = m->index(i);
}

/* Lumel flags (Lumel::m_flags) of any map, for post-process tests on
   arbitrary validity patterns. */
void ref_map_set_flags(void* h, int map, const int* flags) {
    RefCtx* c = (RefCtx*)h;
    Lightmap* m = c->maps[map];
    int n = m->width() * m->height();
    Lumel* L = m->lumels();
    for (int i = 0; i < n; i++) L[i].m_flags = flags[i];
}

/* Lightmap::expand / blur (Lightmap.cpp:167-220) and Lightmap::save
   (:223-283) run by the reference itself. */
void ref_map_expand(void* h, int map) { ((RefCtx*)h)->maps[map]->expand(); }
void ref_map_blur(void* h, int map) { ((RefCtx*)h)->maps[map]->blur(); }
int ref_map_save(void* h, int map, const char* path, int format) {
    return ((RefCtx*)h)->maps[map]->save(path, (StorageFormat)format) ? 1 : 0;
}

/* Photon accumulators (Lumel::m_color, m_photons) of a photonmap. */
void ref_map_set_photons(void* h, int map, const float* color, const int* photons) {
    RefCtx* c = (RefCtx*)h;
    Lightmap* m = c->maps[map];
    int n = m->width() * m->height();
    Lumel* L = m->lumels();
    for (int i = 0; i < n; i++) {
        L[i].m_color = Rgb(color[3 * i], color[3 * i + 1], color[3 * i + 2]);
        L[i].m_photons = photons[i];
    }
}

static bake::BakeIterator* make_iter(int face_mode, int first, int step) {
    if (face_mode) return new bake::FaceBakeIterator(first, step);
    return new bake::LumelBakeIterator(first, step);
}

/* Relight::bakeDirectLight (Relight.cpp:216-227). */
int ref_bake_direct(void* h, int mesh, int face_mode, int first, int step) {
    RefCtx* c = (RefCtx*)h;
    return c->relight->bakeDirectLight(c->scene, c->meshes[mesh], NULL, make_iter(face_mode, first, step));
}

/* Relight::bakeAmbientOcclusion (Relight.cpp:260-271). */
int ref_bake_ao(void* h, int mesh, int samples, float frac, float maxd, float expo, int face_mode, int first,
                int step) {
    RefCtx* c = (RefCtx*)h;
    AmbientOcclusionSettings s = AmbientOcclusionSettings::draft(frac, maxd, expo);
    s.m_samples = samples;
    return c->relight->bakeAmbientOcclusion(c->scene, c->meshes[mesh], NULL, s, make_iter(face_mode, first, step));
}

static IndirectLightSettings make_indirect(int passes, int bounces, float threshold, float pmaxd, int fg_samples,
                                           float fg_maxd, int radius, const float* sky, const float* ambient) {
    IndirectLightSettings s = IndirectLightSettings::draft();
    s.m_photonPassCount = passes;
    s.m_photonBounceCount = bounces;
    s.m_photonEnergyThreshold = threshold;
    s.m_photonMaxDistance = pmaxd;
    s.m_finalGatherSamples = fg_samples;
    s.m_finalGatherDistance = fg_maxd;
    s.m_finalGatherRadius = radius;
    s.m_skyColor = sky ? Rgb(sky[0], sky[1], sky[2]) : Rgb(0, 0, 0);
    s.m_ambientColor = ambient ? Rgb(ambient[0], ambient[1], ambient[2]) : Rgb(0, 0, 0);
    return s;
}

/* Relight::emitPhotons (Relight.cpp:244-257): trace + per-photonmap gather. */
int ref_emit_photons(void* h, int passes, int bounces, float threshold, float maxd, int radius) {
    RefCtx* c = (RefCtx*)h;
    IndirectLightSettings s = make_indirect(passes, bounces, threshold, maxd, 1, 1.0f, radius, nullptr, nullptr);
    return c->relight->emitPhotons(c->scene, s);
}

/* Photonmap::gather(radius) alone (Lightmap.cpp:376-413). */
void ref_photonmap_gather(void* h, int map, int radius) {
    RefCtx* c = (RefCtx*)h;
    ((Photonmap*)c->maps[map])->gather(radius);
}

/* Relight::bakeIndirectLight (Relight.cpp:230-241). */
int ref_bake_indirect(void* h, int mesh, int samples, float maxd, int radius, const float* sky,
                      const float* ambient, int face_mode, int first, int step) {
    RefCtx* c = (RefCtx*)h;
    IndirectLightSettings s = make_indirect(1, 0, 0.0f, 1.0f, samples, maxd, radius, sky, ambient);
    return c->relight->bakeIndirectLight(c->scene, c->meshes[mesh], NULL, s, make_iter(face_mode, first, step));
}

/* ---------------------------------------------------- threaded fan-out */

/* A Worker that runs each pushed job on its own std::thread, as the demo's
   ThreadWorker does (src/demo/Lightmapping.cpp:619-643). */
class StdThreadWorker : public Worker {
public:
    virtual void push(Job* job, JobData* data) {
        data->m_worker = this;
        m_thread = std::thread([job, data]() { job->execute(data); delete data; });
    }
    virtual void wait(void) {
        if (m_thread.joinable()) m_thread.join();
    }
    virtual void notify(const Mesh*, int, int) {}

private:
    std::thread m_thread;
};

struct PassJob : public Job {
    int kind = 0;  /* 0 direct, 1 AO, 2 indirect */
    AmbientOcclusionSettings ao;
    IndirectLightSettings ind;
    virtual void execute(JobData* d) {
        if (kind == 0) d->m_relight->bakeDirectLight(d->m_scene, d->m_mesh, d->m_worker, d->m_iterator);
        else if (kind == 1) d->m_relight->bakeAmbientOcclusion(d->m_scene, d->m_mesh, d->m_worker, ao, d->m_iterator);
        else d->m_relight->bakeIndirectLight(d->m_scene, d->m_mesh, d->m_worker, ind, d->m_iterator);
    }
};

/* Relight::bake(scene, job, root, workers) with `nthreads` thread workers
   (Relight.cpp:205-213 -> FullBakeJob::execute, Worker.cpp:43-83): every
   mesh, face- or lumel-interleaved across the workers. */
int ref_bake_full(void* h, int kind, int nthreads, int ao_samples, float ao_frac, float ao_maxd, float ao_exp,
                  int fg_samples, float fg_maxd, int radius, const float* sky, const float* ambient) {
    RefCtx* c = (RefCtx*)h;
    PassJob* job = new PassJob;
    job->kind = kind;
    job->ao = AmbientOcclusionSettings::draft(ao_frac, ao_maxd, ao_exp);
    job->ao.m_samples = ao_samples;
    job->ind = make_indirect(1, 0, 0.0f, 1.0f, fg_samples, fg_maxd, radius, sky, ambient);
    Workers workers;
    std::vector<StdThreadWorker*> owned;
    for (int i = 0; i < nthreads; i++) { owned.push_back(new StdThreadWorker); workers.push_back(owned.back()); }
    Worker root;  /* the base Worker runs the FullBakeJob inline (Worker.cpp:96-100) */
    c->relight->bake(c->scene, job, &root, workers);
    return 0;
}

/* Sampled fan-out for a bounded CPU baseline: thread j bakes lumels
   j*stride_all ... with LumelBakeIterator(first, step) — the iterator the
   library itself falls back to (Worker.cpp:69-73) — so `1/sample_div` of the
   valid texels are baked, interleaved across the map. */
int ref_bake_sampled(void* h, int kind, int mesh, int nthreads, int sample_div, int ao_samples, float ao_frac,
                     float ao_maxd, float ao_exp, int fg_samples, float fg_maxd, int radius, const float* sky,
                     const float* ambient) {
    RefCtx* c = (RefCtx*)h;
    AmbientOcclusionSettings ao = AmbientOcclusionSettings::draft(ao_frac, ao_maxd, ao_exp);
    ao.m_samples = ao_samples;
    IndirectLightSettings ind = make_indirect(1, 0, 0.0f, 1.0f, fg_samples, fg_maxd, radius, sky, ambient);
    std::vector<std::thread> th;
    for (int j = 0; j < nthreads; j++) {
        th.emplace_back([=]() {
            bake::BakeIterator* it = new bake::LumelBakeIterator(j * sample_div, nthreads * sample_div);
            if (kind == 0) c->relight->bakeDirectLight(c->scene, c->meshes[mesh], NULL, it);
            else if (kind == 1) c->relight->bakeAmbientOcclusion(c->scene, c->meshes[mesh], NULL, ao, it);
            else c->relight->bakeIndirectLight(c->scene, c->meshes[mesh], NULL, ind, it);
        });
    }
    for (auto& t : th) t.join();
    return 0;
}

/* ------------------------------------------------------------ radiosity */

/* RadiosityBuilder::build (radiosity/RadiosityBuilder.cpp:44-58) over every
   scene mesh's radiancemap.  Returns the patch count; *nnz gets the total
   number of form factors. */
int ref_radiosity_build(void* h, float threshold, int max_ff, long long* nnz) {
    RefCtx* c = (RefCtx*)h;
    RadiosityBuilder b(c->scene);
    c->radiosity = b.build(threshold, max_ff);
    long long total = 0;
    for (int i = 0; i < c->radiosity.patchCount(); i++) total += (long long)c->radiosity.patch(i).m_ff.size();
    *nnz = total;
    return c->radiosity.patchCount();
}

/* Form factors as CSR in the reference's own list order; patch positions. */
void ref_radiosity_get(void* h, long long* row_ptr, int* cols, float* vals, float* pos, float* nrm) {
    RefCtx* c = (RefCtx*)h;
    int n = c->radiosity.patchCount();
    const Radiosity::Patch* base = n ? &c->radiosity.patch(0) : nullptr;
    long long k = 0;
    for (int i = 0; i < n; i++) {
        const Radiosity::Patch& p = c->radiosity.patch(i);
        row_ptr[i] = k;
        for (size_t f = 0; f < p.m_ff.size(); f++) {
            cols[k] = (int)(p.m_ff[f].m_patch - base);
            vals[k] = p.m_ff[f].m_weight;
            k++;
        }
        if (pos) { pos[3 * i] = p.m_lumel->m_position.x; pos[3 * i + 1] = p.m_lumel->m_position.y; pos[3 * i + 2] = p.m_lumel->m_position.z; }
        if (nrm) { nrm[3 * i] = p.m_lumel->m_normal.x; nrm[3 * i + 1] = p.m_lumel->m_normal.y; nrm[3 * i + 2] = p.m_lumel->m_normal.z; }
    }
    row_ptr[n] = k;
}

/* Raw segment tracing through the reference's rt::Embree::traceSegment
   (rt/Embree.cpp:145-177): hit flag, point, normal, colour, lightmap uv, mesh. */
void ref_trace_segments(void* h, int n, const float* seg, int flags, int* hit, float* point, float* normal,
                        float* color, float* uv, int* mesh) {
    RefCtx* c = (RefCtx*)h;
    rt::ITracer* tr = c->scene->tracer();
    for (int i = 0; i < n; i++) {
        const float* s = &seg[6 * i];
        rt::Hit r = tr->traceSegment(Vec3(s[0], s[1], s[2]), Vec3(s[3], s[4], s[5]), flags);
        hit[i] = r ? 1 : 0;
        if (point) { point[3 * i] = r.m_point.x; point[3 * i + 1] = r.m_point.y; point[3 * i + 2] = r.m_point.z; }
        if (normal) { normal[3 * i] = r.m_normal.x; normal[3 * i + 1] = r.m_normal.y; normal[3 * i + 2] = r.m_normal.z; }
        if (color) { color[4 * i] = r.m_color.r; color[4 * i + 1] = r.m_color.g; color[4 * i + 2] = r.m_color.b; color[4 * i + 3] = r.m_color.a; }
        if (uv) { uv[2 * i] = r.m_uv.x; uv[2 * i + 1] = r.m_uv.y; }
        if (mesh) {
            int mi = -1;
            for (size_t k = 0; k < c->meshes.size(); k++) if (c->meshes[k] == r.m_mesh) mi = (int)k;
            mesh[i] = mi;
        }
    }
}

}  // extern "C"
