// relight_b200 C++ API (include/relight/Relight.h) over the C ABI
// (include/relight_b200.h).  Scene building follows the reference's float
// arithmetic in order (compiled with -ffp-contract=off): Mesh::transform
// (scene/Mesh.cpp:277-284), area-light face centroids
// (scene/Light.cpp:293-323 via Triangle(const Face&), scene/Mesh.cpp:321-326),
// the directional emitter's plane (scene/Light.cpp:349-352).
#include "../../../include/relight/Relight.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>

#include "../../../include/relight_b200.h"

namespace relight {

// ----------------------------------------------------------------- bounds

void Bounds::add(const Vec3& p) {
    if (p.x < min_.x) min_.x = p.x;
    if (p.y < min_.y) min_.y = p.y;
    if (p.z < min_.z) min_.z = p.z;
    if (p.x > max_.x) max_.x = p.x;
    if (p.y > max_.y) max_.y = p.y;
    if (p.z > max_.z) max_.z = p.z;
}

void Bounds::add(const Bounds& b) {
    add(b.min_);
    add(b.max_);
}

// ---------------------------------------------------------------- texture

Texture::Texture(int w, int h, int c, const unsigned char* px)
    : m_width(w), m_height(h), m_channels(c), m_pixels(px, px + (size_t)w * h * c) {}

Texture* Texture::create(int width, int height, int channels, const unsigned char* pixels) {
    if (width <= 0 || height <= 0 || (channels != 3 && channels != 4) || !pixels) return nullptr;
    return new Texture(width, height, channels, pixels);
}

Texture* Texture::createFromFile(const char* fileName) {
    FILE* f = fopen(fileName, "rb");
    if (!f) return nullptr;
    unsigned char head[12], info[6];
    if (fread(head, 1, 12, f) != 12 || fread(info, 1, 6, f) != 6) {
        fclose(f);
        return nullptr;
    }
    int w = info[1] * 256 + info[0], h = info[3] * 256 + info[2];
    if (w <= 0 || h <= 0 || (info[4] != 24 && info[4] != 32)) {
        fclose(f);
        return nullptr;
    }
    int bpp = info[4] / 8;
    std::vector<unsigned char> px((size_t)w * h * bpp, 0);
    size_t got = fread(px.data(), 1, px.size(), f);
    (void)got;
    fclose(f);
    for (size_t i = 0; i < px.size(); i += bpp) std::swap(px[i], px[i + 2]);
    return new Texture(w, h, bpp, px.data());
}

// ------------------------------------------------------------------- mesh

void Mesh::updateBounds() {
    for (const Vertex& v : m_vertices) m_bounds.add(v.position);
}

Mesh* Mesh::createFromFile(const std::string& fileName) {
    rl_obj_mesh* obj = nullptr;
    if (rl_obj_load(fileName.c_str(), &obj) != RL_OK) return nullptr;
    int32_t nv = 0, ni = 0;
    rl_obj_mesh_counts(obj, &nv, &ni, nullptr);
    std::vector<float> pos(3 * (size_t)nv), nrm(3 * (size_t)nv), uv(2 * (size_t)nv);
    std::vector<int32_t> idx((size_t)ni);
    rl_obj_mesh_arrays(obj, pos.data(), nrm.data(), uv.data(), idx.data());
    rl_obj_mesh_destroy(obj);
    VertexBuffer vertices((size_t)nv);
    for (int32_t i = 0; i < nv; i++) {
        vertices[i].position = Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        vertices[i].normal = Vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
        vertices[i].uv[Vertex::Lightmap] = Uv(uv[2 * i], uv[2 * i + 1]);
    }
    IndexBuffer indices(idx.begin(), idx.end());
    Mesh* m = new Mesh;
    m->addFaces(vertices, indices, nullptr);
    return m;
}

void Mesh::addFaces(const VertexBuffer& vertices, const IndexBuffer& indices, const Material* material) {
    size_t base = m_vertices.size();
    for (Index i : indices) m_indices.push_back((Index)(i + base));
    for (const Vertex& v : vertices) {
        m_vertices.push_back(v);
        m_vertices.back().material = material;
    }
    updateBounds();
}

Mesh* Mesh::transformed(const Matrix4& transform) const {
    Mesh* m = new Mesh;
    m->m_vertices = m_vertices;
    m->m_indices = m_indices;
    for (Vertex& v : m->m_vertices) {
        v.position = transform * v.position;
        v.normal = transform.rotate(v.normal);
        v.normal.normalize();
    }
    m->updateBounds();
    return m;
}

void Mesh::overrideMaterial(const Material* material) {
    for (Vertex& v : m_vertices) v.material = material;
}

// ----------------------------------------------------------------- lights

DirectionalPhotonEmitter::DirectionalPhotonEmitter(const Light* light, const Vec3& direction)
    : PhotonEmitter(light), m_direction(direction) {
    Vec3 p = light ? light->position() : Vec3();
    m_plane[0] = direction.x; m_plane[1] = direction.y; m_plane[2] = direction.z;
    m_plane[3] = -(direction * p);
}

Light::~Light() {
    delete m_cutoff;
    delete m_attenuation;
    delete m_photonEmitter;
    delete m_influence;
}

void Light::setInfluence(LightInfluence* value) { delete m_influence; m_influence = value; }
void Light::setAttenuation(LightAttenuation* value) { delete m_attenuation; m_attenuation = value; }
void Light::setCutoff(LightCutoff* value) { delete m_cutoff; m_cutoff = value; }
void Light::setPhotonEmitter(PhotonEmitter* value) { delete m_photonEmitter; m_photonEmitter = value; }

Light* Light::createPointLight(const Vec3& position, float radius, const Rgb& color, float intensity,
                               bool castsShadow) {
    Light* l = new Light;
    l->setInfluence(new LightInfluence(l));
    l->setAttenuation(new LinearLightAttenuation(l, radius));
    l->setPhotonEmitter(new PhotonEmitter(l));
    l->setCutoff(new LightCutoff(l));
    l->setCastsShadow(castsShadow);
    l->setPosition(position);
    l->setColor(color);
    l->setIntensity(intensity);
    return l;
}

Light* Light::createSpotLight(const Vec3& position, const Vec3& direction, float cutoff, float radius,
                              const Rgb& color, float intensity, bool castsShadow) {
    Light* l = createPointLight(position, radius, color, intensity, castsShadow);
    l->setCutoff(new LightSpotCutoff(l, direction, cutoff, 1.0f));
    return l;
}

Light* Light::createDirectionalLight(const Vec3& direction, const Rgb& color, float intensity, bool castsShadow) {
    Light* l = new Light;
    l->setInfluence(new DirectionalLightInfluence(l, direction));
    l->setPhotonEmitter(new DirectionalPhotonEmitter(l, direction));
    l->setCastsShadow(castsShadow);
    l->setColor(color);
    l->setIntensity(intensity);
    return l;
}

Light* Light::createAreaLight(const Mesh* mesh, const Vec3& position, const Rgb& color, float intensity,
                              bool castsShadow) {
    Light* l = createPointLight(position, 1.0f, color, intensity, castsShadow);
    l->setAttenuation(new LinearLightAttenuation(l, mesh->bounds().volume()));
    for (int f = 0; f < mesh->faceCount(); f++) {
        const Vec3& a = mesh->vertex(mesh->index(3 * f)).position;
        const Vec3& b = mesh->vertex(mesh->index(3 * f + 1)).position;
        const Vec3& c = mesh->vertex(mesh->index(3 * f + 2)).position;
        l->m_vertices.push_back((a + c + b) / 3.0f);
    }
    return l;
}

// ------------------------------------------------------------------- maps

Lightmap::Lightmap(int width, int height, int kind) : m_width(width), m_height(height), m_kind(kind) {
    m_host.resize((size_t)width * height);
}

Lightmap::~Lightmap() {
    if (m_device) rl_map_destroy(m_device);
}

RelightStatus Lightmap::addMesh(const Mesh* mesh) {
    if (!mesh || mesh->lightmap()) return RelightInvalidCall;
    const_cast<Mesh*>(mesh)->m_lightmap = this;
    m_meshes.push_back(mesh);
    return RelightSuccess;
}

RelightStatus Photonmap::addMesh(const Mesh* mesh, bool) {
    if (!mesh || mesh->photonmap()) return RelightInvalidCall;
    const_cast<Mesh*>(mesh)->m_photonmap = this;
    m_meshes.push_back(mesh);
    return RelightSuccess;
}

void Lightmap::attach(rl_scene* scene, const std::vector<const Mesh*>& sceneMeshes) {
    if (m_device) return;
    if (rl_map_create(m_kind, m_width, m_height, &m_device) != RL_OK) return;
    for (const Mesh* m : m_meshes) {
        auto it = std::find(sceneMeshes.begin(), sceneMeshes.end(), m);
        if (it != sceneMeshes.end()) rl_map_add_mesh(m_device, scene, (int)(it - sceneMeshes.begin()), nullptr);
    }
    m_hostStale = true;
}

Lumel* Lightmap::lumels() {
    if (m_device && m_hostStale) {
        size_t n = (size_t)m_width * m_height;
        std::vector<int32_t> flags(n), face(n), photons(n);
        std::vector<float> pos(3 * n), nrm(3 * n), col(3 * n), gat(3 * n);
        if (rl_map_download(m_device, flags.data(), face.data(), pos.data(), nrm.data(), col.data(), photons.data(),
                            gat.data(), nullptr) == RL_OK) {
            for (size_t i = 0; i < n; i++) {
                Lumel& l = m_host[i];
                l.m_flags = flags[i];
                l.m_faceIdx = (Index)face[i];
                l.m_position = Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
                l.m_normal = Vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
                l.m_color = Rgb(col[3 * i], col[3 * i + 1], col[3 * i + 2]);
                l.m_photons = photons[i];
                l.m_gathered = Rgb(gat[3 * i], gat[3 * i + 1], gat[3 * i + 2]);
            }
            m_hostStale = false;
        }
    }
    m_hostEdited = true;  // the caller holds a writable pointer
    return m_host.data();
}

void Lightmap::beforeDevice() {
    if (!m_device || !m_hostEdited || m_hostStale) return;
    size_t n = (size_t)m_width * m_height;
    std::vector<float> col(3 * n);
    std::vector<int32_t> photons(n);
    for (size_t i = 0; i < n; i++) {
        col[3 * i] = m_host[i].m_color.r;
        col[3 * i + 1] = m_host[i].m_color.g;
        col[3 * i + 2] = m_host[i].m_color.b;
        photons[i] = m_host[i].m_photons;
    }
    rl_map_upload(m_device, nullptr, nullptr, nullptr, nullptr, col.data(), m_kind == 1 ? photons.data() : nullptr,
                  nullptr, nullptr);
    cudaStreamSynchronize(nullptr);
    m_hostEdited = false;
}

void Lightmap::afterDevice() { m_hostStale = true; }

float* Lightmap::toHdr() {
    Lumel* l = lumels();
    m_hostEdited = false;
    float* px = new float[(size_t)m_width * m_height * 3];
    for (size_t i = 0; i < (size_t)m_width * m_height; i++) {
        px[3 * i] = l[i].m_color.r;
        px[3 * i + 1] = l[i].m_color.g;
        px[3 * i + 2] = l[i].m_color.b;
    }
    return px;
}

void Lightmap::expand() {
    if (!m_device) return;  // never rasterised: no valid lumel to spread
    beforeDevice();
    rl_map_expand(m_device, nullptr);
    cudaStreamSynchronize(nullptr);
    afterDevice();
}

void Lightmap::blur() {
    if (!m_device) return;
    beforeDevice();
    rl_map_blur(m_device, nullptr);
    cudaStreamSynchronize(nullptr);
    afterDevice();
}

bool Lightmap::save(const std::string& fileName, StorageFormat format) {
    if (m_device) {
        beforeDevice();
        return rl_map_save(m_device, fileName.c_str(), (int)format, nullptr) == RL_OK;
    }
    if (format != RawHdr) return false;
    FILE* f = fopen(fileName.c_str(), "wb");
    if (!f) return false;
    float* px = toHdr();
    fwrite(&m_width, sizeof(int), 1, f);
    fwrite(&m_height, sizeof(int), 1, f);
    fwrite(px, sizeof(float), (size_t)m_width * m_height * 3, f);
    delete[] px;
    fclose(f);
    return true;
}

void Photonmap::gather(int radius) {
    if (!m_device) return;
    beforeDevice();
    rl_photonmap_gather(m_device, radius, nullptr);
    cudaStreamSynchronize(nullptr);
    afterDevice();
}

// ------------------------------------------------------------------ scene

Scene::~Scene() {
    if (m_device) rl_scene_destroy(m_device);
}

RelightStatus Scene::begin() {
    if (m_state != StateInitial) return RelightInvalidCall;
    m_state = StateAddingObjects;
    return RelightSuccess;
}

Mesh* Scene::addMesh(const Mesh* mesh, const Matrix4& transform, const Material* material) {
    Mesh* t = mesh->transformed(transform);
    if (material) t->overrideMaterial(material);
    m_meshes.push_back(t);
    m_bounds = Bounds();
    for (const Mesh* m : m_meshes) m_bounds.add(m->bounds());
    return t;
}

RelightStatus Scene::addLight(const Light* light) {
    m_lights.push_back(light);
    return RelightSuccess;
}

RelightStatus Scene::end() {
    if (m_state != StateAddingObjects) return RelightInvalidCall;
    std::vector<float> pos, nrm, uv0, uv1, mat_rgb;
    std::vector<int32_t> vmat, tris, first(1, 0), lmap, pmap, mat_tex, tex_dims;
    std::vector<int64_t> tex_off;
    std::vector<uint8_t> tex_px;
    std::map<const Material*, int> mats;
    std::map<const Texture*, int> texs;
    std::vector<const Lightmap*> lightmaps, photonmaps;
    int vbase = 0;
    for (const Mesh* m : m_meshes) {
        for (int i = 0; i < m->vertexCount(); i++) {
            const Vertex& v = m->vertex(i);
            pos.insert(pos.end(), {v.position.x, v.position.y, v.position.z});
            nrm.insert(nrm.end(), {v.normal.x, v.normal.y, v.normal.z});
            uv0.insert(uv0.end(), {v.uv[0].x, v.uv[0].y});
            uv1.insert(uv1.end(), {v.uv[1].x, v.uv[1].y});
            int id = -1;
            if (v.material) {
                auto it = mats.find(v.material);
                if (it == mats.end()) {
                    id = (int)mats.size();
                    mats[v.material] = id;
                    const Rgb& c = v.material->color();
                    mat_rgb.insert(mat_rgb.end(), {c.r, c.g, c.b});
                    int tid = -1;
                    if (const Texture* t = v.material->texture()) {
                        auto tt = texs.find(t);
                        if (tt == texs.end()) {
                            tid = (int)texs.size();
                            texs[t] = tid;
                            tex_dims.insert(tex_dims.end(), {t->width(), t->height(), t->channels()});
                            tex_off.push_back((int64_t)tex_px.size());
                            tex_px.insert(tex_px.end(), t->pixels(),
                                          t->pixels() + (size_t)t->width() * t->height() * t->channels());
                        } else {
                            tid = tt->second;
                        }
                    }
                    mat_tex.push_back(tid);
                } else {
                    id = it->second;
                }
            }
            vmat.push_back(id);
        }
        for (int i = 0; i < m->indexCount(); i++) tris.push_back(vbase + m->index(i));
        vbase += m->vertexCount();
        first.push_back(first.back() + m->faceCount());
        int li = -1, pi = -1;
        if (const Lightmap* l = m->lightmap()) {
            auto it = std::find(lightmaps.begin(), lightmaps.end(), l);
            li = (int)(it - lightmaps.begin());
            if (it == lightmaps.end()) lightmaps.push_back(l);
        }
        if (const Photonmap* p = m->photonmap()) {
            auto it = std::find(photonmaps.begin(), photonmaps.end(), (const Lightmap*)p);
            pi = (int)(it - photonmaps.begin());
            if (it == photonmaps.end()) photonmaps.push_back(p);
        }
        lmap.push_back(li);
        pmap.push_back(pi);
    }
    rl_scene_desc d;
    memset(&d, 0, sizeof d);
    d.nverts = vbase;
    d.pos = pos.data(); d.nrm = nrm.data(); d.uv0 = uv0.data(); d.uv1 = uv1.data(); d.vmat = vmat.data();
    d.ntris = (int32_t)(tris.size() / 3);
    d.tris = tris.data();
    d.nmeshes = (int32_t)m_meshes.size();
    d.mesh_first_tri = first.data(); d.mesh_lightmap = lmap.data(); d.mesh_photonmap = pmap.data();
    d.nmats = (int32_t)mats.size();
    d.mat_rgb = mat_rgb.data(); d.mat_tex = mat_tex.data();
    d.ntex = (int32_t)texs.size();
    d.tex_dims = tex_dims.data(); d.tex_offset = tex_off.data(); d.tex_pixels = tex_px.data();
    d.bounds_lo[0] = m_bounds.min().x; d.bounds_lo[1] = m_bounds.min().y; d.bounds_lo[2] = m_bounds.min().z;
    d.bounds_hi[0] = m_bounds.max().x; d.bounds_hi[1] = m_bounds.max().y; d.bounds_hi[2] = m_bounds.max().z;
    if (rl_scene_create(&d, 0, nullptr, &m_device) != RL_OK) return RelightInvalidCall;
    m_state = StateReadyToBake;
    return RelightSuccess;
}

// ----------------------------------------------------------------- settings

static IndirectLightSettings indirect(int passes, int bounces, int samples, const Rgb& sky, const Rgb& ambient,
                                      float pmaxd, float fgd) {
    IndirectLightSettings s;
    s.m_skyColor = sky;
    s.m_ambientColor = ambient;
    s.m_photonPassCount = passes;
    s.m_photonBounceCount = bounces;
    s.m_photonEnergyThreshold = 0.05f;
    s.m_photonMaxDistance = pmaxd;
    s.m_finalGatherSamples = samples;
    s.m_finalGatherDistance = fgd;
    s.m_finalGatherRadius = 7;
    return s;
}

// Relight.cpp:43-120
IndirectLightSettings IndirectLightSettings::draft(const Rgb& s, const Rgb& a, float p, float f) { return indirect(8, 1, 32, s, a, p, f); }
IndirectLightSettings IndirectLightSettings::fast(const Rgb& s, const Rgb& a, float p, float f) { return indirect(16, 3, 64, s, a, p, f); }
IndirectLightSettings IndirectLightSettings::best(const Rgb& s, const Rgb& a, float p, float f) { return indirect(32, 3, 128, s, a, p, f); }
IndirectLightSettings IndirectLightSettings::production(const Rgb& s, const Rgb& a, float p, float f) { return indirect(64, 4, 1024, s, a, p, f); }

static AmbientOcclusionSettings ao(int samples, float frac, float maxd, float expo) {
    AmbientOcclusionSettings s;
    s.m_samples = samples;
    s.m_occludedFraction = frac;
    s.m_maxDistance = maxd;
    s.m_exponent = expo;
    return s;
}

// Relight.cpp:123-172
AmbientOcclusionSettings AmbientOcclusionSettings::draft(float f, float d, float e) { return ao(128, f, d, e); }
AmbientOcclusionSettings AmbientOcclusionSettings::fast(float f, float d, float e) { return ao(256, f, d, e); }
AmbientOcclusionSettings AmbientOcclusionSettings::best(float f, float d, float e) { return ao(1024, f, d, e); }
AmbientOcclusionSettings AmbientOcclusionSettings::production(float f, float d, float e) { return ao(2048, f, d, e); }

// ----------------------------------------------------------------- relight

// ------------------------------------------------------- jobs and workers

void Worker::push(Job* job, JobData* data) {
    data->m_worker = this;
    job->execute(data);
    delete data;
}

FullBakeJob::FullBakeJob(Job* job, const Workers& workers) : m_workers(workers), m_job(job) {}

void FullBakeJob::execute(JobData* data) {
    const int n = (int)m_workers.size();
    std::vector<const Mesh*> meshes;
    for (int i = 0; i < data->m_scene->meshCount(); i++) meshes.push_back(data->m_scene->mesh(i));
    std::stable_sort(meshes.begin(), meshes.end(),
                     [](const Mesh* a, const Mesh* b) { return a->bounds().volume() > b->bounds().volume(); });
    for (const Mesh* mesh : meshes) {
        std::vector<std::unique_ptr<bake::BakeIterator>> iterators;
        for (int j = 0; j < n; j++) {
            JobData* d = new JobData;
            d->m_job = m_job;
            d->m_scene = data->m_scene;
            d->m_relight = data->m_relight;
            d->m_mesh = mesh;
            if (mesh->faceCount() >= n)
                iterators.emplace_back(new bake::FaceBakeIterator(j, n));
            else
                iterators.emplace_back(new bake::LumelBakeIterator(j, n));
            d->m_iterator = iterators.back().get();
            m_workers[j]->push(m_job, d);
        }
        for (int j = 0; j < n; j++) m_workers[j]->wait();
    }
}

void Relight::bake(const Scene* scene, Job* job, Worker* root, const Workers& workers) {
    FullBakeJob* full;
    {
        std::unique_lock<std::mutex> g(m_lock);
        m_jobs.emplace_back(new FullBakeJob(job, workers));
        full = m_jobs.back().get();
    }
    JobData* data = new JobData;
    data->m_scene = scene;
    data->m_relight = this;
    data->m_job = full;
    root->push(full, data);
}

// ----------------------------------------------------------------- relight

uint64_t Relight::nextSeed() {
    m_calls++;
    return m_seed * 0x9E3779B97F4A7C15ull + m_calls;
}

RelightStatus Relight::status(int rc) {
    if (rc == RL_OK) return RelightSuccess;
    char buf[512];
    rl_last_error(buf, sizeof buf);
    m_error = buf;
    return rc == RL_NOT_IMPLEMENTED ? RelightNotImplemented : RelightInvalidCall;
}

// Rasterise every map of the scene's meshes once (Lightmap::addMesh's lumel
// initialisation, deferred to the device).
bool Relight::prepare(const Scene* scene) {
    if (!scene || !scene->m_device) return false;
    if (!scene->m_mapsReady) {
        for (const Mesh* m : scene->m_meshes) {
            if (m->lightmap()) m->lightmap()->attach(scene->m_device, scene->m_meshes);
            if (m->photonmap()) m->photonmap()->attach(scene->m_device, scene->m_meshes);
        }
        const_cast<Scene*>(scene)->m_mapsReady = true;
    }
    return true;
}

struct LightTables {
    std::vector<rl_light> lights;
    std::vector<float> verts;
};

static LightTables light_tables(const Scene* scene) {
    LightTables t;
    for (int i = 0; i < scene->lightCount(); i++) {
        const Light* l = scene->light(i);
        rl_light r;
        memset(&r, 0, sizeof r);
        r.influence = l->influence() ? l->influence()->kind() : 0;
        r.casts_shadow = l->castsShadow();
        r.position[0] = l->position().x; r.position[1] = l->position().y; r.position[2] = l->position().z;
        r.color[0] = l->color().r; r.color[1] = l->color().g; r.color[2] = l->color().b;
        r.intensity = l->intensity();
        if (const DirectionalLightInfluence* d = dynamic_cast<const DirectionalLightInfluence*>(l->influence())) {
            r.direction[0] = d->m_direction.x; r.direction[1] = d->m_direction.y; r.direction[2] = d->m_direction.z;
        }
        if (const LinearLightAttenuation* a = dynamic_cast<const LinearLightAttenuation*>(l->attenuation())) {
            r.attenuation = 1;
            r.att_radius = a->m_radius; r.att_const = a->m_const; r.att_linear = a->m_linear;
            r.att_quadratic = a->m_quadratic;
        }
        if (l->cutoff()) {
            r.cutoff = l->cutoff()->kind();
            if (const LightSpotCutoff* c = dynamic_cast<const LightSpotCutoff*>(l->cutoff())) {
                r.spot_direction[0] = c->m_direction.x; r.spot_direction[1] = c->m_direction.y;
                r.spot_direction[2] = c->m_direction.z;
                r.spot_cutoff = c->m_cutoff;
                r.spot_exponent = c->m_exponent;
            }
        }
        if (l->photonEmitter()) {
            r.emitter = l->photonEmitter()->kind();
            if (const DirectionalPhotonEmitter* e = dynamic_cast<const DirectionalPhotonEmitter*>(l->photonEmitter())) {
                for (int k = 0; k < 4; k++) r.emitter_plane[k] = e->m_plane[k];
                r.direction[0] = e->m_direction.x; r.direction[1] = e->m_direction.y; r.direction[2] = e->m_direction.z;
            }
        }
        if (!l->vertices().empty()) {
            r.vertex_first = (int32_t)(t.verts.size() / 3);
            r.vertex_count = (int32_t)l->vertices().size();
            for (const Vec3& v : l->vertices()) t.verts.insert(t.verts.end(), {v.x, v.y, v.z});
        }
        t.lights.push_back(r);
    }
    return t;
}

static rl_iterator iterator_of(const Scene* scene, const Mesh* mesh, bake::BakeIterator* it) {
    rl_iterator r{0, 0, 1, -1};
    if (!it) return r;
    r.kind = it->kind();
    r.first = it->m_firstIndex;
    r.step = it->m_step;
    if (r.kind == 1)
        for (int i = 0; i < scene->meshCount(); i++)
            if (scene->mesh(i) == mesh) r.mesh = i;
    return r;
}

static std::vector<rl_map*> photon_maps(const Scene* scene) {
    std::vector<rl_map*> maps;
    std::vector<const Photonmap*> seen;
    for (int i = 0; i < scene->meshCount(); i++)
        if (const Photonmap* p = scene->mesh(i)->photonmap())
            if (std::find(seen.begin(), seen.end(), p) == seen.end()) {
                seen.push_back(p);
                maps.push_back(p->device());
            }
    return maps;
}

// Relight::bakeDirectLight (Relight.cpp:216-227) with Baker::bakeMesh's
// checks (baker/Baker.cpp:52-77).
RelightStatus Relight::bakeDirectLight(const Scene* scene, const Mesh* mesh, Progress* progress,
                                       bake::BakeIterator* iterator) {
    std::unique_lock<std::mutex> g(m_lock);
    if (!mesh || mesh->faceCount() == 0 || !mesh->lightmap() || !prepare(scene)) return RelightInvalidCall;
    Lightmap* lm = mesh->lightmap();
    lm->beforeDevice();
    LightTables t = light_tables(scene);
    rl_iterator it = iterator_of(scene, mesh, iterator);
    int rc = rl_bake_direct(scene->device(), lm->device(), t.lights.data(), (int)t.lights.size(), t.verts.data(),
                            (int)(t.verts.size() / 3), &it, nullptr);
    cudaStreamSynchronize(nullptr);
    lm->afterDevice();
    g.unlock();  // the callback may take its own locks
    if (progress) progress->notify(mesh, 1, 1);
    return status(rc);
}

RelightStatus Relight::bakeAmbientOcclusion(const Scene* scene, const Mesh* mesh, Progress* progress,
                                            const AmbientOcclusionSettings& s, bake::BakeIterator* iterator) {
    std::unique_lock<std::mutex> g(m_lock);
    if (!mesh || mesh->faceCount() == 0 || !mesh->lightmap() || !prepare(scene)) return RelightInvalidCall;
    Lightmap* lm = mesh->lightmap();
    lm->beforeDevice();
    rl_iterator it = iterator_of(scene, mesh, iterator);
    int rc = rl_bake_ao(scene->device(), lm->device(), s.m_samples, s.m_occludedFraction, s.m_maxDistance,
                        s.m_exponent, nextSeed(), &it, nullptr);
    cudaStreamSynchronize(nullptr);
    lm->afterDevice();
    g.unlock();  // the callback may take its own locks
    if (progress) progress->notify(mesh, 1, 1);
    return status(rc);
}

// Relight::emitPhotons (Relight.cpp:244-257): trace, then gather each photonmap.
RelightStatus Relight::emitPhotons(const Scene* scene, const IndirectLightSettings& s) {
    std::unique_lock<std::mutex> g(m_lock);
    if (!prepare(scene)) return RelightInvalidCall;
    std::vector<rl_map*> maps = photon_maps(scene);
    LightTables t = light_tables(scene);
    int rc = rl_emit_photons(scene->device(), maps.data(), (int)maps.size(), t.lights.data(), (int)t.lights.size(),
                             s.m_photonPassCount, s.m_photonBounceCount, s.m_photonEnergyThreshold,
                             s.m_photonMaxDistance, nextSeed(), nullptr, nullptr);
    for (rl_map* m : maps)
        if (rc == RL_OK) rc = rl_photonmap_gather(m, s.m_finalGatherRadius, nullptr);
    cudaStreamSynchronize(nullptr);
    for (int i = 0; i < scene->meshCount(); i++)
        if (Photonmap* p = scene->mesh(i)->photonmap()) p->afterDevice();
    return status(rc);
}

RelightStatus Relight::bakeIndirectLight(const Scene* scene, const Mesh* mesh, Progress* progress,
                                         const IndirectLightSettings& s, bake::BakeIterator* iterator) {
    std::unique_lock<std::mutex> g(m_lock);
    if (!mesh || mesh->faceCount() == 0 || !mesh->lightmap() || !prepare(scene)) return RelightInvalidCall;
    Lightmap* lm = mesh->lightmap();
    lm->beforeDevice();
    std::vector<rl_map*> maps = photon_maps(scene);
    rl_iterator it = iterator_of(scene, mesh, iterator);
    float sky[3] = {s.m_skyColor.r, s.m_skyColor.g, s.m_skyColor.b};
    float amb[3] = {s.m_ambientColor.r, s.m_ambientColor.g, s.m_ambientColor.b};
    int rc = rl_bake_indirect(scene->device(), lm->device(), maps.data(), (int)maps.size(), s.m_finalGatherSamples,
                              s.m_finalGatherDistance, sky, amb, nextSeed(), &it, nullptr);
    cudaStreamSynchronize(nullptr);
    lm->afterDevice();
    g.unlock();  // the callback may take its own locks
    if (progress) progress->notify(mesh, 1, 1);
    return status(rc);
}

}  // namespace relight
