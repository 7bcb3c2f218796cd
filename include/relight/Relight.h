/*
 * relight_b200 C++ API — the drop-in for Relight's scene / mesh / light /
 * lightmap baking API (dmsovetov/Relight: Relight.h:82-189, scene/Scene.h,
 * scene/Mesh.h, scene/Light.h, scene/Material.h, Lightmap.h, baker/Baker.h).
 *
 * Class, method and argument names, argument meaning and RelightStatus
 * results are the reference's.  Baking runs on the GPU through the C ABI of
 * include/relight_b200.h:
 *   - Scene::end uploads the scene and builds its BVH on the device;
 *   - the first bake then rasterises every map's lumels on the device
 *     (Lightmap::addMesh records the mesh; the reference rasterises at once);
 *   - Relight::bake* calls run the pass for the iterator's lumels and return
 *     when it is done; Lightmap::lumels() gives the host copy, and host edits
 *     to it are sent back before the map's next bake.
 * Random numbers: each stochastic call draws from its own Philox4x32-10 key
 * (Relight::setSeed), where the reference calls the C library's rand().
 * Threads: the bake calls of one Relight serialise on a lock, so Relight::bake
 * accepts thread workers as the reference does; a GPU bake gains nothing
 * from them (every call is one device pass), and the base Worker, which runs
 * each job at once on the calling thread, is the natural choice.
 */
#ifndef RELIGHT_B200_RELIGHT_H
#define RELIGHT_B200_RELIGHT_H

#include <cmath>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

struct rl_scene;
struct rl_map;

namespace relight {

// ------------------------------------------------------------------ math

// Types.h Vec2 / Vec3 / Rgb / Rgba / Matrix4 / Bounds, the operations the API
// uses, evaluated left to right in float as the reference does.
struct Vec2 {
    float x, y;
    Vec2() : x(0.0f), y(0.0f) {}
    Vec2(float x, float y) : x(x), y(y) {}
};
typedef Vec2 Uv;
typedef Vec2 Barycentric;

struct Vec3 {
    float x, y, z;
    Vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    Vec3(float x, float y, float z) : x(x), y(y), z(z) {}
    Vec3 operator+(const Vec3& o) const { return Vec3(x + o.x, y + o.y, z + o.z); }
    Vec3 operator-(const Vec3& o) const { return Vec3(x - o.x, y - o.y, z - o.z); }
    Vec3 operator-() const { return Vec3(-x, -y, -z); }
    Vec3 operator*(float s) const { return Vec3(x * s, y * s, z * s); }
    Vec3 operator/(float s) const { return Vec3(x / s, y / s, z / s); }
    float operator*(const Vec3& o) const { return x * o.x + y * o.y + z * o.z; }
    float length() const { return std::sqrt(x * x + y * y + z * z); }
    float normalize() {
        float len = length();
        if (len) { x /= len; y /= len; z /= len; }
        return len;
    }
};

struct Rgb {
    float r, g, b;
    Rgb() : r(0.0f), g(0.0f), b(0.0f) {}
    Rgb(float r, float g, float b) : r(r), g(g), b(b) {}
};

struct Rgba {
    float r, g, b, a;
    Rgba() : r(0.0f), g(0.0f), b(0.0f), a(1.0f) {}
    Rgba(float r, float g, float b, float a = 1.0f) : r(r), g(g), b(b), a(a) {}
};

// Row-vector affine matrix: p' = (x, y, z, 1) * M (Types.h:1188-1196).
struct Matrix4 {
    float m[16];
    Matrix4() {
        for (int i = 0; i < 16; i++) m[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    }
    Vec3 operator*(const Vec3& v) const {
        return Vec3(v.x * m[0] + v.y * m[4] + v.z * m[8] + m[12], v.x * m[1] + v.y * m[5] + v.z * m[9] + m[13],
                    v.x * m[2] + v.y * m[6] + v.z * m[10] + m[14]);
    }
    Vec3 rotate(const Vec3& v) const {
        return Vec3(v.x * m[0] + v.y * m[4] + v.z * m[8], v.x * m[1] + v.y * m[5] + v.z * m[9],
                    v.x * m[2] + v.y * m[6] + v.z * m[10]);
    }
    static Matrix4 translation(float x, float y, float z) {
        Matrix4 t;
        t.m[12] = x; t.m[13] = y; t.m[14] = z;
        return t;
    }
};

struct Bounds {
    Vec3 min_, max_;
    Bounds() : min_(3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f), max_(-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f) {}
    void add(const Vec3& p);
    void add(const Bounds& b);
    float volume() const { return (max_.x - min_.x) * (max_.y - min_.y) * (max_.z - min_.z); }
    const Vec3& min() const { return min_; }
    const Vec3& max() const { return max_; }
};

// ---------------------------------------------------------------- status

enum RelightStatus { RelightSuccess, RelightInvalidCall, RelightNotImplemented };

typedef unsigned short Index;

class Scene;
class Mesh;
class Light;
class Material;
class Texture;
class Lightmap;
class Photonmap;
class Relight;
class Worker;
class Job;
struct JobData;

// Relight.h:70-71
typedef std::vector<Worker*> Workers;

// --------------------------------------------------------------- material

class Texture {
public:
    static Texture* create(int width, int height, int channels, const unsigned char* pixels);
    // Uncompressed 24/32-bit TGA, red and blue swapped on load (scene/Material.cpp:154-205).
    static Texture* createFromFile(const char* fileName);
    int width() const { return m_width; }
    int height() const { return m_height; }
    int channels() const { return m_channels; }
    const unsigned char* pixels() const { return m_pixels.data(); }

private:
    Texture(int w, int h, int c, const unsigned char* px);
    int m_width, m_height, m_channels;
    std::vector<unsigned char> m_pixels;
};

class Material {
public:
    explicit Material(const Rgb& color) : m_color(color), m_texture(nullptr) {}
    virtual ~Material() {}
    const Rgb& color() const { return m_color; }
    void setColor(const Rgb& value) { m_color = value; }
    const Texture* texture() const { return m_texture; }

protected:
    Rgb m_color;
    const Texture* m_texture;
};

class TexturedMaterial : public Material {
public:
    TexturedMaterial(const Texture* texture, const Rgb& color) : Material(color) { m_texture = texture; }
};

// ------------------------------------------------------------------- mesh

struct Vertex {
    enum UvLayer { Diffuse, Lightmap, TotalUvLayers };
    Vec3 position;
    Vec3 normal;
    Uv uv[TotalUvLayers];
    const Material* material = nullptr;
};
typedef std::vector<Vertex> VertexBuffer;
typedef std::vector<Index> IndexBuffer;

class Mesh {
public:
    static Mesh* create() { return new Mesh; }
    // Mesh::createFromFile (scene/Mesh.cpp:111-122): a Wavefront OBJ read
    // with MeshLoader's rules (rl_obj_load); NULL if it cannot be loaded.
    static Mesh* createFromFile(const std::string& fileName);
    // Mesh::addFaces (scene/Mesh.cpp:146-165): indices offset by the current
    // vertex count, one material for the added vertices.
    void addFaces(const VertexBuffer& vertices, const IndexBuffer& indices, const Material* material = nullptr);
    int vertexCount() const { return (int)m_vertices.size(); }
    int indexCount() const { return (int)m_indices.size(); }
    int faceCount() const { return (int)m_indices.size() / 3; }
    const Vertex& vertex(int i) const { return m_vertices[i]; }
    Index index(int i) const { return m_indices[i]; }
    const Bounds& bounds() const { return m_bounds; }
    Lightmap* lightmap() const { return m_lightmap; }
    Photonmap* photonmap() const { return m_photonmap; }
    // Mesh::transformed (scene/Mesh.cpp:277-297).
    Mesh* transformed(const Matrix4& transform) const;
    void overrideMaterial(const Material* material);
    void* userData() const { return m_userData; }
    void setUserData(void* value) { m_userData = value; }

private:
    friend class Lightmap;
    friend class Photonmap;
    friend class Scene;
    Mesh() {}
    void updateBounds();
    VertexBuffer m_vertices;
    IndexBuffer m_indices;
    Bounds m_bounds;
    Lightmap* m_lightmap = nullptr;
    Photonmap* m_photonmap = nullptr;
    void* m_userData = nullptr;
};

// ----------------------------------------------------------------- lights

// The light model objects (scene/Light.h:38-223).  They hold parameters;
// the GPU evaluates them.
class LightCutoff {
public:
    explicit LightCutoff(const Light*) {}
    virtual ~LightCutoff() {}
    virtual int kind() const { return 1; }
};
class LightSpotCutoff : public LightCutoff {
public:
    LightSpotCutoff(const Light* light, const Vec3& direction, float cutoff, float exponent)
        : LightCutoff(light), m_direction(direction), m_cutoff(cutoff), m_exponent(exponent) {}
    int kind() const override { return 2; }
    Vec3 m_direction;
    float m_cutoff, m_exponent;
};
class LightAttenuation {
public:
    explicit LightAttenuation(const Light*) {}
    virtual ~LightAttenuation() {}
};
class LinearLightAttenuation : public LightAttenuation {
public:
    LinearLightAttenuation(const Light* light, float radius, float constant = 0.0f, float linear = 0.0f,
                           float quadratic = 25.0f)
        : LightAttenuation(light), m_radius(radius), m_const(constant), m_linear(linear), m_quadratic(quadratic) {}
    float m_radius, m_const, m_linear, m_quadratic;
};
class LightInfluence {
public:
    explicit LightInfluence(const Light*) {}
    virtual ~LightInfluence() {}
    virtual int kind() const { return 1; }
};
class DirectionalLightInfluence : public LightInfluence {
public:
    DirectionalLightInfluence(const Light* light, const Vec3& direction) : LightInfluence(light), m_direction(direction) {}
    int kind() const override { return 2; }
    Vec3 m_direction;
};
class PhotonEmitter {
public:
    explicit PhotonEmitter(const Light*) {}
    virtual ~PhotonEmitter() {}
    virtual int kind() const { return 1; }
};
class DirectionalPhotonEmitter : public PhotonEmitter {
public:
    DirectionalPhotonEmitter(const Light* light, const Vec3& direction);
    int kind() const override { return 2; }
    Vec3 m_direction;
    float m_plane[4];  // Plane::calculate(direction, light position), Types.h:1656-1658
};

class Light {
public:
    virtual ~Light();
    LightInfluence* influence() const { return m_influence; }
    void setInfluence(LightInfluence* value);
    LightAttenuation* attenuation() const { return m_attenuation; }
    void setAttenuation(LightAttenuation* value);
    LightCutoff* cutoff() const { return m_cutoff; }
    void setCutoff(LightCutoff* value);
    PhotonEmitter* photonEmitter() const { return m_photonEmitter; }
    void setPhotonEmitter(PhotonEmitter* value);
    const Vec3& position() const { return m_position; }
    void setPosition(const Vec3& value) { m_position = value; }
    const Rgb& color() const { return m_color; }
    void setColor(const Rgb& value) { m_color = value; }
    float intensity() const { return m_intensity; }
    void setIntensity(float value) { m_intensity = value; }
    bool castsShadow() const { return m_castsShadow; }
    void setCastsShadow(bool value) { m_castsShadow = value; }
    // FaceLightVertexGenerator samples (light-local), empty without a generator.
    const std::vector<Vec3>& vertices() const { return m_vertices; }

    static Light* createPointLight(const Vec3& position, float radius, const Rgb& color = Rgb(1.0f, 1.0f, 1.0f),
                                   float intensity = 1.0f, bool castsShadow = true);
    static Light* createSpotLight(const Vec3& position, const Vec3& direction, float cutoff, float radius,
                                  const Rgb& color = Rgb(1.0f, 1.0f, 1.0f), float intensity = 1.0f,
                                  bool castsShadow = true);
    static Light* createDirectionalLight(const Vec3& direction, const Rgb& color = Rgb(1.0f, 1.0f, 1.0f),
                                         float intensity = 1.0f, bool castsShadow = true);
    static Light* createAreaLight(const Mesh* mesh, const Vec3& position, const Rgb& color = Rgb(1.0f, 1.0f, 1.0f),
                                  float intensity = 1.0f, bool castsShadow = true);

protected:
    Light() {}

private:
    Vec3 m_position;
    Rgb m_color;
    float m_intensity = 0.0f;
    bool m_castsShadow = false;
    LightCutoff* m_cutoff = nullptr;
    LightAttenuation* m_attenuation = nullptr;
    LightInfluence* m_influence = nullptr;
    PhotonEmitter* m_photonEmitter = nullptr;
    std::vector<Vec3> m_vertices;
};

// ------------------------------------------------------------------- maps

// Lightmap.h:35-55.
struct Lumel {
    enum Flags { Valid = 0x1 };
    Index m_faceIdx;
    Vec3 m_position;
    Vec3 m_normal;
    Rgb m_color;
    int m_photons;
    Rgb m_gathered;
    int m_flags;
    Lumel() : m_faceIdx((Index)-1), m_photons(0), m_flags(0) {}
    operator bool() const { return (m_flags & Valid) != 0; }
};

enum StorageFormat { RawHdr, TgaDoubleLdr, TgaRgbm };

class Lightmap {
public:
    virtual ~Lightmap();
    int width() const { return m_width; }
    int height() const { return m_height; }
    // Host copy of the lumels (downloaded from the device after a bake).
    Lumel* lumels();
    Lumel& lumel(int x, int y) { return lumels()[y * m_width + x]; }
    virtual RelightStatus addMesh(const Mesh* mesh);
    // Lightmap::toHdr (Lightmap.cpp:332-349); the caller deletes[] the buffer.
    float* toHdr();
    // Lightmap::save (Lightmap.cpp:223-283): RawHdr, TgaDoubleLdr or TgaRgbm,
    // the reference's file byte for byte (TGA encoding on the device; a
    // lightmap that was never baked saves RawHdr only).
    bool save(const std::string& fileName, StorageFormat format);
    // Lightmap::expand / blur (Lightmap.cpp:167-220), on the device.
    void expand();
    void blur();

    // device side (used by Relight)
    rl_map* device() const { return m_device; }
    int kind() const { return m_kind; }

protected:
    friend class Relight;
    friend class Scene;
    Lightmap(int width, int height, int kind = 0);
    void attach(rl_scene* scene, const std::vector<const Mesh*>& sceneMeshes);
    void beforeDevice();  // host edits -> device
    void afterDevice();   // device changed: host copy is stale
    int m_width, m_height, m_kind;
    std::vector<const Mesh*> m_meshes;
    std::vector<Lumel> m_host;
    bool m_hostStale = true, m_hostEdited = false;
    rl_map* m_device = nullptr;
};

class Photonmap : public Lightmap {
public:
    RelightStatus addMesh(const Mesh* mesh) override { return addMesh(mesh, false); }
    RelightStatus addMesh(const Mesh* mesh, bool copyVertexColor);
    // Photonmap::gather (Lightmap.cpp:376-413), on the device.
    void gather(int radius);

private:
    friend class Relight;
    Photonmap(int width, int height) : Lightmap(width, height, 1) {}
};

// ------------------------------------------------------------------ scene

class Scene {
public:
    ~Scene();
    RelightStatus begin();
    // Scene::end (scene/Scene.cpp:122-142): the scene is uploaded and its BVH
    // built on the device.
    RelightStatus end();
    Mesh* addMesh(const Mesh* mesh, const Matrix4& transform, const Material* material = nullptr);
    RelightStatus addLight(const Light* light);
    int lightCount() const { return (int)m_lights.size(); }
    const Light* light(int index) const { return m_lights[index]; }
    int meshCount() const { return (int)m_meshes.size(); }
    const Mesh* mesh(int index) const { return m_meshes[index]; }
    const Bounds& bounds() const { return m_bounds; }
    rl_scene* device() const { return m_device; }

private:
    friend class Relight;
    Scene() {}
    enum State { StateInitial, StateAddingObjects, StateReadyToBake };
    State m_state = StateInitial;
    std::vector<const Mesh*> m_meshes;
    std::vector<const Light*> m_lights;
    Bounds m_bounds;
    rl_scene* m_device = nullptr;
    bool m_mapsReady = false;
};

// ----------------------------------------------------------------- baking

namespace bake {
// baker/Baker.h:91-155.
class BakeIterator {
public:
    BakeIterator(int first, int step) : m_firstIndex(first), m_step(step) {}
    virtual ~BakeIterator() {}
    virtual int kind() const = 0;
    int m_firstIndex, m_step;
};
class LumelBakeIterator : public BakeIterator {
public:
    LumelBakeIterator(int first, int step) : BakeIterator(first, step) {}
    int kind() const override { return 0; }
};
class FaceBakeIterator : public BakeIterator {
public:
    FaceBakeIterator(int first, int step) : BakeIterator(first, step) {}
    int kind() const override { return 1; }
};
}  // namespace bake

class Progress {
public:
    Progress() {}
    virtual ~Progress() {}
    virtual void notify(const Mesh* instance, int step, int stepCount) {}
};

// ------------------------------------------------------- jobs and workers

// Worker.h:35-42: what a worker is handed for one mesh.
struct JobData {
    Worker* m_worker = nullptr;            // parent worker (set by Worker::push)
    Job* m_job = nullptr;                  // parent job
    Relight* m_relight = nullptr;          // Relight instance
    const Scene* m_scene = nullptr;        // scene to process
    const Mesh* m_mesh = nullptr;          // mesh instance of the scene
    bake::BakeIterator* m_iterator = nullptr;  // the worker's share of the mesh
};

// Worker.h:45-49: user code run for every (mesh, worker) pair, typically a
// sequence of Relight::bake* calls on data->m_mesh with data->m_iterator.
class Job {
public:
    virtual ~Job() {}
    virtual void execute(JobData* data) = 0;
};

// Worker.h:52-69, Worker.cpp:43-83: for every scene mesh, largest bounding
// volume first (ties keep scene order), push `job` to every worker j with
// FaceBakeIterator(j, workers) (LumelBakeIterator(j, workers) for meshes with
// fewer faces than workers), then wait for all workers.
class FullBakeJob : public Job {
public:
    FullBakeJob(Job* job, const Workers& workers);
    void execute(JobData* data) override;

private:
    Workers m_workers;
    Job* m_job;
};

// Worker.h:72-84, Worker.cpp:86-106: the base worker runs a pushed job at
// once on the calling thread (and then frees the JobData it was handed);
// subclasses may run jobs on their own threads and take over the JobData.
class Worker : public Progress {
public:
    Worker() {}
    virtual ~Worker() {}
    virtual void push(Job* job, JobData* data);
    virtual void wait() {}
};

struct IndirectLightSettings {
    int m_photonPassCount;
    int m_photonBounceCount;
    float m_photonEnergyThreshold;
    float m_photonMaxDistance;
    int m_finalGatherSamples;
    float m_finalGatherDistance;
    int m_finalGatherRadius;
    Rgb m_skyColor;
    Rgb m_ambientColor;
    static IndirectLightSettings fast(const Rgb& skyColor = Rgb(0, 0, 0), const Rgb& ambientColor = Rgb(0, 0, 0),
                                      float photonMaxDistance = 10.0f, float finalGatherDistance = 50.0f);
    static IndirectLightSettings draft(const Rgb& skyColor = Rgb(0, 0, 0), const Rgb& ambientColor = Rgb(0, 0, 0),
                                       float photonMaxDistance = 10.0f, float finalGatherDistance = 50.0f);
    static IndirectLightSettings best(const Rgb& skyColor = Rgb(0, 0, 0), const Rgb& ambientColor = Rgb(0, 0, 0),
                                      float photonMaxDistance = 10.0f, float finalGatherDistance = 50.0f);
    static IndirectLightSettings production(const Rgb& skyColor = Rgb(0, 0, 0), const Rgb& ambientColor = Rgb(0, 0, 0),
                                            float photonMaxDistance = 10.0f, float finalGatherDistance = 50.0f);
};

struct AmbientOcclusionSettings {
    int m_samples;
    float m_occludedFraction;
    float m_maxDistance;
    float m_exponent;
    static AmbientOcclusionSettings fast(float occludedFraction = 0.8f, float maxDistance = 0.6f, float exponent = 1.0f);
    static AmbientOcclusionSettings draft(float occludedFraction = 0.8f, float maxDistance = 0.6f, float exponent = 1.0f);
    static AmbientOcclusionSettings best(float occludedFraction = 0.8f, float maxDistance = 0.6f, float exponent = 1.0f);
    static AmbientOcclusionSettings production(float occludedFraction = 0.8f, float maxDistance = 0.6f,
                                               float exponent = 1.0f);
};

class Relight {
public:
    static Relight* create() { return new Relight; }
    Lightmap* createLightmap(int width, int height) const { return new Lightmap(width, height, 0); }
    Photonmap* createPhotonmap(int width, int height) const { return new Photonmap(width, height); }
    Scene* createScene() const { return new Scene; }
    RelightStatus bakeDirectLight(const Scene* scene, const Mesh* mesh, Progress* progress,
                                  bake::BakeIterator* iterator = nullptr);
    RelightStatus bakeIndirectLight(const Scene* scene, const Mesh* mesh, Progress* progress,
                                    const IndirectLightSettings& settings, bake::BakeIterator* iterator = nullptr);
    RelightStatus bakeAmbientOcclusion(const Scene* scene, const Mesh* mesh, Progress* progress,
                                       const AmbientOcclusionSettings& settings, bake::BakeIterator* iterator = nullptr);
    RelightStatus emitPhotons(const Scene* scene, const IndirectLightSettings& settings);
    // Relight::bake (Relight.cpp:204-213): pushes a FullBakeJob over `workers`
    // to `root`.  With the base Worker as root the bake is done on return.
    void bake(const Scene* scene, Job* job, Worker* root, const Workers& workers);
    // Base of the Philox keys of the stochastic passes (no reference counterpart).
    void setSeed(uint64_t seed) { m_seed = seed; m_calls = 0; }
    // Message of the last failed device call.
    const std::string& lastError() const { return m_error; }

private:
    Relight() {}
    uint64_t nextSeed();
    bool prepare(const Scene* scene);
    RelightStatus status(int rc);
    uint64_t m_seed = 0x5EED;
    uint64_t m_calls = 0;
    std::string m_error;
    std::mutex m_lock;  // serialises the bake calls of worker threads
    std::vector<std::unique_ptr<FullBakeJob>> m_jobs;  // freed with the Relight
};

}  // namespace relight

#endif
