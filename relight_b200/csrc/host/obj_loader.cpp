// Wavefront OBJ ingest with Relight's MeshLoader semantics
// (scene/MeshLoader.cpp:44-226, reached through Mesh::createFromFile,
// scene/Mesh.cpp:111-122), as host code behind the C ABI:
//
//   * lines split on '\n'; "vt" / "vn" / "v" lines first commit the faces
//     read since the last commit as one submesh, then append their floats
//     (parsed as scanf's %f does: strtof after whitespace);
//   * a commit clears the normal / uv flags, so a submesh uses normals or
//     uvs only if "vn" / "vt" lines came after the previous submesh;
//   * "f" lines read one triangle with scanf's %i (base-prefixed integers)
//     as "a/b/c a/b/c a/b/c" whenever normals or uvs are flagged, else as
//     "a b c"; further corners are ignored and an unparsed index stays 0;
//   * each corner becomes {position, normal or (0, 1, 0), colour (1, 1, 1),
//     uv clamped to [0, 1]}; corners equal under float comparison share one
//     vertex (first occurrence keeps its bits and its index order);
//   * each submesh is appended like Mesh::addFaces (scene/Mesh.cpp:146-165):
//     indices offset by the vertices already in the mesh, uv in the
//     lightmap layer, no material.
//
// Where the reference's behaviour is undefined this loader reports an
// error instead: a face index outside the parsed arrays (including an
// unparsed 0), or a mesh beyond the 16-bit index range.  A vertex line
// with unparsable numbers stores 0 (the reference stores whatever was on
// the stack), and a corner without uvs has uv (0, 0).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../../include/relight_b200.h"

int rl_internal_fail(int code, const char* msg);

struct rl_obj_mesh {
    std::vector<float> pos, nrm, uv;
    std::vector<int32_t> idx;
    int submeshes = 0;
};

namespace {

enum { kHasUv = 0x2, kHasNormals = 0x4 };  // MeshLoader::MeshDataFlags

const char* skip_ws(const char* p) {
    while (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n' || *p == '\v' || *p == '\f') p++;
    return p;
}

// scanf("%f ...") over up to n floats; unconverted values stay 0.
void scan_floats(const char* p, float* out, int n) {
    for (int k = 0; k < n; k++) out[k] = 0.0f;
    for (int k = 0; k < n; k++) {
        p = skip_ws(p);
        char* end = nullptr;
        float v = strtof(p, &end);
        if (end == p) return;
        out[k] = v;
        p = end;
    }
}

// scanf's %i: whitespace, sign, then a base-0 integer (0x.. hex, 0.. octal).
bool scan_int(const char*& p, int& out) {
    const char* q = skip_ws(p);
    char* end = nullptr;
    errno = 0;
    long v = strtol(q, &end, 0);
    if (end == q) return false;
    out = (int)v;
    p = end;
    return true;
}

// scanf over "%i/%i/%i %i/%i/%i %i/%i/%i" (slashes = 2), "%i %i %i"
// (slashes = 0): fills vals[corner][field] in order until a mismatch.
void scan_face(const char* p, int slashes, int vals[3][3]) {
    for (int c = 0; c < 3; c++) {
        if (c > 0) p = skip_ws(p);  // the format's blank matches any whitespace
        for (int f = 0; f <= slashes; f++) {
            if (f > 0) {
                if (*p != '/') return;
                p++;
            }
            if (!scan_int(p, vals[c][f])) return;
        }
    }
}

struct Key {
    float v[11];
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        uint64_t h = 1469598103934665603ull;
        for (int i = 0; i < 11; i++) {
            float f = k.v[i] == 0.0f ? 0.0f : k.v[i];  // -0 and +0 compare equal
            uint32_t b;
            memcpy(&b, &f, 4);
            h = (h ^ b) * 1099511628211ull;
        }
        return (size_t)h;
    }
};
struct KeyEq {
    bool operator()(const Key& a, const Key& b) const {
        for (int i = 0; i < 11; i++)
            if (!(a.v[i] == b.v[i])) return false;
        return true;
    }
};

struct Loader {
    std::vector<float> xyz, nrm, uv;        // parsed arrays
    std::vector<int> fx, fu, fn;            // per-corner indices (already -1)
    int flags = 0, submesh_faces = 0, total_faces = 0;
    rl_obj_mesh* out = nullptr;
    std::string error;

    // MeshLoader::commit (scene/MeshLoader.cpp:44-118) + Mesh::addFaces.
    bool commit() {
        if (submesh_faces == 0) return true;
        std::unordered_map<Key, int, KeyHash, KeyEq> index;
        std::vector<Key> verts;
        std::vector<int32_t> local;
        local.reserve(3 * submesh_faces);
        for (int i = total_faces - submesh_faces; i < total_faces; i++) {
            for (int j = 0; j < 3; j++) {
                int xi = fx[3 * i + j], ni = fn[3 * i + j], ui = fu[3 * i + j];
                if (xi < 0 || 3 * (size_t)xi + 2 >= xyz.size()) {
                    error = "face " + std::to_string(i) + ": vertex index " + std::to_string(xi + 1) + " out of range";
                    return false;
                }
                Key k;
                k.v[0] = xyz[3 * xi]; k.v[1] = xyz[3 * xi + 1]; k.v[2] = xyz[3 * xi + 2];
                if (flags & kHasNormals) {
                    if (ni < 0 || 3 * (size_t)ni + 2 >= nrm.size()) {
                        error = "face " + std::to_string(i) + ": normal index " + std::to_string(ni + 1) + " out of range";
                        return false;
                    }
                    k.v[3] = nrm[3 * ni]; k.v[4] = nrm[3 * ni + 1]; k.v[5] = nrm[3 * ni + 2];
                } else {
                    k.v[3] = 0.0f; k.v[4] = 1.0f; k.v[5] = 0.0f;
                }
                k.v[6] = k.v[7] = k.v[8] = 1.0f;
                k.v[9] = k.v[10] = 0.0f;
                if (flags & kHasUv) {
                    if (ui < 0 || 2 * (size_t)ui + 1 >= uv.size()) {
                        error = "face " + std::to_string(i) + ": uv index " + std::to_string(ui + 1) + " out of range";
                        return false;
                    }
                    float u = uv[2 * ui], v = uv[2 * ui + 1];
                    if (u > 1.0f) u = 1.0f;
                    if (v > 1.0f) v = 1.0f;
                    if (u < 0.0f) u = 0.0f;
                    if (v < 0.0f) v = 0.0f;
                    k.v[9] = u; k.v[10] = v;
                }
                auto it = index.find(k);
                int id;
                if (it == index.end()) {
                    id = (int)verts.size();
                    index.emplace(k, id);
                    verts.push_back(k);
                } else {
                    id = it->second;
                }
                local.push_back(id);
            }
        }
        size_t base = out->pos.size() / 3;
        if (base + verts.size() > 65536) {
            error = "mesh exceeds the 16-bit index range (" + std::to_string(base + verts.size()) + " vertices)";
            return false;
        }
        for (const Key& k : verts) {
            out->pos.insert(out->pos.end(), {k.v[0], k.v[1], k.v[2]});
            out->nrm.insert(out->nrm.end(), {k.v[3], k.v[4], k.v[5]});
            out->uv.insert(out->uv.end(), {k.v[9], k.v[10]});
        }
        for (int32_t l : local) out->idx.push_back((int32_t)(l + base));
        out->submeshes++;
        submesh_faces = 0;
        flags = 0;
        return true;
    }

    // MeshLoader::load (scene/MeshLoader.cpp:181-226) over the file's text.
    bool run(const std::string& text) {
        size_t pos = 0;
        while (pos <= text.size()) {
            size_t nl = text.find('\n', pos);
            if (nl == std::string::npos) nl = text.size();
            std::string line = text.substr(pos, nl - pos);
            pos = nl + 1;
            const char* s = line.c_str();
            char c1 = s[0], c2 = c1 ? s[1] : '\0';
            if (c1 == 'v' && c2 == 't') {
                if (!commit()) return false;
                float f[2];
                scan_floats(s + 2, f, 2);
                uv.insert(uv.end(), {f[0], f[1]});
                flags |= kHasUv;
            } else if (c1 == 'v' && c2 == 'n') {
                if (!commit()) return false;
                float f[3];
                scan_floats(s + 2, f, 3);
                nrm.insert(nrm.end(), {f[0], f[1], f[2]});
                flags |= kHasNormals;
            } else if (c1 == 'v') {
                if (!commit()) return false;
                float f[3];
                scan_floats(s + 1, f, 3);
                xyz.insert(xyz.end(), {f[0], f[1], f[2]});
            }
            if (c1 == 'f') {
                // MeshLoader::parseFace (:146-178): with normals or uvs flagged,
                // always the full "v/t/n" form
                int vals[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                const char* p = c2 ? s + 2 : s + 1;
                if (flags & (kHasNormals | kHasUv)) {
                    scan_face(p, 2, vals);
                } else {
                    scan_face(p, 0, vals);
                }
                for (int c = 0; c < 3; c++) {
                    fu.push_back(vals[c][1] - 1);
                    fx.push_back(vals[c][0] - 1);
                    fn.push_back(vals[c][2] - 1);
                }
                total_faces++;
                submesh_faces++;
            }
            if (nl == text.size()) break;
        }
        return commit();
    }
};

}  // namespace

extern "C" int rl_obj_load(const char* path, rl_obj_mesh** out) {
    if (!path || !out) return rl_internal_fail(RL_INVALID_CALL, "rl_obj_load: null argument");
    *out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) return rl_internal_fail(RL_INVALID_CALL, "rl_obj_load: cannot open file");
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    fclose(f);
    rl_obj_mesh* m = new (std::nothrow) rl_obj_mesh;
    if (!m) return rl_internal_fail(RL_OUT_OF_MEMORY, "host allocation failed");
    Loader L;
    L.out = m;
    if (!L.run(text)) {
        delete m;
        return rl_internal_fail(RL_INVALID_CALL, ("rl_obj_load: " + L.error).c_str());
    }
    *out = m;
    return RL_OK;
}

extern "C" int rl_obj_mesh_counts(const rl_obj_mesh* m, int32_t* nvertices, int32_t* nindices, int32_t* nsubmeshes) {
    if (!m) return rl_internal_fail(RL_INVALID_CALL, "null mesh");
    if (nvertices) *nvertices = (int32_t)(m->pos.size() / 3);
    if (nindices) *nindices = (int32_t)m->idx.size();
    if (nsubmeshes) *nsubmeshes = m->submeshes;
    return RL_OK;
}

extern "C" int rl_obj_mesh_arrays(const rl_obj_mesh* m, float* positions, float* normals, float* uv_lightmap,
                                  int32_t* indices) {
    if (!m) return rl_internal_fail(RL_INVALID_CALL, "null mesh");
    if (positions && !m->pos.empty()) memcpy(positions, m->pos.data(), m->pos.size() * sizeof(float));
    if (normals && !m->nrm.empty()) memcpy(normals, m->nrm.data(), m->nrm.size() * sizeof(float));
    if (uv_lightmap && !m->uv.empty()) memcpy(uv_lightmap, m->uv.data(), m->uv.size() * sizeof(float));
    if (indices && !m->idx.empty()) memcpy(indices, m->idx.data(), m->idx.size() * sizeof(int32_t));
    return RL_OK;
}

extern "C" int rl_obj_mesh_destroy(rl_obj_mesh* m) {
    delete m;
    return RL_OK;
}
