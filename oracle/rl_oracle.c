/*
 * rl_oracle — plain-C restatement of Relight's ray-bound bake passes.
 * TEST INFRASTRUCTURE ONLY (see rl_oracle.h).  Compile with -ffp-contract=off.
 *
 * File:line citations are to the reference project (dmsovetov/Relight).
 */
#include "rl_oracle.h"
#include "ort.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ vectors */

typedef struct { float x, y, z; } v3;

static inline v3 mk3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 ld3(const float* p) { v3 r = {p[0], p[1], p[2]}; return r; }
static inline void st3(float* p, v3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul3(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline v3 neg3(v3 a) { return mk3(-a.x, -a.y, -a.z); }
/* Vec3::operator*(Vec3) (Types.h:794-796): x*x' + y*y' + z*z', left to right. */
static inline float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* Vec3::length / normalize (Types.h:841-859). */
static inline float len3(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline float normalize3(v3* a) {
    float len = len3(*a);
    if (len) { a->x /= len; a->y /= len; a->z /= len; }
    return len;
}

/* ------------------------------------------------------------- Philox */

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void oro_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0; c1 = lo1; c2 = hi0 ^ c3 ^ k1; c3 = lo0;
        k0 += PHILOX_W0; k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Purpose tags (counter word 3) keep the streams of different draws apart. */
enum { TAG_AO = 1, TAG_FG = 2, TAG_EMIT = 3, TAG_EMIT_POINT = 4, TAG_BOUNCE = 5, TAG_HEMI_FF = 6,
       TAG_AO_F64 = 11, TAG_FG_F64 = 12 };

#define ORO_MAX_ATTEMPTS 64

static inline float u01(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

/* Vec3::randomDirection (Types.h:924-937): cube rejection, then dir / len.
   Attempt a uses the Philox block (item, sample, a, tag). */
static v3 random_direction(uint64_t seed, uint32_t item, uint32_t sample, uint32_t tag) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    v3 dir = mk3(0, 0, 0);
    float len = 0.0f;
    for (uint32_t a = 0; a < ORO_MAX_ATTEMPTS; a++) {
        uint32_t ctr[4] = {item, sample, a, tag}, r[4];
        oro_philox4x32_10(ctr, key, r);
        dir.x = (u01(r[0]) * 2.0f - 1.0f);
        dir.y = (u01(r[1]) * 2.0f - 1.0f);
        dir.z = (u01(r[2]) * 2.0f - 1.0f);
        len = len3(dir);
        if (!(len > 1.0f)) break;
    }
    return mk3(dir.x / len, dir.y / len, dir.z / len);
}

/* Vec3::randomHemisphereDirection (Types.h:940-949). */
static v3 random_hemisphere(v3 normal, uint64_t seed, uint32_t item, uint32_t sample, uint32_t tag) {
    v3 dir = random_direction(seed, item, sample, tag);
    if (dot3(dir, normal) < 0) dir = neg3(dir);
    return dir;
}

/* ------------------------------------------------------------ context */

struct oro_ctx {
    const rl_scene_desc* d;
    ort_scene* bvh;
    int32_t* tri_face;  /* per global triangle: face index within its mesh */
    int32_t* tri_mesh;
    uint64_t stats[3];
};

oro_ctx* oro_create(const rl_scene_desc* d) {
    oro_ctx* c = (oro_ctx*)calloc(1, sizeof(oro_ctx));
    c->d = d;
    c->bvh = ort_create();
    c->tri_face = (int32_t*)malloc(sizeof(int32_t) * (size_t)(d->ntris + 1));
    c->tri_mesh = (int32_t*)malloc(sizeof(int32_t) * (size_t)(d->ntris + 1));
    /* one ort geometry per mesh, registration order = mesh order (rt/Embree.cpp:180-217) */
    for (int m = 0; m < d->nmeshes; m++) {
        int t0 = d->mesh_first_tri[m], t1 = d->mesh_first_tri[m + 1];
        ort_add_mesh(c->bvh, d->pos, 3, d->nverts, d->tris + 3 * (size_t)t0, t1 - t0);
        for (int t = t0; t < t1; t++) { c->tri_face[t] = t - t0; c->tri_mesh[t] = m; }
    }
    ort_commit(c->bvh);
    return c;
}

void oro_destroy(oro_ctx* c) {
    if (!c) return;
    ort_destroy(c->bvh);
    free(c->tri_face); free(c->tri_mesh);
    free(c);
}

void oro_last_stats(const oro_ctx* c, uint64_t out[3]) {
    out[0] = c->stats[0]; out[1] = c->stats[1]; out[2] = c->stats[2];
}

/* -------------------------------------------------- face interpolation */

typedef struct { int a, b, c; } face_t;  /* global vertex ids m_a, m_b, m_c */

static inline face_t face_of(const rl_scene_desc* d, int mesh, int prim) {
    int t = d->mesh_first_tri[mesh] + prim;
    face_t f = {d->tris[3 * t], d->tris[3 * t + 1], d->tris[3 * t + 2]};
    return f;
}

/* Face::normalAt / positionAt (scene/Mesh.cpp:454-475):
   a + (b - a) * uv.y + (c - a) * uv.x, per component, left to right. */
static inline v3 interp3(const float* arr, face_t f, float bx, float by) {
    v3 a = ld3(arr + 3 * f.a), b = ld3(arr + 3 * f.b), c = ld3(arr + 3 * f.c);
    return mk3(a.x + (b.x - a.x) * by + (c.x - a.x) * bx,
               a.y + (b.y - a.y) * by + (c.y - a.y) * bx,
               a.z + (b.z - a.z) * by + (c.z - a.z) * bx);
}

/* Face::uvAt (scene/Mesh.cpp:488-495). */
static inline void interp2(const float* arr, face_t f, float bx, float by, float out[2]) {
    const float* a = arr + 2 * f.a; const float* b = arr + 2 * f.b; const float* c = arr + 2 * f.c;
    out[0] = a[0] + (b[0] - a[0]) * by + (c[0] - a[0]) * bx;
    out[1] = a[1] + (b[1] - a[1]) * by + (c[1] - a[1]) * bx;
}

/* Texture::colorAt (scene/Material.cpp:87-98): nearest texel with wrap. */
static void texture_color(const rl_scene_desc* d, int tex, const float uv[2], float out[4]) {
    int w = d->tex_dims[3 * tex], h = d->tex_dims[3 * tex + 1], ch = d->tex_dims[3 * tex + 2];
    int x = ((int)(uv[0] * (float)w)) % w;
    int y = ((int)(uv[1] * (float)h)) % h;
    if (x >= 0 && x < w && y >= 0 && y < h) {
        const uint8_t* p = d->tex_pixels + d->tex_offset[tex] + ((size_t)y * w * ch + (size_t)x * ch);
        out[0] = p[0] / 255.0f; out[1] = p[1] / 255.0f; out[2] = p[2] / 255.0f;
        out[3] = ch == 4 ? p[3] / 255.0f : 1.0f;
        return;
    }
    out[0] = 1; out[1] = 0; out[2] = 1; out[3] = 1;
}

/* Face::colorAt (scene/Mesh.cpp:478-485) -> Material/TexturedMaterial::colorAt
   (scene/Material.cpp:41-44, 67-70): vertex a's material decides. */
static void face_color(const rl_scene_desc* d, face_t f, float bx, float by, float out[4]) {
    int m = d->vmat ? d->vmat[f.a] : -1;
    if (m < 0) { out[0] = out[1] = out[2] = out[3] = 1.0f; return; }
    float base[4] = {d->mat_rgb[3 * m], d->mat_rgb[3 * m + 1], d->mat_rgb[3 * m + 2], 1.0f};
    int tex = d->mat_tex ? d->mat_tex[m] : -1;
    if (tex < 0) { memcpy(out, base, sizeof base); return; }
    float uv[2], t[4];
    interp2(d->uv0, f, bx, by, uv);
    texture_color(d, tex, uv, t);
    for (int k = 0; k < 4; k++) out[k] = base[k] * t[k];
}

/* ------------------------------------------------------------ tracing */

#define HIT_POINT 1
#define HIT_UV 2
#define HIT_COLOR 4
#define HIT_NORMAL 8
#define HIT_USE_ALPHA 16

typedef struct {
    int hit;
    v3 point, normal;
    float rgba[4];
    float uv[2];
    int mesh, face;
} trace_result;

/* rt::Embree::traceSegment (rt/Embree.cpp:145-177) with initializeRay
   (:107-130): dir = normalize(end - start), tnear 0.01, tfar = |end - start|;
   hit point = start + dir * t; (u, v) passed as Barycentric(u, v), so the
   attributes weight c by u and b by v; alpha <= 0.1 restarts one unit past
   the hit, at most 25 times. */
static void trace_segment(const oro_ctx* c, v3 start, v3 end, int flags, trace_result* res) {
    const rl_scene_desc* d = c->d;
    for (int step = 0;; step++) {
        v3 dir = sub3(end, start);
        float len = normalize3(&dir);
        float o[3] = {start.x, start.y, start.z}, dd[3] = {dir.x, dir.y, dir.z};
        ort_hit h;
        ort_stats st = {0, 0, 0};
        int hit = ort_intersect(c->bvh, o, dd, 0.01f, len, &h, &st);
        ((oro_ctx*)c)->stats[0] += st.rays; ((oro_ctx*)c)->stats[1] += st.box_tests; ((oro_ctx*)c)->stats[2] += st.tri_tests;
        res->hit = 0;
        if (!hit) return;
        v3 point = add3(start, mul3(dir, h.t));
        face_t f = face_of(d, h.geom, h.prim);
        float rgba[4];
        face_color(d, f, h.u, h.v, rgba);
        if ((flags & HIT_USE_ALPHA) && rgba[3] <= 0.1f && step < 25) {
            start = add3(point, dir);
            continue;
        }
        res->hit = 1;
        res->point = point;
        res->mesh = h.geom;
        res->face = h.prim;
        if (flags & HIT_NORMAL) res->normal = interp3(d->nrm, f, h.u, h.v);
        if (flags & HIT_COLOR) memcpy(res->rgba, rgba, sizeof rgba);
        if (flags & HIT_UV) interp2(d->uv1, f, h.u, h.v, res->uv);
        return;
    }
}

void oro_trace_segments(const oro_ctx* c, int n, const float* seg, int flags, int32_t* hit, float* point,
                        float* normal, float* rgba, float* uv, int32_t* mesh, int32_t* face) {
    for (int i = 0; i < n; i++) {
        trace_result r;
        memset(&r, 0, sizeof r);
        trace_segment(c, ld3(seg + 6 * i), ld3(seg + 6 * i + 3), flags, &r);
        if (hit) hit[i] = r.hit;
        if (point) st3(point + 3 * i, r.hit ? r.point : mk3(0, 0, 0));
        if (normal) st3(normal + 3 * i, r.hit && (flags & HIT_NORMAL) ? r.normal : mk3(0, 0, 0));
        if (rgba) for (int k = 0; k < 4; k++) rgba[4 * i + k] = r.hit && (flags & HIT_COLOR) ? r.rgba[k] : 0.0f;
        if (uv) { uv[2 * i] = r.hit && (flags & HIT_UV) ? r.uv[0] : 0.0f; uv[2 * i + 1] = r.hit && (flags & HIT_UV) ? r.uv[1] : 0.0f; }
        if (mesh) mesh[i] = r.hit ? r.mesh : -1;
        if (face) face[i] = r.hit ? r.face : -1;
    }
}

void oro_trace_stats(const oro_ctx* c, int n, const float* seg, int any, uint64_t out[3]) {
    ort_stats st = {0, 0, 0};
    for (int i = 0; i < n; i++) {
        v3 s = ld3(seg + 6 * i), e = ld3(seg + 6 * i + 3);
        v3 dir = sub3(e, s);
        float len = normalize3(&dir);
        float o[3] = {s.x, s.y, s.z}, dd[3] = {dir.x, dir.y, dir.z};
        ort_hit h;
        if (any) ort_occluded(c->bvh, o, dd, 0.01f, len, &st);
        else ort_intersect(c->bvh, o, dd, 0.01f, len, &h, &st);
    }
    out[0] = st.rays; out[1] = st.box_tests; out[2] = st.tri_tests;
}

/* ---------------------------------------------------------- texel init */

/* Face::isUvInside (scene/Mesh.cpp:415-438). */
static int uv_inside(const float* a, const float* b, const float* cc, const float uv[2], float bary[2]) {
    float v0x = cc[0] - a[0], v0y = cc[1] - a[1];
    float v1x = b[0] - a[0], v1y = b[1] - a[1];
    float v2x = uv[0] - a[0], v2y = uv[1] - a[1];
    float dot00 = v0x * v0x + v0y * v0y;
    float dot01 = v0x * v1x + v0y * v1y;
    float dot02 = v0x * v2x + v0y * v2y;
    float dot11 = v1x * v1x + v1y * v1y;
    float dot12 = v1x * v2x + v1y * v2y;
    float invDenom = 1.0f / (dot00 * dot11 - dot01 * dot01);
    float u = (dot11 * dot02 - dot01 * dot12) * invDenom;
    float v = (dot00 * dot12 - dot01 * dot02) * invDenom;
    bary[0] = u; bary[1] = v;
    return (u >= 0.0f) && (v >= 0.0f) && (u + v < 1.0f);
}

static inline float fmin3(float a, float b, float c) { float m = b < c ? b : c; return a < m ? a : m; }
static inline float fmax3(float a, float b, float c) { float m = b > c ? b : c; return a > m ? a : m; }

/* Lightmap::initializeLumels(mesh) -> (face) -> initializeLumel
   (Lightmap.cpp:109-164) with Lightmap::rect (:118-130). */
void oro_init_lumels(const rl_scene_desc* d, int mesh, rl_lumels* lm) {
    int W = lm->width, H = lm->height;
    int t0 = d->mesh_first_tri[mesh], t1 = d->mesh_first_tri[mesh + 1];
    for (int t = t0; t < t1; t++) {
        face_t f = {d->tris[3 * t], d->tris[3 * t + 1], d->tris[3 * t + 2]};
        const float* a = d->uv1 + 2 * f.a; const float* b = d->uv1 + 2 * f.b; const float* cc = d->uv1 + 2 * f.c;
        float minx = fmin3(a[0], b[0], cc[0]), maxx = fmax3(a[0], b[0], cc[0]);
        float miny = fmin3(a[1], b[1], cc[1]), maxy = fmax3(a[1], b[1], cc[1]);
        int uStart = (int)(minx * W), uEnd = (int)(maxx * W);
        int vStart = (int)(miny * H), vEnd = (int)(maxy * H);
        int vmax = vEnd < H - 1 ? vEnd : H - 1, umax = uEnd < W - 1 ? uEnd : W - 1;
        /* a uv below 0 makes the reference index before the map (undefined
           behaviour); such texels are skipped here */
        if (uStart < 0) uStart = 0;
        if (vStart < 0) vStart = 0;
        for (int v = vStart; v <= vmax; v++) {
            for (int u = uStart; u <= umax; u++) {
                float uv[2] = {(u + 0.5f) / (float)W, (v + 0.5f) / (float)H};
                float bary[2];
                if (!uv_inside(a, b, cc, uv, bary)) continue;
                size_t i = (size_t)W * v + u;
                lm->face[i] = t - t0;
                if (lm->mesh) lm->mesh[i] = mesh;
                st3(lm->position + 3 * i, interp3(d->pos, f, bary[0], bary[1]));
                st3(lm->normal + 3 * i, interp3(d->nrm, f, bary[0], bary[1]));
                st3(lm->color + 3 * i, mk3(0, 0, 0));
                lm->flags[i] |= 1;
            }
        }
    }
}

/* ------------------------------------------------------------ iterators */

/* Lumel i's turn under `it`: LumelBakeIterator::next visits i = first,
   first + step, ... (baker/Baker.cpp:176-185); FaceBakeIterator::next visits
   the lumels of faces first, first + step, ... of its mesh whose m_faceIdx is
   that face (:202-234). */
static int iter_visits(const rl_lumels* lm, const rl_iterator* it, int i) {
    if (!(lm->flags[i] & 1)) return 0;
    if (!it || it->kind == 0) {
        int first = it ? it->first : 0, step = it ? it->step : 1;
        return i >= first && (i - first) % step == 0;
    }
    if (!lm->mesh || lm->mesh[i] != it->mesh) return 0;
    int f = lm->face[i];
    return f >= it->first && (f - it->first) % it->step == 0;
}

/* ---------------------------------------------------------- direct light */

/* LightInfluence::lambert (scene/Light.cpp:392-396). */
static inline float lambert(v3 dir, v3 n) { float dp = dot3(dir, n); return dp < 0.0f ? 0.0f : dp; }

/* LightSpotCutoff::cutoffForDirection (scene/Light.cpp:461-476). */
static float spot_cutoff_for_direction(const rl_light* L, v3 direction) {
    float value = dot3(direction, ld3(L->spot_direction));
    if (value <= L->spot_cutoff) return 0.0f;
    value = (1.0f - (1.0f - value) * 1.0f / (1.0f - L->spot_cutoff));
    if (fabsf(1.0f - L->spot_exponent) > 0.01f) value = powf(value, L->spot_exponent);
    return value;
}

/* DirectLight::influenceFromPoint (baker/DirectLight.cpp:101-125) with
   LightInfluence::calculate (scene/Light.cpp:372-389),
   DirectionalLightInfluence::calculate (:407-421), LightCutoff /
   LightSpotCutoff::calculate (:432-458), LinearLightAttenuation (:496-500). */
static float influence_from_point(const oro_ctx* c, v3 lpos, v3 lnrm, v3 point, const rl_light* L) {
    float inf = 0.0f, att = 1.0f, cut = 1.0f, distance = 0.0f;
    if (L->influence == 1) {
        v3 direction = sub3(point, lpos);
        distance = normalize3(&direction);
        float intensity = lambert(direction, lnrm);
        if (intensity <= 0.001f) {
            inf = 0.0f;
        } else {
            if (L->casts_shadow) {
                trace_result r;
                trace_segment(c, lpos, point, HIT_USE_ALPHA, &r);
                intensity *= r.hit ? 0.0f : 1.0f;
            }
            inf = intensity;
        }
    } else if (L->influence == 2) {
        v3 ldir = ld3(L->direction);
        float intensity = lambert(neg3(ldir), lnrm);
        if (intensity <= 0.001f) {
            inf = 0.0f;
        } else {
            if (L->casts_shadow) {
                trace_result r;
                trace_segment(c, lpos, sub3(lpos, mul3(ldir, 1000.0f)), HIT_USE_ALPHA, &r);
                intensity *= r.hit ? 0.0f : 1.0f;
            }
            inf = intensity;
        }
    }
    if (L->cutoff == 2) {
        v3 dir = sub3(lpos, ld3(L->position));
        normalize3(&dir);
        cut = spot_cutoff_for_direction(L, dir);
    }
    if (L->attenuation) {
        float r = distance / L->att_radius;
        float a = 1.0f / (1.0f + L->att_const + L->att_linear * r + L->att_quadratic * r * r);
        att = a > 0.0f ? a : 0.0f;
    }
    return inf * att * cut;
}

/* DirectLight::bakeLumel / lightFromPoint / lightFromPointSet
   (baker/DirectLight.cpp:46-98). */
static void direct_lumel(const oro_ctx* c, const rl_light* lights, int nlights, const float* lverts, v3 pos, v3 nrm,
                         float* color) {
    for (int l = 0; l < nlights; l++) {
        const rl_light* L = &lights[l];
        v3 lc = ld3(L->color);
        v3 infl = mk3(0, 0, 0);
        if (L->vertex_count > 0) {
            v3 acc = mk3(0, 0, 0);
            for (int i = 0; i < L->vertex_count; i++) {
                v3 vp = ld3(lverts + 3 * (size_t)(L->vertex_first + i));
                float inf = influence_from_point(c, pos, nrm, add3(vp, ld3(L->position)), L);
                if (inf > 0.0f) acc = add3(acc, mul3(mul3(lc, L->intensity), inf));
            }
            float n = (float)L->vertex_count;
            infl = mk3(acc.x / n, acc.y / n, acc.z / n);
        } else {
            float inf = influence_from_point(c, pos, nrm, ld3(L->position), L);
            if (inf > 0.0f) infl = mul3(mul3(lc, L->intensity), inf);
        }
        color[0] += infl.x; color[1] += infl.y; color[2] += infl.z;
    }
}

void oro_bake_direct(const oro_ctx* c, const rl_light* lights, int nlights, const float* light_vertices,
                     rl_lumels* lm, const rl_iterator* it) {
    int n = lm->width * lm->height;
    ((oro_ctx*)c)->stats[0] = ((oro_ctx*)c)->stats[1] = ((oro_ctx*)c)->stats[2] = 0;
    for (int i = 0; i < n; i++) {
        if (!iter_visits(lm, it, i)) continue;
        direct_lumel(c, lights, nlights, light_vertices, ld3(lm->position + 3 * (size_t)i),
                     ld3(lm->normal + 3 * (size_t)i), lm->color + 3 * (size_t)i);
    }
}

/* ----------------------------------------------------------- AO */

void oro_bake_ao(const oro_ctx* c, rl_lumels* lm, int samples, float occluded_fraction, float max_distance,
                 float exponent, uint64_t seed, const rl_iterator* it) {
    int n = lm->width * lm->height;
    ((oro_ctx*)c)->stats[0] = ((oro_ctx*)c)->stats[1] = ((oro_ctx*)c)->stats[2] = 0;
    for (int i = 0; i < n; i++) {
        if (!iter_visits(lm, it, i)) continue;
        v3 pos = ld3(lm->position + 3 * (size_t)i), nrm = ld3(lm->normal + 3 * (size_t)i);
        int occluded = 0;
        for (int s = 0; s < samples; s++) {
            v3 dir = random_hemisphere(nrm, seed, (uint32_t)i, (uint32_t)s, TAG_AO);
            trace_result r;
            trace_segment(c, pos, add3(pos, mul3(dir, max_distance)), 0, &r);
            if (r.hit) occluded++;
        }
        float value = 1.0f - occluded / (samples * occluded_fraction);
        if (fabsf(1.0f - exponent) > 0.01f) value = powf(value, exponent);
        float* col = lm->color + 3 * (size_t)i;
        col[0] *= value; col[1] *= value; col[2] *= value;
    }
}

/* ----------------------------------------------------------- photons */

/* Lightmap::lumel(const Uv&) (Lightmap.cpp:61-67): x = int(u * (W - 1)).
   The reference indexes out of range for uv outside [0, 1]; clamped here. */
static inline size_t lumel_at_uv(const rl_lumels* m, const float uv[2]) {
    int x = (int)(uv[0] * (float)(m->width - 1));
    int y = (int)(uv[1] * (float)(m->height - 1));
    if (x < 0) x = 0;
    if (x > m->width - 1) x = m->width - 1;
    if (y < 0) y = 0;
    if (y > m->height - 1) y = m->height - 1;
    return (size_t)y * m->width + x;
}

static inline float luminance(v3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

long long oro_emit_photons(const oro_ctx* c, const rl_light* lights, int nlights, rl_lumels* photonmaps,
                           int pass_count, int max_depth, float energy_threshold, float max_distance,
                           uint64_t seed) {
    return oro_emit_photons_range(c, lights, nlights, photonmaps, pass_count, max_depth, energy_threshold,
                                  max_distance, seed, 0, -1);
}

long long oro_emit_photons_range(const oro_ctx* c, const rl_light* lights, int nlights, rl_lumels* photonmaps,
                                 int pass_count, int max_depth, float energy_threshold, float max_distance,
                                 uint64_t seed, long long first_photon, long long photon_count) {
    const rl_scene_desc* d = c->d;
    long long stored = 0;
    uint32_t photon = 0;
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    ((oro_ctx*)c)->stats[0] = ((oro_ctx*)c)->stats[1] = ((oro_ctx*)c)->stats[2] = 0;
    /* Photons::emit (baker/Photons.cpp:50-65) */
    for (int j = 0; j < pass_count; j++) {
        for (int li = 0; li < nlights; li++) {
            const rl_light* L = &lights[li];
            if (!L->emitter) continue;
            /* PhotonEmitter::photonCount (scene/Light.cpp:334-337) */
            int count = (int)(L->intensity * 25000);
            /* Photons::emitPhotons (baker/Photons.cpp:68-92) */
            for (int k = 0; k < count; k++, photon++) {
                if ((long long)photon < first_photon ||
                    (photon_count >= 0 && (long long)photon >= first_photon + photon_count))
                    continue;
                v3 pos, dir;
                if (L->emitter == 1) {
                    /* PhotonEmitter::emit (scene/Light.cpp:340-344) */
                    pos = ld3(L->position);
                    dir = random_direction(seed, photon, 0, TAG_EMIT);
                } else {
                    /* DirectionalPhotonEmitter::emit (scene/Light.cpp:355-361) with
                       Bounds::randomPointInside (Types.h:1445-1450), lerp (Types.h:75-78)
                       and Plane::operator* (Types.h:1715-1718). */
                    uint32_t ctr[4] = {photon, 0, 0, TAG_EMIT_POINT}, r[4];
                    oro_philox4x32_10(ctr, key, r);
                    float s0 = u01(r[0]), s1 = u01(r[1]), s2 = u01(r[2]);
                    v3 pt = mk3(d->bounds_lo[0] * (1.0f - s0) + d->bounds_hi[0] * s0,
                                d->bounds_lo[1] * (1.0f - s1) + d->bounds_hi[1] * s1,
                                d->bounds_lo[2] * (1.0f - s2) + d->bounds_hi[2] * s2);
                    v3 pn = ld3(L->emitter_plane);
                    float dist = dot3(pn, pt) + L->emitter_plane[3];
                    v3 onplane = sub3(pt, mul3(pn, dist));
                    dir = ld3(L->direction);
                    pos = sub3(onplane, mul3(dir, 5.0f));
                }
                float cut = 1.0f;
                if (L->cutoff == 2) cut = spot_cutoff_for_direction(L, dir);
                if (cut <= 0.0f) continue;
                v3 col = mul3(mul3(ld3(L->color), L->intensity), cut);
                /* Photons::trace (baker/Photons.cpp:95-126), recursion unrolled */
                for (int depth = 0;; depth++) {
                    if (depth > max_depth || luminance(col) < energy_threshold) break;
                    trace_result r;
                    trace_segment(c, pos, add3(pos, mul3(dir, max_distance)), HIT_POINT | HIT_UV | HIT_COLOR | HIT_NORMAL, &r);
                    if (!r.hit) break;
                    /* the attenuation value is computed and discarded (:110-113) */
                    float influence = lambert(neg3(dir), r.normal) * 1.0f;
                    v3 hit_color = mul3(mk3(col.x * r.rgba[0], col.y * r.rgba[1], col.z * r.rgba[2]), influence);
                    /* Photons::store (:129-144) */
                    int pm = d->mesh_photonmap ? d->mesh_photonmap[r.mesh] : -1;
                    if (pm >= 0) {
                        rl_lumels* P = &photonmaps[pm];
                        size_t ti = lumel_at_uv(P, r.uv);
                        if (P->flags[ti] & 1) {
                            float* pc = P->color + 3 * ti;
                            pc[0] += hit_color.x; pc[1] += hit_color.y; pc[2] += hit_color.z;
                            P->photons[ti]++;
                            stored++;
                        }
                    }
                    dir = random_hemisphere(r.normal, seed, photon, (uint32_t)(depth + 1), TAG_BOUNCE);
                    pos = r.point;
                    col = hit_color;
                }
            }
        }
    }
    return stored;
}

/* Photonmap::gather (Lightmap.cpp:376-413), including the x < m_height loop
   bound of :379.  Writes past the end of the map (undefined behaviour in the
   reference when width < height) are skipped. */
void oro_photonmap_gather(rl_lumels* pm, int radius) {
    int W = pm->width, H = pm->height;
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < H; x++) {
            float cr = 0, cg = 0, cb = 0;
            int photons = 0;
            for (int j = y - radius; j <= y + radius; j++) {
                for (int i = x - radius; i <= x + radius; i++) {
                    if (i < 0 || j < 0 || i >= W || j >= H) continue;
                    size_t li = (size_t)j * W + i;
                    float distance = sqrtf((float)((x - i) * (x - i) + (y - j) * (y - j)));
                    if (distance > radius) continue;
                    cr += pm->color[3 * li]; cg += pm->color[3 * li + 1]; cb += pm->color[3 * li + 2];
                    photons += pm->photons[li];
                }
            }
            size_t o = (size_t)y * W + x;
            if (o >= (size_t)W * H) continue;
            if (photons == 0) { pm->gathered[3 * o] = 0; pm->gathered[3 * o + 1] = 0; pm->gathered[3 * o + 2] = 0; }
            else {
                float p = (float)photons;
                pm->gathered[3 * o] = cr / p; pm->gathered[3 * o + 1] = cg / p; pm->gathered[3 * o + 2] = cb / p;
            }
        }
    }
}

/* ------------------------------------------------------- post-process */

void oro_expand(rl_lumels* lm) {
    int W = lm->width, H = lm->height;
    /* Lightmap::expand (Lightmap.cpp:167-182) + fillInvalidAt (:185-193) */
    for (int y = 1; y < H - 1; y++) {
        for (int x = 1; x < W - 1; x++) {
            size_t c = (size_t)y * W + x;
            if (!(lm->flags[c] & 1)) continue;
            const int dx[4] = {-1, -1, 1, 1}, dy[4] = {-1, 1, -1, 1};
            for (int k = 0; k < 4; k++) {
                size_t t = (size_t)(y + dy[k]) * W + (x + dx[k]);
                if (lm->flags[t] & 1) continue;
                lm->color[3 * t] = lm->color[3 * c];
                lm->color[3 * t + 1] = lm->color[3 * c + 1];
                lm->color[3 * t + 2] = lm->color[3 * c + 2];
            }
        }
    }
}

void oro_blur(rl_lumels* lm) {
    int W = lm->width, H = lm->height;
    /* Lightmap::blur (Lightmap.cpp:196-220) */
    for (int y = 1; y < H - 1; y++) {
        for (int x = 1; x < W - 1; x++) {
            float r = 0.0f, g = 0.0f, b = 0.0f;
            int count = 0;
            for (int j = y - 1; j <= y + 1; j++) {
                for (int i = x - 1; i <= x + 1; i++) {
                    size_t l = (size_t)j * W + i;
                    if (lm->flags[l] & 1) {
                        r += lm->color[3 * l]; g += lm->color[3 * l + 1]; b += lm->color[3 * l + 2];
                        count++;
                    }
                }
            }
            if (count) {
                float inv = 1.0f / (float)count;
                size_t o = (size_t)y * W + x;
                lm->color[3 * o] = r * inv; lm->color[3 * o + 1] = g * inv; lm->color[3 * o + 2] = b * inv;
            }
        }
    }
}

uint8_t oro_f2u8(float v) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return 0;
    return (uint8_t)(uint32_t)(int32_t)v;
}

static float min2f(float a, float b) { return a < b ? a : b; }   /* Types.h:87-89 */
static float max2f(float a, float b) { return a > b ? a : b; }   /* Types.h:99-101 */

void oro_to_double_ldr(const rl_lumels* lm, uint8_t* out) {
    size_t n = (size_t)lm->width * lm->height;
    /* Rgb::doubleLdr (Types.h:215-221) */
    for (size_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) out[3 * i + k] = oro_f2u8(min2f(255.0f, lm->color[3 * i + k] * 0.5f * 255.0f));
}

void oro_to_rgbm(const rl_lumels* lm, uint8_t* out) {
    int W = lm->width, H = lm->height;
    size_t stride = (size_t)W * 4;
    /* Lightmap::toRgbmLdr (Lightmap.cpp:288-308), Rgb::rgbm (Types.h:224-235) */
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            const float* c = lm->color + 3 * ((size_t)y * W + x);
            float m = 255.0f / max2f(c[0], max2f(c[1], c[2]));
            uint8_t* px = out + (size_t)y * stride + (size_t)x * 3;
            px[0] = oro_f2u8(min2f(255.0f, c[0] / m * 255.0f));
            px[1] = oro_f2u8(min2f(255.0f, c[1] / m * 255.0f));
            px[2] = oro_f2u8(min2f(255.0f, c[2] / m * 255.0f));
            px[3] = oro_f2u8(min2f(255.0f, m * 255.0f));
        }
    }
}

/* ---------------------------------------------------------- final gather */

void oro_bake_indirect(const oro_ctx* c, rl_lumels* lm, const rl_lumels* photonmaps, int samples,
                       float max_distance, const float sky[3], const float ambient[3], uint64_t seed,
                       const rl_iterator* it) {
    const rl_scene_desc* d = c->d;
    int n = lm->width * lm->height;
    ((oro_ctx*)c)->stats[0] = ((oro_ctx*)c)->stats[1] = ((oro_ctx*)c)->stats[2] = 0;
    /* IndirectLight::bakeLumel (baker/IndirectLight.cpp:47-75) */
    for (int i = 0; i < n; i++) {
        if (!iter_visits(lm, it, i)) continue;
        v3 pos = ld3(lm->position + 3 * (size_t)i), nrm = ld3(lm->normal + 3 * (size_t)i);
        float gr = 0, gg = 0, gb = 0;
        for (int k = 0; k < samples; k++) {
            v3 dir = random_hemisphere(nrm, seed, (uint32_t)i, (uint32_t)k, TAG_FG);
            float dp = dot3(nrm, dir);
            float influence = dp > 0.0f ? dp : 0.0f;
            trace_result r;
            trace_segment(c, pos, add3(pos, mul3(dir, max_distance)), HIT_UV | HIT_NORMAL, &r);
            if (!r.hit) {
                gr += sky[0] * influence + ambient[0];
                gg += sky[1] * influence + ambient[1];
                gb += sky[2] * influence + ambient[2];
                continue;
            }
            if (dot3(dir, r.normal) >= 0.0f) continue;
            int pm = d->mesh_photonmap ? d->mesh_photonmap[r.mesh] : -1;
            if (pm >= 0) {
                const rl_lumels* P = &photonmaps[pm];
                size_t ti = lumel_at_uv(P, r.uv);
                gr += P->gathered[3 * ti] * influence + ambient[0];
                gg += P->gathered[3 * ti + 1] * influence + ambient[1];
                gb += P->gathered[3 * ti + 2] * influence + ambient[2];
            }
        }
        float s = (float)samples;
        float* col = lm->color + 3 * (size_t)i;
        col[0] += gr / s; col[1] += gg / s; col[2] += gb / s;
    }
}

/* ------------------------------------------------------------ radiosity */

typedef struct { int32_t i, j; float w; } ff_pair;

/* RadiosityBuilder::computeFormFactors (radiosity/RadiosityBuilder.cpp:126-139),
   distanceFormFactor (:142-176) and refineFormFactors (:99-123). */
long long oro_ff_pairwise(const oro_ctx* c, int n, const float* pos, const float* nrm, float threshold,
                          int64_t* row_ptr, int32_t* cols, float* vals) {
    const float Pi = 3.1415926535897932f;  /* Types.h:58 */
    size_t cap = 1024, np = 0;
    ff_pair* pairs = (ff_pair*)malloc(sizeof(ff_pair) * cap);
    ((oro_ctx*)c)->stats[0] = ((oro_ctx*)c)->stats[1] = ((oro_ctx*)c)->stats[2] = 0;
    for (int i = 0; i < n; i++) {
        v3 rPos = ld3(pos + 3 * (size_t)i), rN = ld3(nrm + 3 * (size_t)i);
        for (int j = i + 1; j < n; j++) {
            v3 sPos = ld3(pos + 3 * (size_t)j), sN = ld3(nrm + 3 * (size_t)j);
            v3 dir = sub3(sPos, rPos);
            float r = normalize3(&dir);
            float cosBA = dot3(dir, rN);
            float cosAB = -(dot3(dir, sN));
            if (r == 0.0f || cosAB < 0.0f || cosBA < 0.0f) continue;
            float wBA = ((cosBA * cosAB) / (Pi * r * r));
            float wAB = ((cosAB * cosBA) / (Pi * r * r));
            if (wBA < threshold && wAB < threshold) continue;
            trace_result h;
            trace_segment(c, rPos, sPos, HIT_POINT | HIT_UV | HIT_COLOR | HIT_NORMAL, &h);
            if (h.hit) continue;
            if (np == cap) { cap *= 2; pairs = (ff_pair*)realloc(pairs, sizeof(ff_pair) * cap); }
            /* wBA == wAB bit for bit (commutative product); both pushes share it */
            pairs[np].i = i; pairs[np].j = j; pairs[np].w = wBA; np++;
        }
    }
    long long nnz = 2 * (long long)np;
    if (!cols) { free(pairs); return nnz; }
    /* Pairs arrive in (i asc, j asc) order, so appending both directions in
       pair order lists every row's partners in ascending order — the
       reference's push_back order. */
    int64_t* fill = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (size_t p = 0; p < np; p++) { fill[pairs[p].i + 1]++; fill[pairs[p].j + 1]++; }
    for (int i = 0; i < n; i++) fill[i + 1] += fill[i];
    memcpy(row_ptr, fill, sizeof(int64_t) * ((size_t)n + 1));
    for (size_t p = 0; p < np; p++) {
        int64_t a = fill[pairs[p].i]++;
        cols[a] = pairs[p].j; vals[a] = pairs[p].w;
        int64_t b = fill[pairs[p].j]++;
        cols[b] = pairs[p].i; vals[b] = pairs[p].w;
    }
    for (int i = 0; i < n; i++) {
        float sum = 0.0f;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) sum += vals[k];
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) vals[k] /= sum;
    }
    free(fill); free(pairs);
    return nnz;
}

/* Orthonormal basis from a unit normal: Duff, Burgess, Christensen, Hery,
   Kensler, Liani, Villemin, "Building an Orthonormal Basis, Revisited",
   JCGT 6(1), 2017. */
static void onb(v3 n, v3* b1, v3* b2) {
    float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    *b1 = mk3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
    *b2 = mk3(b, sign + n.y * n.y * a, -n.y);
}

/* Cosine-weighted hemisphere direction by Malley's method with disc rejection
   (no trigonometry, so CPU and GPU agree bit for bit). */
static v3 cosine_direction(v3 n, uint64_t seed, uint32_t item, uint32_t sample) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    float x = 0, y = 0;
    for (uint32_t a = 0; a < ORO_MAX_ATTEMPTS; a++) {
        uint32_t ctr[4] = {item, sample, a, TAG_HEMI_FF}, r[4];
        oro_philox4x32_10(ctr, key, r);
        x = u01(r[0]) * 2.0f - 1.0f;
        y = u01(r[1]) * 2.0f - 1.0f;
        if (x * x + y * y <= 1.0f) break;
    }
    float zz = 1.0f - x * x - y * y;
    float z = sqrtf(zz > 0.0f ? zz : 0.0f);
    v3 b1, b2;
    onb(n, &b1, &b2);
    return mk3(b1.x * x + b2.x * y + n.x * z, b1.y * x + b2.y * y + n.y * z, b1.z * x + b2.z * y + n.z * z);
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

long long oro_ff_hemisphere(const oro_ctx* c, int n, const float* pos, const float* nrm, int rays,
                            float max_distance, uint64_t seed, const int32_t* mesh_map, const int32_t* map_dims,
                            const int64_t* map_base, const int32_t* patch_of_texel, int64_t* row_ptr,
                            int32_t* cols, float* vals) {
    int32_t* hits = (int32_t*)malloc(sizeof(int32_t) * (size_t)rays);
    long long nnz = 0;
    for (int i = 0; i < n; i++) {
        v3 p = ld3(pos + 3 * (size_t)i), nn = ld3(nrm + 3 * (size_t)i);
        int nh = 0;
        for (int r = 0; r < rays; r++) {
            v3 dir = cosine_direction(nn, seed, (uint32_t)i, (uint32_t)r);
            trace_result h;
            trace_segment(c, p, add3(p, mul3(dir, max_distance)), HIT_UV, &h);
            if (!h.hit) continue;
            int map = mesh_map[h.mesh];
            if (map < 0) continue;
            rl_lumels tmp;
            tmp.width = map_dims[2 * map]; tmp.height = map_dims[2 * map + 1];
            size_t ti = lumel_at_uv(&tmp, h.uv);
            int32_t pj = patch_of_texel[map_base[map] + (int64_t)ti];
            if (pj < 0) continue;
            hits[nh++] = pj;
        }
        qsort(hits, (size_t)nh, sizeof(int32_t), cmp_i32);
        if (row_ptr) row_ptr[i] = nnz;
        for (int k = 0; k < nh;) {
            int e = k;
            while (e < nh && hits[e] == hits[k]) e++;
            if (cols) { cols[nnz] = hits[k]; vals[nnz] = (float)(e - k) / (float)rays; }
            nnz++;
            k = e;
        }
    }
    if (row_ptr) row_ptr[n] = nnz;
    free(hits);
    return nnz;
}

void oro_jacobi_f64(int n, const int64_t* row_ptr, const int32_t* cols, const float* vals, const float* E,
                    const float* rho, int iters, double* B) {
    double* nb = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    for (int i = 0; i < 3 * n; i++) B[i] = E[i];
    for (int it = 0; it < iters; it++) {
        for (int i = 0; i < n; i++) {
            double s0 = 0, s1 = 0, s2 = 0;
            for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
                double w = vals[k];
                const double* b = B + 3 * (size_t)cols[k];
                s0 += w * b[0]; s1 += w * b[1]; s2 += w * b[2];
            }
            nb[3 * i] = E[3 * i] + rho[3 * i] * s0;
            nb[3 * i + 1] = E[3 * i + 1] + rho[3 * i + 1] * s1;
            nb[3 * i + 2] = E[3 * i + 2] + rho[3 * i + 2] * s2;
        }
        memcpy(B, nb, sizeof(double) * 3 * (size_t)n);
    }
    free(nb);
}

void oro_jacobi_f32(int n, const int64_t* row_ptr, const int32_t* cols, const float* vals, const float* E,
                    const float* rho, int iters, float* B) {
    float* nb = (float*)malloc(sizeof(float) * 3 * (size_t)n);
    for (int i = 0; i < 3 * n; i++) B[i] = E[i];
    for (int it = 0; it < iters; it++) {
        for (int i = 0; i < n; i++) {
            float s0 = 0, s1 = 0, s2 = 0;
            for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
                float w = vals[k];
                const float* b = B + 3 * (size_t)cols[k];
                s0 += w * b[0]; s1 += w * b[1]; s2 += w * b[2];
            }
            nb[3 * i] = E[3 * i] + rho[3 * i] * s0;
            nb[3 * i + 1] = E[3 * i + 1] + rho[3 * i + 1] * s1;
            nb[3 * i + 2] = E[3 * i + 2] + rho[3 * i + 2] * s2;
        }
        memcpy(B, nb, sizeof(float) * 3 * (size_t)n);
    }
    free(nb);
}

/* ------------------------------------------------- FP64 expectations */

static void random_hemisphere_f64(const double n[3], uint64_t seed, uint32_t item, uint32_t sample, uint32_t tag,
                                  double out[3]) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    double x = 0, y = 0, z = 0, len = 0;
    for (uint32_t a = 0; a < ORO_MAX_ATTEMPTS; a++) {
        uint32_t ctr[4] = {item, sample, a, tag}, r[4];
        oro_philox4x32_10(ctr, key, r);
        x = ((double)r[0] + 0.5) * (2.0 / 4294967296.0) - 1.0;
        y = ((double)r[1] + 0.5) * (2.0 / 4294967296.0) - 1.0;
        z = ((double)r[2] + 0.5) * (2.0 / 4294967296.0) - 1.0;
        len = sqrt(x * x + y * y + z * z);
        if (len <= 1.0) break;
    }
    x /= len; y /= len; z /= len;
    if (x * n[0] + y * n[1] + z * n[2] < 0) { x = -x; y = -y; z = -z; }
    out[0] = x; out[1] = y; out[2] = z;
}

void oro_ao_expect_f64(const oro_ctx* c, const rl_lumels* lm, int ntexels, const int32_t* texels, int samples,
                       float occluded_fraction, float max_distance, uint64_t seed, double* out_value) {
    for (int t = 0; t < ntexels; t++) {
        size_t i = (size_t)texels[t];
        double p[3] = {lm->position[3 * i], lm->position[3 * i + 1], lm->position[3 * i + 2]};
        double n[3] = {lm->normal[3 * i], lm->normal[3 * i + 1], lm->normal[3 * i + 2]};
        long occ = 0;
        for (int s = 0; s < samples; s++) {
            double d[3], tt, uu, vv; int g, pr;
            random_hemisphere_f64(n, seed, (uint32_t)i, (uint32_t)s, TAG_AO_F64, d);
            if (ort_intersect_f64(c->bvh, p, d, 0.01, (double)max_distance, &tt, &uu, &vv, &g, &pr)) occ++;
        }
        out_value[t] = 1.0 - (double)occ / ((double)samples * (double)occluded_fraction);
    }
}

void oro_fg_expect_f64(const oro_ctx* c, const rl_lumels* lm, const rl_lumels* photonmaps, int ntexels,
                       const int32_t* texels, int samples, float max_distance, const float sky[3],
                       const float ambient[3], uint64_t seed, double* out_rgb) {
    const rl_scene_desc* d = c->d;
    for (int t = 0; t < ntexels; t++) {
        size_t i = (size_t)texels[t];
        double p[3] = {lm->position[3 * i], lm->position[3 * i + 1], lm->position[3 * i + 2]};
        double n[3] = {lm->normal[3 * i], lm->normal[3 * i + 1], lm->normal[3 * i + 2]};
        double g[3] = {0, 0, 0};
        for (int s = 0; s < samples; s++) {
            double dir[3], tt, uu, vv; int gm, pr;
            random_hemisphere_f64(n, seed, (uint32_t)i, (uint32_t)s, TAG_FG_F64, dir);
            double dp = n[0] * dir[0] + n[1] * dir[1] + n[2] * dir[2];
            double infl = dp > 0 ? dp : 0;
            if (!ort_intersect_f64(c->bvh, p, dir, 0.01, (double)max_distance, &tt, &uu, &vv, &gm, &pr)) {
                for (int k = 0; k < 3; k++) g[k] += sky[k] * infl + ambient[k];
                continue;
            }
            face_t f = face_of(d, gm, pr);
            double hn[3], uv[2];
            for (int k = 0; k < 3; k++) {
                double a = d->nrm[3 * f.a + k], b = d->nrm[3 * f.b + k], cc = d->nrm[3 * f.c + k];
                hn[k] = a + (b - a) * vv + (cc - a) * uu;
            }
            for (int k = 0; k < 2; k++) {
                double a = d->uv1[2 * f.a + k], b = d->uv1[2 * f.b + k], cc = d->uv1[2 * f.c + k];
                uv[k] = a + (b - a) * vv + (cc - a) * uu;
            }
            if (dir[0] * hn[0] + dir[1] * hn[1] + dir[2] * hn[2] >= 0) continue;
            int pm = d->mesh_photonmap ? d->mesh_photonmap[gm] : -1;
            if (pm < 0) continue;
            const rl_lumels* P = &photonmaps[pm];
            float uvf[2] = {(float)uv[0], (float)uv[1]};
            size_t ti = lumel_at_uv(P, uvf);
            for (int k = 0; k < 3; k++) g[k] += P->gathered[3 * ti + k] * infl + ambient[k];
        }
        for (int k = 0; k < 3; k++) out_rgb[3 * t + k] = g[k] / samples;
    }
}
