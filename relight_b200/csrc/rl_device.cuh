// Device-side building blocks of the B200 baker: scene view, vector math in
// the reference's evaluation order, Philox4x32-10, material lookup and BVH
// traversal.
//
// Floating point: this library is compiled with --fmad=false, so an
// expression written `a * b + c` rounds twice exactly as the reference's C++
// does (Types.h vector operators, evaluated left to right).  Fused
// multiply-adds appear only where they are written out as __fmaf_rn(): in
// the BVH slab test (conservative by construction) and in the triangle test,
// whose fixed fmaf sequence defines this tracer's arithmetic.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rl {

// ------------------------------------------------------------------ scene

// BVH node, 64 bytes, both children's boxes in the parent (four float4):
//   n0 = c0.lo.x c0.hi.x c0.lo.y c0.hi.y
//   n1 = c1.lo.x c1.hi.x c1.lo.y c1.hi.y
//   n2 = c0.lo.z c0.hi.z c1.lo.z c1.hi.z
//   n3 = child0, child1 (int bits), 0, 0
// child >= 0: inner node index; child < 0: leaf, ~child = first_tri << 3 | (count - 1).
// Triangles, 48 bytes in leaf order: t0 = v0.xyz | gid bits, t1 = e1.xyz, t2 = e2.xyz.
struct DevScene {
    const float4* nodes;
    const float4* nodes4;       // 4-wide nodes, 128 B: lo.x hi.x lo.y hi.y lo.z hi.z (4 children each), codes, pad
    const float4* tris;
    const int4* tri_vidx;       // per global triangle id: a, b, c, mesh
    const float4* shade;        // per global triangle id: 4 float4, normals + lightmap uv + photonmap slot
    const uint4* nodes8;        // compressed 8-wide nodes, 80 B (rl_bvh.cpp), or null
    const float4* tris8;        // triangle records in 8-wide node order
    const float* pos;
    const float* nrm;
    const float* uv0;
    const float* uv1;
    const int* vmat;
    const int* mesh_first_tri;
    const int* mesh_photonmap;
    const float* mat_rgb;
    const int* mat_tex;
    const int* tex_dims;
    const long long* tex_offset;
    const unsigned char* tex_pixels;
    float bounds_lo[3];
    float bounds_hi[3];
    int ntris;
    int nmeshes;
    int has_alpha;              // some material can have alpha <= 0.1 (RGBA texture)
};

// SoA lumel arrays of one map (Lightmap.h:35-55).
struct DevMap {
    int width, height;
    int* flags;
    int* face;
    int* mesh;  // scene mesh whose faces rasterised the lumel, -1 none
    float* position;
    float* normal;
    float* color;
    int* photons;
    float* gathered;
};

// bake::LumelBakeIterator / FaceBakeIterator (baker/Baker.h:91-155) as a
// predicate over lumels: kind 0 visits lumels first, first + step, ...; kind 1
// visits every lumel rasterised from face first, first + step, ... of `mesh`.
struct Iter {
    int kind, first, step, mesh;
};

// Thread k's lumel i under `it`, and whether it is to be baked.  Kind 2 is
// the whole map in 8x8 lumel tiles (it.first tiles per row): 64 consecutive
// threads cover one tile and a warp an 8x4 half, so a warp's rays start
// close together; threads past the map's edge bake nothing.
__device__ __forceinline__ bool iter_lumel(const DevMap& m, const Iter& it, long long k, long long& i) {
    if (it.kind == 2) {
        const long long tile = k >> 6;
        const int t = (int)(k & 63);
        const int x = (int)(tile % it.first) * 8 + (t & 7), y = (int)(tile / it.first) * 8 + (t >> 3);
        if (x >= m.width || y >= m.height) {
            i = 0;
            return false;
        }
        i = (long long)y * m.width + x;
        return (m.flags[i] & 1) != 0;
    }
    if (it.kind == 0) {
        i = it.first + k * it.step;
        return (m.flags[i] & 1) != 0;
    }
    i = k;
    if (!(m.flags[i] & 1) || m.mesh[i] != it.mesh) return false;
    int f = m.face[i];
    return f >= it.first && (f - it.first) % it.step == 0;
}

constexpr int kHitPoint = 1, kHitUv = 2, kHitColor = 4, kHitNormal = 8, kHitUseAlpha = 16;
constexpr int kStackSize = 64;

// ------------------------------------------------------------------ vectors

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 mk3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(float* p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 mul3(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 neg3(V3 a) { return V3{-a.x, -a.y, -a.z}; }
// Vec3::operator*(Vec3) (Types.h:794-796)
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// Vec3::length / normalize (Types.h:841-859)
__device__ __forceinline__ float len3(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ float normalize3(V3& a) {
    float len = len3(a);
    if (len != 0.0f) {
        a.x = a.x / len; a.y = a.y / len; a.z = a.z / len;
    }
    return len;
}

// ------------------------------------------------------------------ Philox

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Purpose tags (counter word 3) keep the streams of different draws apart.
enum : uint32_t { kTagAO = 1, kTagFG = 2, kTagEmit = 3, kTagEmitPoint = 4, kTagBounce = 5, kTagHemiFF = 6 };
constexpr int kMaxAttempts = 64;

__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

// Vec3::randomDirection (Types.h:924-937): uniform cube rejection, dir / len.
__device__ __forceinline__ V3 random_direction(uint2 key, uint32_t item, uint32_t sample, uint32_t tag) {
    V3 dir = mk3(0.f, 0.f, 0.f);
    float len = 0.0f;
    for (uint32_t a = 0; a < kMaxAttempts; a++) {
        uint4 r = philox(make_uint4(item, sample, a, tag), key);
        dir.x = (u01(r.x) * 2.0f - 1.0f);
        dir.y = (u01(r.y) * 2.0f - 1.0f);
        dir.z = (u01(r.z) * 2.0f - 1.0f);
        len = len3(dir);
        if (!(len > 1.0f)) break;
    }
    return mk3(dir.x / len, dir.y / len, dir.z / len);
}

// Vec3::randomHemisphereDirection (Types.h:940-949).
__device__ __forceinline__ V3 random_hemisphere(V3 n, uint2 key, uint32_t item, uint32_t sample, uint32_t tag) {
    V3 d = random_direction(key, item, sample, tag);
    if (dot3(d, n) < 0.0f) d = neg3(d);
    return d;
}

// ---------------------------------------------------------- face attributes

// Face::normalAt / positionAt (scene/Mesh.cpp:454-475): a + (b-a)*y + (c-a)*x.
__device__ __forceinline__ V3 interp3(const float* arr, int4 f, float bx, float by) {
    V3 a = ld3(arr + 3 * f.x), b = ld3(arr + 3 * f.y), c = ld3(arr + 3 * f.z);
    return mk3(a.x + (b.x - a.x) * by + (c.x - a.x) * bx, a.y + (b.y - a.y) * by + (c.y - a.y) * bx,
               a.z + (b.z - a.z) * by + (c.z - a.z) * bx);
}

// Face::uvAt (scene/Mesh.cpp:488-495).
__device__ __forceinline__ float2 interp2(const float* arr, int4 f, float bx, float by) {
    const float* a = arr + 2 * f.x;
    const float* b = arr + 2 * f.y;
    const float* c = arr + 2 * f.z;
    return make_float2(a[0] + (b[0] - a[0]) * by + (c[0] - a[0]) * bx, a[1] + (b[1] - a[1]) * by + (c[1] - a[1]) * bx);
}

// Face::colorAt -> Material / TexturedMaterial / Texture::colorAt
// (scene/Mesh.cpp:478-485, scene/Material.cpp:41-98).
__device__ __forceinline__ float4 face_color(const DevScene& s, int4 f, float bx, float by) {
    int m = s.vmat[f.x];
    if (m < 0) return make_float4(1.f, 1.f, 1.f, 1.f);
    float4 base = make_float4(s.mat_rgb[3 * m], s.mat_rgb[3 * m + 1], s.mat_rgb[3 * m + 2], 1.0f);
    int tex = s.mat_tex[m];
    if (tex < 0) return base;
    float2 uv = interp2(s.uv0, f, bx, by);
    int w = s.tex_dims[3 * tex], h = s.tex_dims[3 * tex + 1], ch = s.tex_dims[3 * tex + 2];
    int x = ((int)(uv.x * (float)w)) % w;
    int y = ((int)(uv.y * (float)h)) % h;
    float4 t = make_float4(1.f, 0.f, 1.f, 1.f);
    if (x >= 0 && x < w && y >= 0 && y < h) {
        const unsigned char* p = s.tex_pixels + s.tex_offset[tex] + ((long long)y * w * ch + (long long)x * ch);
        t = make_float4(p[0] / 255.0f, p[1] / 255.0f, p[2] / 255.0f, ch == 4 ? p[3] / 255.0f : 1.0f);
    }
    return make_float4(base.x * t.x, base.y * t.y, base.z * t.z, base.w * t.w);
}

// Lightmap::lumel(const Uv&) (Lightmap.cpp:61-67): x = int(u * (W - 1)).
// Out-of-range uvs (undefined behaviour in the reference) are clamped.
__device__ __forceinline__ int lumel_at_uv(int w, int h, float2 uv) {
    int x = (int)(uv.x * (float)(w - 1));
    int y = (int)(uv.y * (float)(h - 1));
    x = x < 0 ? 0 : (x > w - 1 ? w - 1 : x);
    y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
    return y * w + x;
}

// ---------------------------------------------------------------- traversal

// Moeller-Trumbore over v0, e1, e2 with the oracle tracer's exact fmaf
// sequence (hit on the open interval tnear < t < tfar).
__device__ __forceinline__ bool tri_test(float4 t0, float4 t1, float4 t2, V3 o, V3 d, float tnear, float tfar,
                                         float& t_out, float& u_out, float& v_out) {
    float px = __fmaf_rn(d.y, t2.z, -(d.z * t2.y));
    float py = __fmaf_rn(d.z, t2.x, -(d.x * t2.z));
    float pz = __fmaf_rn(d.x, t2.y, -(d.y * t2.x));
    float det = __fmaf_rn(t1.x, px, __fmaf_rn(t1.y, py, t1.z * pz));
    if (det == 0.0f) return false;
    float inv = 1.0f / det;
    float tx = o.x - t0.x, ty = o.y - t0.y, tz = o.z - t0.z;
    float u = __fmaf_rn(tx, px, __fmaf_rn(ty, py, tz * pz)) * inv;
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    float qx = __fmaf_rn(ty, t1.z, -(tz * t1.y));
    float qy = __fmaf_rn(tz, t1.x, -(tx * t1.z));
    float qz = __fmaf_rn(tx, t1.y, -(ty * t1.x));
    float v = __fmaf_rn(d.x, qx, __fmaf_rn(d.y, qy, d.z * qz)) * inv;
    if (!(v >= 0.0f && u + v <= 1.0f)) return false;
    float t = __fmaf_rn(t2.x, qx, __fmaf_rn(t2.y, qy, t2.z * qz)) * inv;
    if (!(t > tnear && t < tfar)) return false;
    t_out = t; u_out = u; v_out = v;
    return true;
}

struct RayHit {
    float t, u, v;
    int gid;  // global triangle id, -1 = miss
};

__device__ __forceinline__ float safe_inv(float d) {
    // keep the slab test finite: |d| below 1e-20 is treated as +-1e-20
    float a = fabsf(d) < 1e-20f ? copysignf(1e-20f, d) : d;
    return 1.0f / a;
}

// Three-input minimum / maximum (one instruction on sm_100).  Min and max
// round nothing, so these equal the two-input cascades exactly (the slab
// operands are never NaN: safe_inv keeps 1/d finite).
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Slab test of both children of a node against [tnear, tmax]; returns the
// entry distances.  Conservative: boxes were padded at build and the exit
// bound is widened by a few ulps.
__device__ __forceinline__ void slab2(float4 n0, float4 n1, float4 n2, V3 idir, V3 ood, float tnear, float tmax,
                                      bool& h0, bool& h1, float& e0, float& e1) {
    float a0 = __fmaf_rn(n0.x, idir.x, -ood.x), a1 = __fmaf_rn(n0.y, idir.x, -ood.x);
    float b0 = __fmaf_rn(n0.z, idir.y, -ood.y), b1 = __fmaf_rn(n0.w, idir.y, -ood.y);
    float c0 = __fmaf_rn(n2.x, idir.z, -ood.z), c1 = __fmaf_rn(n2.y, idir.z, -ood.z);
    float lo0 = fmax3(fminf(a0, a1), fminf(b0, b1), fmaxf(fminf(c0, c1), tnear));
    float hi0 = fmin3(fmaxf(a0, a1), fmaxf(b0, b1), fminf(fmaxf(c0, c1), tmax));
    float d0 = __fmaf_rn(n1.x, idir.x, -ood.x), d1 = __fmaf_rn(n1.y, idir.x, -ood.x);
    float f0 = __fmaf_rn(n1.z, idir.y, -ood.y), f1 = __fmaf_rn(n1.w, idir.y, -ood.y);
    float g0 = __fmaf_rn(n2.z, idir.z, -ood.z), g1 = __fmaf_rn(n2.w, idir.z, -ood.z);
    float lo1 = fmax3(fminf(d0, d1), fminf(f0, f1), fmaxf(fminf(g0, g1), tnear));
    float hi1 = fmin3(fmaxf(d0, d1), fmaxf(f0, f1), fminf(fmaxf(g0, g1), tmax));
    h0 = lo0 <= hi0 * 1.0000003f;
    h1 = lo1 <= hi1 * 1.0000003f;
    e0 = lo0;
    e1 = lo1;
}

// Closest hit (any = false) or first hit (any = true) on (tnear, tfar).
// Ties in t go to the smaller global triangle id, so the answer does not
// depend on the BVH's shape.
template <bool kAny>
__device__ __forceinline__ bool traverse(const DevScene& s, V3 o, V3 d, float tnear, float tfar, RayHit& hit,
                                         int* overflow) {
    hit.gid = -1;
    if (s.ntris == 0) return false;
    V3 idir = mk3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    V3 ood = mk3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
    int stack[kStackSize];
    int sp = 0;
    int node = 0;
    float best = tfar;
    int best_gid = 0x7fffffff;
    for (;;) {
        while (node >= 0) {
            const float4* np = s.nodes + 4 * (size_t)node;
            float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
            bool h0, h1;
            float e0, e1;
            slab2(n0, n1, n2, idir, ood, tnear, best, h0, h1, e0, e1);
            int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                int nearc = c0, farc = c1;
                if (e1 < e0) { nearc = c1; farc = c0; }
                if (sp < kStackSize) stack[sp++] = farc;
                else if (overflow) *overflow = 1;
                node = nearc;
            } else if (h0) {
                node = c0;
            } else if (h1) {
                node = c1;
            } else {
                if (sp == 0) return hit.gid >= 0;
                node = stack[--sp];
            }
        }
        // leaf
        int code = ~node;
        int first = code >> 3, count = (code & 7) + 1;
        for (int i = first; i < first + count; i++) {
            const float4* tp = s.tris + 3 * (size_t)i;
            float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
            float t, u, v;
            if (tri_test(t0, t1, t2, o, d, tnear, tfar, t, u, v)) {
                int gid = __float_as_int(t0.w);
                if (t < best || (t == best && gid < best_gid)) {
                    best = t; best_gid = gid;
                    hit.t = t; hit.u = u; hit.v = v; hit.gid = gid;
                    if (kAny) return true;
                }
            }
        }
        if (sp == 0) return hit.gid >= 0;
        node = stack[--sp];
    }
}

// ------------------------------------------------------------ ray loop

constexpr int kNodeDone = (int)0x80000000;  // never a leaf code: ntris < 2^28

// Persistent per-lane ray loop.  A generator `g` supplies this lane's rays
// one after another (g.next) and consumes each result (g.finish).  A lane
// starts its next ray as soon as its current one terminates, so lanes of a
// warp never wait for each other between rays — only inside one traversal
// step (the inner-node loop, then one leaf).  Results are the same as
// traverse<kAny>() per ray: closest hit with the smaller-id tie-break, or
// first hit.
template <bool kAny, typename Gen>
__device__ __forceinline__ void ray_loop(const DevScene& s, Gen& g, int refill, int* overflow) {
    V3 o = mk3(0.f, 0.f, 0.f), d = o, idir = o, ood = o;
    float tnear = 0.f, tfar = 0.f, best = 0.f;
    int best_gid = 0x7fffffff;
    RayHit hit;
    hit.gid = -1; hit.t = hit.u = hit.v = 0.f;
    int stack[kStackSize];
    int sp = 0;
    int node = kNodeDone;
    bool have = false, exhausted = false;
    const unsigned mask = __activemask();
    for (;;) {
        // Lanes whose ray ended wait until `refill` of the warp's live lanes
        // (or all of them) have ended, then start their next rays together,
        // so ray generation and hit shading run on many lanes at once.
        bool need = node == kNodeDone && !exhausted;
        unsigned alive = __ballot_sync(mask, !exhausted);
        if (alive == 0) break;
        unsigned needm = __ballot_sync(mask, need);
        if (need && (__popc(needm) >= refill || needm == alive)) {
            if (have) {
                g.finish(hit);
                have = false;
            }
            if (g.next(o, d, tnear, tfar)) {
                have = true;
                idir = mk3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
                ood = mk3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
                best = tfar;
                best_gid = 0x7fffffff;
                hit.gid = -1;
                sp = 0;
                node = s.ntris > 0 ? 0 : kNodeDone;
            } else {
                exhausted = true;
            }
        }
        if (node == kNodeDone) continue;
        // inner nodes until a leaf (or the end of the walk)
        while (node >= 0) {
            const float4* np = s.nodes + 4 * (size_t)node;
            float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
            bool h0, h1;
            float e0, e1;
            slab2(n0, n1, n2, idir, ood, tnear, best, h0, h1, e0, e1);
            int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                int nearc = c0, farc = c1;
                if (e1 < e0) { nearc = c1; farc = c0; }
                if (sp < kStackSize) stack[sp++] = farc;
                else if (overflow) *overflow = 1;
                node = nearc;
            } else if (h0) {
                node = c0;
            } else if (h1) {
                node = c1;
            } else {
                node = sp > 0 ? stack[--sp] : kNodeDone;
            }
        }
        if (node == kNodeDone) continue;
        // one leaf
        int code = ~node;
        int first = code >> 3, count = (code & 7) + 1;
        bool stop = false;
        for (int i = first; i < first + count; i++) {
            const float4* tp = s.tris + 3 * (size_t)i;
            float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
            float t, u, v;
            if (tri_test(t0, t1, t2, o, d, tnear, tfar, t, u, v)) {
                int gid = __float_as_int(t0.w);
                if (t < best || (t == best && gid < best_gid)) {
                    best = t; best_gid = gid;
                    hit.t = t; hit.u = u; hit.v = v; hit.gid = gid;
                    if (kAny) { stop = true; break; }
                }
            }
        }
        node = (!stop && sp > 0) ? stack[--sp] : kNodeDone;
    }
}

// ray_loop over a shared list of work items (lumels) instead of one per
// lane: a lane whose item has no rays left takes the next item from its
// warp's pool, and the warp refills the pool from `src` (src.claim(lo, hi):
// called by the whole warp, gives the same [lo, hi) to every lane, false
// when the source is dry).  Lanes therefore keep tracing until the source
// runs dry, instead of idling until the warp's slowest item is done, and a
// persistent grid has no wave tail.  Neighbouring items of a chunk stay in
// one warp (coherent rays).  Each item is still one lane's rays in order,
// so results are those of ray_loop.  The generator adds:
//   has_more()        the current item has rays left
//   end_item()        the current item is done (write its result); no-op
//                     when the lane holds none
//   start_item(k)     take item k; false if k is not to be baked (then the
//                     lane takes another)

// A source of `chunk` consecutive items [0, count) from a global counter.
struct CounterSource {
    unsigned long long* counter;
    long long count;
    int chunk;
    __device__ __forceinline__ bool claim(long long& lo, long long& hi) {
        unsigned long long base = 0;
        if ((threadIdx.x & 31) == 0) base = atomicAdd(counter, (unsigned long long)chunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((long long)base >= count) return false;
        lo = (long long)base;
        hi = lo + chunk < count ? lo + chunk : count;
        return true;
    }
};

template <bool kAny, typename Gen, typename Src>
__device__ __forceinline__ void ray_loop_pool(const DevScene& s, Gen& g, int refill, int* overflow, Src& src) {
    V3 o = mk3(0.f, 0.f, 0.f), d = o, idir = o, ood = o;
    float tnear = 0.f, tfar = 0.f, best = 0.f;
    int best_gid = 0x7fffffff;
    RayHit hit;
    hit.gid = -1; hit.t = hit.u = hit.v = 0.f;
    int stack[kStackSize];
    int sp = 0;
    int node = kNodeDone;
    bool have = false, exhausted = false;
    const unsigned lanes_below = (1u << (threadIdx.x & 31)) - 1u;
    long long pool_next = 0, pool_end = 0;  // warp-uniform: items claimed, not yet handed out
    bool dry = false;                       // warp-uniform: the list is used up
    for (;;) {
        const bool need = node == kNodeDone && !exhausted;
        const unsigned alive = __ballot_sync(0xffffffffu, !exhausted);
        if (alive == 0) break;
        const unsigned needm = __ballot_sync(0xffffffffu, need);
        if (needm && (__popc(needm) >= refill || needm == alive)) {
            if (need && have) {
                g.finish(hit);
                have = false;
            }
            bool want = need && !g.has_more();
            if (want) g.end_item();
            unsigned wm = __ballot_sync(0xffffffffu, want);
            while (wm) {
                if (pool_next >= pool_end) {
                    if (dry) break;
                    if (!src.claim(pool_next, pool_end)) {
                        dry = true;
                        break;
                    }
                }
                const long long item = pool_next + __popc(wm & lanes_below);
                if (want && item < pool_end && g.start_item(item)) want = false;
                const long long handed = __popc(wm);
                pool_next = pool_end - pool_next < handed ? pool_end : pool_next + handed;
                wm = __ballot_sync(0xffffffffu, want);
            }
            if (want) exhausted = true;
            if (need && !exhausted) {
                g.next(o, d, tnear, tfar);
                have = true;
                idir = mk3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
                ood = mk3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
                best = tfar;
                best_gid = 0x7fffffff;
                hit.gid = -1;
                sp = 0;
                node = s.ntris > 0 ? 0 : kNodeDone;
            }
        }
        if (node == kNodeDone) continue;
        // inner nodes until a leaf (or the end of the walk)
        while (node >= 0) {
            const float4* np = s.nodes + 4 * (size_t)node;
            float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
            bool h0, h1;
            float e0, e1;
            slab2(n0, n1, n2, idir, ood, tnear, best, h0, h1, e0, e1);
            int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                int nearc = c0, farc = c1;
                if (e1 < e0) { nearc = c1; farc = c0; }
                if (sp < kStackSize) stack[sp++] = farc;
                else if (overflow) *overflow = 1;
                node = nearc;
            } else if (h0) {
                node = c0;
            } else if (h1) {
                node = c1;
            } else {
                node = sp > 0 ? stack[--sp] : kNodeDone;
            }
        }
        if (node == kNodeDone) continue;
        // one leaf
        int code = ~node;
        int first = code >> 3, count_tris = (code & 7) + 1;
        bool stop = false;
        for (int i = first; i < first + count_tris; i++) {
            const float4* tp = s.tris + 3 * (size_t)i;
            float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
            float t, u, v;
            if (tri_test(t0, t1, t2, o, d, tnear, tfar, t, u, v)) {
                int gid = __float_as_int(t0.w);
                if (t < best || (t == best && gid < best_gid)) {
                    best = t; best_gid = gid;
                    hit.t = t; hit.u = u; hit.v = v; hit.gid = gid;
                    if (kAny) { stop = true; break; }
                }
            }
        }
        node = (!stop && sp > 0) ? stack[--sp] : kNodeDone;
    }
}

template <bool kAny, typename Gen>
__device__ __forceinline__ void ray_loop_spec(const DevScene& s, Gen& g, int refill, int* overflow) {
    V3 o = mk3(0.f, 0.f, 0.f), d = o, idir = o, ood = o;
    float tnear = 0.f, tfar = 0.f, best = 0.f;
    int best_gid = 0x7fffffff;
    RayHit hit;
    hit.gid = -1; hit.t = hit.u = hit.v = 0.f;
    int stack[kStackSize];
    int sp = 0;
    int node = kNodeDone;
    bool have = false, exhausted = false;
    const unsigned mask = __activemask();
    for (;;) {
        // Lanes whose ray ended wait until `refill` of the warp's live lanes
        // (or all of them) have ended, then start their next rays together,
        // so ray generation and hit shading run on many lanes at once.
        bool need = node == kNodeDone && !exhausted;
        unsigned alive = __ballot_sync(mask, !exhausted);
        if (alive == 0) break;
        unsigned needm = __ballot_sync(mask, need);
        if (need && (__popc(needm) >= refill || needm == alive)) {
            if (have) {
                g.finish(hit);
                have = false;
            }
            if (g.next(o, d, tnear, tfar)) {
                have = true;
                idir = mk3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
                ood = mk3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
                best = tfar;
                best_gid = 0x7fffffff;
                hit.gid = -1;
                sp = 0;
                node = s.ntris > 0 ? 0 : kNodeDone;
            } else {
                exhausted = true;
            }
        }
        if (node == kNodeDone) continue;
        // Inner nodes with speculative leaf postponing (Aila & Laine, "Understanding
        // the efficiency of ray traversal on GPUs", HPG 2009): a lane that reaches
        // a leaf parks it and keeps descending until every lane of the warp has a
        // leaf, then all lanes test their leaves together.
        int leaf = 0;  // 0: none parked; otherwise a leaf code
        while (node >= 0) {
            const float4* np = s.nodes + 4 * (size_t)node;
            float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
            bool h0, h1;
            float e0, e1;
            slab2(n0, n1, n2, idir, ood, tnear, best, h0, h1, e0, e1);
            int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            if (h0 && h1) {
                int nearc = c0, farc = c1;
                if (e1 < e0) { nearc = c1; farc = c0; }
                if (sp < kStackSize) stack[sp++] = farc;
                else if (overflow) *overflow = 1;
                node = nearc;
            } else if (h0) {
                node = c0;
            } else if (h1) {
                node = c1;
            } else {
                node = sp > 0 ? stack[--sp] : kNodeDone;
            }
            if (node < 0 && node != kNodeDone && leaf == 0) {
                leaf = node;
                node = sp > 0 ? stack[--sp] : kNodeDone;
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;
        }
        // the parked leaf, then a leaf met right after it
        bool stop = false;
        while (leaf != 0) {
            int code = ~leaf;
            int first = code >> 3, count = (code & 7) + 1;
            for (int i = first; i < first + count; i++) {
                const float4* tp = s.tris + 3 * (size_t)i;
                float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
                float t, u, v;
                if (tri_test(t0, t1, t2, o, d, tnear, tfar, t, u, v)) {
                    int gid = __float_as_int(t0.w);
                    if (t < best || (t == best && gid < best_gid)) {
                        best = t; best_gid = gid;
                        hit.t = t; hit.u = u; hit.v = v; hit.gid = gid;
                        if (kAny) { stop = true; break; }
                    }
                }
            }
            if (stop) break;
            if (node < 0 && node != kNodeDone) {
                leaf = node;
                node = sp > 0 ? stack[--sp] : kNodeDone;
            } else {
                leaf = 0;
            }
        }
        if (stop) node = kNodeDone;
    }
}

// Entry distance of one child of a 4-wide node, or kMissKey when the ray
// misses its box (or the slot is empty).  Same conservative slab test as slab2.
constexpr float kMissKey = 3.0e38f;

__device__ __forceinline__ float child_entry(float lx, float hx, float ly, float hy, float lz, float hz, V3 idir,
                                             V3 ood, float tnear, float tmax, int code) {
    float a0 = __fmaf_rn(lx, idir.x, -ood.x), a1 = __fmaf_rn(hx, idir.x, -ood.x);
    float b0 = __fmaf_rn(ly, idir.y, -ood.y), b1 = __fmaf_rn(hy, idir.y, -ood.y);
    float c0 = __fmaf_rn(lz, idir.z, -ood.z), c1 = __fmaf_rn(hz, idir.z, -ood.z);
    float lo = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), tnear));
    float hi = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), tmax));
    return (lo <= hi * 1.0000003f && code != kNodeDone) ? lo : kMissKey;
}

__device__ __forceinline__ void cswap(float& ka, int& ca, float& kb, int& cb) {
    bool sw = kb < ka;
    float tk = sw ? kb : ka;
    int tc = sw ? cb : ca;
    kb = sw ? ka : kb;
    cb = sw ? ca : cb;
    ka = tk;
    ca = tc;
}

template <bool kAny, typename Gen>
__device__ __forceinline__ void ray_loop4(const DevScene& s, Gen& g, int refill, int* overflow) {
    V3 o = mk3(0.f, 0.f, 0.f), d = o, idir = o, ood = o;
    float tnear = 0.f, tfar = 0.f, best = 0.f;
    int best_gid = 0x7fffffff;
    RayHit hit;
    hit.gid = -1; hit.t = hit.u = hit.v = 0.f;
    int stack[kStackSize];
    int sp = 0;
    int node = kNodeDone;
    bool have = false, exhausted = false;
    const unsigned mask = __activemask();
    for (;;) {
        // Lanes whose ray ended wait until `refill` of the warp's live lanes
        // (or all of them) have ended, then start their next rays together,
        // so ray generation and hit shading run on many lanes at once.
        bool need = node == kNodeDone && !exhausted;
        unsigned alive = __ballot_sync(mask, !exhausted);
        if (alive == 0) break;
        unsigned needm = __ballot_sync(mask, need);
        if (need && (__popc(needm) >= refill || needm == alive)) {
            if (have) {
                g.finish(hit);
                have = false;
            }
            if (g.next(o, d, tnear, tfar)) {
                have = true;
                idir = mk3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
                ood = mk3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
                best = tfar;
                best_gid = 0x7fffffff;
                hit.gid = -1;
                sp = 0;
                node = s.ntris > 0 ? 0 : kNodeDone;
            } else {
                exhausted = true;
            }
        }
        if (node == kNodeDone) continue;
        // 4-wide inner nodes until a leaf (or the end of the walk)
        while (node >= 0) {
            const float4* np = s.nodes4 + 8 * (size_t)node;
            float4 lx = __ldg(np), hx = __ldg(np + 1), ly = __ldg(np + 2), hy = __ldg(np + 3);
            float4 lz = __ldg(np + 4), hz = __ldg(np + 5);
            int4 cc = __ldg(reinterpret_cast<const int4*>(np + 6));
            float k0 = child_entry(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, idir, ood, tnear, best, cc.x);
            float k1 = child_entry(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, idir, ood, tnear, best, cc.y);
            float k2 = child_entry(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, idir, ood, tnear, best, cc.z);
            float k3 = child_entry(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, idir, ood, tnear, best, cc.w);
            int c0 = cc.x, c1 = cc.y, c2 = cc.z, c3 = cc.w;
            // sort (entry, child) ascending: 5 compare-exchanges
            cswap(k0, c0, k1, c1);
            cswap(k2, c2, k3, c3);
            cswap(k0, c0, k2, c2);
            cswap(k1, c1, k3, c3);
            cswap(k1, c1, k2, c2);
            int nh = (k0 < kMissKey) + (k1 < kMissKey) + (k2 < kMissKey) + (k3 < kMissKey);
            if (nh == 0) {
                node = sp > 0 ? stack[--sp] : kNodeDone;
                continue;
            }
            if (sp + nh - 1 > kStackSize) {
                if (overflow) *overflow = 1;
                nh = 1 + (kStackSize - sp > 0 ? kStackSize - sp : 0);
                if (nh > 4) nh = 4;
            }
            if (nh > 3) stack[sp++] = c3;
            if (nh > 2) stack[sp++] = c2;
            if (nh > 1) stack[sp++] = c1;
            node = c0;
        }
        if (node == kNodeDone) continue;
        // one leaf
        int code = ~node;
        int first = code >> 3, count = (code & 7) + 1;
        bool stop = false;
        for (int i = first; i < first + count; i++) {
            const float4* tp = s.tris + 3 * (size_t)i;
            float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
            float t, u, v;
            if (tri_test(t0, t1, t2, o, d, tnear, tfar, t, u, v)) {
                int gid = __float_as_int(t0.w);
                if (t < best || (t == best && gid < best_gid)) {
                    best = t; best_gid = gid;
                    hit.t = t; hit.u = u; hit.v = v; hit.gid = gid;
                    if (kAny) { stop = true; break; }
                }
            }
        }
        node = (!stop && sp > 0) ? stack[--sp] : kNodeDone;
    }
}

// Ray setup of rt::Embree::initializeRay (rt/Embree.cpp:107-130) for the
// segment start -> start + dir * length.
__device__ __forceinline__ void segment_ray(V3 start, V3 dir, float length, V3& o, V3& d, float& tnear,
                                            float& tfar) {
    V3 end = add3(start, mul3(dir, length));
    d = sub3(end, start);
    tfar = normalize3(d);
    o = start;
    tnear = 0.01f;
}

// Result of the reference's traceSegment post-processing.
struct SegHit {
    bool hit;
    V3 point;
    V3 normal;
    float4 rgba;
    float2 uv;
    int mesh, face;
    float t, u, v;
};

// rt::Embree::traceSegment + initializeRay (rt/Embree.cpp:107-177).
__device__ __forceinline__ void trace_segment(const DevScene& s, V3 start, V3 end, int flags, SegHit& r,
                                              int* overflow) {
    r.hit = false;
    for (int step = 0;; step++) {
        V3 dir = sub3(end, start);
        float len = normalize3(dir);
        RayHit h;
        if (!traverse<false>(s, start, dir, 0.01f, len, h, overflow)) return;
        V3 point = add3(start, mul3(dir, h.t));
        int4 f = __ldg(s.tri_vidx + h.gid);
        float4 rgba = make_float4(1.f, 1.f, 1.f, 1.f);
        if ((flags & (kHitColor | kHitUseAlpha)) != 0) rgba = face_color(s, f, h.u, h.v);
        if ((flags & kHitUseAlpha) && rgba.w <= 0.1f && step < 25) {
            start = add3(point, dir);
            continue;
        }
        r.hit = true;
        r.point = point;
        r.mesh = f.w;
        r.face = h.gid - s.mesh_first_tri[f.w];
        r.t = h.t; r.u = h.u; r.v = h.v;
        if (flags & kHitNormal) r.normal = interp3(s.nrm, f, h.u, h.v);
        if (flags & kHitColor) r.rgba = rgba;
        if (flags & kHitUv) r.uv = interp2(s.uv1, f, h.u, h.v);
        return;
    }
}

// Hit / miss of a segment as the reference sees it (traceSegment's bool).
// Without alpha in play a first-hit walk gives the same answer.
__device__ __forceinline__ bool segment_blocked(const DevScene& s, V3 start, V3 end, int flags, int* overflow) {
    if (!(flags & kHitUseAlpha) || !s.has_alpha) {
        V3 dir = sub3(end, start);
        float len = normalize3(dir);
        RayHit h;
        return traverse<true>(s, start, dir, 0.01f, len, h, overflow);
    }
    SegHit r;
    trace_segment(s, start, end, flags, r, overflow);
    return r.hit;
}


// ----------------------------------------------------- compressed 8-wide walk

constexpr int kStack8 = 32;

__device__ __forceinline__ float qbyte(uint32_t lo4, uint32_t hi4, int c) {
    return (float)(((c < 4 ? lo4 : hi4) >> ((c & 3) * 8)) & 0xffu);
}

// One compressed 8-wide node (rl_bvh.cpp): decode the eight child boxes
// (p + q * 2^e, exact product, one rounding: the builder's decode) and run
// slab2's conservative test on each.  Returns the internal children hit as
// key bits (bit slot ^ oct) and the triangle slots of the leaf children hit.
__device__ __forceinline__ void visit8(const DevScene& s, int node, V3 idir, V3 ood, float tnear, float tmax,
                                       uint32_t oct, uint32_t& child_base, uint32_t& keys, uint32_t& imask,
                                       uint32_t& tri_base, uint32_t& tmask) {
    const uint4* np = s.nodes8 + 5 * (size_t)node;
    const uint4 q0 = __ldg(np), q1 = __ldg(np + 1), q2 = __ldg(np + 2), q3 = __ldg(np + 3), q4 = __ldg(np + 4);
    const float px = __uint_as_float(q0.x), py = __uint_as_float(q0.y), pz = __uint_as_float(q0.z);
    const float sx = __uint_as_float((q0.w & 0xffu) << 23), sy = __uint_as_float(((q0.w >> 8) & 0xffu) << 23),
                sz = __uint_as_float(((q0.w >> 16) & 0xffu) << 23);
    imask = q0.w >> 24;
    child_base = q1.x;
    tri_base = q1.y;
    uint32_t k = 0, t = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const uint32_t meta = ((c < 4 ? q1.z : q1.w) >> ((c & 3) * 8)) & 0xffu;
        const bool inner = (imask >> c) & 1u;
        if (!inner && meta == 0u) continue;
        const float lx = __fmaf_rn(qbyte(q2.x, q2.y, c), sx, px), hx = __fmaf_rn(qbyte(q3.z, q3.w, c), sx, px);
        const float ly = __fmaf_rn(qbyte(q2.z, q2.w, c), sy, py), hy = __fmaf_rn(qbyte(q4.x, q4.y, c), sy, py);
        const float lz = __fmaf_rn(qbyte(q3.x, q3.y, c), sz, pz), hz = __fmaf_rn(qbyte(q4.z, q4.w, c), sz, pz);
        const float a0 = __fmaf_rn(lx, idir.x, -ood.x), a1 = __fmaf_rn(hx, idir.x, -ood.x);
        const float b0 = __fmaf_rn(ly, idir.y, -ood.y), b1 = __fmaf_rn(hy, idir.y, -ood.y);
        const float c0 = __fmaf_rn(lz, idir.z, -ood.z), c1 = __fmaf_rn(hz, idir.z, -ood.z);
        const float lo = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fmaxf(fminf(c0, c1), tnear));
        const float hi = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fminf(fmaxf(c0, c1), tmax));
        if (!(lo <= hi * 1.0000003f)) continue;
        if (inner) k |= 1u << (c ^ oct);
        else t |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
    }
    keys = k;
    tmask = t;
}

// ray_loop over the compressed 8-wide tree: node groups (a node's internal
// children hit, as key bits, with its child base) on the stack instead of
// single nodes, and the triangles of the leaf children hit tested in the
// following step (Ylitie, Karras & Laine, "Efficient incoherent ray traversal
// on GPUs through compressed wide BVHs", HPG 2017).  Same warp refill and
// same closest-hit / tie-break rule as ray_loop, so the hits are identical.
// On the terrain final gather it measured 2.3x slower than the binary walk
// (116 vs 51 ms): each visit decodes and tests eight boxes and the octant
// order culls less than ray_loop's distance order, so it is opt-in.
template <bool kAny, typename Gen>
__device__ __forceinline__ void ray_loop8(const DevScene& s, Gen& g, int refill, int* overflow) {
    V3 o = mk3(0.f, 0.f, 0.f), d = o, idir = o, ood = o;
    float tnear = 0.f, tfar = 0.f, best = 0.f;
    int best_gid = 0x7fffffff;
    RayHit hit;
    hit.gid = -1; hit.t = hit.u = hit.v = 0.f;
    uint2 stack[kStack8];
    int sp = 0;
    uint32_t gbase = 0, gkeys = 0, gimask = 0;  // current node group
    uint32_t tbase = 0, tmask = 0;              // current triangle group
    uint32_t oct = 0;
    bool root = false, walking = false, have = false, exhausted = false;
    const unsigned mask = __activemask();
    for (;;) {
        bool need = !walking && !exhausted;
        unsigned alive = __ballot_sync(mask, !exhausted);
        if (alive == 0) break;
        unsigned needm = __ballot_sync(mask, need);
        if (need && (__popc(needm) >= refill || needm == alive)) {
            if (have) {
                g.finish(hit);
                have = false;
            }
            if (g.next(o, d, tnear, tfar)) {
                have = true;
                idir = mk3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
                ood = mk3(o.x * idir.x, o.y * idir.y, o.z * idir.z);
                oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
                best = tfar;
                best_gid = 0x7fffffff;
                hit.gid = -1;
                sp = 0;
                gkeys = 0;
                tmask = 0;
                root = s.ntris > 0;
                walking = root;
            } else {
                exhausted = true;
            }
        }
        if (!walking) continue;
        // nodes until there are triangles to test (or the walk ends)
        while (tmask == 0u) {
            int node;
            if (root) {
                node = 0;
                root = false;
            } else if (gkeys) {
                const uint32_t key = __ffs(gkeys) - 1;
                gkeys &= gkeys - 1u;
                const uint32_t slot = key ^ oct;
                node = (int)(gbase + __popc(gimask & ((1u << slot) - 1u)));
            } else if (sp > 0) {
                const uint2 e = stack[--sp];
                gbase = e.x;
                gkeys = e.y & 0xffu;
                gimask = e.y >> 8;
                continue;
            } else {
                walking = false;
                break;
            }
            uint32_t cb, keys, im, tb, tm;
            visit8(s, node, idir, ood, tnear, best, oct, cb, keys, im, tb, tm);
            if (keys) {
                if (gkeys) {
                    if (sp < kStack8) stack[sp++] = make_uint2(gbase, gkeys | (gimask << 8));
                    else if (overflow) *overflow = 1;
                }
                gbase = cb;
                gkeys = keys;
                gimask = im;
            }
            if (tm) {
                tbase = tb;
                tmask = tm;
            }
        }
        if (!walking) continue;
        // every triangle of the group
        while (tmask) {
        const int i = (int)(tbase + __ffs(tmask) - 1);
        tmask &= tmask - 1u;
        const float4* tp = s.tris8 + 3 * (size_t)i;
        float4 t0 = __ldg(tp), t1 = __ldg(tp + 1), t2 = __ldg(tp + 2);
        float t, u, v;
        if (tri_test(t0, t1, t2, o, d, tnear, tfar, t, u, v)) {
            int gid = __float_as_int(t0.w);
            if (t < best || (t == best && gid < best_gid)) {
                best = t; best_gid = gid;
                hit.t = t; hit.u = u; hit.v = v; hit.gid = gid;
                if (kAny) {
                    walking = false;
                    tmask = 0;
                }
            }
        }
        }
    }
}

}  // namespace rl
