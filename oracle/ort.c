/*
 * ort — the oracle's CPU ray tracer (binned-SAH binary BVH + Moeller-Trumbore).
 * TEST INFRASTRUCTURE ONLY (see ort.h).  Compile with -ffp-contract=off.
 *
 * It stands in for Intel Embree 2's rtcCommit/rtcIntersect/rtcOccluded, which
 * the reference calls at rt/Embree.cpp:57,151,139.  The BVH here is the
 * "canonical binary SAH BVH" whose box/triangle test counts feed the per-ray
 * byte model of the benchmark's roofline.
 */
#include "ort.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    float lo[3], hi[3];
    int   left;   /* inner: first child index; leaf: first triangle slot */
    int   count;  /* 0 for inner nodes (children are left, left+1)       */
} ort_node;

typedef struct {
    float v0[3], e1[3], e2[3];
    int   geom, prim, gid;
} ort_tri;

struct ort_scene {
    /* staged meshes */
    float* pos;     /* 3 floats per vertex, all meshes */
    int    npos, cap_pos;
    int*   idx;     /* 3 global vertex ids per triangle */
    int*   tgeom;
    int*   tprim;
    int    ntri, cap_tri;
    int    nmesh;
    /* built */
    ort_tri*  tris;     /* in leaf order */
    double*   tri64;    /* 9 doubles per tri: p0, p1, p2 in leaf order */
    ort_node* nodes;
    int       nnodes;
};

ort_scene* ort_create(void) {
    ort_scene* s = (ort_scene*)calloc(1, sizeof(ort_scene));
    return s;
}

void ort_destroy(ort_scene* s) {
    if (!s) return;
    free(s->pos); free(s->idx); free(s->tgeom); free(s->tprim);
    free(s->tris); free(s->tri64); free(s->nodes);
    free(s);
}

int ort_triangle_count(const ort_scene* s) { return s->ntri; }

int ort_add_mesh(ort_scene* s, const float* verts, int vstride, int nverts, const int* tris, int ntris) {
    int base = s->npos;
    if (nverts < 0 || ntris < 0) return -1;
    if (s->npos + nverts > s->cap_pos) {
        size_t cap = ((size_t)s->npos + (size_t)nverts) * 2 + 16;
        s->pos = (float*)realloc(s->pos, sizeof(float) * 3 * cap);
        s->cap_pos = (int)cap;
    }
    for (int i = 0; i < nverts; i++) {
        s->pos[3 * (base + i) + 0] = verts[(size_t)i * vstride + 0];
        s->pos[3 * (base + i) + 1] = verts[(size_t)i * vstride + 1];
        s->pos[3 * (base + i) + 2] = verts[(size_t)i * vstride + 2];
    }
    s->npos += nverts;
    if (s->ntri + ntris > s->cap_tri) {
        size_t cap = ((size_t)s->ntri + (size_t)ntris) * 2 + 16;
        s->idx = (int*)realloc(s->idx, sizeof(int) * 3 * cap);
        s->tgeom = (int*)realloc(s->tgeom, sizeof(int) * cap);
        s->tprim = (int*)realloc(s->tprim, sizeof(int) * cap);
        s->cap_tri = (int)cap;
    }
    for (int t = 0; t < ntris; t++) {
        for (int k = 0; k < 3; k++) s->idx[3 * (s->ntri + t) + k] = base + tris[3 * t + k];
        s->tgeom[s->ntri + t] = s->nmesh;
        s->tprim[s->ntri + t] = t;
    }
    s->ntri += ntris;
    return s->nmesh++;
}

/* ------------------------------------------------------------------ build */

typedef struct { float lo[3], hi[3]; } box3;

static void box_empty(box3* b) {
    for (int k = 0; k < 3; k++) { b->lo[k] = FLT_MAX; b->hi[k] = -FLT_MAX; }
}
static void box_grow_pt(box3* b, const float* p) {
    for (int k = 0; k < 3; k++) {
        if (p[k] < b->lo[k]) b->lo[k] = p[k];
        if (p[k] > b->hi[k]) b->hi[k] = p[k];
    }
}
static void box_grow(box3* b, const box3* o) {
    for (int k = 0; k < 3; k++) {
        if (o->lo[k] < b->lo[k]) b->lo[k] = o->lo[k];
        if (o->hi[k] > b->hi[k]) b->hi[k] = o->hi[k];
    }
}
static float box_area(const box3* b) {
    float dx = b->hi[0] - b->lo[0], dy = b->hi[1] - b->lo[1], dz = b->hi[2] - b->lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

typedef struct {
    box3*  tbox;   /* per triangle */
    float* cent;   /* 3 per triangle */
    int*   order;  /* triangle permutation */
    ort_node* nodes;
    int nnodes, cap;
} builder;

#define ORT_BINS 32
#define ORT_MAX_LEAF 4

static int new_node(builder* b) {
    if (b->nnodes == b->cap) {
        b->cap = b->cap * 2 + 64;
        b->nodes = (ort_node*)realloc(b->nodes, sizeof(ort_node) * (size_t)b->cap);
    }
    return b->nnodes++;
}

static void build_rec(builder* b, int ni, int first, int count) {
    box3 nb, cb;
    box_empty(&nb); box_empty(&cb);
    for (int i = first; i < first + count; i++) {
        int t = b->order[i];
        box_grow(&nb, &b->tbox[t]);
        box_grow_pt(&cb, &b->cent[3 * t]);
    }
    for (int k = 0; k < 3; k++) { b->nodes[ni].lo[k] = nb.lo[k]; b->nodes[ni].hi[k] = nb.hi[k]; }
    if (count <= 2) {
        b->nodes[ni].left = first; b->nodes[ni].count = count;
        return;
    }
    /* binned SAH over all three axes */
    float best_cost = FLT_MAX; int best_axis = -1, best_split = -1;
    for (int axis = 0; axis < 3; axis++) {
        float ext = cb.hi[axis] - cb.lo[axis];
        if (!(ext > 0.0f)) continue;
        box3 bb[ORT_BINS]; int bc[ORT_BINS];
        for (int i = 0; i < ORT_BINS; i++) { box_empty(&bb[i]); bc[i] = 0; }
        float scale = (float)ORT_BINS / ext;
        for (int i = first; i < first + count; i++) {
            int t = b->order[i];
            int bi = (int)((b->cent[3 * t + axis] - cb.lo[axis]) * scale);
            if (bi >= ORT_BINS) bi = ORT_BINS - 1;
            if (bi < 0) bi = 0;
            bc[bi]++; box_grow(&bb[bi], &b->tbox[t]);
        }
        float larea[ORT_BINS]; int lcnt[ORT_BINS];
        box3 acc; box_empty(&acc); int n = 0;
        for (int i = 0; i < ORT_BINS - 1; i++) {
            box_grow(&acc, &bb[i]); n += bc[i];
            larea[i] = box_area(&acc); lcnt[i] = n;
        }
        box_empty(&acc); n = 0;
        for (int i = ORT_BINS - 1; i > 0; i--) {
            box_grow(&acc, &bb[i]); n += bc[i];
            if (lcnt[i - 1] == 0 || n == 0) continue;
            float cost = larea[i - 1] * (float)lcnt[i - 1] + box_area(&acc) * (float)n;
            if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = i; }
        }
    }
    float leaf_cost = box_area(&nb) * (float)count;
    int mid;
    if (best_axis < 0) {
        if (count <= ORT_MAX_LEAF) { b->nodes[ni].left = first; b->nodes[ni].count = count; return; }
        mid = first + count / 2;  /* all centroids coincide: split by index */
    } else {
        if (count <= ORT_MAX_LEAF && best_cost >= leaf_cost) {
            b->nodes[ni].left = first; b->nodes[ni].count = count; return;
        }
        float ext = cb.hi[best_axis] - cb.lo[best_axis];
        float scale = (float)ORT_BINS / ext;
        int i = first, j = first + count - 1;
        while (i <= j) {
            int t = b->order[i];
            int bi = (int)((b->cent[3 * t + best_axis] - cb.lo[best_axis]) * scale);
            if (bi >= ORT_BINS) bi = ORT_BINS - 1;
            if (bi < best_split) i++;
            else { int tmp = b->order[i]; b->order[i] = b->order[j]; b->order[j] = tmp; j--; }
        }
        mid = i;
        if (mid == first || mid == first + count) mid = first + count / 2;
    }
    int l = new_node(b);
    int r = new_node(b);
    (void)r;
    b->nodes[ni].left = l; b->nodes[ni].count = 0;
    build_rec(b, l, first, mid - first);
    build_rec(b, l + 1, mid, first + count - mid);
}

void ort_commit(ort_scene* s) {
    int n = s->ntri > 0 ? s->ntri : 0;
    builder b;
    memset(&b, 0, sizeof(b));
    b.tbox = (box3*)malloc(sizeof(box3) * (size_t)(n > 0 ? n : 1));
    b.cent = (float*)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
    b.order = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int t = 0; t < n; t++) {
        box3* bx = &b.tbox[t];
        box_empty(bx);
        for (int k = 0; k < 3; k++) box_grow_pt(bx, &s->pos[3 * s->idx[3 * t + k]]);
        /* Pad outward so that a Moeller-Trumbore hit whose computed t carries
           rounding error still lies inside every ancestor box. */
        for (int k = 0; k < 3; k++) {
            float m = fmaxf(fabsf(bx->lo[k]), fabsf(bx->hi[k]));
            float pad = 1e-5f * (m > 1.0f ? m : 1.0f);
            bx->lo[k] -= pad; bx->hi[k] += pad;
        }
        for (int k = 0; k < 3; k++) b.cent[3 * t + k] = 0.5f * (bx->lo[k] + bx->hi[k]);
        b.order[t] = t;
    }
    free(s->nodes); free(s->tris); free(s->tri64);
    int root = new_node(&b);
    if (n > 0) build_rec(&b, root, 0, n);
    else { box3 e; box_empty(&e); memcpy(b.nodes[0].lo, e.lo, sizeof e.lo); memcpy(b.nodes[0].hi, e.hi, sizeof e.hi); b.nodes[0].left = 0; b.nodes[0].count = 0; }
    s->nodes = b.nodes; s->nnodes = b.nnodes;
    s->tris = (ort_tri*)malloc(sizeof(ort_tri) * (size_t)(n > 0 ? n : 1));
    s->tri64 = (double*)malloc(sizeof(double) * 9 * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) {
        int t = b.order[i];
        const float* p0 = &s->pos[3 * s->idx[3 * t + 0]];
        const float* p1 = &s->pos[3 * s->idx[3 * t + 1]];
        const float* p2 = &s->pos[3 * s->idx[3 * t + 2]];
        ort_tri* tr = &s->tris[i];
        for (int k = 0; k < 3; k++) {
            tr->v0[k] = p0[k];
            tr->e1[k] = p1[k] - p0[k];
            tr->e2[k] = p2[k] - p0[k];
            s->tri64[9 * i + k] = p0[k];
            s->tri64[9 * i + 3 + k] = p1[k];
            s->tri64[9 * i + 6 + k] = p2[k];
        }
        tr->geom = s->tgeom[t]; tr->prim = s->tprim[t]; tr->gid = t;
    }
    free(b.tbox); free(b.cent); free(b.order);
}

/* -------------------------------------------------------------- traversal */

int ort_triangle_test(const float v0[3], const float e1[3], const float e2[3],
                      const float o[3], const float d[3], float tnear, float tfar,
                      float* t_out, float* u_out, float* v_out) {
    /* pvec = d x e2 */
    float px = fmaf(d[1], e2[2], -(d[2] * e2[1]));
    float py = fmaf(d[2], e2[0], -(d[0] * e2[2]));
    float pz = fmaf(d[0], e2[1], -(d[1] * e2[0]));
    float det = fmaf(e1[0], px, fmaf(e1[1], py, e1[2] * pz));
    if (det == 0.0f) return 0;
    float inv = 1.0f / det;
    float tx = o[0] - v0[0], ty = o[1] - v0[1], tz = o[2] - v0[2];
    float u = fmaf(tx, px, fmaf(ty, py, tz * pz)) * inv;
    if (!(u >= 0.0f && u <= 1.0f)) return 0;
    /* qvec = tvec x e1 */
    float qx = fmaf(ty, e1[2], -(tz * e1[1]));
    float qy = fmaf(tz, e1[0], -(tx * e1[2]));
    float qz = fmaf(tx, e1[1], -(ty * e1[0]));
    float v = fmaf(d[0], qx, fmaf(d[1], qy, d[2] * qz)) * inv;
    if (!(v >= 0.0f && u + v <= 1.0f)) return 0;
    float t = fmaf(e2[0], qx, fmaf(e2[1], qy, e2[2] * qz)) * inv;
    if (!(t > tnear && t < tfar)) return 0;
    *t_out = t; *u_out = u; *v_out = v;
    return 1;
}

static inline int slab(const ort_node* n, const float o[3], const float id[3], float tnear, float tfar, float* tentry) {
    float tmin = tnear, tmax = tfar;
    for (int k = 0; k < 3; k++) {
        float a = (n->lo[k] - o[k]) * id[k];
        float b = (n->hi[k] - o[k]) * id[k];
        float lo = fminf(a, b), hi = fmaxf(a, b);
        tmin = fmaxf(tmin, lo);
        tmax = fminf(tmax, hi);
    }
    *tentry = tmin;
    return tmin <= tmax * 1.0000002f;
}

#define ORT_STACK 128

static int traverse(const ort_scene* s, const float o[3], const float d[3], float tnear, float tfar,
                    int any, ort_hit* best, ort_stats* st) {
    if (s->ntri == 0) return 0;
    float id[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    int stack[ORT_STACK]; int sp = 0;
    int found = 0;
    float best_t = tfar; int best_gid = 0x7fffffff;
    float te;
    if (st) st->rays++;
    if (st) st->box_tests++;
    if (!slab(&s->nodes[0], o, id, tnear, tfar, &te)) return 0;
    int ni = 0;
    for (;;) {
        const ort_node* n = &s->nodes[ni];
        if (n->count == 0) {
            const ort_node* a = &s->nodes[n->left];
            const ort_node* b = &s->nodes[n->left + 1];
            float ta, tb;
            /* inclusive upper bound: a tie at best_t may still win on gid */
            int ha = slab(a, o, id, tnear, best_t, &ta);
            int hb = slab(b, o, id, tnear, best_t, &tb);
            if (st) st->box_tests += 2;
            if (ha && hb) {
                int nearc = n->left, farc = n->left + 1;
                if (tb < ta) { nearc = n->left + 1; farc = n->left; }
                if (sp < ORT_STACK) stack[sp++] = farc;
                ni = nearc; continue;
            } else if (ha) { ni = n->left; continue; }
            else if (hb) { ni = n->left + 1; continue; }
        } else {
            for (int i = n->left; i < n->left + n->count; i++) {
                const ort_tri* tr = &s->tris[i];
                float t, u, v;
                if (st) st->tri_tests++;
                /* tfar for the test is the original segment end; best_t only
                   filters afterwards so that ties resolve on gid. */
                if (ort_triangle_test(tr->v0, tr->e1, tr->e2, o, d, tnear, tfar, &t, &u, &v)) {
                    if (t < best_t || (t == best_t && tr->gid < best_gid)) {
                        best_t = t; best_gid = tr->gid;
                        best->t = t; best->u = u; best->v = v; best->geom = tr->geom; best->prim = tr->prim;
                        found = 1;
                        if (any) return 1;
                    }
                }
            }
        }
        /* pop, re-testing against the shrunken best_t */
        for (;;) {
            if (sp == 0) return found;
            ni = stack[--sp];
            if (!found) break;
            if (st) st->box_tests++;
            if (slab(&s->nodes[ni], o, id, tnear, best_t, &te)) break;
        }
    }
}

int ort_intersect(const ort_scene* s, const float o[3], const float d[3], float tnear, float tfar,
                  ort_hit* hit, ort_stats* stats) {
    return traverse(s, o, d, tnear, tfar, 0, hit, stats);
}

int ort_occluded(const ort_scene* s, const float o[3], const float d[3], float tnear, float tfar,
                 ort_stats* stats) {
    ort_hit h;
    return traverse(s, o, d, tnear, tfar, 1, &h, stats);
}

/* FP64 Moeller-Trumbore on the exact (widened) vertices. */
static int tri_test_f64(const double* p, const double o[3], const double d[3], double tnear, double tfar,
                        double* t_out, double* u_out, double* v_out) {
    double e1[3] = {p[3] - p[0], p[4] - p[1], p[5] - p[2]};
    double e2[3] = {p[6] - p[0], p[7] - p[1], p[8] - p[2]};
    double px = d[1] * e2[2] - d[2] * e2[1];
    double py = d[2] * e2[0] - d[0] * e2[2];
    double pz = d[0] * e2[1] - d[1] * e2[0];
    double det = e1[0] * px + e1[1] * py + e1[2] * pz;
    if (det == 0.0) return 0;
    double inv = 1.0 / det;
    double tx = o[0] - p[0], ty = o[1] - p[1], tz = o[2] - p[2];
    double u = (tx * px + ty * py + tz * pz) * inv;
    if (!(u >= 0.0 && u <= 1.0)) return 0;
    double qx = ty * e1[2] - tz * e1[1];
    double qy = tz * e1[0] - tx * e1[2];
    double qz = tx * e1[1] - ty * e1[0];
    double v = (d[0] * qx + d[1] * qy + d[2] * qz) * inv;
    if (!(v >= 0.0 && u + v <= 1.0)) return 0;
    double t = (e2[0] * qx + e2[1] * qy + e2[2] * qz) * inv;
    if (!(t > tnear && t < tfar)) return 0;
    *t_out = t; *u_out = u; *v_out = v;
    return 1;
}

int ort_intersect_f64(const ort_scene* s, const double o[3], const double d[3], double tnear, double tfar,
                      double* t_out, double* u_out, double* v_out, int* geom, int* prim) {
    if (s->ntri == 0) return 0;
    /* Boxes are padded float boxes: conservative for the exact double test too. */
    float of[3] = {(float)o[0], (float)o[1], (float)o[2]};
    double dn = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    float df[3] = {(float)(d[0] / dn), (float)(d[1] / dn), (float)(d[2] / dn)};
    float id[3] = {1.0f / df[0], 1.0f / df[1], 1.0f / df[2]};
    int stack[ORT_STACK]; int sp = 0;
    int found = 0; double best_t = tfar; int best_gid = 0x7fffffff;
    float te;
    /* widen the float interval a little: the origin was rounded to float */
    float fnear = (float)(tnear * dn) * 0.999f - 1e-3f, ffar = (float)(tfar * dn) * 1.001f + 1e-3f;
    stack[sp++] = 0;
    while (sp) {
        const ort_node* n = &s->nodes[stack[--sp]];
        if (!slab(n, of, id, fnear, (float)(best_t * dn) * 1.001f + 1e-3f, &te)) continue;
        (void)ffar;
        if (n->count == 0) {
            if (sp + 2 <= ORT_STACK) { stack[sp++] = n->left; stack[sp++] = n->left + 1; }
        } else {
            for (int i = n->left; i < n->left + n->count; i++) {
                double t, u, v;
                if (tri_test_f64(&s->tri64[9 * i], o, d, tnear, tfar, &t, &u, &v)) {
                    const ort_tri* tr = &s->tris[i];
                    if (t < best_t || (t == best_t && tr->gid < best_gid)) {
                        best_t = t; best_gid = tr->gid; *t_out = t; *u_out = u; *v_out = v;
                        *geom = tr->geom; *prim = tr->prim; found = 1;
                    }
                }
            }
        }
    }
    return found;
}
