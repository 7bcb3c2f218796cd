/*
 * ort — the oracle's CPU ray tracer.  TEST INFRASTRUCTURE ONLY: nothing in the
 * product (relight_b200/) links, loads or calls this code.  It is used by
 *   - oracle/embree2_cpu.cpp, which implements the Embree 2 C API that the
 *     reference's rt/Embree.cpp calls (so the reference baker runs unchanged),
 *   - oracle/rl_oracle.c, the plain-C restatement of the bake passes,
 * as the checker of the CUDA traversal kernels.
 *
 * Semantics it defines (Embree 2 is a closed binary, so these are restated
 * from its public API contract in embree2/rtcore_ray.h:24-51 and the call
 * sites in rt/Embree.cpp:107-177):
 *   - closest hit on the OPEN interval tnear < t < tfar,
 *   - (u, v) with hit = (1-u-v)*p0 + u*p1 + v*p2 (p0/p1/p2 = index-buffer order),
 *   - geomID = registration order of meshes, primID = triangle index in mesh,
 *   - ties in t go to the smaller (geomID, primID).
 *
 * Triangle test: Moeller-Trumbore (Moeller & Trumbore 1997, "Fast, minimum
 * storage ray/triangle intersection") over precomputed v0, e1 = p1-p0,
 * e2 = p2-p0, with every fused multiply-add written out as fmaf() so that a
 * CUDA kernel that writes the same __fmaf_rn() sequence gets bit-identical
 * t, u, v.  The file must be compiled with -ffp-contract=off.
 */
#ifndef ORACLE_ORT_H
#define ORACLE_ORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ort_scene ort_scene;

typedef struct {
    float t, u, v;
    int   geom, prim;
} ort_hit;

/* Traversal counters for the roofline's per-ray byte model. */
typedef struct {
    uint64_t rays, box_tests, tri_tests;
} ort_stats;

ort_scene* ort_create(void);
void       ort_destroy(ort_scene* s);
/* verts: nverts points, `vstride` floats apart (x,y,z first); tris: 3 ints per triangle. */
int        ort_add_mesh(ort_scene* s, const float* verts, int vstride, int nverts, const int* tris, int ntris);
void       ort_commit(ort_scene* s);
int        ort_triangle_count(const ort_scene* s);

/* Closest hit in (tnear, tfar).  Returns 1 and fills *hit on a hit. */
int ort_intersect(const ort_scene* s, const float o[3], const float d[3], float tnear, float tfar,
                  ort_hit* hit, ort_stats* stats);
/* Any hit in (tnear, tfar) (same triangle test, first hit ends the walk). */
int ort_occluded(const ort_scene* s, const float o[3], const float d[3], float tnear, float tfar,
                 ort_stats* stats);
/* FP64 closest hit on the same triangles (vertices widened exactly to double). */
int ort_intersect_f64(const ort_scene* s, const double o[3], const double d[3], double tnear, double tfar,
                      double* t, double* u, double* v, int* geom, int* prim);

/* The Moeller-Trumbore test used by every traversal above (exposed for tests). */
int ort_triangle_test(const float v0[3], const float e1[3], const float e2[3],
                      const float o[3], const float d[3], float tnear, float tfar,
                      float* t, float* u, float* v);

#ifdef __cplusplus
}
#endif
#endif
