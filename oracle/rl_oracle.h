/*
 * rl_oracle — plain-C restatement of Relight's four ray-bound bake passes.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels in relight_b200/.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * oracle/liboracle.so; the product never links or calls it.
 *
 * Each function cites the reference file:line it restates.  Floating-point
 * expressions keep the reference's evaluation order and are compiled with
 * -ffp-contract=off, so that (a) the deterministic direct-light pass matches
 * the compiled reference bit for bit, and (b) a CUDA kernel compiled with
 * --fmad=false that follows the same order produces bit-identical results.
 *
 * Random numbers: the reference calls the C library's global rand()
 * (Types.h:110-113), which no other implementation can reproduce.  Here every
 * random draw comes from Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)
 * keyed by (seed) with a counter naming (item, sample, attempt, purpose), so a
 * GPU kernel keyed the same way draws the same numbers.  The distributions are
 * the reference's (uniform cube rejection, uniform hemisphere flip).
 */
#ifndef ORACLE_RL_ORACLE_H
#define ORACLE_RL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat scene: all meshes concatenated, already in scene space (i.e. after
   Scene::addMesh's Mesh::transformed, scene/Scene.cpp:98-107). */
typedef struct {
    int32_t nverts;
    const float* pos;          /* [nverts][3] */
    const float* nrm;          /* [nverts][3] */
    const float* uv0;          /* [nverts][2] diffuse uv layer */
    const float* uv1;          /* [nverts][2] lightmap uv layer */
    const int32_t* vmat;       /* [nverts] material index or -1 */
    int32_t ntris;
    const int32_t* tris;       /* [ntris][3] global vertex ids, index-buffer order (a, b, c) */
    int32_t nmeshes;
    const int32_t* mesh_first_tri;  /* [nmeshes + 1] */
    const int32_t* mesh_lightmap;   /* [nmeshes] map id or -1 */
    const int32_t* mesh_photonmap;  /* [nmeshes] map id or -1 */
    int32_t nmats;
    const float* mat_rgb;      /* [nmats][3] */
    const int32_t* mat_tex;    /* [nmats] texture id or -1 */
    int32_t ntex;
    const int32_t* tex_dims;   /* [ntex][3]: width, height, channels */
    const int64_t* tex_offset; /* [ntex] byte offset into tex_pixels */
    const uint8_t* tex_pixels;
    float bounds_lo[3];        /* Scene::bounds() */
    float bounds_hi[3];
} rl_scene_desc;

/* One light, as the reference's Light + its model objects (scene/Light.h). */
typedef struct {
    int32_t influence;        /* 0 none, 1 LightInfluence, 2 DirectionalLightInfluence */
    int32_t casts_shadow;
    float position[3];
    float color[3];
    float intensity;
    float direction[3];       /* DirectionalLightInfluence / DirectionalPhotonEmitter direction */
    int32_t attenuation;      /* 0 none, 1 LinearLightAttenuation */
    float att_radius, att_const, att_linear, att_quadratic;
    int32_t cutoff;           /* 0 none, 1 LightCutoff (always 1), 2 LightSpotCutoff */
    float spot_direction[3];
    float spot_cutoff, spot_exponent;
    int32_t emitter;          /* 0 none, 1 PhotonEmitter, 2 DirectionalPhotonEmitter */
    float emitter_plane[4];   /* DirectionalPhotonEmitter::m_plane: normal xyz, distance */
    int32_t vertex_first;     /* light-vertex samples (light-local points) in the pool */
    int32_t vertex_count;     /* 0: no vertex generator (point sample at position) */
} rl_light;

/* A lightmap / photonmap / radiancemap as SoA lumel arrays (Lightmap.h:35-55). */
typedef struct {
    int32_t width, height;
    int32_t* flags;    /* [w*h] Lumel::m_flags (bit 0 = Valid) */
    int32_t* face;     /* [w*h] Lumel::m_faceIdx */
    float* position;   /* [w*h][3] */
    float* normal;     /* [w*h][3] */
    float* color;      /* [w*h][3] */
    int32_t* photons;  /* [w*h] */
    float* gathered;   /* [w*h][3] */
    int32_t* mesh;     /* [w*h] scene mesh that rasterised the lumel, -1 none */
} rl_lumels;

/* bake::LumelBakeIterator (kind 0) / FaceBakeIterator (kind 1, over `mesh`)
   (baker/Baker.h:91-155, baker/Baker.cpp:176-234); NULL = LumelBakeIterator(0, 1). */
typedef struct {
    int32_t kind, first, step, mesh;
} rl_iterator;

typedef struct oro_ctx oro_ctx;

oro_ctx* oro_create(const rl_scene_desc* desc);
void oro_destroy(oro_ctx* c);

/* Philox4x32-10 block (exposed for known-answer tests). */
void oro_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Lightmap::addMesh -> initializeLumels (Lightmap.cpp:93-164). */
void oro_init_lumels(const rl_scene_desc* d, int mesh, rl_lumels* lm);

/* rt::Embree::traceSegment (rt/Embree.cpp:107-177).  seg: [n][6] start, end.
   Outputs (any may be NULL): hit flag, point, normal, rgba, lightmap uv, mesh,
   face, t of the final segment. */
void oro_trace_segments(const oro_ctx* c, int n, const float* seg, int flags, int32_t* hit, float* point,
                        float* normal, float* rgba, float* uv, int32_t* mesh, int32_t* face);

/* Relight::bakeDirectLight with a bake iterator
   (Relight.cpp:216-227, baker/DirectLight.cpp:46-125). */
void oro_bake_direct(const oro_ctx* c, const rl_light* lights, int nlights, const float* light_vertices,
                     rl_lumels* lm, const rl_iterator* it);

/* Relight::bakeAmbientOcclusion (baker/AmbientOcclusion.cpp:46-66). */
void oro_bake_ao(const oro_ctx* c, rl_lumels* lm, int samples, float occluded_fraction, float max_distance,
                 float exponent, uint64_t seed, const rl_iterator* it);

/* Relight::emitPhotons minus the gather (baker/Photons.cpp:50-144).
   photonmaps[k] is map id k; deposits go to the hit mesh's photonmap.
   Returns the number of photons stored. */
long long oro_emit_photons(const oro_ctx* c, const rl_light* lights, int nlights, rl_lumels* photonmaps,
                           int pass_count, int max_depth, float energy_threshold, float max_distance,
                           uint64_t seed);

/* The photons with global index in [first_photon, first_photon + count)
   (count < 0: to the end), in the pass / light / photon loop order above. */
long long oro_emit_photons_range(const oro_ctx* c, const rl_light* lights, int nlights, rl_lumels* photonmaps,
                                 int pass_count, int max_depth, float energy_threshold, float max_distance,
                                 uint64_t seed, long long first_photon, long long photon_count);

/* Photonmap::gather(radius) (Lightmap.cpp:376-413). */
void oro_photonmap_gather(rl_lumels* pm, int radius);

/* Lightmap::expand (Lightmap.cpp:167-193): every valid interior lumel copies
   its colour into its invalid diagonal neighbours, in scan order (the last
   writer wins), in place. */
void oro_expand(rl_lumels* lm);
/* Lightmap::blur (Lightmap.cpp:196-220): each interior texel becomes the mean
   of the valid texels of its 3x3 window, computed in place in scan order, so
   the window's upper row and left neighbour are already blurred. */
void oro_blur(rl_lumels* lm);
/* Lightmap::toDoubleLdr / toRgbmLdr (Lightmap.cpp:288-330) with
   Rgb::doubleLdr / Rgb::rgbm (Types.h:215-235).  DoubleLdr: out[w*h*3].
   RGBM: out[w*h*4] with the reference's pixel offset x*3 inside a row of
   stride w*4, so each pixel's m byte is overwritten by the next pixel's r
   and the bytes past 3w+1 of a row are never written (left as they are). */
void oro_to_double_ldr(const rl_lumels* lm, uint8_t* out);
void oro_to_rgbm(const rl_lumels* lm, uint8_t* out);
/* static_cast<unsigned char>(float) as x86-64 code performs it: truncate to
   a 32-bit integer (the out-of-range / NaN result is 0x80000000) and keep
   the low byte. */
uint8_t oro_f2u8(float v);

/* Relight::bakeIndirectLight (baker/IndirectLight.cpp:47-75). */
void oro_bake_indirect(const oro_ctx* c, rl_lumels* lm, const rl_lumels* photonmaps, int samples,
                       float max_distance, const float sky[3], const float ambient[3], uint64_t seed,
                       const rl_iterator* it);

/* RadiosityBuilder::computeFormFactors with distanceFormFactor and
   refineFormFactors, maxFormFactors = 0 (radiosity/RadiosityBuilder.cpp:99-176).
   Two calls: with cols == NULL it returns nnz; then it fills row_ptr/cols/vals. */
long long oro_ff_pairwise(const oro_ctx* c, int n, const float* pos, const float* nrm, float threshold,
                          int64_t* row_ptr, int32_t* cols, float* vals);

/* Hemisphere-cast form factors (no reference counterpart: the
   cosine-weighted hemisphere variant): `rays` cosine-weighted rays per patch, F_ij = hits/rays. */
long long oro_ff_hemisphere(const oro_ctx* c, int n, const float* pos, const float* nrm, int rays,
                            float max_distance, uint64_t seed, const int32_t* mesh_map, const int32_t* map_dims,
                            const int64_t* map_base, const int32_t* patch_of_texel, int64_t* row_ptr,
                            int32_t* cols, float* vals);

/* Jacobi gather iterations B <- E + rho .* (F B) over RGB, B0 = E
   (the gather of src/relight/Radiosity.cpp:130-146, iterated). */
void oro_jacobi_f64(int n, const int64_t* row_ptr, const int32_t* cols, const float* vals, const float* E,
                    const float* rho, int iters, double* B);
void oro_jacobi_f32(int n, const int64_t* row_ptr, const int32_t* cols, const float* vals, const float* E,
                    const float* rho, int iters, float* B);

/* FP64 high-sample expectations for Monte-Carlo parity (project-written). */
void oro_ao_expect_f64(const oro_ctx* c, const rl_lumels* lm, int ntexels, const int32_t* texels, int samples,
                       float occluded_fraction, float max_distance, uint64_t seed, double* out_value);
void oro_fg_expect_f64(const oro_ctx* c, const rl_lumels* lm, const rl_lumels* photonmaps, int ntexels,
                       const int32_t* texels, int samples, float max_distance, const float sky[3],
                       const float ambient[3], uint64_t seed, double* out_rgb);

/* Ray statistics of the last oracle pass (rays, box tests, triangle tests). */
void oro_last_stats(const oro_ctx* c, uint64_t out[3]);
/* Closest-hit / any-hit traversal statistics for an explicit ray set. */
void oro_trace_stats(const oro_ctx* c, int n, const float* seg, int any, uint64_t out[3]);

#ifdef __cplusplus
}
#endif
#endif
