/*
 * relight_b200 — C ABI of the B200 (sm_100a) lightmap baker.
 *
 * This is the drop-in boundary for Relight's ray-bound bake passes.  Every
 * entry point replaces one reference interface, cited beside it
 * (dmsovetov/Relight, path:line).  Signatures use plain pointers, sizes and
 * opaque handles only.  Every call returns an int status (RL_OK = 0), and
 * rl_last_error() gives the message of the calling thread's last failure.
 * No exception crosses the ABI.
 *
 * Memory: an rl_scene owns the device copy of the geometry and its BVH.  An
 * rl_map owns the device lumel arrays of one lightmap, photonmap or
 * radiancemap.  Host pointers passed in are borrowed for the duration of the
 * call only.  Device pointers (`d_*`) stay owned by the caller.
 *
 * Streams: `stream` is a cudaStream_t (NULL = legacy default stream).  Work is
 * enqueued on it, so a call may return before its kernels finish.  The calls
 * that return data in host memory (rl_map_download, rl_ff_*,
 * rl_radiosity_solve) synchronise the stream.  One handle must not be used
 * from two threads at once.
 */
#ifndef RELIGHT_B200_H
#define RELIGHT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */

/* RelightStatus (Relight.h:82-86) plus the errors a GPU call can raise. */
enum {
    RL_OK = 0,              /* RelightSuccess */
    RL_INVALID_CALL = 1,    /* RelightInvalidCall: bad handle/argument or state */
    RL_NOT_IMPLEMENTED = 2, /* RelightNotImplemented */
    RL_OUT_OF_MEMORY = 3,
    RL_CUDA_ERROR = 4,
    RL_CAPACITY = 5         /* an output did not fit the caller's capacity */
};

/* rt::HitFlags (rt/Tracer.h:65-72). */
enum {
    RL_HIT_POINT = 1,
    RL_HIT_UV = 2,
    RL_HIT_COLOR = 4,
    RL_HIT_NORMAL = 8,
    RL_HIT_USE_ALPHA = 16,
    RL_HIT_ALL = 15
};

/* Message of the calling thread's last failed call ("" if none). */
int rl_last_error(char* buf, size_t len);
/* Library version string and the device the library was built for. */
const char* rl_version(void);

/* ------------------------------------------------------------- scene */

/* The flat scene: all meshes concatenated, in scene space (after
   Scene::addMesh's Mesh::transformed, scene/Scene.cpp:98-107).  Replaces
   the per-mesh registration of rt::Embree::addMesh (rt/Embree.cpp:180-217):
   geometry id = mesh index, primitive id = face index within the mesh. */
typedef struct {
    int32_t nverts;
    const float* pos;          /* [nverts][3] Vertex::position */
    const float* nrm;          /* [nverts][3] Vertex::normal */
    const float* uv0;          /* [nverts][2] Vertex::uv[Diffuse] */
    const float* uv1;          /* [nverts][2] Vertex::uv[Lightmap] */
    const int32_t* vmat;       /* [nverts] material index or -1 (Vertex::material) */
    int32_t ntris;
    const int32_t* tris;       /* [ntris][3] global vertex ids in index-buffer order */
    int32_t nmeshes;
    const int32_t* mesh_first_tri;  /* [nmeshes + 1] */
    const int32_t* mesh_lightmap;   /* [nmeshes] lightmap slot or -1 (Mesh::lightmap) */
    const int32_t* mesh_photonmap;  /* [nmeshes] photonmap slot or -1 (Mesh::photonmap) */
    int32_t nmats;
    const float* mat_rgb;      /* [nmats][3] Material::color */
    const int32_t* mat_tex;    /* [nmats] texture index or -1 (TexturedMaterial) */
    int32_t ntex;
    const int32_t* tex_dims;   /* [ntex][3] width, height, channels (3 or 4) */
    const int64_t* tex_offset; /* [ntex] byte offset into tex_pixels */
    const uint8_t* tex_pixels;
    float bounds_lo[3];        /* Scene::bounds() (scene/Scene.cpp:81-88) */
    float bounds_hi[3];
} rl_scene_desc;

/* A light with its model objects (scene/Light.h:228-336). */
typedef struct {
    int32_t influence;        /* 0 none, 1 LightInfluence, 2 DirectionalLightInfluence */
    int32_t casts_shadow;
    float position[3];
    float color[3];
    float intensity;
    float direction[3];       /* directional influence / emitter direction */
    int32_t attenuation;      /* 0 none, 1 LinearLightAttenuation */
    float att_radius, att_const, att_linear, att_quadratic;
    int32_t cutoff;           /* 0 none, 1 LightCutoff, 2 LightSpotCutoff */
    float spot_direction[3];
    float spot_cutoff, spot_exponent;
    int32_t emitter;          /* 0 none, 1 PhotonEmitter, 2 DirectionalPhotonEmitter */
    float emitter_plane[4];   /* DirectionalPhotonEmitter plane: normal, distance */
    int32_t vertex_first;     /* LightVertexGenerator samples in the light-vertex pool */
    int32_t vertex_count;     /* 0 = no vertex generator */
} rl_light;

typedef struct rl_scene rl_scene;

/* Scene::end -> new rt::Embree; addMesh...; rtcCommit (scene/Scene.cpp:122-142,
   rt/Embree.cpp:49-58): upload the geometry and build the BVH on the device.
   `builder`: 0 = binned SAH on the host (the better tree: the bake default),
   1 = LBVH on the device (Karras 2012; the fast build for many or changing
   scenes).  Hits do not depend on the builder (closest hit, ties to the
   smaller triangle id). */
int rl_scene_create(const rl_scene_desc* desc, int builder, void* stream, rl_scene** out);
int rl_scene_destroy(rl_scene* scene);
/* BVH statistics: node count, leaf count, max depth, SAH cost. */
int rl_scene_bvh_stats(const rl_scene* scene, int64_t* nodes, int64_t* leaves, int32_t* depth, double* sah);
/* The scene's traversal status word, read after the work queued on `stream`
   (waits for it): bit 0 = a traversal stack overflowed (a ray may have
   skipped part of the tree).  `clear` != 0 resets it.  Embree reports no
   such condition (rtcIntersect has no failure path); this is the check
   behind every bake of a scene. */
int rl_scene_status(rl_scene* scene, int clear, int32_t* flags, void* stream);

/* ------------------------------------------------------------ tracing */

/* rt::ITracer::traceSegment (rt/Tracer.h:87; rt::Embree::traceSegment +
   initializeRay, rt/Embree.cpp:107-177) for a batch of segments:
   closest hit on (0.01, |end - start|), with the reference's hit
   post-processing (point = start + dir * t, Barycentric(u, v) attribute
   interpolation, HitUseAlpha restarts).  Device arrays:
     d_seg     [n][6]  start xyz, end xyz
     d_hit     [n]     1 hit / 0 miss
     d_t_uv    [n][3]  t, u, v of the final segment (may be NULL)
     d_mesh_face [n][2] mesh, face (-1 on a miss) (may be NULL)
     d_point, d_normal [n][3], d_rgba [n][4], d_uv [n][2] (may be NULL) */
int rl_trace_segments(const rl_scene* scene, int64_t n, const float* d_seg, int flags, int32_t* d_hit,
                      float* d_t_uv, int32_t* d_mesh_face, float* d_point, float* d_normal, float* d_rgba,
                      float* d_uv, void* stream);

/* rtcIntersect / rtcOccluded (Embree 2, embree2/rtcore_ray.h:24-51 and
   rtcore_scene.h; called at rt/Embree.cpp:139,151) for a batch of rays in
   Embree's own terms: the closest hit (any_hit = 0) or some hit (any_hit =
   1) on the open interval (tnear, tfar) of org + t * dir, ties to the
   smaller (geomID, primID).  The Embree-level seam: the reference's
   rt::Embree runs unchanged with these answering its Embree calls.
     d_rays      [n][8]  org xyz, tnear, dir xyz, tfar (16-byte aligned)
     d_geom_prim [n][2]  geomID (scene mesh), primID (face); -1, -1 on a miss
     d_t_uv      [n][3]  t, u, v of the hit (may be NULL)
   rl_intersect_rays_host is the same call on host arrays: it stages them
   through a device buffer of the calling thread (kept for its next call),
   runs on that thread's own stream and returns when the results are in
   host memory, so several host threads may call it at once. */
int rl_intersect_rays(const rl_scene* scene, int64_t n, const float* d_rays, int any_hit, int32_t* d_geom_prim,
                      float* d_t_uv, void* stream);
int rl_intersect_rays_host(const rl_scene* scene, int64_t n, const float* rays, int any_hit, int32_t* geom_prim,
                           float* t_uv);

/* ----------------------------------------------------------- lumel maps */

typedef struct rl_map rl_map;

/* Relight::createLightmap / createPhotonmap (Relight.cpp:193-202); kind
   0 = Lightmap, 1 = Photonmap, 2 = Radiancemap (Lightmap.h:58-184). */
int rl_map_create(int kind, int width, int height, rl_map** out);
int rl_map_destroy(rl_map* map);
/* The same map as one stream-ordered block (cudaMallocAsync, initialised by
   a kernel on `stream`), and its stream-ordered release: neither call waits
   for the device, so a serving loop can admit and retire lightmaps while
   other bakes run.  rl_map_bytes gives the block size of a width x height
   map (the unit of an HBM budget).  No reference counterpart. */
int rl_map_bytes(int width, int height, int64_t* bytes);
/* Those blocks (and batch tables) come from the library's memory pool on
   the current device, which keeps freed memory for reuse instead of
   returning it at every synchronisation.  rl_pool_trim returns all but
   `keep_bytes` of the unused memory; rl_pool_bytes reports the pool's
   reserved and in-use bytes (either pointer may be NULL). */
int rl_pool_trim(int64_t keep_bytes);
int rl_pool_bytes(int64_t* reserved, int64_t* used);
int rl_map_create_async(int kind, int width, int height, void* stream, rl_map** out);
int rl_map_destroy_async(rl_map* map, void* stream);
/* Lightmap::addMesh / Photonmap::addMesh -> initializeLumels
   (Lightmap.cpp:93-164, 360-373): rasterise the mesh's faces into lumels
   (last face wins).  Call once per mesh, in the reference's addMesh order. */
int rl_map_add_mesh(rl_map* map, const rl_scene* scene, int mesh, void* stream);
/* Lumel read-back / upload (Lightmap::lumels(), Lightmap.cpp:55-58, and
   toHdr(), :332-349).  Host arrays [w*h] or [w*h][3]; any may be NULL. */
int rl_map_download(const rl_map* map, int32_t* flags, int32_t* face, float* position, float* normal, float* color,
                    int32_t* photons, float* gathered, void* stream);
/* The baked colours ([w*h][3]) copied to `color` in stream order, without
   waiting: the data is there once `stream` has reached this point (pinned
   host memory for a truly asynchronous copy).  No reference counterpart. */
int rl_map_download_async(const rl_map* map, float* color, void* stream);
int rl_map_upload(rl_map* map, const int32_t* flags, const int32_t* face, const float* position,
                  const float* normal, const float* color, const int32_t* photons, const float* gathered,
                  void* stream);
/* Lightmap::expand (Lightmap.cpp:167-193) and Lightmap::blur (:196-220) on
   the device, bit-identical to the reference's in-place scan-order loops
   (blur runs as a one-block wavefront). */
int rl_map_expand(rl_map* map, void* stream);
int rl_map_blur(rl_map* map, void* stream);
/* relight::StorageFormat (Relight.h:89-93). */
enum { RL_RAW_HDR = 0, RL_TGA_DOUBLE_LDR = 1, RL_TGA_RGBM = 2 };
/* The pixel buffer Lightmap::toHdr / toDoubleLdr / toRgbmLdr
   (Lightmap.cpp:288-349) returns, encoded on the device and copied to host
   `out` (w*h*12, w*h*3 or w*h*4 bytes; waits for `stream`).  RGBM keeps the
   reference's row layout (pixel offset x*3 in rows of w*4 bytes); the bytes
   the reference leaves uninitialised are 0. */
int rl_map_encode(const rl_map* map, int format, uint8_t* out, void* stream);
/* Lightmap::save (Lightmap.cpp:223-283): the same file, byte for byte. */
int rl_map_save(const rl_map* map, const char* path, int format, void* stream);
/* Set every lumel colour / photon accumulator to zero. */
int rl_map_clear(rl_map* map, int colors, int photons, void* stream);
/* Device pointers of the lumel arrays (SoA, [w*h] or [w*h][3]); any may be NULL. */
int rl_map_device_arrays(const rl_map* map, int32_t** flags, float** position, float** normal, float** color,
                         int32_t** photons, float** gathered);
/* Number of valid lumels (after rl_map_add_mesh). */
int rl_map_valid_count(const rl_map* map, int64_t* count);

/* --------------------------------------------------------------- passes */

/* bake::LumelBakeIterator / bake::FaceBakeIterator (baker/Baker.h:91-155,
   baker/Baker.cpp:176-234): which lumels of the map a bake call visits.
     kind 0  LumelBakeIterator(first, step): lumels first, first + step, ...
             of the whole map, whichever mesh rasterised them;
     kind 1  FaceBakeIterator(first, step) on `mesh`: the lumels rasterised
             from faces first, first + step, ... of that scene mesh.
   A NULL iterator means LumelBakeIterator(0, 1), the default of the
   Relight::bake* calls (Relight.cpp:218-220). */
typedef struct {
    int32_t kind;
    int32_t first;
    int32_t step;
    int32_t mesh;
} rl_iterator;

/* Relight::bakeDirectLight with a bake iterator
   (Relight.cpp:216-227; baker/DirectLight.cpp:46-125;
   scene/Light.cpp:372-500).  Adds every light's influence to the lumel
   colours.  `lights` and `light_vertices` ([nverts][3]) are host arrays. */
int rl_bake_direct(const rl_scene* scene, rl_map* lightmap, const rl_light* lights, int nlights,
                   const float* light_vertices, int nlight_vertices, const rl_iterator* iterator, void* stream);

/* Relight::bakeAmbientOcclusion (Relight.cpp:260-271;
   baker/AmbientOcclusion.cpp:46-66): colour *= 1 - occluded/(samples*fraction),
   optionally raised to `exponent`.  Directions are Philox-keyed by (seed,
   lumel index, sample). */
int rl_bake_ao(const rl_scene* scene, rl_map* lightmap, int samples, float occluded_fraction, float max_distance,
               float exponent, uint64_t seed, const rl_iterator* iterator, void* stream);

/* Relight::emitPhotons minus the gather (Relight.cpp:244-250;
   baker/Photons.cpp:50-144; scene/Light.cpp:334-361): trace
   pass_count x sum_l int(intensity*25000) photons and deposit colour+count
   into each hit mesh's photonmap (maps[] indexed by the scene's photonmap
   slot).  *stored (host, may be NULL) receives the deposit count. */
int rl_emit_photons(const rl_scene* scene, rl_map* const* photonmaps, int nmaps, const rl_light* lights,
                    int nlights, int pass_count, int max_depth, float energy_threshold, float max_distance,
                    uint64_t seed, int64_t* stored, void* stream);

/* The same photons, restricted to the global photon indices
   [first_photon, first_photon + photon_count) of the reference's
   pass / light / photon loop order: a GPU's share when one bake's photons
   are split across GPUs.  The shares' photonmap accumulators (colour, count)
   summed over GPUs equal the unsplit emission's. */
int rl_emit_photons_range(const rl_scene* scene, rl_map* const* photonmaps, int nmaps, const rl_light* lights,
                          int nlights, int pass_count, int max_depth, float energy_threshold, float max_distance,
                          uint64_t seed, int64_t first_photon, int64_t photon_count, int64_t* stored, void* stream);
/* Number of photons one emission traces: pass_count x sum over emitting
   lights of int(intensity * 25000) (PhotonEmitter::photonCount,
   scene/Light.cpp:334-337). */
int rl_photon_count(const rl_light* lights, int nlights, int pass_count, int64_t* total);

/* k-nearest-neighbour photon estimate (no reference counterpart: the
   reference has only the texel-space disc gather, Photonmap::gather,
   Lightmap.cpp:376-413).  rl_emit_photons_records is rl_emit_photons that
   also keeps every deposit Photons::store makes (baker/Photons.cpp:119-126)
   as a world-space record in `records` (cleared first; deposits beyond its
   capacity are counted but not kept).  rl_photonmap_gather_knn then sets,
   at every valid lumel of the photonmap in `slot`, gathered = the mean
   colour of the k nearest deposits of that photonmap within `radius` world
   units of the lumel position (ties by photon number and bounce; 0 when
   none), over a uniform grid of cells RL_TUNE_KNN_CELL / 64 of the radius
   wide.  The colours are summed exactly in 64-bit fixed point (2^s per unit,
   2^53 <= s-scaled largest colour < 2^54) and the mean is taken in double
   precision, so the value depends only on which deposits are nearest.  Run
   it after rl_photonmap_gather: lumels that are not valid keep the disc's
   value. */
typedef struct rl_photons rl_photons;
int rl_photons_create(int64_t capacity, rl_photons** out);
int rl_photons_destroy(rl_photons* records);
/* Deposits of the last emission (may exceed the capacity). */
int rl_photons_count(const rl_photons* records, int64_t* deposits);
/* The kept records, in no particular order: xyzrgb [n][6], photon [n],
   depth_slot [n][2] (any may be NULL; n = min(count, capacity)). */
int rl_photons_download(const rl_photons* records, float* xyzrgb, uint32_t* photon, int32_t* depth_slot);
/* Replaces the records with n given ones (same layout as the download;
   depth and slot in [0, 65535]), as if an emission had kept them: records
   from another emitter, or planted cases.  No reference counterpart. */
int rl_photons_upload(rl_photons* records, int64_t n, const float* xyzrgb, const uint32_t* photon,
                      const int32_t* depth_slot);
int rl_emit_photons_records(const rl_scene* scene, rl_map* const* photonmaps, int nmaps, const rl_light* lights,
                            int nlights, int pass_count, int max_depth, float threshold, float max_distance,
                            uint64_t seed, rl_photons* records, int64_t* stored, void* stream);
/* k in [1, 128]; fails with RL_CAPACITY if the records overflowed. */
int rl_photonmap_gather_knn(rl_map* photonmap, int slot, rl_photons* records, int k, float radius, void* stream);

/* Photonmap::gather(radius) (Lightmap.cpp:376-413), the loop-bound quirk
   of :379 included. */
int rl_photonmap_gather(rl_map* photonmap, int radius, void* stream);

/* Relight::bakeIndirectLight (Relight.cpp:230-241;
   baker/IndirectLight.cpp:47-75): final gather against the gathered
   photonmaps (maps[] by photonmap slot). */
int rl_bake_indirect(const rl_scene* scene, rl_map* lightmap, rl_map* const* photonmaps, int nmaps, int samples,
                     float max_distance, const float sky[3], const float ambient[3], uint64_t seed,
                     const rl_iterator* iterator, void* stream);

/* ------------------------------------------------------------ OBJ ingest */

/* Mesh::createFromFile -> MeshLoader::load (scene/Mesh.cpp:111-122,
   scene/MeshLoader.cpp:44-226): Wavefront OBJ with the reference's
   submesh commits, face forms, float-equality vertex sharing and uv clamp.
   Host-only (no device needed).  Face indices outside the parsed arrays and
   meshes beyond 16-bit indices fail with RL_INVALID_CALL (undefined in the
   reference). */
typedef struct rl_obj_mesh rl_obj_mesh;
int rl_obj_load(const char* path, rl_obj_mesh** out);
int rl_obj_mesh_counts(const rl_obj_mesh* mesh, int32_t* nvertices, int32_t* nindices, int32_t* nsubmeshes);
/* positions/normals [n][3], uv_lightmap [n][2] (uv[Vertex::Lightmap]; the
   diffuse layer is 0), indices [nindices]; any may be NULL. */
int rl_obj_mesh_arrays(const rl_obj_mesh* mesh, float* positions, float* normals, float* uv_lightmap,
                       int32_t* indices);
int rl_obj_mesh_destroy(rl_obj_mesh* mesh);

/* ------------------------------------------------------------- denoiser */

/* Building blocks of the lightmap denoiser (no reference counterpart: the
   reference has no denoiser).  Tensors are device NHWC BF16 arrays whose
   channel stride is a multiple of 16; convolutions run on the tensor cores
   (tcgen05, FP32 accumulation).  `d_err` (device int, may be NULL) gets a
   nonzero bit if a kernel's bounded wait ran out.

   rl_dn_conv3x3: out = act(conv3x3(concat(in0, in1)) + bias) with zero
   padding; c0 / c1 are the inputs' stored channel counts (multiples of 8).
   `weights` is BF16 [9][K/8][ncols][8] (16-byte aligned), K = 16*(ceil(c0/16)
   + ceil(c1/16)): tap = 3*(dy+1) + (dx+1), then blocks of 8 input channels
   (segment 0's, zero-padded to a multiple of 16, then segment 1's), then
   output channels, then the 8 channels of the block.  Accumulator columns
   [outK_c0, outK_c0 + outK_cn) go to outK (channel stride outK_cs), times
   (maskK > 0 ? 1 : slope) when maskK is given; relu != 0 applies a leaky
   ReLU of negative slope `slope` (0: ReLU); in1/out1 may be NULL. */
int rl_dn_conv3x3(const void* in0, int c0, const void* in1, int c1, int width, int height, int images,
                  const void* weights, int ncols, const float* bias, int relu, float slope, void* out0, int out0_c0,
                  int out0_cn, int out0_cs, const void* mask0, void* out1, int out1_c0, int out1_cn, int out1_cs,
                  const void* mask1, int* d_err, void* stream);
/* dw[co][tap][ci_off + ci] += sum_p grad[p][co] * in[p + offset(tap)][ci]
   (FP32, accumulated), co < cout <= 128, ci < cin. */
int rl_dn_conv3x3_wgrad(const void* grad, int cout, int grad_cs, const void* in, int cin, int in_cs, int width,
                        int height, int images, float* dw, int ci_off, int ci_total, int* d_err, void* stream);

/* The denoiser network: 8 convolutions over 4 levels (32, 64, 96, 128
   channels, leaky ReLU; 2x2 average pooling, nearest upsampling, skip
   concatenation),
   input features [h][w][16] = (log1p noisy rgb, normal, albedo, valid, 0),
   output = residual on log1p rgb.  Parameters are FP32 masters updated by
   Adam; the convolutions run in BF16 on the tensor cores. */
typedef struct rl_denoiser rl_denoiser;
int rl_denoiser_create(uint64_t seed, rl_denoiser** out);
int rl_denoiser_destroy(rl_denoiser* dn);
int rl_denoiser_param_count(const rl_denoiser* dn, int64_t* count);
/* Per layer: weights [cout][9][k] (k = input channels padded per segment to
   64) then biases [cout], as one FP32 host array. */
int rl_denoiser_get_params(const rl_denoiser* dn, float* host);
int rl_denoiser_set_params(rl_denoiser* dn, const float* host);
int rl_denoiser_get_grads(rl_denoiser* dn, float* host);
/* Features of a baked lightmap (d_x: BF16 [h][w][16]) and training targets
   (d_t: FP32 [h][w][4] = log1p rgb, valid). */
int rl_denoiser_features(const rl_scene* scene, const rl_map* lightmap, void* d_x, void* stream);
int rl_denoiser_targets(const rl_map* lightmap, float* d_t, void* stream);
/* One Adam step on a batch of square patches; *d_loss += the batch's mean L1
   (log space) when d_loss is not NULL.  lr < 0: accumulate the gradients
   only, for rl_denoiser_get_grads (which returns and clears them). */
int rl_denoiser_train_step(rl_denoiser* dn, const void* d_x, const float* d_t, int batch, int patch, float lr,
                           float* d_loss, void* stream);
/* Denoise a lightmap in place: colour = base + expm1(prediction) on valid
   lumels (d_base [w*h][3] or NULL for 0). */
int rl_denoiser_apply(rl_denoiser* dn, const rl_scene* scene, rl_map* lightmap, const float* d_base, void* stream);
/* Raw network output (BF16 [n][h][w][16]) for features d_x. */
int rl_denoiser_forward(rl_denoiser* dn, const void* d_x, int images, int height, int width, void* d_y,
                        void* stream);
/* Size the working buffers for inputs up to images x height x width (and the
   training gradients when train != 0), so later calls do not allocate. */
int rl_denoiser_reserve(rl_denoiser* dn, int images, int height, int width, int train);
/* Bits set by bounded waits that ran out in the denoiser's kernels (0 = none). */
int rl_denoiser_status(rl_denoiser* dn, int* flags);

/* --------------------------------------------------------------- batches */

/* Many bake jobs — any scenes, lightmaps, passes — in one persistent launch
   (no counterpart in the reference, whose Worker/Job fan-out,
   Worker.cpp:43-83, runs jobs one after another per thread).  Each job is a
   single-job bake call (rl_bake_direct / rl_bake_ao / rl_bake_indirect)
   restricted to the slice [begin, end) of its iterator's visits (end < 0:
   all), with the same Philox keys, so a batch bakes bit-identical lumels.
   Passes apply in the order direct light, AO, final gather (as a bake applies
   them to one lightmap); two jobs of one pass may share a lightmap only over
   provably disjoint lumels (different face-iterator meshes, lumel iterators
   of one step with different residues, or disjoint slices of one iterator),
   else rl_batch_create fails with RL_INVALID_CALL. */
typedef struct {
    int32_t kind;                     /* 0 direct light, 1 ambient occlusion, 2 final gather */
    const rl_scene* scene;
    rl_map* lightmap;
    rl_map* const* photonmaps;        /* final gather: maps by photonmap slot */
    int32_t nmaps;
    const rl_light* lights;           /* direct light */
    int32_t nlights;
    const float* light_vertices;
    int32_t nlight_vertices;
    int32_t samples;                  /* AO / final gather */
    float occluded_fraction;          /* AO */
    float max_distance;               /* AO / final gather */
    float exponent;                   /* AO */
    float sky[3], ambient[3];         /* final gather */
    uint64_t seed;                    /* AO / final gather */
    rl_iterator iterator;
    int64_t begin, end;
} rl_batch_job;

typedef struct rl_batch rl_batch;

/* Upload a job table (host arrays are read before the call returns). */
int rl_batch_create(const rl_batch_job* jobs, int njobs, rl_batch** out);
/* Replace the job table, asynchronously on `stream` (host arrays are read
   before the call returns; the copy runs in stream order, after the launches
   already enqueued there).  A captured graph stays valid: its kernels read
   the table from a fixed device header at run time.  Update and launch or
   replay on the same stream.  On error the previous table stays. */
int rl_batch_update(rl_batch* batch, const rl_batch_job* jobs, int njobs, void* stream);
/* One persistent launch per pass kind over every job's lumels (warps take
   32 lumels at a time from a shared counter).  Launches of one batch must
   not overlap on the GPU (they share the counters). */
int rl_batch_launch(rl_batch* batch, void* stream);
/* Capture the launch into a CUDA graph on `stream` (non-default), then
   replay it; the batch reads its lightmaps' current contents at each replay. */
int rl_batch_capture(rl_batch* batch, void* stream);
int rl_batch_replay(rl_batch* batch, void* stream);
/* Number of lumel work items of the current table (summed over jobs). */
int rl_batch_work_items(const rl_batch* batch, int64_t* items);
int rl_batch_destroy(rl_batch* batch);

/* ------------------------------------------------------------- radiosity */

/* RadiosityBuilder::computeFormFactors + distanceFormFactor +
   refineFormFactors with maxFormFactors = 0
   (radiosity/RadiosityBuilder.cpp:99-176): pairwise point-to-point form
   factors over `n` patches (device arrays d_pos, d_nrm [n][3]), visibility
   by segment, each row normalised to sum 1.  Output CSR in host memory,
   columns ascending (the reference's list order).  Call with cols == NULL
   to get *nnz only; then with arrays of that capacity. */
int rl_ff_pairwise(const rl_scene* scene, int n, const float* d_pos, const float* d_nrm, float threshold,
                   int64_t* row_ptr, int32_t* cols, float* vals, int64_t capacity, int64_t* nnz, void* stream);

/* Hemisphere-cast form factors (no reference counterpart; cosine-weighted
   variant of the form factors above): `rays` cosine-distributed rays per
   patch; F_ij = (rays from i whose hit maps to patch j) / rays.  A hit maps
   to a patch through the hit mesh's map (mesh_map[mesh], map_dims[map] =
   w,h), the lumel at the hit's lightmap uv (Lightmap::lumel(const Uv&),
   Lightmap.cpp:61-67) and patch_of_texel[map_base[map] + texel] (-1 none).
   All arrays are host arrays.  Output CSR as for rl_ff_pairwise. */
int rl_ff_hemisphere(const rl_scene* scene, int n, const float* d_pos, const float* d_nrm, int rays,
                     float max_distance, uint64_t seed, const int32_t* mesh_map, int nmaps, const int32_t* map_dims,
                     const int64_t* map_base, const int32_t* patch_of_texel, int64_t ntexels, int64_t* row_ptr,
                     int32_t* cols, float* vals, int64_t capacity, int64_t* nnz, void* stream);
/* The same form factors with the CSR left in device memory (d_row_ptr
   [n + 1], d_cols and d_vals of `capacity` entries), ready for
   rl_radiosity_solve without a trip through host memory.  With d_cols NULL
   it only reports *nnz.  The CSR is written in stream order; n * rays is
   always enough capacity.  No reference counterpart. */
int rl_ff_hemisphere_device(const rl_scene* scene, int n, const float* d_pos, const float* d_nrm, int rays,
                            float max_distance, uint64_t seed, const int32_t* mesh_map, int nmaps,
                            const int32_t* map_dims, const int64_t* map_base, const int32_t* patch_of_texel,
                            int64_t ntexels, int64_t* d_row_ptr, int32_t* d_cols, float* d_vals, int64_t capacity,
                            int64_t* nnz, void* stream);

/* Radiosity gather iterations (RadiositySolver::solve is an empty stub,
   radiosity/RadiositySolver.cpp:34-36; the gather math is the legacy
   cRadiositySolver::Solve, src/relight/Radiosity.cpp:130-146, iterated):
   B <- E + rho .* (F B) over RGB, B0 = E, `iters` Jacobi steps.  CSR and
   vectors are device arrays; d_B [n][3] receives the result. */
int rl_radiosity_solve(int n, const int64_t* d_row_ptr, const int32_t* d_cols, const float* d_vals,
                       const float* d_E, const float* d_rho, int iters, float* d_B, void* stream);

/* One Jacobi step restricted to rows [row_begin, row_end):
   d_B_next[row] = E[row] + rho[row] * sum_k F[row][k] d_B[k] ([n][3] arrays,
   rows written at their own index).  The unit of a row-sharded solve across
   GPUs (each GPU steps its rows, then the rows are all-gathered into d_B).
   Each row uses rl_radiosity_solve's arithmetic (the same 16-byte-load
   choice for aligned d_cols / d_vals), so iterating it over all rows gives
   rl_radiosity_solve's bits. */
int rl_radiosity_step(int row_begin, int row_end, const int64_t* d_row_ptr, const int32_t* d_cols,
                      const float* d_vals, const float* d_E, const float* d_rho, const float* d_B, float* d_B_next,
                      void* stream);

/* The same solve for callers that cannot allocate device memory: a plugin
   inside a host application (a game engine or an editor) that owns every
   device allocation itself, or a bake server that reserved its HBM when the
   request was admitted.  This entry point calls no cudaMalloc, cudaFree or
   allocating routine.  Its two ping-pong iterates live in a fixed device
   array of 2 x RL_SOLVE_NOALLOC_MAX_PATCHES float4 (2 MiB), committed on a
   device when this library's solver module first loads there (the first
   launch of one of its kernels, or the first call of this entry point; a
   call with n = 0 is enough) and held until the process exits.  Callers
   that budget HBM up front make that warm-up call first.  Larger `n` is
   rejected with RL_INVALID_CALL.  The first call on a device looks the
   array's address up (once per device, with that device current); make it
   before any stream capture.  It runs the same kernels in the same order as
   rl_radiosity_solve, so both give the same bits, and d_B may alias d_E or
   d_rho (it is written last).  All calls share the one array, so calls
   whose work overlaps on the GPU race; run them on one stream or one at a
   time.  No counterpart in the reference. */
#define RL_SOLVE_NOALLOC_MAX_PATCHES 65536
int rl_radiosity_solve_noalloc(int n, const int64_t* d_row_ptr, const int32_t* d_cols, const float* d_vals,
                               const float* d_E, const float* d_rho, int iters, float* d_B, void* stream);

/* ---------------------------------------------------------------- tuning */

/* Launch parameters of the ray-stream kernels (final gather, AO), chosen by
   the autotuner (relight_b200/autotune.py); process-wide.  They change
   scheduling only, never results.  No counterpart in the reference.
     *_REFILL: a warp restarts finished lanes' rays once this many of its
               live lanes (1..32) have finished;
     *_BLOCK:  threads per block (64, 128 or 256);
     RL_TUNE_BVH_WIDTH: 2 (binary nodes), 4 (4-wide nodes) or 8 (compressed
                        8-wide nodes, built for scenes created while it is
                        selected);
     RL_TUNE_SPECULATIVE: 1 = binary traversal parks leaves until the whole
                          warp has one (speculative traversal), 0 = off;
     RL_TUNE_KNN_CELL: cell width of rl_photonmap_gather_knn's grid in 64ths
                       of its radius (8..256, default 80);
     RL_TUNE_AO_SPLIT: lanes that share one lumel's AO samples (1, 2, 4 or 8;
                       0 = chosen from the map size, the default);
     RL_TUNE_FG_POOL: 1 = final gather, unsplit AO and the batch kernels on
                      a persistent grid whose lanes take lumels from their
                      warp's pool as they finish one; 0 = one lumel per
                      thread (the default: measured faster on the terrain
                      final gather, where the pool's lanes lose ray
                      coherence);
     RL_TUNE_FG_CHUNK: lumels a warp claims for its pool at a time (8..256). */
enum {
    RL_TUNE_FG_REFILL = 0,
    RL_TUNE_FG_BLOCK = 1,
    RL_TUNE_AO_REFILL = 2,
    RL_TUNE_AO_BLOCK = 3,
    RL_TUNE_BVH_WIDTH = 4,
    RL_TUNE_SPECULATIVE = 5,
    RL_TUNE_KNN_CELL = 6,
    RL_TUNE_AO_SPLIT = 7,
    RL_TUNE_FG_POOL = 8,
    RL_TUNE_FG_CHUNK = 9
};
int rl_tune_set(int param, int value);
int rl_tune_get(int param, int* value);

/* ------------------------------------------------------------ measurement */

/* Device read bandwidth (GB/s) of `bytes` streamed `iters` times with 16-byte
   loads; below the L2 size this is the L2 bandwidth the traversal kernels
   draw on.  A measurement utility with no counterpart in the reference. */
int rl_measure_read_bandwidth(size_t bytes, int iters, double* gbs);
/* L1 read bandwidth (GB/s, whole GPU): every block re-reads the same
   `bytes_per_block` (a multiple of 16 KiB, at most 128 KiB) `iters` times
   with 16-byte cached
   loads, so after the first pass the loads hit each SM's L1 — the level a
   tree of a few hundred triangles lives in.  No counterpart in the
   reference. */
int rl_measure_l1_read_bandwidth(size_t bytes_per_block, int iters, double* gbs);

#ifdef __cplusplus
}
#endif
#endif /* RELIGHT_B200_H */
