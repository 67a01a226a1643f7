/*
 * slimtracer_b200.h -- C ABI of the B200 (sm_100a) per-pixel trace path.
 *
 * Drop-in for the GPU seam of SlimTracin's renderer: the reference compiles
 * renderer/renderer_GPU.h into the app when built with nvcc
 * (renderer/renderer.h:7-17) and calls its hooks from
 * RayTracingRenderer's constructor and render() (renderer/renderer.h:60,
 * 69-81).  This library exports the same hooks as plain C functions taking
 * pointers to POD mirrors of the reference's structs, laid out byte for
 * byte like the reference's own types on LP64 with 4-byte u32
 * (static-asserted below), so an app passes `(const SlimSceneData*)&scene`.
 *
 * Differences from the reference's hooks, all deliberate:
 *   - every call returns an int status (SLIM_OK == 0) instead of printing
 *     and exit()ing (core/base.h:17-27) or silently ignoring errors in
 *     release builds (core/base.h:46); slimGetLastError() describes it;
 *   - the library never falls back to a CPU path: without a usable CUDA
 *     device every call fails with SLIM_ERR_CUDA.
 */
#ifndef SLIMTRACER_B200_H
#define SLIMTRACER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SLIM_OK              0
#define SLIM_ERR_ARGUMENT    1   /* null pointer, bad count or size          */
#define SLIM_ERR_CUDA        2   /* CUDA runtime error (no device, OOM, ...) */
#define SLIM_ERR_STATE       3   /* call order (e.g. render before init)     */
#define SLIM_ERR_LIMIT       4   /* a fixed capacity would be exceeded       */
#define SLIM_ERR_IO          5   /* file missing, truncated or malformed     */
#define SLIM_ERR_STACK       6   /* a traversal stack overflowed (device)    */
#define SLIM_ERR_TIMEOUT     7   /* a bounded device wait gave up            */

/* ---- enums and flags (core/base.h:137-149,402-414,626-633,655-660) ----- */
enum { SLIM_GEOMETRY_NONE = 0, SLIM_GEOMETRY_MESH, SLIM_GEOMETRY_GRID, SLIM_GEOMETRY_BOX,
       SLIM_GEOMETRY_CURVE, SLIM_GEOMETRY_TET, SLIM_GEOMETRY_QUAD, SLIM_GEOMETRY_SPHERE,
       SLIM_GEOMETRY_LIGHT };
enum { SLIM_BRDF_LAMBERT = 0, SLIM_BRDF_BLINN, SLIM_BRDF_PHONG, SLIM_BRDF_COOK_TORRANCE };
enum { SLIM_RENDER_NORMALS = 0, SLIM_RENDER_NORMAL_MAP, SLIM_RENDER_BEAUTY, SLIM_RENDER_DEPTH,
       SLIM_RENDER_MIP_LEVEL, SLIM_RENDER_UVS };
enum { SLIM_AA_NONE = 0, SLIM_AA_MSAA, SLIM_AA_SSAA };
#define SLIM_MATERIAL_IS_REFLECTIVE   1u
#define SLIM_MATERIAL_IS_REFRACTIVE   2u
#define SLIM_MATERIAL_IS_EMISSIVE     4u
#define SLIM_MATERIAL_HAS_ALBEDO_MAP 16u
#define SLIM_MATERIAL_HAS_NORMAL_MAP 32u
#define SLIM_GEOMETRY_IS_VISIBLE      1u
#define SLIM_GEOMETRY_IS_SHADOWING    2u
#define SLIM_GEOMETRY_IS_TRANSPARENT  4u
#define SLIM_LIGHT_IS_DIRECTIONAL     1u   /* scene/material.h:10-15 */
#define SLIM_LIGHT_IS_SHADOWING       2u
#define SLIM_SCENE_HAD_EMISSIVE_QUADS 1u   /* scene/scene.h:27 */
/* ImageInfo.flags bits (core/base.h:1264-1276) */
#define SLIM_IMAGE_ALPHA    (1u << 0)
#define SLIM_IMAGE_LINEAR   (1u << 1)
#define SLIM_IMAGE_TILE     (1u << 2)
#define SLIM_IMAGE_CHANNEL  (1u << 3)
#define SLIM_IMAGE_MIPMAP   (1u << 4)
#define SLIM_IMAGE_FLIP     (1u << 5)
#define SLIM_IMAGE_WRAP     (1u << 6)
#define SLIM_IMAGE_NORMAL   (1u << 7)
#define SLIM_IMAGE_CUBEMAP  (1u << 8)

/* ---- POD mirrors of the reference structs ------------------------------ */
typedef struct { float x, y, z; } SlimVec3;                       /* math/vec3.h:5   */
typedef struct { float x, y; } SlimVec2;                          /* math/vec2.h:255 */
typedef struct { SlimVec3 min, max; } SlimAABB;                   /* math/vec3.h:423 */

/* OrientationUsingQuaternion = quat{axis, amount} + Orientation's euler
 * cache x,y,z (math/quat.h:3-6, core/base.h:546-622). */
typedef struct { SlimVec3 axis; float amount; float euler[3]; } SlimOrientation;
typedef struct { SlimOrientation orientation; SlimVec3 position, scale; } SlimTransform;   /* core/transform.h:5-8  */
typedef struct {                                                                          /* core/transform.h:59-65 */
    SlimTransform transform;
    int32_t type;           /* SLIM_GEOMETRY_*                      */
    uint32_t material_id;
    uint32_t id;            /* mesh index for SLIM_GEOMETRY_MESH    */
    uint8_t flags;          /* SLIM_GEOMETRY_IS_*                   */
    uint8_t _pad[3];
    int32_t color;          /* ColorID, unused by the tracer        */
} SlimGeometry;
typedef struct {                                                                          /* scene/material.h:93-110 */
    float albedo[3];
    float roughness;
    uint8_t flags, texture_count, texture_ids[2];
    int32_t brdf;
    float normal_magnitude;
    SlimVec2 uv_repeat;
    float emission[3];
    float IOR;
    float reflectivity[3];
    float metalness;
} SlimMaterial;
typedef struct {                                                                          /* scene/material.h:17-21 */
    float color[3];
    SlimVec3 position_or_direction;
    float intensity;
    uint8_t flags;
    uint8_t _pad[3];
} SlimLight;
typedef struct {                                                                          /* scene/bvh.h:5-16 */
    SlimAABB aabb;
    uint32_t first_index;
    uint16_t leaf_count;
    uint8_t depth, flags;
} SlimBVHNode;
typedef struct { SlimBVHNode *nodes; uint32_t node_count; uint8_t height; uint8_t _pad[3]; } SlimBVH;  /* scene/bvh.h:18-21 */
typedef struct {                                                                          /* scene/mesh.h:19-23 */
    float local_to_tangent[9];   /* mat3 columns X, Y, Z */
    SlimVec3 position, normal, n1, n2, n3;
    SlimVec2 uv1, uv2, uv3;
    float uv_coverage, padding;
} SlimTriangle;
typedef struct {                                                                          /* scene/mesh.h:25-41 */
    SlimAABB aabb;
    SlimBVH bvh;
    SlimTriangle *triangles;
    SlimVec3 *vertex_positions, *vertex_normals;
    SlimVec2 *vertex_uvs;
    uint32_t *vertex_position_indices, *vertex_normal_indices, *vertex_uvs_indices;  /* [triangle][3] */
    uint32_t *edge_vertex_indices;                                                     /* [edge][2]     */
    uint32_t triangle_count, vertex_count, edge_count, normals_count, uvs_count;
    uint32_t _pad;
} SlimMesh;
typedef struct { uint8_t R[4], G[4], B[4]; } SlimTexelQuad;   /* {TL,TR,BL,BR} per channel, core/texture.h:5-11 */
typedef struct { uint32_t width, height; SlimTexelQuad *texel_quads; } SlimTextureMip;   /* core/texture.h:13-15 */
typedef struct {                                              /* ImageInfo + mips, core/base.h:1233-1284, core/texture.h:44-45 */
    uint32_t width, height, size, stride, tile_width, tile_height;
    uint32_t mip_count;
    uint32_t flags;          /* SLIM_IMAGE_* */
    SlimTextureMip *mips;
} SlimTexture;
typedef struct {                                              /* scene/scene.h:17-19 */
    uint32_t geometries, cameras, lights, materials, textures, meshes, grids, boxes, tets, quads, curves;
} SlimSceneCounts;
typedef struct {                                              /* scene/scene.h:35-56 */
    SlimSceneCounts counts;
    uint16_t flags, mesh_stack_size;
    SlimGeometry *geometries;
    void *cameras;
    SlimLight *lights;
    SlimMaterial *materials;
    SlimTexture *textures;
    SlimMesh *meshes;
    void *grids, *boxes, *tets, *quads, *curves;
    SlimAABB *aabbs;
    void *io, *bvh_builder;
    uint32_t *bvh_leaf_geometry_indices;
    SlimBVH bvh;
} SlimSceneData;
typedef struct {                                              /* core/base.h:1300-1311 */
    uint32_t width_times_height;
    float width_over_height, height_over_width, f_width, f_height, h_width, h_height;
    uint16_t width, height, stride, _pad;
} SlimDimensions;
typedef struct { float r, g, b, opacity; } SlimPixel;          /* core/base.h:1081-1083 */
typedef struct {                                              /* draw/canvas.h:11-17 */
    SlimDimensions dimensions;
    int32_t antialias;       /* SLIM_AA_* */
    SlimPixel *pixels;
    float *depths;
} SlimCanvasData;
typedef struct {                                              /* scene/camera.h:58-63 */
    float inverted_camera_rotation[9];
    SlimVec3 start, right, down, camera_position;
    SlimVec2 C_start;
    float squared_distance_to_projection_plane;
    float sample_size;
} SlimCameraRayProjection;
typedef struct {                                              /* renderer/ray_tracer.h:10-17 */
    uint8_t max_depth;
    int8_t skybox_color_texture_id, skybox_radiance_texture_id, skybox_irradiance_texture_id;
    int32_t render_mode;     /* SLIM_RENDER_* */
    int32_t mip_level_colors[9];
} SlimRayTracerSettings;

/* Options with no reference counterpart (B200 execution choices). */
enum { SLIM_ENGINE_WAVEFRONT = 0, SLIM_ENGINE_MEGAKERNEL = 1, SLIM_ENGINE_AUTO = 2 };
enum { SLIM_CONES_REFERENCE = 0, SLIM_CONES_PER_PIXEL = 1 };
enum { SLIM_SCENE_BVH_UPLOADED = 0, SLIM_SCENE_BVH_REFIT = 1 };
typedef struct {
    int32_t engine;          /* SLIM_ENGINE_*: wavefront queues, one fused kernel, or AUTO --
                                the library's setting until the first slimSetRenderOptions (a
                                zeroed struct selects WAVEFRONT): the fused kernel for frames of
                                scenes without meshes whose paths end at their first hit (max
                                depth 1, or no reflective or refractive material) or that have
                                fewer than 2^19 samples, the wavefront engine for the rest and
                                for radiance-cache frames.  Both engines write the same pixels;
                                the choice is speed only (fused: one launch, no queues; wavefront:
                                split BVH walks that keep warps full on long or divergent paths) */
    int32_t ray_cones;       /* SLIM_CONES_REFERENCE (default): the reference's effective ray
                                cone (mip 0: its copy of the aux hit clears the per-pixel
                                spread); SLIM_CONES_PER_PIXEL: per-pixel spread */
    int32_t scene_bvh;       /* SLIM_SCENE_BVH_UPLOADED (default) or GPU refit of its topology */
    int32_t block_size;      /* threads per block (multiple of 32, at most 256), 0 = tuned default */
    int32_t count_work;      /* non-zero: accumulate per-frame work counters (slower) */
    int32_t profile_stages;  /* non-zero: time every stage launch with CUDA events */
    int32_t shadow_queue_mb; /* wavefront shadow-ray queue budget in MiB, 0 = 1024 */
    int32_t radiance_cache;  /* SLIM_CACHE_*: with the wavefront engine and a configured
                                radiance cache, paths stop at the cache depth and take the
                                cache's answer.  OFF (default); ON: the network; TRUNCATE:
                                nothing (the method without the network); EXACT: every
                                query traced on to max_depth by the tracer (a check of the
                                cache plumbing: equals the plain frame up to rounding) */
    int32_t row_bands;       /* wavefront frames render in this many row bands, two in flight
                                at once (the caller's stream and a second one), so one
                                band's launch tails overlap the other's work; into a pinned
                                host canvas each band downloads while the next renders.
                                0 = default (2 from 512x512 samples up, else 1), 1 = whole
                                frame, at most 64.  The fused engine, and radiance-cache
                                frames other than ON with overlapped training, use one
                                band; banded cache frames gather every band's queries and
                                answer them in one cache phase.  Plain frames' pixels are
                                the same for any band count. */
} SlimRenderOptions;
enum { SLIM_CACHE_OFF = 0, SLIM_CACHE_ON = 1, SLIM_CACHE_TRUNCATE = 2, SLIM_CACHE_EXACT = 3 };

/* Work counters of the last frame (rays traced and memory records touched).
 * The shadow_* fields are the parts of the node, triangle and geometry
 * tests spent in any-hit (shadow-ray) traversals; only the fused engine,
 * which walks every ray in the reference's order, splits them out. */
typedef struct {
    uint64_t primary_rays, shadow_rays, bounce_rays;
    uint64_t scene_node_tests, mesh_node_tests, triangle_tests;
    uint64_t geometry_tests, mesh_hit_fetches, texel_taps;
    uint64_t pixels;
    uint64_t shadow_scene_node_tests, shadow_mesh_node_tests, shadow_triangle_tests, shadow_geometry_tests;
} SlimWorkCounters;

#ifdef __cplusplus
#define SLIM_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define SLIM_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
SLIM_STATIC_ASSERT(sizeof(SlimGeometry) == 72, "Geometry is 72 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimMaterial) == 68, "Material is 68 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimLight) == 32, "Light is 32 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimBVHNode) == 32, "BVHNode is 32 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimTriangle) == 128, "Triangle is 128 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimTexelQuad) == 12, "TexelQuad is 12 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimTextureMip) == 16, "TextureMip is 16 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimTexture) == 40, "Texture is 40 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimMesh) == 128, "Mesh is 128 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimSceneData) == 184, "SceneData is 184 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimCanvasData) == 56, "CanvasData is 56 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimCameraRayProjection) == 100, "CameraRayProjection is 100 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimRayTracerSettings) == 44, "RayTracerSettings is 44 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimRenderOptions) == 36, "RenderOptions is 36 bytes");

/* ======================================================================== *
 * Drop-in hooks (renderer/renderer_GPU.h)                                   *
 * ======================================================================== */

/* Replaces initDataOnGPU(const Scene&) (renderer/renderer_GPU.h:80-181):
 * one-time deep copy of the scene -- geometries, materials, lights, scene
 * BVH, meshes (triangles + BVH nodes) and textures (mips + texel quads) --
 * into the device layout.  Mesh and texture topology is frozen afterwards,
 * as in the reference.  May be called again to replace the scene. */
int slimInitDataOnGPU(const SlimSceneData *scene);

/* Replace uploadLights/uploadCameras/uploadGeometries/uploadMaterials/
 * uploadSceneBVH(const Scene&) (renderer/renderer_GPU.h:70-78): re-upload
 * the per-frame mutable parts.  Counts must equal those given to
 * slimInitDataOnGPU (SLIM_ERR_STATE otherwise). */
int slimUploadLights(const SlimSceneData *scene);
int slimUploadCameras(const SlimSceneData *scene);
int slimUploadGeometries(const SlimSceneData *scene);
int slimUploadMaterials(const SlimSceneData *scene);
int slimUploadSceneBVH(const SlimSceneData *scene);

/* Replaces renderOnGPU(const Canvas&, const CameraRayProjection&,
 * const RayTracerSettings&) (renderer/renderer_GPU.h:48-68): traces every
 * pixel (every sub-sample under SSAA) and writes canvas->pixels (Pixel
 * {clamp(c)^2, 1}) and canvas->depths synchronously, like the reference.
 * Into pinned host memory (cudaHostAlloc) the rows download while later
 * bounces still render; a pageable canvas of 4 MB of pixels or more goes
 * through the library's own pinned staging buffer and a host copy. */
int slimRenderOnGPU(const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                    const SlimRayTracerSettings *settings);

/* ======================================================================== *
 * Extensions (no reference counterpart unless cited)                        *
 * ======================================================================== */

const char *slimGetLastError(void);
int slimGetVersion(void);

/* Waits for `stream` and reports what the device flagged since the last
 * check (stack overflow, bad index, a timed-out wait) and, with
 * options.count_work, the work counters of the last frame or batch. */
int slimSynchronize(void *stream);

/* Kernels this library has launched since it was loaded (a replayed batch
 * graph counts its kernel nodes). */
int slimGetLaunchCount(uint64_t *count);

int slimSetRenderOptions(const SlimRenderOptions *options);
int slimGetRenderOptions(SlimRenderOptions *options);

/* Device-resident render: same work as slimRenderOnGPU, but the frame stays
 * in device memory (d_pixels: float4 per sample, d_depths: float per
 * sample, both allocated by the caller with room for every sample) and the
 * call is asynchronous on `stream` (a cudaStream_t, 0 = legacy default). */
int slimRenderToDevice(const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                       const SlimRayTracerSettings *settings, void *d_pixels, void *d_depths,
                       void *stream);

/* No counterpart in the reference.  Same frame as slimRenderToDevice with
 * the wavefront engine, but allocates nothing: for callers that cannot
 * enter the CUDA allocator from their per-frame hook -- e.g. while another
 * thread captures a CUDA graph in global capture mode, which makes
 * cudaMalloc/cudaFree fail process-wide, or inside a host engine that
 * reserves all device memory up front.  The queues live in one file-scope
 * __device__ array of 64 MiB that every GPU loading the library holds until
 * exit; frames needing more (about 250 bytes per sample, e.g. 640x360 with
 * several lights fits, 1080p does not) fail with SLIM_ERR_LIMIT.  The first
 * call on each device looks up the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream
 * capture, with the scene's device current (another current device is
 * refused with SLIM_ERR_STATE).  Every call shares the one array: calls
 * whose work overlaps on the GPU (different streams, or threads without
 * ordering) race and corrupt each other's frames.  Debug render modes and
 * max_depth 0 use no scratch and have no size limit.  The radiance cache and
 * work counting are refused (SLIM_ERR_STATE): switch them off with
 * slimSetRenderOptions first.  The call only enqueues work, so a device-side
 * error of its kernels (a traversal stack overflow, say) is reported by the
 * next synchronous call of the library (slimSynchronize, for one), as for
 * slimRenderToDevice. */
int slimRenderToDeviceNoAlloc(const SlimCanvasData *canvas, const SlimCameraRayProjection *projection,
                              const SlimRayTracerSettings *settings, void *d_pixels, void *d_depths, void *stream);

/* Closest hit of every primary ray (renderer/ray_tracer.h:36-45 ->
 * scene/scene_tracer.h:26-98) into device buffers of width*height entries:
 * geometry index (-1 = miss), mesh triangle id in leaf order (0 for
 * implicit primitives), hit distance, hit-from-behind flag. */
int slimTracePrimary(const SlimCameraRayProjection *projection, int width, int height,
                     void *d_geometry_ids, void *d_primitive_ids, void *d_distances,
                     void *d_from_behind, void *stream);

/* Selection::manipulate's pick (scene/selection.h:36-80): the geometry
 * behind pixel (x, y) and the point light whose selection sphere the ray
 * reaches first (light >= 0 wins over the geometry, as in the reference).
 * Synchronous. */
typedef struct {
    int32_t geometry;          /* closest geometry index, -1 on a miss */
    int32_t light;             /* picked light index, -1 for none */
    uint32_t triangle;         /* mesh triangle id in leaf order (0 for implicit primitives) */
    float distance;            /* hit distance along the normalised ray (INF on a miss) */
    float position[3];         /* world position of the hit */
    uint32_t from_behind;
} SlimPick;
int slimPick(const SlimCameraRayProjection *projection, int x, int y, SlimPick *out);

/* Work counters of the last frame rendered with options.count_work set. */
int slimGetWorkCounters(SlimWorkCounters *counters);

/* Per-stage launch statistics accumulated while options.profile_stages is
 * set (stage names: fused, extend, shadow_gen, shadow, shade, refit):
 * launches, summed CUDA-event milliseconds and -- with count_work -- the
 * work counters of the last frame.  Fills up to `capacity` entries. */
typedef struct {
    char name[24];
    uint32_t launches;
    float total_ms;
    SlimWorkCounters work;
} SlimStageStats;
int slimGetStageStats(SlimStageStats *stats, int capacity, int *count);
int slimResetStageStats(void);

/* Re-fits the device copy of the scene BVH to the current geometries
 * (GPU), keeping the topology last uploaded: scene/scene.h:165-191 rebuilds
 * it from scratch on the host every frame instead. */
int slimRefitSceneBVH(void *stream);

/* No counterpart in the reference (its scene BVH only lives on the host).
 * Copies the device copy of the scene BVH -- as the last upload or refit
 * left it -- into scene->bvh.nodes, whose node_count must equal the
 * uploaded one.  Synchronous: waits for the last refit. */
int slimDownloadSceneBVH(SlimSceneData *scene);

/* ---- Neural radiance cache.  No counterpart in the reference. ----------
 * A 96-64-64-64-64-3 MLP (ReLU, exp output; bf16 weights and activations,
 * f32 accumulation on the sm_100a tensor cores) that stands in for the rest
 * of a path from the cache depth on.  Inputs per sample, 16 floats:
 *   (p.xyz, roughness) (direction.xyz, 0) (normal.xyz, 0) (albedo.xyz, 0)
 * with p the hit position mapped to [0,1]^3 by the scene box.  It is
 * encoded as 12-octave sin/cos of p, bands 0..3 spherical harmonics of the
 * direction, normal, roughness, albedo and a constant 1.  Parameters: one
 * f32 vector of SLIM_NRC_PARAMS, W0 [64][96], W1..W3 [64][64], W4 [3][64]
 * (row = output unit).  Training: L2 on log(radiance + 0.01) against the
 * exp output's argument, Adam; the cache answers max(exp(z) - 0.01, 0). */
#define SLIM_NRC_PARAMS 18624
#define SLIM_NRC_FEATURES 16
typedef struct {
    uint32_t cache_depth;    /* path vertex the cache answers at (>= 2) */
    uint32_t train_samples;  /* training paths per frame (65536) */
    uint32_t batch;          /* samples per Adam step (16384) */
    uint32_t seed;           /* weight initialisation, per-frame sample selection */
    float learning_rate;     /* 1e-2 */
    float beta1, beta2, epsilon;   /* 0.9, 0.99, 1e-8 */
    uint32_t train;          /* non-zero: train online every rendered frame */
    uint32_t overlap;        /* non-zero: trace the training paths and take the Adam steps
                                on a second stream, one frame behind: a frame's queries are
                                answered with the weights trained through the previous frame,
                                while its own training overlaps the next frame's rays */
    uint32_t train_suffix;   /* 0: every training path is traced to max_depth (its target is
                                the tracer's full-depth radiance).  k > 0: a training path is
                                traced k bounces past the cache vertex and, where it is still
                                going there, ends in the cache's own answer for that vertex
                                (self-training: targets cost k rounds instead of
                                max_depth - cache_depth + 1); max_depth still ends paths */
    uint32_t _reserved;
} SlimRadianceCacheConfig;
typedef struct {
    uint64_t frames, steps;  /* frames rendered with the cache, Adam steps taken */
    uint32_t queries;        /* cache queries of the last frame */
    uint32_t train_samples;  /* training samples of the last frame */
    float loss;              /* mean log-radiance L2 loss of the last step */
    float _pad;
} SlimRadianceCacheStats;

/* Allocates the cache (needs slimInitDataOnGPU), initialises the weights
 * from config->seed and clears the Adam state. */
int slimRadianceCacheConfigure(const SlimRadianceCacheConfig *config);
int slimRadianceCacheGetConfig(SlimRadianceCacheConfig *config);
/* f32 master weights (host arrays of SLIM_NRC_PARAMS); setting them clears
 * the Adam moments and step count. */
int slimRadianceCacheSetWeights(const float *params, uint32_t count);
int slimRadianceCacheGetWeights(float *params, uint32_t count);
/* Mean-loss gradient of the last training step. */
int slimRadianceCacheGetGradients(float *grad, uint32_t count);

/* Training checkpoint: what online training continues from.  A state of
 * SLIM_NRC_STATE_BYTES is this header, then the f32 master weights, Adam's
 * first moments and Adam's second moments, SLIM_NRC_PARAMS floats each.
 * Save waits for training in flight.  Load (needs slimInitDataOnGPU)
 * configures the cache from the header's config, then restores the weights,
 * the moments and both counters, so the next step and the next frame's
 * training-set selection continue as if training had never stopped. */
#define SLIM_NRC_STATE_MAGIC 0x4B43524Eu
typedef struct {
    uint32_t magic;          /* SLIM_NRC_STATE_MAGIC */
    uint32_t params;         /* SLIM_NRC_PARAMS */
    uint32_t steps;          /* Adam steps taken (the bias corrections' exponent) */
    uint32_t frames;         /* cache frames rendered (offsets the training-set selection) */
    SlimRadianceCacheConfig config;
} SlimRadianceCacheStateHeader;
#define SLIM_NRC_STATE_BYTES (sizeof(SlimRadianceCacheStateHeader) + 3u * SLIM_NRC_PARAMS * sizeof(float))
int slimRadianceCacheSaveState(void *state, uint64_t bytes);
int slimRadianceCacheLoadState(const void *state, uint64_t bytes);
/* Device pointers: radiance (float4 per sample, rgb) of `count` samples of
 * SLIM_NRC_FEATURES floats.  Asynchronous on `stream`. */
int slimRadianceCacheQuery(const void *d_features, uint32_t count, void *d_radiance, void *stream);
/* One Adam step over `count` (features, target float4 rgb) device samples. */
int slimRadianceCacheTrain(const void *d_features, const void *d_targets, uint32_t count, void *stream);
/* Makes `stream` wait for the cache's overlapped training (no-op without). */
int slimRadianceCacheJoin(void *stream);
int slimRadianceCacheGetStats(SlimRadianceCacheStats *stats);

/* ---- Batched requests.  No counterpart in the reference. ----------------
 * Many render requests, each with its own scene, camera, settings and
 * canvas, traced together: their pixels are cut into tiles, consecutive
 * tiles fill waves of up to `queue_capacity` paths, and every wave runs the
 * wavefront stage kernels once for all of its requests (each path looks up
 * its request's scene and canvas).  The whole batch is captured into a CUDA
 * graph on the first slimBatchRender and replayed afterwards.  Mesh and
 * texture ids of every request refer to the assets uploaded by
 * slimInitDataOnGPU (a request's scene->meshes / ->textures are not read). */
typedef struct {
    const SlimSceneData *scene;        /* geometries, materials, lights, scene BVH + leaf indices, flags */
    SlimCameraRayProjection projection;
    SlimRayTracerSettings settings;    /* beauty mode only */
    uint32_t width, height;            /* canvas pixels (no SSAA in a batch) */
    int32_t radiance_cache;            /* SLIM_CACHE_OFF or SLIM_CACHE_ON (needs a configured cache) */
    uint32_t _pad;
    void *d_pixels;                    /* device: float4 per pixel */
    void *d_depths;                    /* device: float per pixel */
} SlimRenderRequest;

typedef struct {
    uint32_t queue_capacity;   /* path slots per wave */
    uint32_t tile_pixels;      /* pixels per tile (a tile never spans two waves) */
    int32_t block_size;        /* threads per block of the stage kernels (32..256) */
    uint32_t waves;            /* out: waves of the current requests */
    float batch_ms;            /* out: one batch with this plan, when it was tuned */
    uint32_t candidates;       /* out: plans the tuner timed */
    uint32_t graph_nodes;      /* out: kernel nodes of the captured graph (0 before the first render) */
    uint32_t tuned;            /* out: non-zero when slimBatchTune chose the plan */
    uint32_t persistent;       /* non-zero: the requests without the radiance cache are rendered by
                                  one persistent launch that pulls their pixels from a device work
                                  queue (warps refill finished paths), beside the waves of the
                                  requests with the cache; 0: every request goes through the waves */
    uint32_t _pad;
} SlimBatchPlan;

/* Uploads the requests (validated like slimInitDataOnGPU) and drops any
 * captured graph.  At most 512 requests of at most 2^23 pixels each. */
int slimBatchSetRequests(const SlimRenderRequest *requests, uint32_t count);
/* Project autotuner: times candidate plans (queue capacity, tile size, block
 * size) on the current requests with CUDA events and keeps the fastest. */
int slimBatchTune(void *stream);
int slimBatchSetPlan(const SlimBatchPlan *plan);
int slimBatchGetPlan(SlimBatchPlan *plan);
/* Renders every request (asynchronous on `stream`): the first call after
 * slimBatchSetRequests / slimBatchSetPlan captures the batch into a CUDA
 * graph, later calls replay it. */
int slimBatchRender(void *stream);

SLIM_STATIC_ASSERT(sizeof(SlimRadianceCacheConfig) == 48, "RadianceCacheConfig is 48 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimRadianceCacheStateHeader) == 64, "RadianceCacheStateHeader is 64 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimRadianceCacheStats) == 32, "RadianceCacheStats is 32 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimRenderRequest) == 184, "RenderRequest is 184 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimBatchPlan) == 40, "BatchPlan is 40 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimPick) == 32, "Pick is 32 bytes");

/* Host-side helpers: the reference's own host algorithms, restated. */

/* CameraRayProjection::reset (scene/camera.h:69-83); orientation given as
 * the camera matrix columns X (right), Y (up), Z (forward). */
int slimProjectionReset(const float orientation9[9], const float position3[3], float focal_length,
                        int width, int height, int antialias_ssaa, SlimCameraRayProjection *out);

/* Scene::updateAABBs + updateBVH (scene/scene.h:165-191, full SAH build with
 * one geometry per leaf, scene/bvh_builder.h:10-263) into scene->bvh.nodes
 * (capacity 2*geometries), scene->bvh_leaf_geometry_indices and
 * scene->flags (SLIM_SCENE_HAD_EMISSIVE_QUADS, scene/scene.h:156-159). */
int slimBuildSceneBVH(SlimSceneData *scene);

/* obj2mesh after parsing (obj2mesh.cpp:201-231 with scale 1, no rotation)
 * and BVHBuilder::buildMesh (scene/bvh_builder.h:265-341): recentres the
 * positions (in place) on the AABB centre, builds the SAH BVH (at most 2
 * triangles per leaf) and the leaf-ordered Triangle records.  Caller sizes
 * out_triangles for triangle_count and out_nodes for 2*triangle_count. */
int slimBuildMesh(float *positions, uint32_t vertex_count, const uint32_t *position_indices,
                  uint32_t triangle_count, const float *normals, uint32_t normals_count,
                  const uint32_t *normal_indices, const float *uvs, uint32_t uvs_count,
                  const uint32_t *uv_indices, SlimTriangle *out_triangles, SlimBVHNode *out_nodes,
                  uint32_t *out_node_count, uint32_t *out_height, float out_aabb6[6]);

/* .mesh file I/O (serialization/mesh.h:56-163).  slimReadMeshHeader fills
 * the counts; the caller then allocates the arrays it points the mesh at
 * (triangles, positions, index arrays, edges, uvs, normals, bvh.nodes) and
 * calls slimReadMesh.  Edge indices may be null on write (edge_count 0). */
int slimReadMeshHeader(const char *path, SlimMesh *mesh);
int slimReadMesh(const char *path, SlimMesh *mesh);
int slimWriteMesh(const char *path, const SlimMesh *mesh);

/* .texture file I/O (core/base.h:1544-1609, serialization/texture.h:7-62). */
int slimReadTextureHeader(const char *path, SlimTexture *texture, uint32_t *total_texel_quads);
int slimReadTexture(const char *path, SlimTexture *texture, SlimTextureMip *mips,
                    SlimTexelQuad *texel_quads);
int slimWriteTexture(const char *path, const SlimTexture *texture);

/* Whole-scene files: save/load(Scene&, SceneIO&) (serialization/scene.h:5-109).
 * A scene file holds SlimSceneCounts (44 bytes); every mesh's .mesh header
 * (7 u32: vertex, triangle, edge, uv and normal counts, BVH node count and
 * height); every texture's ImageInfo (32 bytes); per camera focal_length,
 * zoom_amount, dolly_amount, target_distance (f32 each), current_velocity,
 * position (vec3) and the orientation (48 bytes); the geometries (72 bytes
 * each); the viewport overlay's grids, boxes and curves (records of
 * SLIM_GRID_BYTES, SLIM_BOX_BYTES and SLIM_CURVE_BYTES, kept opaque here);
 * then every mesh's content (a .mesh file after its header) and every
 * texture's mips (a .texture file after its ImageInfo).  Lights and
 * materials are not in the file, as in the reference. */
typedef struct {                                              /* scene/camera.h:6-13 */
    float orientation[9];    /* OrientationUsing3x3Matrix: columns X (right), Y (up), Z (forward) */
    float rotation[3];       /* its x, y, z angles (radians) */
    SlimVec3 position, current_velocity;
    float focal_length, zoom_amount, target_distance, dolly_amount;
} SlimCamera;
#define SLIM_GRID_BYTES  9700   /* sizeof(Grid),  scene/grid.h  */
#define SLIM_BOX_BYTES    384   /* sizeof(Box),   scene/box.h   */
#define SLIM_CURVE_BYTES   12   /* sizeof(Curve), core/base.h   */
typedef struct {
    SlimSceneCounts counts;  /* of the arrays below (lights, materials, tets, quads: not in the file) */
    uint32_t _pad;
    SlimCamera *cameras;
    SlimGeometry *geometries;
    SlimMesh *meshes;        /* records whose arrays the caller allocates */
    SlimTexture *textures;   /* records with caller-allocated mips and texel quads */
    void *grids, *boxes, *curves;
} SlimSceneFile;
SLIM_STATIC_ASSERT(sizeof(SlimCamera) == 88, "Camera is 88 bytes");
SLIM_STATIC_ASSERT(sizeof(SlimSceneFile) == 104, "SceneFile is 104 bytes");

int slimSaveScene(const char *path, const SlimSceneFile *scene);
/* Sizing pass of a load.  Fills scene->counts; when scene->meshes and
 * scene->textures are given (records for counts.meshes / counts.textures),
 * also every mesh's counts (vertex ... normals counts, bvh.node_count,
 * bvh.height) and every texture's ImageInfo fields and mip_count, and, when
 * texel_quad_counts is given, the texel quads of each texture's mips. */
int slimReadSceneHeader(const char *path, SlimSceneFile *scene, uint32_t *texel_quad_counts);
/* Reads the whole file into the caller's arrays: cameras, geometries,
 * grids, boxes, curves, and every mesh's and texture's arrays (texture
 * mips point into one texel-quad array per texture, as slimReadTexture
 * sets them).  The counts must equal the file's. */
int slimLoadScene(const char *path, SlimSceneFile *scene);

/* bmp2texture's texel-quad baker (bmp2texture.cpp:24-237,255-335) from
 * 8-bit BGR(A) rows as a BMP stores them after its own flip handling.
 * flags: SLIM_IMAGE_* (LINEAR, MIPMAP, WRAP, NORMAL, CUBEMAP as the
 * -l -m -w -n -c switches).  First call with texel_quads == NULL to get
 * mip_count and the texel-quad count, then again with buffers. */
int slimBakeTexture(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels,
                    uint32_t flags, SlimTexture *texture, SlimTextureMip *mips,
                    SlimTexelQuad *texel_quads, uint32_t *mip_count, uint32_t *texel_quad_count);

/* The same bake on the GPU (the converter bmp2texture.cpp:24-335 runs on the
 * host in the reference): same arguments, same two-call protocol, the same
 * bytes as slimBakeTexture.  Host buffers in and out; the image crosses to
 * the device, the texel quads come back before the call returns. */
int slimBakeTextureOnGPU(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels,
                         uint32_t flags, SlimTexture *texture, SlimTextureMip *mips,
                         SlimTexelQuad *texel_quads, uint32_t *mip_count, uint32_t *texel_quad_count);

#ifdef __cplusplus
}
#endif
#endif /* SLIMTRACER_B200_H */
