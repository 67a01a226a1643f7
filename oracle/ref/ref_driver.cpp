/*
 * oracle/ref/ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A thin C-ABI driver around the UNMODIFIED algorithms of the reference
 * renderer (HardCoreCodin/SlimTracinCpp, header-only C++), compiled by
 * oracle/build_ref.sh from a patched temporary copy of the reference sources
 * into oracle/_ref/libslimref.so.  Nothing in the product links this file;
 * only tests/, __graft_entry__.smoke() and bench.py's reference / cpu
 * baseline legs load the resulting library, as the checker and the timed
 * CPU baseline.
 *
 * Entry points:
 *   ref_projection_reset  CameraRayProjection::reset        scene/camera.h:69-83
 *   ref_build_scene_bvh   Scene::updateAABBs + updateBVH    scene/scene.h:156-191
 *   ref_build_mesh        obj2mesh post-parse + BVHBuilder::buildMesh
 *                                                           obj2mesh.cpp:201-231,
 *                                                           scene/bvh_builder.h:265-341
 *   ref_render            per-pixel body of d_render (renderer/renderer_GPU.h:22-46)
 *                         run on host threads: renderPixel + Canvas::setPixel
 *   ref_render_cpu        the unmodified single-threaded renderOnCPU
 *                         (renderer/renderer.h:87-100)
 *   ref_trace_primary     SceneTracer::trace of each primary ray
 *                         (renderer/ray_tracer.h:36-45, scene/scene_tracer.h:26-98)
 *   ref_save_scene / ref_load_scene   save/load(Scene&, SceneIO&)
 *                         (serialization/scene.h:5-109), ref_scene_record_sizes
 */
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>
#include <thread>
#include <vector>

#include "slim/math/vec2.h"
#include "slim/renderer/renderer.h"
#include "slim/serialization/scene.h"

static_assert(sizeof(u32) == 4, "reference u32 must be 4 bytes");
static_assert(sizeof(Geometry) == 72, "Geometry layout");
static_assert(sizeof(Material) == 68, "Material layout");
static_assert(sizeof(Light) == 32, "Light layout");
static_assert(sizeof(BVHNode) == 32, "BVHNode layout");
static_assert(sizeof(Triangle) == 128, "Triangle layout");
static_assert(sizeof(TexelQuad) == 12, "TexelQuad layout");
static_assert(sizeof(TextureMip) == 16, "TextureMip layout");
static_assert(sizeof(Texture) == 40, "Texture layout");
static_assert(sizeof(Mesh) == 128, "Mesh layout");
static_assert(sizeof(SceneData) == 184, "SceneData layout");
static_assert(sizeof(CanvasData) == 56, "CanvasData layout");
static_assert(sizeof(CameraRayProjection) == 100, "CameraRayProjection layout");
static_assert(sizeof(RayTracerSettings) == 44, "RayTracerSettings layout");

// ---------------------------------------------------------------------------
// POSIX definitions of the platform functions base.h declares
// (core/base.h:1354-1366); the reference defines them for Win32 only.
// getMemory hands out zeroed memory, as VirtualAlloc(MEM_COMMIT) does.
void* os::getMemory(u64 size, u64) { return calloc(1, size ? size : 1); }
void os::setWindowTitle(char*) {}
void os::setWindowCapture(bool) {}
void os::setCursorVisibility(bool) {}
void os::closeFile(void *handle) { if (handle) fclose((FILE*)handle); }
void* os::openFileForReading(const char* path) { return fopen(path, "rb"); }
void* os::openFileForWriting(const char* path) { return fopen(path, "wb"); }
bool os::readFromFile(void *out, unsigned long size, void *handle) {
    return fread(out, 1, size, (FILE*)handle) == size;
}
bool os::writeToFile(void *out, unsigned long size, void *handle) {
    return fwrite(out, 1, size, (FILE*)handle) == size;
}
u64 timers::getTicks() {
    timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    return (u64)ts.tv_sec * 1000000000ull + (u64)ts.tv_nsec;
}

// ---------------------------------------------------------------------------
// Per-thread tracer state.  d_render constructs a fresh SceneTracer,
// SurfaceShader, Ray and RayHit for every pixel; the reference CPU app owns
// them inside a value-initialised (zeroed) app object.  Members the
// reference never writes (e.g. SceneTracer::aux_hit.scaling_factor) are
// therefore zero here, exactly as in the CPU app.
namespace {
constexpr u32 kStack = 256;

struct PixelContext {
    alignas(64) u32 scene_stack[kStack];
    alignas(64) u32 mesh_stack[kStack];
    alignas(64) unsigned char tracer_mem[sizeof(SceneTracer)];
    alignas(64) unsigned char surface_mem[sizeof(SurfaceShader)];
    alignas(64) unsigned char ray_mem[sizeof(Ray)];
    alignas(64) unsigned char hit_mem[sizeof(RayHit)];
    SceneTracer *tracer;
    SurfaceShader *surface;
    Ray *ray;
    RayHit *hit;

    void fresh() {
        memset(tracer_mem, 0, sizeof(tracer_mem));
        memset(surface_mem, 0, sizeof(surface_mem));
        memset(ray_mem, 0, sizeof(ray_mem));
        memset(hit_mem, 0, sizeof(hit_mem));
        tracer = new (tracer_mem) SceneTracer{scene_stack, mesh_stack};
        surface = new (surface_mem) SurfaceShader{};
        ray = new (ray_mem) Ray{};
        hit = new (hit_mem) RayHit{};
    }
};

// Runs fn(y0, y1) over [0, rows) on `threads` host threads.  Rows are
// claimed dynamically in chunks of 4 (an atomic counter), so threads whose
// rows are cheap (sky) take more of them and the frame ends when the work
// does, not when the most expensive static band does.
// A zeroed context: the reference app's tracer stacks come from zeroed
// pages (os::getMemory), and its traversal may read a stack slot it has not
// written in this pixel, so they must start as zero here too.
PixelContext *new_context() {
    PixelContext *ctx = (PixelContext*)aligned_alloc(64, sizeof(PixelContext));
    if (ctx) memset((void*)ctx, 0, sizeof(PixelContext));
    return ctx;
}

template <typename Fn>
void parallel_rows(int rows, int threads, Fn fn) {
    if (threads <= 1) { fn(0, rows); return; }
    constexpr int kChunk = 4;
    std::atomic<int> next{0};
    auto worker = [&]() {
        for (;;) {
            int y0 = next.fetch_add(kChunk);
            if (y0 >= rows) break;
            fn(y0, y0 + kChunk < rows ? y0 + kChunk : rows);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; t++) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
}
}  // namespace

extern "C" {

int ref_abi_version() { return 1; }

// CameraRayProjection::reset (scene/camera.h:69-83) from an orientation
// matrix given column-wise as X(right), Y(up), Z(forward).
int ref_projection_reset(const float *orientation9, const float *position3, float focal_length,
                         int width, int height, int antialias_ssaa, void *out_projection) {
    Camera camera;
    mat3 m{orientation9[0], orientation9[1], orientation9[2],
           orientation9[3], orientation9[4], orientation9[5],
           orientation9[6], orientation9[7], orientation9[8]};
    camera.orientation = m;
    camera.position = vec3{position3[0], position3[1], position3[2]};
    camera.focal_length = focal_length;
    Dimensions dim;
    dim.update((u16)width, (u16)height);
    CameraRayProjection projection;
    projection.reset(camera, dim, antialias_ssaa != 0);
    memcpy(out_projection, &projection, sizeof(projection));
    return 0;
}

// Scene::Scene's AABB/BVH pass (scene/scene.h:156-191): fills scene->bvh.nodes
// (capacity 2*geometries), bvh.node_count/height, bvh_leaf_geometry_indices
// and the SCENE_HAD_EMISSIVE_QUADS flag of a caller-owned SceneData.
int ref_build_scene_bvh(void *scene_data) {
    SceneData *sd = (SceneData*)scene_data;
    if (!sd || !sd->counts.geometries) return 1;
    SceneCounts counts;
    counts.geometries = sd->counts.geometries;
    counts.cameras = sd->counts.cameras;
    counts.lights = sd->counts.lights;
    counts.materials = sd->counts.materials;
    // Meshes/textures are attached in memory already; the constructor would
    // otherwise try to load them from files.
    Scene *scene = new Scene{counts, sd->geometries, sd->cameras, sd->lights, sd->materials,
                             nullptr, nullptr, sd->meshes, nullptr};
    memcpy(sd->bvh.nodes, scene->bvh.nodes, sizeof(BVHNode) * scene->bvh.node_count);
    sd->bvh.node_count = scene->bvh.node_count;
    sd->bvh.height = scene->bvh.height;
    memcpy(sd->bvh_leaf_geometry_indices, scene->bvh_leaf_geometry_indices,
           sizeof(u32) * sd->counts.geometries);
    sd->flags = scene->flags;
    // The Scene's arena was taken from os::getMemory and is never released
    // by the reference; the wrapper object itself is freed here.
    ::operator delete(scene);
    return 0;
}

// obj2mesh after parsing (obj2mesh.cpp:201-231, scale 1, no rotation):
// recentre on the AABB centre, then BVHBuilder::buildMesh.  Outputs the
// leaf-ordered triangles, the BVH nodes and the centred AABB.
int ref_build_mesh(const float *positions, u32 vertex_count, const u32 *position_indices,
                   u32 triangle_count, const float *normals, u32 normals_count,
                   const u32 *normal_indices, const float *uvs, u32 uvs_count,
                   const u32 *uv_indices, void *out_triangles, void *out_nodes,
                   u32 *out_node_count, u32 *out_height, float *out_aabb6,
                   float *out_positions) {
    Mesh mesh;
    mesh.triangle_count = triangle_count;
    mesh.vertex_count = vertex_count;
    mesh.normals_count = normals_count;
    mesh.uvs_count = uvs_count;
    mesh.edge_count = 0;
    std::vector<vec3> pos(vertex_count);
    for (u32 i = 0; i < vertex_count; i++) pos[i] = vec3{positions[3*i], positions[3*i+1], positions[3*i+2]};
    std::vector<vec3> nrm(normals_count);
    for (u32 i = 0; i < normals_count; i++) nrm[i] = vec3{normals[3*i], normals[3*i+1], normals[3*i+2]};
    std::vector<vec2> uv(uvs_count);
    for (u32 i = 0; i < uvs_count; i++) uv[i] = vec2{uvs[2*i], uvs[2*i+1]};
    std::vector<TriangleVertexIndices> pidx(triangle_count), nidx(triangle_count), uidx(triangle_count);
    for (u32 i = 0; i < triangle_count; i++)
        for (int k = 0; k < 3; k++) {
            pidx[i].ids[k] = position_indices[3*i+k];
            if (normals_count) nidx[i].ids[k] = normal_indices[3*i+k];
            if (uvs_count) uidx[i].ids[k] = uv_indices[3*i+k];
        }
    mesh.vertex_positions = pos.data();
    mesh.vertex_normals = normals_count ? nrm.data() : nullptr;
    mesh.vertex_uvs = uvs_count ? uv.data() : nullptr;
    mesh.vertex_position_indices = pidx.data();
    mesh.vertex_normal_indices = normals_count ? nidx.data() : nullptr;
    mesh.vertex_uvs_indices = uvs_count ? uidx.data() : nullptr;

    std::vector<Triangle> tris(triangle_count);
    std::vector<BVHNode> nodes(triangle_count * 2 + 2);
    mesh.triangles = tris.data();
    mesh.bvh.nodes = nodes.data();
    mesh.bvh.node_count = triangle_count * 2;
    mesh.bvh.height = (u8)triangle_count;

    f32 scale = 1;
    mesh.aabb.min = INFINITY;
    mesh.aabb.max = -INFINITY;
    for (u32 i = 0; i < mesh.vertex_count; i++) {
        vec3 &position = mesh.vertex_positions[i];
        position *= scale;
        mesh.aabb.min = minimum(mesh.aabb.min, position);
        mesh.aabb.max = maximum(mesh.aabb.max, position);
    }
    vec3 centroid = (mesh.aabb.min + mesh.aabb.max) / 2.0f;
    if (centroid.nonZero()) {
        mesh.aabb.min -= centroid;
        mesh.aabb.max -= centroid;
        for (u32 i = 0; i < mesh.vertex_count; i++)
            mesh.vertex_positions[i] -= centroid;
    }

    u64 builder_bytes = BVHBuilder::getSizeInBytes(triangle_count * 2);
    memory::MonotonicAllocator allocator{builder_bytes};
    BVHBuilder builder{triangle_count * 2, &allocator};
    builder.buildMesh(mesh);

    memcpy(out_triangles, tris.data(), sizeof(Triangle) * triangle_count);
    memcpy(out_nodes, nodes.data(), sizeof(BVHNode) * mesh.bvh.node_count);
    *out_node_count = mesh.bvh.node_count;
    *out_height = mesh.bvh.height;
    out_aabb6[0] = mesh.aabb.min.x; out_aabb6[1] = mesh.aabb.min.y; out_aabb6[2] = mesh.aabb.min.z;
    out_aabb6[3] = mesh.aabb.max.x; out_aabb6[4] = mesh.aabb.max.y; out_aabb6[5] = mesh.aabb.max.z;
    if (out_positions) memcpy(out_positions, pos.data(), sizeof(vec3) * vertex_count);
    free(allocator.address - allocator.occupied);
    return 0;
}

// The per-pixel body of d_render (renderer/renderer_GPU.h:22-46) on host
// threads: primary direction start + down*y + right*x, the d_render
// scaling factor, renderPixel (renderer/ray_tracer.h:144) and
// Canvas::setPixel(x, y, color, -1, depth) (draw/canvas.h:128-185).
// Rows [row_begin, row_end) of the (SSAA-doubled) sample grid are rendered.
int ref_render(const void *scene_data, const void *canvas_data, const void *projection_data,
               const void *settings_data, int row_begin, int row_end, int threads) {
    const Scene &scene = *(const Scene*)scene_data;
    const Canvas &canvas = *(const Canvas*)canvas_data;
    const CameraRayProjection &projection = *(const CameraRayProjection*)projection_data;
    const RayTracerSettings &settings = *(const RayTracerSettings*)settings_data;
    u32 s = canvas.antialias == SSAA ? 2 : 1;
    i32 width = (i32)canvas.dimensions.width * (i32)s;
    i32 height = (i32)canvas.dimensions.height * (i32)s;
    if (row_end > height) row_end = height;
    if (row_begin < 0) row_begin = 0;
    if (row_begin >= row_end) return 0;
    parallel_rows(row_end - row_begin, threads, [&](int y0, int y1) {
        PixelContext *ctx = new_context();
        Color color;
        f32 depth;
        for (i32 y = row_begin + y0; y < row_begin + y1; y++)
            for (i32 x = 0; x < width; x++) {
                ctx->fresh();
                ctx->ray->pixel_coords.x = x;
                ctx->ray->pixel_coords.y = y;
                ctx->hit->scaling_factor = 1.0f / sqrtf(projection.squared_distance_to_projection_plane +
                    vec2{(f32)x, (f32)-y}.scaleAdd(projection.sample_size, projection.C_start).squaredLength());
                renderPixel(settings, projection, (Scene&)scene, *ctx->tracer, *ctx->surface,
                            *ctx->ray, *ctx->hit, projection.getRayDirectionAt(x, y), color, depth);
                canvas.setPixel(x, y, color, -1, depth);
            }
        free(ctx);
    });
    return 0;
}

// The unmodified single-threaded CPU path RayTracingRenderer::renderOnCPU
// (renderer/renderer.h:87-100): incremental ray directions, one persistent
// tracer/shader/ray/hit for the whole frame.  The projection is copied
// because renderOnCPU advances projection.start row by row.
int ref_render_cpu(const void *scene_data, const void *canvas_data, const void *projection_data,
                   const void *settings_data) {
    Scene &scene = *(Scene*)scene_data;
    const Canvas &canvas = *(const Canvas*)canvas_data;
    CameraRayProjection projection = *(const CameraRayProjection*)projection_data;
    const RayTracerSettings &settings = *(const RayTracerSettings*)settings_data;
    PixelContext *ctx = new_context();
    ctx->fresh();
    void *renderer_mem = calloc(1, sizeof(RayTracingRenderer));
    RayTracingRenderer *renderer = new (renderer_mem) RayTracingRenderer{
        scene, *ctx->tracer, projection, settings.max_depth,
        settings.skybox_color_texture_id, settings.skybox_radiance_texture_id,
        settings.skybox_irradiance_texture_id, settings.render_mode};
    renderer->settings = settings;
    renderer->renderOnCPU(canvas);
    free(renderer_mem);
    free(ctx);
    return 0;
}

// Closest hit of every primary ray, as renderPixelBeauty's first trace
// (renderer/ray_tracer.h:36-45): geometry index (-1 on miss), the mesh
// triangle id in leaf order (0 for implicit primitives), the hit distance
// and whether the surface was hit from behind.
int ref_trace_primary(const void *scene_data, const void *projection_data, int width, int height,
                      int *geometry_ids, unsigned *primitive_ids, float *distances,
                      unsigned char *from_behind, int threads) {
    const Scene &scene = *(const Scene*)scene_data;
    const CameraRayProjection &projection = *(const CameraRayProjection*)projection_data;
    parallel_rows(height, threads, [&](int y0, int y1) {
        PixelContext *ctx = new_context();
        for (i32 y = y0; y < y1; y++)
            for (i32 x = 0; x < width; x++) {
                ctx->fresh();
                ctx->ray->reset(projection.camera_position, projection.getRayDirectionAt(x, y).normalized());
                ctx->ray->depth = ctx->tracer->aux_ray.depth = 1;
                Geometry *geo = ctx->tracer->trace(*ctx->ray, *ctx->hit, (Scene&)scene);
                size_t o = (size_t)y * width + x;
                if (geo) {
                    geometry_ids[o] = (int)(geo - scene.geometries);
                    primitive_ids[o] = geo->type == GeometryType_Mesh ? ctx->hit->id : 0;
                    distances[o] = ctx->hit->distance;
                    from_behind[o] = ctx->hit->from_behind;
                } else {
                    geometry_ids[o] = -1;
                    primitive_ids[o] = 0;
                    distances[o] = INFINITY;
                    from_behind[o] = 0;
                }
            }
        free(ctx);
    });
    return 0;
}

// Sizes of the records a scene file holds (serialization/scene.h:5-109):
// Camera, its OrientationUsing3x3Matrix, Grid, Box, Curve, SceneCounts,
// ImageInfo, Geometry.
int ref_scene_record_sizes(unsigned *out) {
    out[0] = sizeof(Camera); out[1] = sizeof(OrientationUsing3x3Matrix); out[2] = sizeof(Grid);
    out[3] = sizeof(Box); out[4] = sizeof(Curve); out[5] = sizeof(SceneCountsData); out[6] = sizeof(ImageInfo);
    out[7] = sizeof(Geometry);
    return 0;
}

// save(Scene&, SceneIO&) (serialization/scene.h:59-109) on a caller-owned
// SceneData (counts, cameras, geometries, grids, boxes, curves, meshes,
// textures are the members it reads).
int ref_save_scene(void *scene_data, const char *path) {
    SceneIO io;
    io.file_path = String(path);
    save(*(Scene*)scene_data, io);
    return 0;
}

// load(Scene&, SceneIO&) (serialization/scene.h:5-57) into caller-allocated
// arrays sized from the file (the reference's own app sizes them from the
// mesh and texture files it loads first).
int ref_load_scene(void *scene_data, const char *path) {
    SceneIO io;
    io.file_path = String(path);
    load(*(Scene*)scene_data, io);
    return 0;
}

}  // extern "C"
