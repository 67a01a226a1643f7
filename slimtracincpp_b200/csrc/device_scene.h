// Device-side (HBM) layout of a scene for the B200 trace kernels.
//
// Everything is stored as 16-byte vectors so a record is one or a few
// 128-bit loads:
//   geometry       4 x float4   rotation quat | position,type | scale,material | 1/scale,flags+mesh
//   BVH node       2 x float4   the reference's 32-byte BVHNode bytes unchanged
//                               (min.xyz, max.x | max.yz, first_index, leaf_count/depth/flags)
//   triangle hot   3 x float4   position, normal and the two rows of local_to_tangent
//                               the hit test reads (48 B of the reference's 128 B)
//   triangle cold  4 x float4   n1..n3, uv1..uv3, uv_coverage (read once per mesh hit)
//   texel quad     1 x uint4    R, G, B byte quads + 4 bytes padding (one load per bilinear tap)
// Mesh and texture arrays of all assets are concatenated; per-asset offsets
// live in DevMesh / DevTexture / DevMip.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "slimtracer_b200.h"

namespace slim {

constexpr int kStackCapacity = 64;
// Mesh-BVH leaves waiting in the persistent mesh kernels are packed as
// first triangle | count << kLeafCountShift: meshes hold fewer than 2^26
// triangles and leaves below the root fewer than 64 (checked on upload; the
// reference's builder makes leaves of at most two).
constexpr uint32_t kLeafCountShift = 26;        // per-ray traversal stack entries (scene and mesh)
constexpr int kMaxLights = 64;            // lights a shadow mask can track
constexpr uint32_t kErrStack = 1u;        // device error bits
constexpr uint32_t kErrIndex = 2u;

struct DevMesh {
    float aabb_min[3], aabb_max[3];
    uint32_t node_offset;     // into mesh_nodes (in nodes)
    uint32_t tri_offset;      // into tri_hot / tri_cold (in triangles)
    uint32_t tri_count;
    uint32_t node_count;
    uint32_t has_normals, has_uvs;
};

struct DevMip {
    uint32_t width, height;
    uint32_t quad_offset;     // into quads
    uint32_t _pad;
};

struct DevTexture {
    uint32_t width, height, mip_count, flags;
    uint32_t mip_base;        // into mips
    uint32_t _pad[3];
};

struct DevScene {
    const float4 *geometries;      // 4 float4 per geometry
    const SlimMaterial *materials;
    const SlimLight *lights;
    const float4 *scene_nodes;     // 2 float4 per node
    const uint32_t *leaf_geometry; // bvh_leaf_geometry_indices
    const DevMesh *meshes;
    const float4 *mesh_nodes;
    const float4 *tri_hot;
    const float4 *tri_cold;
    const DevTexture *textures;
    const DevMip *mips;
    const uint4 *quads;
    const uint32_t *emissive_quads; // geometry ids of emissive quads, in geometry order
    uint32_t geometry_count, material_count, light_count, texture_count, mesh_count;
    uint32_t emissive_quad_count;
    uint32_t flags;                // SLIM_SCENE_HAD_EMISSIVE_QUADS
    uint32_t scene_node_count;
};

// Per-frame parameters of a render launch.
struct DevFrame {
    SlimCameraRayProjection projection;
    SlimRayTracerSettings settings;
    uint32_t width, height;        // sample grid (doubled under SSAA)
    uint32_t row_begin, rows;      // the sample rows [row_begin, row_begin + rows) this launch renders
    uint32_t stride;               // canvas stride in pixels
    int32_t antialias;
    int32_t cones_per_pixel;
    float4 *pixels;
    float *depths;
    uint32_t *error_flags;
    unsigned long long *counters;  // SlimWorkCounters fields, or null
    uint32_t cache_depth;          // batched requests: path vertex answered by the radiance cache (0 = none)
};

}  // namespace slim
