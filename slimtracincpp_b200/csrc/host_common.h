// Shared host-side declarations of libslimtracer_b200 (error state and the
// host algorithms in host_assets.cpp / texture_baker.cpp).
#pragma once
#include <cstdint>
#include "slimtracer_b200.h"

namespace slim {

// Records a message for slimGetLastError() and returns `code`.
int set_error(int code, const char *message);
const char *last_error();

void geometry_world_box(const SlimSceneData &s, uint32_t g, float out_min[3], float out_max[3]);
int build_scene_bvh(SlimSceneData *s);
int build_mesh(float *positions, uint32_t vertex_count, const uint32_t *pidx, uint32_t tri_count,
               const float *normals, uint32_t normals_count, const uint32_t *nidx, const float *uvs,
               uint32_t uvs_count, const uint32_t *uidx, SlimTriangle *out_tris, SlimBVHNode *out_nodes,
               uint32_t *out_node_count, uint32_t *out_height, float out_aabb6[6]);
int projection_reset(const float o[9], const float p[3], float focal_length, int width, int height,
                     int ssaa, SlimCameraRayProjection *out);
int read_mesh_header(const char *path, SlimMesh *m);
int read_mesh(const char *path, SlimMesh *m);
int write_mesh(const char *path, const SlimMesh *m);
int read_texture_header(const char *path, SlimTexture *t, uint32_t *total_quads);
int read_texture(const char *path, SlimTexture *t, SlimTextureMip *mips, SlimTexelQuad *quads);
int write_texture(const char *path, const SlimTexture *t);
int save_scene(const char *path, const SlimSceneFile *scene);
int read_scene_header(const char *path, SlimSceneFile *scene, uint32_t *texel_quad_counts);
int load_scene(const char *path, SlimSceneFile *scene);
int bake_texture(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels, uint32_t flags,
                 SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *quads, uint32_t *mip_count,
                 uint32_t *quad_count);
float bake_component(uint8_t c, bool linear);

}  // namespace slim
