"""numpy mirrors of the POD structs in include/slimtracer_b200.h.

Each dtype has the byte layout of the reference's struct on LP64 with a
4-byte u32 (the C header static-asserts the same sizes), so arrays of these
dtypes are passed to the C ABI by pointer.
"""
from __future__ import annotations

import numpy as np

# ---- enums / flags (core/base.h, scene/material.h, scene/scene.h) ---------
GEOMETRY_NONE, GEOMETRY_MESH, GEOMETRY_GRID, GEOMETRY_BOX, GEOMETRY_CURVE, GEOMETRY_TET, GEOMETRY_QUAD, \
    GEOMETRY_SPHERE, GEOMETRY_LIGHT = range(9)
BRDF_LAMBERT, BRDF_BLINN, BRDF_PHONG, BRDF_COOK_TORRANCE = range(4)
RENDER_NORMALS, RENDER_NORMAL_MAP, RENDER_BEAUTY, RENDER_DEPTH, RENDER_MIP_LEVEL, RENDER_UVS = range(6)
AA_NONE, AA_MSAA, AA_SSAA = range(3)
MATERIAL_IS_REFLECTIVE = 1
MATERIAL_IS_REFRACTIVE = 2
MATERIAL_IS_EMISSIVE = 4
MATERIAL_HAS_ALBEDO_MAP = 16
MATERIAL_HAS_NORMAL_MAP = 32
GEOMETRY_IS_VISIBLE = 1
GEOMETRY_IS_SHADOWING = 2
GEOMETRY_IS_TRANSPARENT = 4
LIGHT_IS_DIRECTIONAL = 1
LIGHT_IS_SHADOWING = 2
SCENE_HAD_EMISSIVE_QUADS = 1
IMAGE_ALPHA, IMAGE_LINEAR, IMAGE_TILE, IMAGE_CHANNEL, IMAGE_MIPMAP, IMAGE_FLIP, IMAGE_WRAP, IMAGE_NORMAL, \
    IMAGE_CUBEMAP = (1 << i for i in range(9))
ENGINE_WAVEFRONT, ENGINE_MEGAKERNEL, ENGINE_AUTO = 0, 1, 2
CONES_REFERENCE, CONES_PER_PIXEL = 0, 1
SCENE_BVH_UPLOADED, SCENE_BVH_REFIT = 0, 1

# ColorID values used by RayTracerSettings.mip_level_colors (core/base.h:626-662)
BRIGHT_RED, BRIGHT_GREEN, BRIGHT_BLUE, BRIGHT_GREY = 13, 14, 15, 16
BRIGHT_CYAN, BRIGHT_MAGENTA, BRIGHT_YELLOW = 17, 18, 19
GREY, DARK_GREY = 2, 12
F0_DEFAULT, F0_GLASS_LOW, F0_ALUMINIUM = 23, 25, 34
IOR_AIR = np.float32(1.0003)
IOR_GLASS = np.float32(1.52)

f4, u4, i4, u2, u1, i1, u8 = "<f4", "<u4", "<i4", "<u2", "u1", "i1", "<u8"


def _dt(fields, itemsize):
    names = [f[0] for f in fields]
    formats = [f[1] for f in fields]
    offsets = [f[2] for f in fields]
    dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": itemsize})
    return dt


GEOMETRY = _dt([("axis", (f4, 3), 0), ("amount", f4, 12), ("euler", (f4, 3), 16), ("position", (f4, 3), 28),
                ("scale", (f4, 3), 40), ("type", i4, 52), ("material_id", u4, 56), ("id", u4, 60),
                ("flags", u1, 64), ("color", i4, 68)], 72)
MATERIAL = _dt([("albedo", (f4, 3), 0), ("roughness", f4, 12), ("flags", u1, 16), ("texture_count", u1, 17),
                ("texture_ids", (u1, 2), 18), ("brdf", i4, 20), ("normal_magnitude", f4, 24),
                ("uv_repeat", (f4, 2), 28), ("emission", (f4, 3), 36), ("IOR", f4, 48),
                ("reflectivity", (f4, 3), 52), ("metalness", f4, 64)], 68)
LIGHT = _dt([("color", (f4, 3), 0), ("position", (f4, 3), 12), ("intensity", f4, 24), ("flags", u1, 28)], 32)
BVH_NODE = _dt([("min", (f4, 3), 0), ("max", (f4, 3), 12), ("first_index", u4, 24), ("leaf_count", u2, 28),
                ("depth", u1, 30), ("flags", u1, 31)], 32)
TRIANGLE = _dt([("local_to_tangent", (f4, 9), 0), ("position", (f4, 3), 36), ("normal", (f4, 3), 48),
                ("n1", (f4, 3), 60), ("n2", (f4, 3), 72), ("n3", (f4, 3), 84), ("uv1", (f4, 2), 96),
                ("uv2", (f4, 2), 104), ("uv3", (f4, 2), 112), ("uv_coverage", f4, 120), ("padding", f4, 124)], 128)
TEXEL_QUAD = _dt([("R", (u1, 4), 0), ("G", (u1, 4), 4), ("B", (u1, 4), 8)], 12)
TEXTURE_MIP = _dt([("width", u4, 0), ("height", u4, 4), ("texel_quads", u8, 8)], 16)
TEXTURE = _dt([("width", u4, 0), ("height", u4, 4), ("size", u4, 8), ("stride", u4, 12), ("tile_width", u4, 16),
               ("tile_height", u4, 20), ("mip_count", u4, 24), ("flags", u4, 28), ("mips", u8, 32)], 40)
MESH = _dt([("aabb_min", (f4, 3), 0), ("aabb_max", (f4, 3), 12), ("bvh_nodes", u8, 24), ("bvh_node_count", u4, 32),
            ("bvh_height", u1, 36), ("triangles", u8, 40), ("vertex_positions", u8, 48), ("vertex_normals", u8, 56),
            ("vertex_uvs", u8, 64), ("vertex_position_indices", u8, 72), ("vertex_normal_indices", u8, 80),
            ("vertex_uvs_indices", u8, 88), ("edge_vertex_indices", u8, 96), ("triangle_count", u4, 104),
            ("vertex_count", u4, 108), ("edge_count", u4, 112), ("normals_count", u4, 116), ("uvs_count", u4, 120)], 128)
SCENE_DATA = _dt([("counts", (u4, 11), 0), ("flags", u2, 44), ("mesh_stack_size", u2, 46), ("geometries", u8, 48),
                  ("cameras", u8, 56), ("lights", u8, 64), ("materials", u8, 72), ("textures", u8, 80),
                  ("meshes", u8, 88), ("grids", u8, 96), ("boxes", u8, 104), ("tets", u8, 112), ("quads", u8, 120),
                  ("curves", u8, 128), ("aabbs", u8, 136), ("io", u8, 144), ("bvh_builder", u8, 152),
                  ("bvh_leaf_geometry_indices", u8, 160), ("bvh_nodes", u8, 168), ("bvh_node_count", u4, 176),
                  ("bvh_height", u1, 180)], 184)
CAMERA = _dt([("orientation", (f4, 9), 0), ("rotation", (f4, 3), 36), ("position", (f4, 3), 48),
              ("current_velocity", (f4, 3), 60), ("focal_length", f4, 72), ("zoom_amount", f4, 76),
              ("target_distance", f4, 80), ("dolly_amount", f4, 84)], 88)
SCENE_FILE = _dt([("counts", (u4, 11), 0), ("cameras", u8, 48), ("geometries", u8, 56), ("meshes", u8, 64),
                  ("textures", u8, 72), ("grids", u8, 80), ("boxes", u8, 88), ("curves", u8, 96)], 104)
GRID_BYTES, BOX_BYTES, CURVE_BYTES = 9700, 384, 12
COUNT_GEOMETRIES, COUNT_CAMERAS, COUNT_LIGHTS, COUNT_MATERIALS, COUNT_TEXTURES, COUNT_MESHES = 0, 1, 2, 3, 4, 5
COUNT_GRIDS, COUNT_BOXES, COUNT_TETS, COUNT_QUADS, COUNT_CURVES = 6, 7, 8, 9, 10
CANVAS_DATA = _dt([("width_times_height", u4, 0), ("width_over_height", f4, 4), ("height_over_width", f4, 8),
                   ("f_width", f4, 12), ("f_height", f4, 16), ("h_width", f4, 20), ("h_height", f4, 24),
                   ("width", u2, 28), ("height", u2, 30), ("stride", u2, 32), ("antialias", i4, 36),
                   ("pixels", u8, 40), ("depths", u8, 48)], 56)
PROJECTION = _dt([("inverted_camera_rotation", (f4, 9), 0), ("start", (f4, 3), 36), ("right", (f4, 3), 48),
                  ("down", (f4, 3), 60), ("camera_position", (f4, 3), 72), ("C_start", (f4, 2), 84),
                  ("squared_distance_to_projection_plane", f4, 92), ("sample_size", f4, 96)], 100)
SETTINGS = _dt([("max_depth", u1, 0), ("skybox_color_texture_id", i1, 1), ("skybox_radiance_texture_id", i1, 2),
                ("skybox_irradiance_texture_id", i1, 3), ("render_mode", i4, 4), ("mip_level_colors", (i4, 9), 8)], 44)
RENDER_OPTIONS = _dt([("engine", i4, 0), ("ray_cones", i4, 4), ("scene_bvh", i4, 8), ("block_size", i4, 12),
                      ("count_work", i4, 16), ("profile_stages", i4, 20), ("shadow_queue_mb", i4, 24),
                      ("radiance_cache", i4, 28), ("row_bands", i4, 32)], 36)
CACHE_CONFIG = _dt([("cache_depth", u4, 0), ("train_samples", u4, 4), ("batch", u4, 8), ("seed", u4, 12),
                    ("learning_rate", f4, 16), ("beta1", f4, 20), ("beta2", f4, 24), ("epsilon", f4, 28),
                    ("train", u4, 32), ("overlap", u4, 36), ("train_suffix", u4, 40), ("_reserved", u4, 44)], 48)
CACHE_STATE_HEADER = _dt([("magic", u4, 0), ("params", u4, 4), ("steps", u4, 8), ("frames", u4, 12),
                          ("config", CACHE_CONFIG, 16)], 64)
CACHE_STATS = _dt([("frames", u8, 0), ("steps", u8, 8), ("queries", u4, 16), ("train_samples", u4, 20),
                   ("loss", f4, 24), ("_pad", f4, 28)], 32)
CACHE_OFF, CACHE_ON, CACHE_TRUNCATE, CACHE_EXACT = 0, 1, 2, 3
RENDER_REQUEST = _dt([("scene", u8, 0), ("projection", PROJECTION, 8), ("settings", SETTINGS, 108),
                      ("width", u4, 152), ("height", u4, 156), ("radiance_cache", i4, 160), ("_pad", u4, 164),
                      ("d_pixels", u8, 168), ("d_depths", u8, 176)], 184)
PICK = _dt([("geometry", i4, 0), ("light", i4, 4), ("triangle", u4, 8), ("distance", f4, 12),
            ("position", (f4, 3), 16), ("from_behind", u4, 28)], 32)
BATCH_PLAN = _dt([("queue_capacity", u4, 0), ("tile_pixels", u4, 4), ("block_size", i4, 8), ("waves", u4, 12),
                  ("batch_ms", f4, 16), ("candidates", u4, 20), ("graph_nodes", u4, 24), ("tuned", u4, 28),
                  ("persistent", u4, 32), ("_pad", u4, 36)], 40)
NRC_PARAMS = 18624
NRC_STATE_MAGIC = 0x4B43524E
NRC_STATE_BYTES = 64 + 3 * NRC_PARAMS * 4
NRC_FEATURES = 16
WORK_COUNTERS = _dt([(n, u8, 8 * i) for i, n in enumerate(
    ["primary_rays", "shadow_rays", "bounce_rays", "scene_node_tests", "mesh_node_tests", "triangle_tests",
     "geometry_tests", "mesh_hit_fetches", "texel_taps", "pixels", "shadow_scene_node_tests",
     "shadow_mesh_node_tests", "shadow_triangle_tests", "shadow_geometry_tests"])], 112)
STAGE_STATS = _dt([("name", "S24", 0), ("launches", u4, 24), ("total_ms", f4, 28), ("work", WORK_COUNTERS, 32)], 144)

for _name, _dtype, _size in [("GEOMETRY", GEOMETRY, 72), ("MATERIAL", MATERIAL, 68), ("LIGHT", LIGHT, 32),
                             ("BVH_NODE", BVH_NODE, 32), ("TRIANGLE", TRIANGLE, 128), ("TEXEL_QUAD", TEXEL_QUAD, 12),
                             ("TEXTURE_MIP", TEXTURE_MIP, 16), ("TEXTURE", TEXTURE, 40), ("MESH", MESH, 128),
                             ("SCENE_DATA", SCENE_DATA, 184), ("CANVAS_DATA", CANVAS_DATA, 56),
                             ("PROJECTION", PROJECTION, 100), ("SETTINGS", SETTINGS, 44)]:
    assert _dtype.itemsize == _size, (_name, _dtype.itemsize)


def default_material(albedo=1.0, roughness=1.0, flags=0, brdf=BRDF_COOK_TORRANCE, texture_ids=(), normal_magnitude=1.0,
                     uv_repeat=(1.0, 1.0), emission=0.0, ior=1.0, reflectivity=0.04, metalness=0.0):
    """A Material record with the reference's defaults (scene/material.h:93-110)."""
    m = np.zeros((), MATERIAL)
    m["albedo"] = np.broadcast_to(np.float32(albedo), 3)
    m["roughness"] = roughness
    m["flags"] = flags
    m["texture_count"] = len(texture_ids)
    ids = list(texture_ids) + [0] * (2 - len(texture_ids))
    m["texture_ids"] = ids[:2]
    m["brdf"] = brdf
    m["normal_magnitude"] = normal_magnitude
    m["uv_repeat"] = uv_repeat
    m["emission"] = np.broadcast_to(np.float32(emission), 3)
    m["IOR"] = ior
    m["reflectivity"] = np.broadcast_to(np.float32(reflectivity), 3)
    m["metalness"] = metalness
    return m


def default_settings(max_depth=3, skybox_color=-1, skybox_radiance=-1, skybox_irradiance=-1,
                     render_mode=RENDER_BEAUTY):
    """RayTracerSettings as RayTracingRenderer's constructor fills it
    (renderer/renderer.h:36-61)."""
    s = np.zeros((), SETTINGS)
    s["max_depth"] = max_depth
    s["skybox_color_texture_id"] = skybox_color
    s["skybox_radiance_texture_id"] = skybox_radiance
    s["skybox_irradiance_texture_id"] = skybox_irradiance
    s["render_mode"] = render_mode
    s["mip_level_colors"] = [BRIGHT_RED, BRIGHT_YELLOW, BRIGHT_GREEN, BRIGHT_MAGENTA, BRIGHT_CYAN, BRIGHT_BLUE,
                             BRIGHT_GREY, GREY, DARK_GREY]
    return s
