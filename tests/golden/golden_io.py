"""Serialisation of golden cases: a scene's input arrays plus the
reference's outputs for it, in one compressed .npz per case."""
from __future__ import annotations

import numpy as np

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200.scene import Camera, MeshAsset, Scene, TextureAsset


def scene_arrays(scene: Scene, camera: Camera, prefix=""):
    out = {
        "geometries": scene.geometries.view(np.uint8),
        "materials": scene.materials.view(np.uint8),
        "lights": scene.lights.view(np.uint8),
        "camera_orientation": camera.orientation,
        "camera_position": camera.position,
        "camera_focal": np.float32(camera.focal_length),
        "mesh_count": np.int32(len(scene.meshes)),
        "texture_count": np.int32(len(scene.textures)),
    }
    for i, t in enumerate(scene.textures):
        out[f"texture{i}_header"] = t.header.reshape(1).view(np.uint8)
        out[f"texture{i}_mips"] = np.array(t.mip_sizes, np.uint32).reshape(-1, 2)
        out[f"texture{i}_quads"] = t.quads.view(np.uint8)
    for i, m in enumerate(scene.meshes):
        out[f"mesh{i}_triangles"] = m.triangles.view(np.uint8)
        out[f"mesh{i}_nodes"] = m.nodes.view(np.uint8)
        out[f"mesh{i}_aabb"] = np.concatenate([m.aabb_min, m.aabb_max])
        out[f"mesh{i}_height"] = np.int32(m.height)
        out[f"mesh{i}_positions"] = m.positions
        out[f"mesh{i}_indices"] = m.position_indices
        if m.normals is not None:
            out[f"mesh{i}_normals"] = m.normals
            out[f"mesh{i}_normal_indices"] = m.normal_indices
        if m.uvs is not None:
            out[f"mesh{i}_uvs"] = m.uvs
            out[f"mesh{i}_uv_indices"] = m.uv_indices
    return {prefix + k: v for k, v in out.items()}


def load_scene(z):
    meshes = []
    for i in range(int(z["mesh_count"])):
        g = lambda k: z[f"mesh{i}_{k}"] if f"mesh{i}_{k}" in z else None
        aabb = z[f"mesh{i}_aabb"]
        meshes.append(MeshAsset(z[f"mesh{i}_triangles"].view(L.TRIANGLE), z[f"mesh{i}_nodes"].view(L.BVH_NODE),
                                aabb[:3], aabb[3:], int(z[f"mesh{i}_height"]), g("positions"), g("indices"),
                                g("normals"), g("normal_indices"), g("uvs"), g("uv_indices")))
    textures = []
    for i in range(int(z["texture_count"]) if "texture_count" in z else 0):
        textures.append(TextureAsset(z[f"texture{i}_header"].view(L.TEXTURE).reshape(()),
                                     [tuple(m) for m in z[f"texture{i}_mips"]], z[f"texture{i}_quads"].view(L.TEXEL_QUAD)))
    scene = Scene(z["geometries"].view(L.GEOMETRY), z["materials"].view(L.MATERIAL), z["lights"].view(L.LIGHT),
                  meshes=meshes, textures=textures)
    cam = Camera(z["camera_orientation"], z["camera_position"], float(z["camera_focal"]))
    return scene, cam
