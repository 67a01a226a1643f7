#!/usr/bin/env python3
"""Regenerates the golden cases in tests/golden/ from the REFERENCE itself.

Each case stores a seeded scene's input arrays together with what the
reference's own code (oracle/_ref/libslimref.so, compiled from the
reference's sources by oracle/build_ref.sh) computes for it:

  render_*.npz   Canvas pixels + depths of the per-pixel path
                 (renderPixel + Canvas::setPixel, renderer/ray_tracer.h:144)
                 and the primary-ray hit ids/distances (scene/scene_tracer.h:26)
  bvh_*.npz      Scene::updateBVH output (scene/scene.h:176-191)
  mesh_*.npz     obj2mesh's BVHBuilder::buildMesh output (scene/bvh_builder.h:265)
  projection.npz CameraRayProjection::reset for several cameras (scene/camera.h:69)

Run on a machine holding the reference sources:
    bash oracle/build_ref.sh && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from golden_io import scene_arrays  # noqa: E402
from oracle import bindings as O  # noqa: E402
from slimtracincpp_b200 import layout as L  # noqa: E402
from slimtracincpp_b200 import scenes  # noqa: E402
from slimtracincpp_b200.scene import Camera, Scene, geometry  # noqa: E402

RENDER_CASES = {
    "render_config1": lambda: (scenes.config1(11, 80, 45), L.AA_NONE, None),
    "render_config1_ssaa": lambda: (scenes.config1(12, 40, 24), L.AA_SSAA, None),
    "render_mesh": lambda: (scenes.small_mesh_scene(5, 80, 45), L.AA_NONE, None),
    "render_mesh_normals": lambda: (scenes.small_mesh_scene(6, 64, 36), L.AA_NONE, L.RENDER_NORMALS),
    "render_features": lambda: (scenes.feature_scene(7, 96, 54), L.AA_NONE, None),
    "render_features_depth": lambda: (scenes.feature_scene(8, 64, 36), L.AA_NONE, L.RENDER_DEPTH),
    "render_textured_ibl": lambda: (scenes.small_textured_scene(9, 64, 36), L.AA_NONE, None),
}


def render_case(name, make):
    w, aa, mode = make()
    settings = w.settings.copy()
    if mode is not None:
        settings["render_mode"] = mode
    ssaa = aa == L.AA_SSAA
    proj = O.reference_projection(w.camera, w.width, w.height, ssaa, L)
    pix, dep = O.reference_render(w.scene, proj, settings, w.width, w.height, antialias=aa, layout=L)
    g, p, d, b = O.reference_trace_primary(w.scene, proj, w.width * (2 if ssaa else 1), w.height * (2 if ssaa else 1))
    np.savez_compressed(HERE / f"{name}.npz", **scene_arrays(w.scene, w.camera), settings=settings.reshape(1).view(np.uint8),
                        width=w.width, height=w.height, antialias=aa, projection=proj.reshape(1).view(np.uint8),
                        pixels=pix, depths=dep, geometry_ids=g, primitive_ids=p, distances=d, from_behind=b)


def bvh_case(name, seed, count):
    rng = np.random.default_rng(seed)
    geos = []
    kinds = [L.GEOMETRY_BOX, L.GEOMETRY_SPHERE, L.GEOMETRY_TET, L.GEOMETRY_QUAD]
    for i in range(count):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        s = rng.uniform(0.2, 3.0, 3).astype(np.float32)
        geos.append(geometry(kinds[i % 4], 0, rng.uniform(-20, 20, 3), s, q[:3], q[3]))
    # ties: a column of identical unit boxes
    for k in range(4):
        geos.append(geometry(L.GEOMETRY_BOX, 0, (0.0, 2.0 * k, 0.0), (1, 1, 1)))
    scene = Scene(np.array(geos), np.array([L.default_material()]))
    nodes, leaf, flags, height = O.reference_scene_bvh(scene, L)
    np.savez_compressed(HERE / f"{name}.npz", geometries=scene.geometries.view(np.uint8), nodes=nodes.view(np.uint8),
                        leaf_ids=leaf, flags=flags, height=height)


def mesh_case(name, pos, idx, nrm=None, nidx=None, uv=None, uidx=None):
    tris, nodes, height, aabb, out_pos = O.reference_build_mesh(pos, idx, nrm, nidx, uv, uidx, layout=L)
    extra = {}
    if nrm is not None:
        extra.update(normals=nrm, normal_indices=nidx)
    if uv is not None:
        extra.update(uvs=uv, uv_indices=uidx)
    np.savez_compressed(HERE / f"{name}.npz", positions=pos, indices=idx, triangles=tris.view(np.uint8),
                        nodes=nodes.view(np.uint8), height=height, aabb=aabb, centred_positions=out_pos, **extra)


def projection_case():
    rng = np.random.default_rng(21)
    out = {}
    for i, (w, h, ssaa) in enumerate([(640, 360, False), (1920, 1080, False), (97, 61, True), (3840, 2160, False)]):
        cam = Camera.look_at(rng.uniform(-10, 10, 3), rng.uniform(-2, 2, 3), float(rng.uniform(30, 90)))
        proj = O.reference_projection(cam, w, h, ssaa, L)
        out[f"cam{i}_orientation"] = cam.orientation
        out[f"cam{i}_position"] = cam.position
        out[f"cam{i}_focal"] = np.float32(cam.focal_length)
        out[f"cam{i}_size"] = np.array([w, h, int(ssaa)])
        out[f"cam{i}_projection"] = proj.reshape(1).view(np.uint8)
    np.savez_compressed(HERE / "projection.npz", **out)


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libslimref.so is missing: run oracle/build_ref.sh first")
    for name, make in RENDER_CASES.items():
        render_case(name, make)
    bvh_case("bvh_scene40", 31, 40)
    bvh_case("bvh_scene7", 32, 7)
    ico = scenes.icosphere(2)
    mesh_case("mesh_icosphere2", ico[0], ico[1], ico[2], ico[1])
    hf = scenes.heightfield(np.random.default_rng(3), 12, 0.3)
    uv = (hf[0][:, [0, 2]] * 0.5 + 0.5).astype(np.float32)
    mesh_case("mesh_heightfield12_uv", hf[0], hf[1], hf[2], hf[1], uv, hf[1])
    rng = np.random.default_rng(5)
    soup = rng.uniform(-1, 1, (90, 3)).astype(np.float32)
    mesh_case("mesh_soup30", soup, np.arange(90, dtype=np.uint32).reshape(30, 3))
    projection_case()
    print("golden cases written to", HERE)


if __name__ == "__main__":
    main()
