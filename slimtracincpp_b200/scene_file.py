"""Whole-scene files: the reference's save/load(Scene&, SceneIO&)
(serialization/scene.h:5-109) over slimSaveScene / slimReadSceneHeader /
slimLoadScene.

    SceneFile(geometries, meshes, textures, cameras).save("level.scene")
    f = SceneFile.load("level.scene")        # f.geometries, f.meshes, ...

A scene file holds the counts, cameras, geometries, the viewport overlay's
grids, boxes and curves (opaque records here), and every mesh and texture
in full.  Lights and materials are not part of it, as in the reference.
"""
from __future__ import annotations

import numpy as np

from . import layout as L
from .native import check, lib, ptr
from .scene import MeshAsset, TextureAsset


def camera_record(camera, zoom_amount=None, target_distance=10.0, dolly_amount=0.0, rotation=(0.0, 0.0, 0.0),
                  velocity=(0.0, 0.0, 0.0)):
    """A Camera record (scene/camera.h:6-13) from a scene.Camera pose."""
    c = np.zeros((), L.CAMERA)
    c["orientation"], c["position"], c["focal_length"] = camera.orientation, camera.position, camera.focal_length
    c["zoom_amount"] = camera.focal_length if zoom_amount is None else zoom_amount
    c["target_distance"], c["dolly_amount"] = target_distance, dolly_amount
    c["rotation"], c["current_velocity"] = rotation, velocity
    return c


class SceneFile:
    def __init__(self, geometries, meshes=(), textures=(), cameras=None, grids=None, boxes=None, curves=None):
        self.geometries = np.ascontiguousarray(geometries, dtype=L.GEOMETRY)
        self.meshes = list(meshes)
        self.textures = list(textures)
        self.cameras = np.zeros(0, L.CAMERA) if cameras is None else np.ascontiguousarray(cameras, dtype=L.CAMERA)
        self.grids = _opaque(grids, L.GRID_BYTES)
        self.boxes = _opaque(boxes, L.BOX_BYTES)
        self.curves = _opaque(curves, L.CURVE_BYTES)

    def record(self):
        """The SlimSceneFile record; keeps the mesh and texture records alive
        on the instance while it is in use."""
        self._mesh_records = np.zeros(max(1, len(self.meshes)), L.MESH)
        for i, m in enumerate(self.meshes):
            self._mesh_records[i] = m.record()
        self._texture_records = np.zeros(max(1, len(self.textures)), L.TEXTURE)
        for i, t in enumerate(self.textures):
            self._texture_records[i] = t.record()
        r = np.zeros((), L.SCENE_FILE)
        counts = np.zeros(11, np.uint32)
        counts[L.COUNT_GEOMETRIES], counts[L.COUNT_CAMERAS] = len(self.geometries), len(self.cameras)
        counts[L.COUNT_TEXTURES], counts[L.COUNT_MESHES] = len(self.textures), len(self.meshes)
        counts[L.COUNT_GRIDS], counts[L.COUNT_BOXES], counts[L.COUNT_CURVES] = len(self.grids), len(self.boxes), len(self.curves)
        r["counts"] = counts
        r["cameras"], r["geometries"] = _addr(self.cameras), _addr(self.geometries)
        r["meshes"] = ptr(self._mesh_records) if self.meshes else 0
        r["textures"] = ptr(self._texture_records) if self.textures else 0
        r["grids"], r["boxes"], r["curves"] = _addr(self.grids), _addr(self.boxes), _addr(self.curves)
        return r

    def save(self, path):
        r = self.record()
        check(lib().slimSaveScene(str(path).encode(), ptr(r)))

    @classmethod
    def load(cls, path):
        path_b = str(path).encode()
        r = np.zeros((), L.SCENE_FILE)
        check(lib().slimReadSceneHeader(path_b, ptr(r), 0))
        counts = r["counts"].copy()
        nm, nt = int(counts[L.COUNT_MESHES]), int(counts[L.COUNT_TEXTURES])
        mesh_records = np.zeros(max(1, nm), L.MESH)
        tex_records = np.zeros(max(1, nt), L.TEXTURE)
        quad_counts = np.zeros(max(1, nt), np.uint32)
        r["meshes"], r["textures"] = ptr(mesh_records), ptr(tex_records)
        check(lib().slimReadSceneHeader(path_b, ptr(r), ptr(quad_counts)))
        keep = []
        for i in range(nm):
            h = mesh_records[i]
            t, v, e = int(h["triangle_count"]), int(h["vertex_count"]), int(h["edge_count"])
            nn, nu = int(h["normals_count"]), int(h["uvs_count"])
            arrays = {"triangles": np.zeros(t, L.TRIANGLE), "nodes": np.zeros(int(h["bvh_node_count"]), L.BVH_NODE),
                      "positions": np.zeros((v, 3), np.float32), "pidx": np.zeros((t, 3), np.uint32),
                      "edges": np.zeros((e, 2), np.uint32),
                      "nrm": np.zeros((nn, 3), np.float32) if nn else None,
                      "nidx": np.zeros((t, 3), np.uint32) if nn else None,
                      "uv": np.zeros((nu, 2), np.float32) if nu else None,
                      "uidx": np.zeros((t, 3), np.uint32) if nu else None}
            h["triangles"], h["bvh_nodes"] = ptr(arrays["triangles"]), ptr(arrays["nodes"])
            h["vertex_positions"], h["vertex_position_indices"] = ptr(arrays["positions"]), ptr(arrays["pidx"])
            h["edge_vertex_indices"] = ptr(arrays["edges"])
            h["vertex_normals"], h["vertex_normal_indices"] = ptr(arrays["nrm"]), ptr(arrays["nidx"])
            h["vertex_uvs"], h["vertex_uvs_indices"] = ptr(arrays["uv"]), ptr(arrays["uidx"])
            keep.append(arrays)
        tex_arrays = []
        for i in range(nt):
            mips = np.zeros(int(tex_records[i]["mip_count"]), L.TEXTURE_MIP)
            quads = np.zeros(int(quad_counts[i]), L.TEXEL_QUAD)
            mips[0]["texel_quads"] = ptr(quads)
            tex_records[i]["mips"] = ptr(mips)
            tex_arrays.append((mips, quads))
        geos = np.zeros(int(counts[L.COUNT_GEOMETRIES]), L.GEOMETRY)
        cams = np.zeros(int(counts[L.COUNT_CAMERAS]), L.CAMERA)
        grids = np.zeros((int(counts[L.COUNT_GRIDS]), L.GRID_BYTES), np.uint8)
        boxes = np.zeros((int(counts[L.COUNT_BOXES]), L.BOX_BYTES), np.uint8)
        curves = np.zeros((int(counts[L.COUNT_CURVES]), L.CURVE_BYTES), np.uint8)
        r["counts"] = counts
        r["geometries"], r["cameras"] = _addr(geos), _addr(cams)
        r["grids"], r["boxes"], r["curves"] = _addr(grids), _addr(boxes), _addr(curves)
        check(lib().slimLoadScene(path_b, ptr(r)))
        meshes = []
        for i, a in enumerate(keep):
            h = mesh_records[i]
            meshes.append(MeshAsset(a["triangles"], a["nodes"], h["aabb_min"].copy(), h["aabb_max"].copy(),
                                    int(h["bvh_height"]), a["positions"], a["pidx"], a["nrm"], a["nidx"], a["uv"],
                                    a["uidx"], a["edges"]))
        textures = []
        for i, (mips, quads) in enumerate(tex_arrays):
            textures.append(TextureAsset(tex_records[i], [(m["width"], m["height"]) for m in mips], quads))
        return cls(geos, meshes, textures, cams, grids, boxes, curves)


def _opaque(records, size):
    if records is None:
        return np.zeros((0, size), np.uint8)
    a = np.ascontiguousarray(records, dtype=np.uint8)
    return a.reshape(-1, size)


def _addr(a):
    return ptr(a) if len(a) else 0
