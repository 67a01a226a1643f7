"""Whole-scene files (serialization/scene.h:5-109): slimSaveScene /
slimReadSceneHeader / slimLoadScene against the reference's own save and
load, compiled from its sources into oracle/_ref.

  * the record sizes the format stores equal the reference's;
  * a scene with meshes (normals, uvs), textures (mip chains, a cube map),
    cameras, geometries and overlay records saves to the reference's bytes;
  * each side loads the other's file to the same arrays;
  * save -> load -> save is the identity; truncated files and mismatched
    counts are errors, never a crash.
"""
import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.scene import Camera, MeshAsset, TextureAsset
from slimtracincpp_b200.scene_file import SceneFile, camera_record
from oracle import bindings as O

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (needs the reference sources)")


def sample_scene(seed=0):
    rng = np.random.default_rng(seed)
    w = scenes.small_mesh_scene(seed, 32, 18)
    pos, idx, nrm = scenes.icosphere(1)
    uv = rng.random((len(pos), 2)).astype(np.float32)
    with_uv = MeshAsset.build(pos, idx, nrm, idx, uv, idx)
    meshes = list(w.scene.meshes) + [with_uv]
    img = rng.integers(0, 256, (32, 32, 3), dtype=np.uint8)
    tex = [TextureAsset.bake(img, L.IMAGE_MIPMAP | L.IMAGE_WRAP),
           TextureAsset.bake(rng.integers(0, 256, (8, 48, 3), dtype=np.uint8), L.IMAGE_CUBEMAP | L.IMAGE_LINEAR)]
    cams = np.zeros(2, L.CAMERA)
    cams[0] = camera_record(w.camera, target_distance=7.5, dolly_amount=-3.0, rotation=(0.1, -0.4, 0.0),
                            velocity=(0.5, 0.0, -0.25))
    cams[1] = camera_record(Camera.look_at((2.0, 3.0, -4.0), (0.0, 0.0, 0.0), 45.0))
    grids = rng.integers(0, 256, (2, L.GRID_BYTES), dtype=np.uint8)
    boxes = rng.integers(0, 256, (3, L.BOX_BYTES), dtype=np.uint8)
    curves = rng.integers(0, 256, (1, L.CURVE_BYTES), dtype=np.uint8)
    return SceneFile(w.scene.geometries, meshes, tex, cams, grids, boxes, curves)


def assert_same(a, b):
    assert a.geometries.tobytes() == b.geometries.tobytes()
    assert a.cameras.tobytes() == b.cameras.tobytes()
    for k in ("grids", "boxes", "curves"):
        assert getattr(a, k).tobytes() == getattr(b, k).tobytes(), k
    assert len(a.meshes) == len(b.meshes)
    for m, n in zip(a.meshes, b.meshes):
        assert m.triangles.tobytes() == n.triangles.tobytes()
        assert m.nodes.tobytes() == n.nodes.tobytes()
        assert m.positions.tobytes() == n.positions.tobytes()
        assert m.position_indices.tobytes() == n.position_indices.tobytes()
        assert m.edges.tobytes() == n.edges.tobytes()
        for k in ("normals", "normal_indices", "uvs", "uv_indices"):
            x, y = getattr(m, k), getattr(n, k)
            assert (x is None) == (y is None), k
            if x is not None:
                assert x.tobytes() == y.tobytes(), k
        assert np.array_equal(m.aabb_min, n.aabb_min) and np.array_equal(m.aabb_max, n.aabb_max)
        assert m.height == n.height
    assert len(a.textures) == len(b.textures)
    for t, u in zip(a.textures, b.textures):
        assert t.quads.tobytes() == u.quads.tobytes()
        assert t.mip_sizes == u.mip_sizes
        assert t.header.tobytes()[:32] == u.header.tobytes()[:32]


@needs_ref
def test_record_sizes_match_reference():
    cam, orient, grid, box, curve, counts, image, geo = O.reference_scene_record_sizes()
    assert (cam, orient) == (L.CAMERA.itemsize, 48)
    assert (grid, box, curve) == (L.GRID_BYTES, L.BOX_BYTES, L.CURVE_BYTES)
    assert (counts, image, geo) == (44, 32, L.GEOMETRY.itemsize)


@needs_ref
def test_save_writes_the_reference_bytes(tmp_path):
    f = sample_scene(0)
    f.save(tmp_path / "ours.scene")
    O.reference_save_scene(f, tmp_path / "ref.scene", L)
    assert (tmp_path / "ours.scene").read_bytes() == (tmp_path / "ref.scene").read_bytes()


@needs_ref
def test_each_side_loads_the_others_file(tmp_path):
    f = sample_scene(1)
    O.reference_save_scene(f, tmp_path / "ref.scene", L)
    assert_same(SceneFile.load(tmp_path / "ref.scene"), f)
    f.save(tmp_path / "ours.scene")
    assert_same(O.reference_load_scene(tmp_path / "ours.scene", f, L), f)


def test_round_trip_and_empty_sections(tmp_path):
    f = sample_scene(2)
    f.save(tmp_path / "a.scene")
    g = SceneFile.load(tmp_path / "a.scene")
    assert_same(g, f)
    g.save(tmp_path / "b.scene")
    assert (tmp_path / "a.scene").read_bytes() == (tmp_path / "b.scene").read_bytes()
    bare = SceneFile(f.geometries[:1])
    bare.save(tmp_path / "c.scene")
    h = SceneFile.load(tmp_path / "c.scene")
    assert h.geometries.tobytes() == f.geometries[:1].tobytes() and not h.meshes and not h.textures
    assert (tmp_path / "c.scene").stat().st_size == 44 + L.GEOMETRY.itemsize


def test_truncated_and_mismatched_files_are_errors(tmp_path):
    f = sample_scene(3)
    f.save(tmp_path / "a.scene")
    data = (tmp_path / "a.scene").read_bytes()
    for cut in (10, 200, len(data) // 2, len(data) - 5):
        (tmp_path / "t.scene").write_bytes(data[:cut])
        with pytest.raises(native.SlimError) as e:
            SceneFile.load(tmp_path / "t.scene")
        assert e.value.code in (1, 5)
    r = f.record()
    r["counts"][L.COUNT_GEOMETRIES] += 1
    rc = native.lib().slimLoadScene(str(tmp_path / "a.scene").encode(), native.ptr(r))
    assert rc == 1
    with pytest.raises(native.SlimError):
        SceneFile.load(tmp_path / "missing.scene")
