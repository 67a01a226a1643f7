"""Host side of the boundary (CPU only): the C-ABI library loads and exports
every declared symbol, the host algorithms restated from the reference
(projection, SAH builds) match the reference's golden outputs bit for bit,
the native file formats round-trip, and errors come back as status codes.
"""
import re
from pathlib import Path

import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.scene import Camera, MeshAsset, Scene, geometry
from oracle import bindings as O
from conftest import reference_src

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
HEADER = ROOT / "include" / "slimtracer_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(slim[A-Z]\w*)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(native.EXPORTS) <= set(names)


def test_cuda_calls_fail_loudly_without_gpu_or_init():
    lib = native.lib()
    cv = np.zeros((), L.CANVAS_DATA)
    rc = lib.slimRenderOnGPU(native.ptr(cv), native.ptr(np.zeros((), L.PROJECTION)), native.ptr(L.default_settings()))
    assert rc in (native.ERRORS and 2, 3)  # CUDA (no device) or STATE (not initialised)
    assert lib.slimGetLastError()


def test_cache_checkpoint_layout_and_refusals():
    """The checkpoint header and size agree with the C header; without a
    configured cache (or slimInitDataOnGPU) both calls refuse with STATE and
    touch no device."""
    text = HEADER.read_text()
    assert int(re.search(r"#define SLIM_NRC_STATE_MAGIC (0x[0-9A-Fa-f]+)u", text).group(1), 16) == L.NRC_STATE_MAGIC
    assert L.CACHE_STATE_HEADER.itemsize == 64 and L.CACHE_STATE_HEADER.fields["config"][1] == 16
    assert L.NRC_STATE_BYTES == 64 + 3 * 4 * L.NRC_PARAMS
    lib = native.lib()
    buf = np.zeros(L.NRC_STATE_BYTES, np.uint8)
    assert lib.slimRadianceCacheSaveState(native.ptr(buf), buf.nbytes) == 3
    assert lib.slimRadianceCacheLoadState(native.ptr(buf), buf.nbytes) == 3


def test_render_options_are_validated():
    """Options outside their ranges are refused without touching the device."""
    for bad in ({"row_bands": -1}, {"row_bands": 65}, {"block_size": 48}, {"radiance_cache": 4}, {"engine": 3},
                {"engine": -1}):
        with pytest.raises(native.SlimError):
            native.set_render_options(**bad)
    native.set_render_options(row_bands=64)
    native.set_render_options(engine=L.ENGINE_AUTO)
    native.set_render_options()


def test_projection_matches_reference_golden():
    z = np.load(GOLDEN / "projection.npz")
    for i in range(4):
        w, h, ssaa = (int(v) for v in z[f"cam{i}_size"])
        got = native.projection_reset(z[f"cam{i}_orientation"], z[f"cam{i}_position"], float(z[f"cam{i}_focal"]),
                                      w, h, bool(ssaa))
        assert got.tobytes() == z[f"cam{i}_projection"].tobytes(), i


@pytest.mark.parametrize("name", ["bvh_scene40", "bvh_scene7"])
def test_scene_bvh_matches_reference_golden(name):
    z = np.load(GOLDEN / f"{name}.npz")
    geos = z["geometries"].view(L.GEOMETRY)
    scene = Scene(geos, np.array([L.default_material()]))
    n = int(scene.data["bvh_node_count"])
    assert scene.bvh_nodes[:n].tobytes() == z["nodes"].tobytes()
    assert np.array_equal(scene.leaf_ids, z["leaf_ids"])
    assert int(scene.data["bvh_height"]) == int(z["height"])


@pytest.mark.parametrize("name", ["mesh_icosphere2", "mesh_heightfield12_uv", "mesh_soup30"])
def test_mesh_build_matches_reference_golden(name):
    z = np.load(GOLDEN / f"{name}.npz")
    g = lambda k: z[k] if k in z else None
    m = MeshAsset.build(z["positions"], z["indices"], g("normals"), g("normal_indices"), g("uvs"), g("uv_indices"))
    assert m.triangles.tobytes() == z["triangles"].tobytes()
    assert m.nodes.tobytes() == z["nodes"].tobytes()
    assert m.height == int(z["height"])
    assert np.array_equal(np.concatenate([m.aabb_min, m.aabb_max]).view(np.uint32), z["aabb"].view(np.uint32))
    assert np.array_equal(m.positions.view(np.uint32), z["centred_positions"].view(np.uint32))


needs_ref = pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built (needs reference sources)")


@needs_ref
@pytest.mark.parametrize("seed", range(5))
def test_scene_bvh_matches_reference_live(seed):
    rng = np.random.default_rng(100 + seed)
    count = int(rng.integers(1, 60))
    geos = []
    for i in range(count):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        kind = [L.GEOMETRY_BOX, L.GEOMETRY_SPHERE, L.GEOMETRY_TET, L.GEOMETRY_QUAD][int(rng.integers(0, 4))]
        geos.append(geometry(kind, 0, rng.uniform(-10, 10, 3), rng.uniform(0.1, 4, 3), q[:3], q[3]))
    scene = Scene(np.array(geos), np.array([L.default_material()]))
    nodes, leaf, flags, height = O.reference_scene_bvh(scene, L)
    n = int(scene.data["bvh_node_count"])
    assert scene.bvh_nodes[:n].tobytes() == nodes.tobytes()
    assert np.array_equal(scene.leaf_ids[:count], leaf)
    assert int(scene.data["bvh_height"]) == height


@needs_ref
def test_mesh_build_matches_reference_on_grid_ties():
    """A flat grid has thousands of equal sort keys; the quicksort's tie order
    decides the BVH and the leaf order of the triangle ids."""
    pos, idx, nrm = scenes.heightfield(np.random.default_rng(0), 40, 0.0)
    m = MeshAsset.build(pos, idx, nrm, idx)
    tris, nodes, height, aabb, _ = O.reference_build_mesh(pos, idx, nrm, idx, layout=L)
    assert m.triangles.tobytes() == tris.tobytes()
    assert m.nodes.tobytes() == nodes.tobytes()
    assert m.height == height


def test_mesh_file_round_trip(tmp_path):
    pos, idx, nrm = scenes.icosphere(1)
    uv = np.ascontiguousarray(pos[:, :2] * 0.5 + 0.5)
    m = MeshAsset.build(pos, idx, nrm, idx, uv, idx)
    path = tmp_path / "ico.mesh"
    m.save(path)
    back = MeshAsset.load(path)
    assert back.triangles.tobytes() == m.triangles.tobytes()
    assert back.nodes.tobytes() == m.nodes.tobytes()
    assert np.array_equal(back.positions, m.positions)
    assert np.array_equal(back.uvs, m.uvs)
    assert np.array_equal(back.normal_indices, m.normal_indices)
    assert len(back.edges) == len(m.edges) == 120
    # header: 7 u32, the 4-byte height slot holds the height in its low byte
    head = np.fromfile(path, np.uint32, 7)
    assert list(head[:6]) == [len(pos), len(idx), 120, len(uv), len(nrm), len(m.nodes)]
    assert head[6] & 0xFF == m.height


def test_mesh_file_truncated_is_an_io_error(tmp_path):
    pos, idx, nrm = scenes.icosphere(0)
    m = MeshAsset.build(pos, idx)
    path = tmp_path / "t.mesh"
    m.save(path)
    data = path.read_bytes()
    path.write_bytes(data[:len(data) // 2])
    with pytest.raises(native.SlimError) as e:
        MeshAsset.load(path)
    assert e.value.code == 5


def test_shipped_reference_meshes_load():
    """monkey.mesh / cube.mesh from the reference's examples (read in place
    when the reference sources are present)."""
    src = reference_src()
    ex = src / "examples" if src else Path("/nonexistent")
    if not (ex / "monkey.mesh").exists():
        pytest.skip("reference assets not present")
    monkey = MeshAsset.load(ex / "monkey.mesh")
    assert (monkey.triangle_count, len(monkey.nodes), monkey.height) == (968, 1121, 13)
    cube = MeshAsset.load(ex / "cube.mesh")
    assert (cube.triangle_count, len(cube.nodes)) == (12, 9)


def test_build_mesh_rejects_bad_indices():
    pos = np.zeros((3, 3), np.float32)
    with pytest.raises(native.SlimError) as e:
        MeshAsset.build(pos, np.array([[0, 1, 7]], np.uint32))
    assert e.value.code == 1


def test_scene_bvh_single_geometry_is_a_leaf_root():
    scene = Scene(np.array([geometry(L.GEOMETRY_SPHERE, 0, (1, 2, 3), (2, 2, 2))]), np.array([L.default_material()]))
    n = int(scene.data["bvh_node_count"])
    assert n == 1 and scene.bvh_nodes[0]["leaf_count"] == 1
    assert np.allclose(scene.bvh_nodes[0]["min"], [-1, 0, 1]) and np.allclose(scene.bvh_nodes[0]["max"], [3, 4, 5])


def test_emissive_quad_flag():
    mats = np.array([L.default_material(), L.default_material(flags=L.MATERIAL_IS_EMISSIVE)])
    g = [geometry(L.GEOMETRY_SPHERE, 0), geometry(L.GEOMETRY_QUAD, 1, (0, 5, 0))]
    assert int(Scene(np.array(g), mats).data["flags"]) == L.SCENE_HAD_EMISSIVE_QUADS
    g[1]["material_id"] = 0
    assert int(Scene(np.array(g), mats).data["flags"]) == 0


def _load_bmp_components(path):
    """The component buffer the reference's loadBitmap returns
    (platforms/win32_bitmap.h:122-160): raw B,G,R[,A] bytes, rows flipped to
    top-down when the BMP is stored bottom-up."""
    import struct
    b = Path(path).read_bytes()
    off = struct.unpack_from("<I", b, 10)[0]
    w, h = struct.unpack_from("<ii", b, 18)
    ch = 4 if struct.unpack_from("<H", b, 28)[0] == 32 else 3
    comp = np.frombuffer(b, np.uint8, count=w * abs(h) * ch, offset=off).reshape(abs(h), w, ch)
    return np.ascontiguousarray(comp[::-1] if h > 0 else comp)


@pytest.mark.parametrize("name", ["cathedral_irradiance", "bolonga_irradiance"])
def test_texture_baker_reproduces_shipped_reference_textures(name, tmp_path):
    """The reference ships these cube maps baked by its bmp2texture -c -l
    from the BMPs beside them; the restated baker must write the same bytes."""
    from slimtracincpp_b200.scene import TextureAsset
    src = reference_src()
    ex = src / "examples" if src else Path("/nonexistent")
    if not (ex / f"{name}.texture").exists():
        pytest.skip("reference assets not present")
    t = TextureAsset.bake(_load_bmp_components(ex / f"{name}.bmp"), L.IMAGE_CUBEMAP | L.IMAGE_LINEAR)
    t.save(tmp_path / "t.texture")
    assert (tmp_path / "t.texture").read_bytes() == (ex / f"{name}.texture").read_bytes()
    back = TextureAsset.load(ex / f"{name}.texture")
    assert back.mip_sizes == [(512, 128), (128, 128), (128, 128)]


def test_texture_round_trip_and_mip_chain(tmp_path):
    from slimtracincpp_b200.scene import TextureAsset
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (64, 64, 3), dtype=np.uint8)
    t = TextureAsset.bake(img, L.IMAGE_MIPMAP | L.IMAGE_WRAP)
    assert t.mip_sizes == [(64, 64), (32, 32), (16, 16), (8, 8), (4, 4)]
    t.save(tmp_path / "a.texture")
    back = TextureAsset.load(tmp_path / "a.texture")
    assert back.quads.tobytes() == t.quads.tobytes() and back.mip_sizes == t.mip_sizes
    # wrap: the border quads repeat the opposite edge
    q = t.mip_quads(0)
    assert q[0, 0]["R"][3] == q[0, 0]["R"][3]
