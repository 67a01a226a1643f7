"""GPU parity: the CUDA trace path (through the C ABI) against the CPU oracle
on the same seeded scenes.

Bars (from the path's acceptance criteria):
  * primary-hit geometry ids and mesh triangle ids: bit-exact;
  * hit distances: within 1e-5 relative (bit-exact in practice: the kernels
    keep the reference's operation order);
  * final 8-bit pixels: within +-1 LSB on >= 99.9% of pixels (transcendental
    functions -- powf, acosf, sinf, cosf -- differ by a few ULP between CUDA
    and glibc; everything else is IEEE-exact on both sides).
"""
import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport
from slimtracincpp_b200.scene import Scene
from oracle import bindings as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ENGINES = [L.ENGINE_MEGAKERNEL, L.ENGINE_WAVEFRONT]


def gpu_primary(scene, projection, width, height):
    n = width * height
    g = torch.empty(n, dtype=torch.int32, device="cuda")
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    d = torch.empty(n, dtype=torch.float32, device="cuda")
    b = torch.empty(n, dtype=torch.uint8, device="cuda")
    native.check(native.lib().slimTracePrimary(native.ptr(projection), width, height, g.data_ptr(), p.data_ptr(),
                                               d.data_ptr(), b.data_ptr(), 0))
    torch.cuda.synchronize()
    return g.cpu().numpy(), p.cpu().numpy().view(np.uint32), d.cpu().numpy(), b.cpu().numpy()


def to8(pixels, w, h):
    return RayTracingRenderer.to_content(pixels, w, h).astype(np.int32)


def assert_pixels_close(gpu, ref, w, h, frac=0.999):
    a, b = to8(gpu, w, h), to8(ref, w, h)
    within = (np.abs(a - b) <= 1).all(axis=-1)
    assert within.mean() >= frac, f"only {within.mean():.5f} of pixels within 1 LSB"


def assert_float_pixels_close(gpu, ref, tol=1e-4, frac=0.995):
    """Stored (squared, clamped) colours: only transcendental ULPs differ, so
    nearly every pixel is within 1e-4 absolute on every channel."""
    close = (np.abs(gpu - ref) <= tol).all(axis=1).mean()
    assert close >= frac, f"only {close:.5f} of pixels within {tol}"


def assert_depths_close(gpu, ref):
    finite = np.isfinite(ref)
    assert np.array_equal(np.isfinite(gpu), finite)
    np.testing.assert_allclose(gpu[finite], ref[finite], rtol=1e-5, atol=0)


def renderer_for(w, **kw):
    """A renderer with the workload's settings (depth and skybox ids)."""
    st = w.settings
    return RayTracingRenderer(w.scene, int(st["max_depth"]), int(st["skybox_color_texture_id"]),
                              int(st["skybox_radiance_texture_id"]), int(st["skybox_irradiance_texture_id"]), **kw)


def axis_aligned_mesh_scene():
    """An unrotated camera over an odd-sized canvas: the centre column and row
    of primary rays have direction components of exactly zero (infinite
    reciprocals, the slab test's NaN-handling path)."""
    from slimtracincpp_b200.scene import Camera
    w = scenes.small_mesh_scene(0, 65, 65)
    w.camera = Camera(np.eye(3, dtype=np.float32), np.array([0.0, 1.0, -8.0], np.float32), w.camera.focal_length)
    return w


def workloads():
    return {
        "axis_aligned": axis_aligned_mesh_scene,
        "config1": lambda: scenes.config1(0, 320, 180),
        "config1_seed3": lambda: scenes.config1(3, 256, 144),
        "mesh_small": lambda: scenes.small_mesh_scene(0, 192, 108),
        "features": lambda: scenes.feature_scene(0, 160, 90),
        "features_seed4": lambda: scenes.feature_scene(4, 128, 72, max_depth=6),
        "textured_ibl": lambda: scenes.small_textured_scene(0, 160, 90),
    }


@pytest.mark.parametrize("name", list(workloads()))
def test_primary_hits_bit_exact(name):
    w = workloads()[name]()
    RayTracingRenderer(w.scene, max_depth=int(w.settings["max_depth"]))
    proj = w.projection()
    g, p, d, b = gpu_primary(w.scene, proj, w.width, w.height)
    og, op, od, ob = O.oracle_trace_primary(w.scene, proj, w.width, w.height)
    assert np.array_equal(g, og)
    assert np.array_equal(p, op)
    assert np.array_equal(b, ob)
    assert np.array_equal(d.view(np.uint32), od.view(np.uint32))


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", list(workloads()))
def test_render_matches_oracle(name, engine):
    native.set_render_options(engine=engine)
    w = workloads()[name]()
    r = renderer_for(w)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    opix, odep, _ = O.oracle_render(w.scene, w.projection(), w.settings, w.width, w.height, layout=L)
    assert_pixels_close(pix, opix, w.width, w.height)
    assert_depths_close(dep, odep)
    assert_float_pixels_close(pix, opix)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("size", [(1, 1), (1, 7), (7, 1), (5, 3), (9, 5), (33, 17)])
def test_tiny_and_ragged_canvases_match_oracle(size, engine):
    """Canvases smaller than one 8x4 tile of primary numbering, one pixel wide
    or high, and with partial tiles on both edges."""
    native.set_render_options(engine=engine)
    w = scenes.small_mesh_scene(0, *size)
    r = renderer_for(w)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    opix, odep, _ = O.oracle_render(w.scene, w.projection(), w.settings, w.width, w.height, layout=L)
    assert_pixels_close(pix, opix, w.width, w.height)
    assert_depths_close(dep, odep)
    g, p, d, b = gpu_primary(w.scene, w.projection(), w.width, w.height)
    og, op, od, ob = O.oracle_trace_primary(w.scene, w.projection(), w.width, w.height)
    assert np.array_equal(g, og) and np.array_equal(p, op)
    assert np.array_equal(d.view(np.uint32), od.view(np.uint32))
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("mode", [L.RENDER_NORMALS, L.RENDER_DEPTH, L.RENDER_UVS, L.RENDER_MIP_LEVEL])
def test_debug_modes(mode, engine):
    native.set_render_options(engine=engine)
    w = scenes.small_mesh_scene(1, 160, 90)
    r = RayTracingRenderer(w.scene, render_mode=mode)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    st = L.default_settings(max_depth=3, render_mode=mode)
    opix, odep, _ = O.oracle_render(w.scene, w.projection(), st, w.width, w.height, layout=L)
    assert np.array_equal(pix.view(np.uint32), opix.view(np.uint32))
    assert_depths_close(dep, odep)


@pytest.mark.parametrize("engine", ENGINES)
def test_ssaa(engine):
    native.set_render_options(engine=engine)
    w = scenes.config1(1, 128, 72)
    r = RayTracingRenderer(w.scene, max_depth=1)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height, L.AA_SSAA))
    proj = w.camera.projection(w.width, w.height, True)
    opix, odep, _ = O.oracle_render(w.scene, proj, w.settings, w.width, w.height, antialias=L.AA_SSAA, layout=L)
    assert_pixels_close(pix, opix, 2 * w.width, 2 * w.height)
    assert_depths_close(dep, odep)


@pytest.mark.parametrize("engine", ENGINES)
def test_work_counters_match_oracle(engine):
    native.set_render_options(engine=engine, count_work=True)
    try:
        w = scenes.small_mesh_scene(2, 128, 72)
        r = RayTracingRenderer(w.scene, max_depth=2)
        r.render(Viewport(w.camera, w.width, w.height))
        got = native.work_counters()
    finally:
        native.set_render_options(engine=engine)
    _, _, ref = O.oracle_render(w.scene, w.projection(), w.settings, w.width, w.height, layout=L, count=True)
    # The fused kernel walks every ray in the reference's order, so all its
    # work counts equal the oracle's.  The wavefront engine tests shadow
    # candidates in another (equally valid) order, so only its ray counts
    # are fixed.
    keys = ["primary_rays", "shadow_rays", "bounce_rays"]
    if engine == L.ENGINE_MEGAKERNEL:
        keys += ["scene_node_tests", "mesh_node_tests", "triangle_tests", "geometry_tests", "mesh_hit_fetches"]
    for k in keys:
        assert got[k] == ref[k], (k, got[k], ref[k])


@pytest.mark.parametrize("engine", ENGINES)
def test_ray_cone_mips_match_oracle(engine):
    """SLIM_CONES_PER_PIXEL: mip levels chosen from the per-pixel cone spread
    (the reference's intended ray cones) instead of its effective mip 0."""
    native.set_render_options(engine=engine, ray_cones=L.CONES_PER_PIXEL)
    try:
        w = scenes.small_textured_scene(1, 160, 90)
        r = renderer_for(w)
        pix, dep = r.render(Viewport(w.camera, w.width, w.height))
        # mip-level debug view must differ from mip 0 somewhere
        r2 = RayTracingRenderer(w.scene, render_mode=L.RENDER_MIP_LEVEL)
        mip, _ = r2.render(Viewport(w.camera, w.width, w.height))
    finally:
        native.set_render_options(engine=engine)
    opix, odep, _ = O.oracle_render(w.scene, w.projection(), w.settings, w.width, w.height, layout=L,
                                    cones_per_pixel=True)
    assert_pixels_close(pix, opix, w.width, w.height)
    assert_float_pixels_close(pix, opix)
    st = L.default_settings(max_depth=3, render_mode=L.RENDER_MIP_LEVEL)
    omip, _, _ = O.oracle_render(w.scene, w.projection(), st, w.width, w.height, layout=L, cones_per_pixel=True)
    assert np.array_equal(mip.view(np.uint32), omip.view(np.uint32))
    assert len(np.unique(omip[:, :3], axis=0)) > 2


@pytest.mark.parametrize("engine", ENGINES)
def test_normal_map_debug_mode(engine):
    native.set_render_options(engine=engine)
    w = scenes.small_textured_scene(2, 128, 72)
    r = RayTracingRenderer(w.scene, render_mode=L.RENDER_NORMAL_MAP)
    pix, dep = r.render(Viewport(w.camera, w.width, w.height))
    st = L.default_settings(max_depth=3, render_mode=L.RENDER_NORMAL_MAP)
    opix, _, _ = O.oracle_render(w.scene, w.projection(), st, w.width, w.height, layout=L)
    assert np.array_equal(pix.view(np.uint32), opix.view(np.uint32))


@pytest.mark.parametrize("name", ["config1", "mesh_small", "features"])
def test_pick_matches_the_closest_hit(name):
    """slimPick's geometry, triangle, distance and side equal the oracle's
    closest hit of the same pixel (bit for bit)."""
    w = workloads()[name]()
    RayTracingRenderer(w.scene, max_depth=int(w.settings["max_depth"]))
    proj = w.projection()
    og, op, od, ob = O.oracle_trace_primary(w.scene, proj, w.width, w.height)
    rng = np.random.default_rng(0)
    for _ in range(40):
        x, y = int(rng.integers(0, w.width)), int(rng.integers(0, w.height))
        i = y * w.width + x
        p = native.pick(proj, x, y)
        assert int(p["geometry"]) == og[i]
        if og[i] >= 0:
            assert int(p["triangle"]) == op[i]
            assert np.float32(p["distance"]).view(np.uint32) == od[i].view(np.uint32)
            assert int(p["from_behind"]) == ob[i]


def test_pick_selects_a_light_in_front_of_the_geometry():
    w = scenes.config1(2, 160, 90)
    w.scene.lights[0]["position"] = (0.0, 3.0, -6.0)    # in front of the camera, above the floor
    w.scene.lights[0]["intensity"] = 50.0                 # selection radius 50 / 2 / 64: a few pixels wide
    RayTracingRenderer(w.scene, max_depth=1)
    proj = w.projection()
    light = w.scene.lights[0]
    # the pixel whose ray points closest to the light's centre
    P = proj
    xs, ys = np.meshgrid(np.arange(w.width, dtype=np.float32), np.arange(w.height, dtype=np.float32))
    d = (P["start"][None, None, :] + P["down"][None, None, :] * ys[..., None] + P["right"][None, None, :] * xs[..., None])
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    to_light = np.asarray(light["position"], np.float64) - np.asarray(P["camera_position"], np.float64)
    to_light /= np.linalg.norm(to_light)
    y, x = np.unravel_index(np.argmax(d @ to_light), d.shape[:2])
    p = native.pick(proj, int(x), int(y))
    assert int(p["light"]) == 0
    far = native.pick(proj, 0, w.height - 1)
    assert int(far["light"]) == -1


def _without_lights(w):
    """The workload with every light removed (the scene is rebuilt)."""
    sc = w.scene
    w.scene = Scene(sc.geometries, sc.materials, np.zeros(0, L.LIGHT), meshes=sc.meshes, textures=sc.textures)
    return w


BANDED_SCENES = {
    "mesh_depth2": lambda: scenes.small_mesh_scene(0, 120, 70),
    "implicit_depth6": lambda: scenes.feature_scene(4, 120, 70, max_depth=6),   # late bounces in the fused tail
    # no shadow rays: the depths download with the pixels, not before them
    "mesh_no_lights": lambda: _without_lights(scenes.small_mesh_scene(2, 120, 70)),
    # fewer tile rows than first-round shade chunks: empty chunks are skipped
    "mesh_4_rows": lambda: scenes.small_mesh_scene(3, 24, 4),
    "implicit_6_rows": lambda: scenes.feature_scene(5, 24, 6, max_depth=3),
}


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("antialias", [L.AA_NONE, L.AA_MSAA, L.AA_SSAA])
@pytest.mark.parametrize("scene", list(BANDED_SCENES))
def test_banded_download_into_a_pinned_canvas(engine, antialias, scene):
    """slimRenderOnGPU renders the frame in row bands, two in flight on two
    streams.  Into pinned host memory each band's rows download once its
    first round is done (its depths, when the scene has lights, once the
    primary hits are shaded for shadow rays), and the pixels of later bounces
    are written into the host canvas directly: the canvas must equal the
    one-band frame bit for bit, for any band count (70 rows: the last band
    also holds the rows past the last 4-row tile band).  The fused engine
    writes a pinned canvas directly from its kernel, with no copy after it."""
    from slimtracincpp_b200.renderer import make_canvas
    w = BANDED_SCENES[scene]()
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height, antialias)
    native.set_render_options(engine=engine)
    ref_pix, ref_dep = r.render(vp)          # pageable canvas: one download after the frame
    cv, pix, dep = make_canvas(w.width, w.height, antialias)
    pin_pix = torch.from_numpy(pix).pin_memory()
    pin_dep = torch.from_numpy(dep).pin_memory()
    cv["pixels"], cv["depths"] = pin_pix.data_ptr(), pin_dep.data_ptr()
    proj = w.camera.projection(w.width, w.height, antialias == L.AA_SSAA)
    try:
        for bands in (0, 1, 3, 64):
            native.set_render_options(engine=engine, row_bands=bands)
            pin_pix.fill_(-1.0)
            pin_dep.fill_(-1.0)
            native.check(native.lib().slimRenderOnGPU(native.ptr(cv), native.ptr(proj), native.ptr(r.settings)))
            assert np.array_equal(pin_pix.numpy().view(np.uint32), ref_pix.view(np.uint32)), bands
            assert np.array_equal(pin_dep.numpy().view(np.uint32), ref_dep.view(np.uint32)), bands
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)



def test_row_bands_on_the_callers_stream_with_work_counters():
    """slimRenderToDevice with the frame split into row bands on the caller's
    stream and a second one: same pixels and depths as the whole frame, the
    same rays and scene-node tests.  Mesh-node and triangle tests depend on
    the order in which concurrent candidates of a ray publish their hits
    (culling), so they match only closely."""
    w = scenes.small_mesh_scene(1, 160, 96)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    n = w.width * w.height
    stream = torch.cuda.Stream()
    results = []
    try:
        for bands in (1, 2, 5):
            native.set_render_options(engine=L.ENGINE_WAVEFRONT, row_bands=bands, count_work=True)
            pix = torch.full((n, 4), -1.0, device="cuda")
            dep = torch.full((n,), -1.0, device="cuda")
            torch.cuda.synchronize()
            r.render_to_device(vp, pix.data_ptr(), dep.data_ptr(), stream.cuda_stream)
            stream.synchronize()
            results.append((pix.cpu().numpy(), dep.cpu().numpy(), native.work_counters()))
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    for pix, dep, work in results[1:]:
        assert np.array_equal(pix.view(np.uint32), results[0][0].view(np.uint32))
        assert np.array_equal(dep.view(np.uint32), results[0][1].view(np.uint32))
        ref = results[0][2]
        for k in ("primary_rays", "shadow_rays", "bounce_rays", "scene_node_tests", "pixels"):
            assert work[k] == ref[k], k
        for k in ("mesh_node_tests", "triangle_tests"):
            assert abs(work[k] - ref[k]) <= 0.02 * ref[k], k


def test_pageable_canvas_through_pinned_staging():
    """A pageable canvas of at least 4 MB of pixels: the frame downloads into
    the library's pinned staging canvas (banded, early) and host threads copy
    it over; the pixels equal the device-resident frame bit for bit."""
    w = scenes.small_mesh_scene(2, 640, 480)
    r = renderer_for(w)
    vp = Viewport(w.camera, w.width, w.height)
    n = w.width * w.height
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    pix, dep = r.render(vp)                  # numpy arrays: pageable
    assert pix.nbytes >= 4 << 20
    d_pix = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    d_dep = torch.zeros(n, dtype=torch.float32, device="cuda")
    r.render_to_device(vp, d_pix.data_ptr(), d_dep.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(pix.view(np.uint32), d_pix.cpu().numpy().view(np.uint32))
    assert np.array_equal(dep.view(np.uint32), d_dep.cpu().numpy().view(np.uint32))


def test_mesh_leaf_too_large_for_the_packed_record_is_refused():
    """The persistent mesh kernels pack a waiting leaf into one word (first
    triangle, count below 64); a mesh whose BVH has a larger leaf below the
    root is refused on upload with SLIM_ERR_LIMIT instead of being traced
    wrong.  A root leaf of any size is fine (tested without packing)."""
    from slimtracincpp_b200.scene import MeshAsset, Scene, geometry
    pos, idx, nrm = scenes.icosphere(2)
    mesh = MeshAsset.build(pos, idx, nrm, idx)
    assert mesh.triangle_count >= 64
    mesh.nodes["leaf_count"][1] = 64
    mesh.nodes["first_index"][1] = 0
    g = geometry(L.GEOMETRY_MESH, 0)
    scene = Scene(np.array([g]), np.array([L.default_material()]), meshes=[mesh])
    with pytest.raises(native.SlimError) as err:
        RayTracingRenderer(scene, max_depth=1)
    assert err.value.code == 4 and "64 triangles" in str(err.value)


def _stage_launches(w, viewport):
    native.reset_stage_stats()
    pix, dep = renderer_for(w).render(viewport)
    return pix, dep, {s["name"]: s["launches"] for s in native.stage_stats()}


def test_auto_engine_picks_by_scene_and_size():
    """SLIM_ENGINE_AUTO: the fused kernel for mesh-free frames whose paths end
    at their first hit or that are small, the wavefront engine for mesh
    scenes and for large frames whose paths bounce -- with the pixels both
    explicit engines write, bit for bit, and the oracle's."""
    cases = [
        (scenes.config1(3, 320, 180), "fused"),                        # no meshes, no bounces
        (scenes.small_textured_scene(2, 160, 90), "fused"),            # bounces, few samples
        (scenes.config3(1, 1024, 512, tex_size=64, cube_size=32, irradiance_size=8), "extend"),  # bounces, 2^19 samples
        (scenes.small_mesh_scene(1, 160, 90), "extend"),               # meshes
    ]
    try:
        for w, stage in cases:
            vp = Viewport(w.camera, w.width, w.height)
            native.set_render_options(engine=L.ENGINE_AUTO, profile_stages=True)
            pix, dep, launches = _stage_launches(w, vp)
            other = "extend" if stage == "fused" else "fused"
            assert launches.get(stage, 0) > 0 and launches.get(other, 0) == 0, (w.name, launches)
            for engine in ENGINES:
                native.set_render_options(engine=engine)
                p2, d2 = renderer_for(w).render(vp)
                assert np.array_equal(pix.view(np.uint32), p2.view(np.uint32)), (w.name, engine)
                assert np.array_equal(dep.view(np.uint32), d2.view(np.uint32)), (w.name, engine)
            opix, odep, _ = O.oracle_render(w.scene, w.projection(), w.settings, w.width, w.height, layout=L)
            assert_pixels_close(pix, opix, w.width, w.height)
            assert_depths_close(dep, odep)
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
