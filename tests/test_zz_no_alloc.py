"""slimRenderToDeviceNoAlloc: the render entry point for callers that cannot
allocate device memory from their frame hook (another thread capturing a
CUDA graph in global mode, or a host engine that owns all device memory).
Its queues live in a fixed 64 MiB device array inside the library, so the
test checks that two calls in a row -- the second reusing the array the
first one left behind -- produce the same frames as slimRenderToDevice,
and that a frame too large for the array is refused.

Collected last (file name) so a failure here never hides other tests.
"""
import numpy as np
import pytest

from slimtracincpp_b200 import layout as L
from slimtracincpp_b200 import native, scenes
from slimtracincpp_b200.renderer import RayTracingRenderer, make_canvas

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _canvas(width, height, antialias=L.AA_NONE):
    cv, _, _ = make_canvas(1, 1, antialias)
    cv["width"], cv["height"], cv["stride"] = width, height, width
    cv["width_times_height"] = width * height
    return cv


def _same_frames(lib, cv, proj, settings, n):
    got = _frame(lib.slimRenderToDeviceNoAlloc, cv, proj, settings, n)
    want = _frame(lib.slimRenderToDevice, cv, proj, settings, n)
    assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
    assert np.array_equal(got[1].view(np.uint32), want[1].view(np.uint32))
    return got


def _frame(fn, cv, proj, settings, n):
    pix = torch.full((n, 4), -1.0, dtype=torch.float32, device="cuda")
    dep = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
    native.check(fn(native.ptr(cv), native.ptr(proj), native.ptr(settings), pix.data_ptr(), dep.data_ptr(), 0))
    torch.cuda.synchronize()
    return pix.cpu().numpy(), dep.cpu().numpy()


def test_no_alloc_frames_match_allocating_entry_point():
    lib = native.lib()
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    w = scenes.feature_scene(5, 320, 180)
    r = RayTracingRenderer(w.scene, max_depth=int(w.settings["max_depth"]))
    views = [(w.camera, 320, 180), (scenes.Camera.look_at((4.0, 6.0, -7.0), (0.0, 1.0, 2.0), 50.0), 256, 144)]
    for cam, width, height in views:      # two calls in a row on the shared scratch
        cv = _canvas(width, height)
        proj = cam.projection(width, height)
        n = width * height
        got = _frame(lib.slimRenderToDeviceNoAlloc, cv, proj, r.settings, n)
        want = _frame(lib.slimRenderToDevice, cv, proj, r.settings, n)
        assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32))
        assert np.array_equal(got[1].view(np.uint32), want[1].view(np.uint32))
        assert (got[0][:, 3] == 1.0).all()   # every pixel written


def test_no_alloc_rejects_frames_beyond_its_array():
    lib = native.lib()
    w = scenes.config1(0, 64, 36)
    r = RayTracingRenderer(w.scene, max_depth=1)
    width, height = 1920, 1080
    cv = _canvas(width, height)
    proj = w.camera.projection(width, height)
    pix = torch.empty((width * height, 4), dtype=torch.float32, device="cuda")
    dep = torch.empty(width * height, dtype=torch.float32, device="cuda")
    rc = lib.slimRenderToDeviceNoAlloc(native.ptr(cv), native.ptr(proj), native.ptr(r.settings), pix.data_ptr(),
                                       dep.data_ptr(), 0)
    assert rc == 4   # SLIM_ERR_LIMIT
    assert b"no-alloc scratch" in lib.slimGetLastError()


def test_no_alloc_ssaa_and_light_batches():
    """Four samples per pixel (SSAA), and a scene with 16 lights at a size
    where the 64 MiB array holds the shadow rays of only some of them per
    batch (every light batch then reuses the shadow queue), both bit for bit
    against slimRenderToDevice."""
    from slimtracincpp_b200.scene import Scene, light
    lib = native.lib()
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    w = scenes.feature_scene(6, 320, 180)
    r = RayTracingRenderer(w.scene, max_depth=int(w.settings["max_depth"]))
    width, height = 320, 180
    cv = _canvas(width, height, L.AA_SSAA)
    proj = w.camera.projection(width, height, True)
    _same_frames(lib, cv, proj, r.settings, 4 * width * height)
    rng = np.random.default_rng(3)
    lights = [light(rng.uniform(0.3, 1.0, 3), (rng.uniform(-6, 6), rng.uniform(3, 7), rng.uniform(-6, 6)),
                    rng.uniform(5, 15)) for _ in range(16)]
    s2 = w.scene
    many = Scene(s2.geometries, s2.materials, np.array(lights), meshes=s2.meshes)
    r2 = RayTracingRenderer(many, max_depth=3)
    n = width * height
    per_sample, per_light = 152, 80      # scratch bytes: path state and queues; shadow ray + candidate pair
    assert ((64 << 20) - per_sample * n) // (per_light * n) < 16   # the lights do not fit one batch
    cv = _canvas(width, height)
    for cam in (w.camera, scenes.Camera.look_at((3.0, 7.0, -8.0), (0.0, 1.0, 1.0), 55.0)):
        got = _same_frames(lib, cv, cam.projection(width, height), r2.settings, n)
        assert (got[0][:, 3] == 1.0).all()


def test_no_alloc_full_hd_without_queues():
    """Debug render modes and max_depth 0 run the fused kernel, which needs
    no scratch: a 1920x1080 frame is accepted and equals slimRenderToDevice."""
    lib = native.lib()
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    w = scenes.config1(0, 64, 36)
    width, height = 1920, 1080
    cv = _canvas(width, height)
    proj = w.camera.projection(width, height)
    for settings in (L.default_settings(max_depth=0), L.default_settings(max_depth=2, render_mode=L.RENDER_NORMALS)):
        RayTracingRenderer(w.scene, max_depth=int(settings["max_depth"]))
        _same_frames(lib, cv, proj, settings, width * height)


def test_no_alloc_refuses_cache_and_work_counting():
    """The radiance cache and work counting need state this entry point does
    not keep: both are refused with SLIM_ERR_STATE instead of silently giving
    a different frame."""
    lib = native.lib()
    w = scenes.config1(0, 64, 36)
    r = RayTracingRenderer(w.scene, max_depth=1)
    cv = _canvas(64, 36)
    proj = w.camera.projection(64, 36)
    pix = torch.empty((64 * 36, 4), dtype=torch.float32, device="cuda")
    dep = torch.empty(64 * 36, dtype=torch.float32, device="cuda")
    try:
        for opts in ({"radiance_cache": L.CACHE_ON}, {"count_work": True}):
            native.set_render_options(engine=L.ENGINE_WAVEFRONT, **opts)
            rc = lib.slimRenderToDeviceNoAlloc(native.ptr(cv), native.ptr(proj), native.ptr(r.settings),
                                               pix.data_ptr(), dep.data_ptr(), 0)
            assert rc == 3, opts    # SLIM_ERR_STATE
    finally:
        native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    native.check(lib.slimRenderToDeviceNoAlloc(native.ptr(cv), native.ptr(proj), native.ptr(r.settings),
                                               pix.data_ptr(), dep.data_ptr(), 0))
    torch.cuda.synchronize()
