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


def _canvas(width, height):
    cv, _, _ = make_canvas(1, 1, L.AA_NONE)
    cv["width"], cv["height"], cv["stride"] = width, height, width
    cv["width_times_height"] = width * height
    return cv


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
