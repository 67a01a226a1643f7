"""RayTracingRenderer: the reference's renderer interface
(renderer/renderer.h:24-100) over the B200 library.

    renderer = RayTracingRenderer(scene, max_depth=2)
    pixels, depths = renderer.render(viewport)          # host arrays

`render(viewport, update_scene=True)` does what the reference's render()
does on its GPU branch: rebuild the scene AABBs/BVH on the host, upload
lights, cameras, geometries and the scene BVH, trace every pixel on the
GPU and copy the frame back.  There is no CPU branch: use_GPU=False is
rejected rather than silently run elsewhere.
"""
from __future__ import annotations

import numpy as np

from . import layout as L
from .native import check, lib, ptr


class Viewport:
    """Canvas size/antialiasing plus the camera (viewport/viewport.h:7-12)."""

    def __init__(self, camera, width, height, antialias=L.AA_NONE):
        self.camera, self.width, self.height, self.antialias = camera, int(width), int(height), antialias

    @property
    def ssaa(self):
        return self.antialias == L.AA_SSAA


def make_canvas(width, height, antialias):
    s = 2 if antialias == L.AA_SSAA else 1
    pixels = np.zeros((height * s * width * s, 4), np.float32)
    depths = np.full(height * width * (1 if antialias == L.AA_NONE else 4), np.inf, np.float32)
    cv = np.zeros((), L.CANVAS_DATA)
    cv["width_times_height"] = width * height
    cv["f_width"], cv["f_height"] = width, height
    cv["h_width"], cv["h_height"] = width * 0.5, height * 0.5
    cv["width_over_height"], cv["height_over_width"] = width / height, height / width
    cv["width"], cv["height"], cv["stride"] = width, height, width
    cv["antialias"] = antialias
    cv["pixels"], cv["depths"] = pixels.ctypes.data, depths.ctypes.data
    return cv, pixels, depths


class RayTracingRenderer:
    def __init__(self, scene, max_depth=3, skybox_color_texture_id=-1, skybox_radiance_texture_id=-1,
                 skybox_irradiance_texture_id=-1, render_mode=L.RENDER_BEAUTY):
        self.scene = scene
        self.settings = L.default_settings(max_depth, skybox_color_texture_id, skybox_radiance_texture_id,
                                           skybox_irradiance_texture_id, render_mode)
        check(lib().slimInitDataOnGPU(scene.ptr))

    def upload(self):
        """The per-frame uploads of render(update_scene=True)."""
        h = lib()
        check(h.slimUploadLights(self.scene.ptr))
        check(h.slimUploadCameras(self.scene.ptr))
        check(h.slimUploadGeometries(self.scene.ptr))
        check(h.slimUploadSceneBVH(self.scene.ptr))

    def upload_materials(self):
        check(lib().slimUploadMaterials(self.scene.ptr))

    def render(self, viewport, update_scene=True, use_GPU=True):
        if not use_GPU:
            raise ValueError("the B200 renderer has no CPU path (use_GPU=False)")
        if update_scene:
            self.scene.build_bvh()
            self.upload()
        cv, pixels, depths = make_canvas(viewport.width, viewport.height, viewport.antialias)
        proj = viewport.camera.projection(viewport.width, viewport.height, viewport.ssaa)
        check(lib().slimRenderOnGPU(ptr(cv), ptr(proj), ptr(self.settings)))
        return pixels, depths

    def render_to_device(self, viewport, d_pixels, d_depths, stream=0):
        """Frame into caller-owned device buffers (e.g. torch tensors),
        asynchronously on `stream`."""
        cv, _, _ = make_canvas(1, 1, viewport.antialias)
        cv["width"], cv["height"], cv["stride"] = viewport.width, viewport.height, viewport.width
        cv["width_times_height"] = viewport.width * viewport.height
        proj = viewport.camera.projection(viewport.width, viewport.height, viewport.ssaa)
        check(lib().slimRenderToDevice(ptr(cv), ptr(proj), ptr(self.settings), int(d_pixels), int(d_depths), int(stream)))

    @staticmethod
    def to_content(pixels, width, height):
        """Pixel::asContent (core/base.h:1166-1171): 8-bit R, G, B per pixel
        from the stored squared colour (no SSAA resolve)."""
        c = pixels[:, :3].reshape(height, width, 3).astype(np.float32)
        v = np.float32(255.0) * np.sqrt(np.maximum(c, np.float32(0)))
        return np.where(c > np.float32(1.0), np.float32(255), v).astype(np.uint8)
