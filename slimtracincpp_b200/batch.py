"""Batched rendering over the library's slimBatch* entry points.

    assets = Scene(..., meshes=shared_meshes, textures=shared_textures)
    batch = BatchRenderer(assets)                 # uploads the shared assets
    batch.set_requests(requests, outputs)         # per request: scene, camera, size, depth
    batch.tune()                                  # project autotuner picks the plan
    batch.render(); batch.synchronize()           # one captured CUDA graph per batch

Every request's canvas is a caller-owned device buffer pair (float4 pixels,
float depths), e.g. torch tensors.
"""
from __future__ import annotations

import numpy as np

from . import layout as L
from .native import check, lib, ptr
from .scene import Scene


class BatchRenderer:
    def __init__(self, assets: Scene):
        self.assets = assets
        check(lib().slimInitDataOnGPU(assets.ptr))

    def set_requests(self, requests, outputs):
        """requests: scenes.Request list; outputs: (d_pixels, d_depths) device addresses per request."""
        arr = np.zeros(len(requests), L.RENDER_REQUEST)
        self._keep = []
        for i, (q, (pix, dep)) in enumerate(zip(requests, outputs)):
            q.scene.build_bvh()
            self._keep.append(q.scene)
            arr[i]["scene"] = q.scene.ptr
            arr[i]["projection"] = q.projection()
            arr[i]["settings"] = q.settings
            arr[i]["width"], arr[i]["height"] = q.width, q.height
            arr[i]["radiance_cache"] = q.radiance_cache
            arr[i]["d_pixels"], arr[i]["d_depths"] = int(pix), int(dep)
        check(lib().slimBatchSetRequests(ptr(arr), len(arr)))

    def tune(self, stream=0):
        check(lib().slimBatchTune(int(stream)))
        return self.plan()

    def set_plan(self, queue_capacity, tile_pixels, block_size=256, persistent=False):
        """persistent: the requests without the radiance cache render in one
        persistent launch fed by a device pixel queue (the others in waves)."""
        p = np.zeros((), L.BATCH_PLAN)
        p["queue_capacity"], p["tile_pixels"], p["block_size"] = queue_capacity, tile_pixels, block_size
        p["persistent"] = int(bool(persistent))
        check(lib().slimBatchSetPlan(ptr(p)))

    def plan(self):
        p = np.zeros((), L.BATCH_PLAN)
        check(lib().slimBatchGetPlan(ptr(p)))
        return {k: p[k].item() for k in L.BATCH_PLAN.names}

    def render(self, stream=0):
        check(lib().slimBatchRender(int(stream)))

    def synchronize(self, stream=0):
        check(lib().slimSynchronize(int(stream)))
