"""ctypes binding of libslimtracer_b200.so (the C ABI in include/slimtracer_b200.h).

The library is the only compute path: there is no Python or CPU fallback.
Loading fails loudly when the in-tree build is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import layout as L

# SLIMTRACER_LIB points at another build of the same library (packaging).
LIB_PATH = Path(os.environ.get("SLIMTRACER_LIB", Path(__file__).resolve().parent / "_native" / "libslimtracer_b200.so"))

SLIM_OK = 0
ERRORS = {1: "ARGUMENT", 2: "CUDA", 3: "STATE", 4: "LIMIT", 5: "IO", 6: "STACK", 7: "TIMEOUT"}

EXPORTS = [
    "slimInitDataOnGPU", "slimUploadLights", "slimUploadCameras", "slimUploadGeometries", "slimUploadMaterials",
    "slimUploadSceneBVH", "slimRenderOnGPU", "slimGetLastError", "slimGetVersion", "slimSetRenderOptions",
    "slimGetRenderOptions", "slimRenderToDevice", "slimTracePrimary", "slimGetWorkCounters", "slimRefitSceneBVH",
    "slimProjectionReset", "slimBuildSceneBVH", "slimBuildMesh", "slimReadMeshHeader", "slimReadMesh",
    "slimWriteMesh", "slimReadTextureHeader", "slimReadTexture", "slimWriteTexture", "slimBakeTexture",
    "slimBakeTextureOnGPU",
    "slimGetStageStats", "slimResetStageStats", "slimRenderToDeviceNoAlloc",
    "slimRadianceCacheConfigure", "slimRadianceCacheGetConfig", "slimRadianceCacheSetWeights",
    "slimRadianceCacheGetWeights", "slimRadianceCacheGetGradients", "slimRadianceCacheQuery",
    "slimRadianceCacheTrain", "slimRadianceCacheGetStats", "slimRadianceCacheJoin", "slimRadianceCacheSaveState",
    "slimRadianceCacheLoadState", "slimSynchronize",
    "slimGetLaunchCount", "slimPick", "slimDownloadSceneBVH", "slimSaveScene", "slimReadSceneHeader", "slimLoadScene",
    "slimBatchSetRequests", "slimBatchTune", "slimBatchSetPlan", "slimBatchGetPlan", "slimBatchRender",
]


class SlimError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"SLIM_ERR_{ERRORS.get(code, code)}: {message}")
        self.code = code


_lib = None
P = C.c_void_p


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m slimtracincpp_b200.build` "
                           "(the trace path has no CPU fallback)")
    h = C.CDLL(str(LIB_PATH))
    for name in EXPORTS:
        getattr(h, name)
    h.slimGetLastError.restype = C.c_char_p
    h.slimGetLastError.argtypes = []
    for name in ["slimInitDataOnGPU", "slimUploadLights", "slimUploadCameras", "slimUploadGeometries",
                 "slimUploadMaterials", "slimUploadSceneBVH", "slimBuildSceneBVH", "slimSetRenderOptions",
                 "slimGetRenderOptions", "slimGetWorkCounters", "slimRefitSceneBVH", "slimDownloadSceneBVH"]:
        getattr(h, name).argtypes = [P]
        getattr(h, name).restype = C.c_int
    h.slimRenderOnGPU.argtypes = [P, P, P]
    h.slimRenderToDevice.argtypes = [P, P, P, P, P, P]
    h.slimRenderToDeviceNoAlloc.argtypes = [P, P, P, P, P, P]
    h.slimTracePrimary.argtypes = [P, C.c_int, C.c_int, P, P, P, P, P]
    h.slimProjectionReset.argtypes = [P, P, C.c_float, C.c_int, C.c_int, C.c_int, P]
    h.slimBuildMesh.argtypes = [P, C.c_uint32, P, C.c_uint32, P, C.c_uint32, P, P, C.c_uint32, P, P, P, P, P, P]
    h.slimReadMeshHeader.argtypes = [C.c_char_p, P]
    h.slimReadMesh.argtypes = [C.c_char_p, P]
    h.slimWriteMesh.argtypes = [C.c_char_p, P]
    h.slimReadTextureHeader.argtypes = [C.c_char_p, P, P]
    h.slimReadTexture.argtypes = [C.c_char_p, P, P, P]
    h.slimWriteTexture.argtypes = [C.c_char_p, P]
    h.slimSaveScene.argtypes = [C.c_char_p, P]
    h.slimReadSceneHeader.argtypes = [C.c_char_p, P, P]
    h.slimLoadScene.argtypes = [C.c_char_p, P]
    h.slimBakeTexture.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P, P, P, P, P]
    h.slimBakeTextureOnGPU.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P, P, P, P, P]
    h.slimGetStageStats.argtypes = [P, C.c_int, P]
    h.slimResetStageStats.argtypes = []
    for name in ["slimRadianceCacheConfigure", "slimRadianceCacheGetConfig", "slimRadianceCacheGetStats"]:
        getattr(h, name).argtypes = [P]
    for name in ["slimRadianceCacheSetWeights", "slimRadianceCacheGetWeights", "slimRadianceCacheGetGradients"]:
        getattr(h, name).argtypes = [P, C.c_uint32]
    h.slimRadianceCacheQuery.argtypes = [P, C.c_uint32, P, P]
    h.slimRadianceCacheSaveState.argtypes = [P, C.c_uint64]
    h.slimRadianceCacheLoadState.argtypes = [P, C.c_uint64]
    for name in ["slimSynchronize", "slimRadianceCacheJoin", "slimGetLaunchCount", "slimBatchTune", "slimBatchSetPlan", "slimBatchGetPlan", "slimBatchRender"]:
        getattr(h, name).argtypes = [P]
    h.slimBatchSetRequests.argtypes = [P, C.c_uint32]
    h.slimPick.argtypes = [P, C.c_int, C.c_int, P]
    h.slimRadianceCacheTrain.argtypes = [P, P, C.c_uint32, P]
    for name in EXPORTS:
        if name not in ("slimGetLastError",):
            getattr(h, name).restype = C.c_int
    _lib = h
    return h


def check(rc):
    if rc != SLIM_OK:
        msg = lib().slimGetLastError().decode(errors="replace")
        raise SlimError(rc, msg)
    return rc


def ptr(a) -> int:
    """Address of a numpy array (or 0 for None)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a)


def projection_reset(orientation9, position3, focal_length, width, height, ssaa=False):
    """CameraRayProjection::reset (scene/camera.h:69-83)."""
    out = np.zeros((), L.PROJECTION)
    o = np.ascontiguousarray(orientation9, dtype=np.float32)
    p = np.ascontiguousarray(position3, dtype=np.float32)
    check(lib().slimProjectionReset(ptr(o), ptr(p), C.c_float(focal_length), width, height, int(bool(ssaa)), ptr(out)))
    return out


def set_render_options(engine=L.ENGINE_WAVEFRONT, ray_cones=L.CONES_REFERENCE, scene_bvh=L.SCENE_BVH_UPLOADED,
                       block_size=0, count_work=False, profile_stages=False, shadow_queue_mb=0,
                       radiance_cache=L.CACHE_OFF, row_bands=0):
    o = np.zeros((), L.RENDER_OPTIONS)
    o["engine"], o["ray_cones"], o["scene_bvh"] = engine, ray_cones, scene_bvh
    o["block_size"], o["count_work"] = block_size, int(bool(count_work))
    o["profile_stages"], o["shadow_queue_mb"] = int(bool(profile_stages)), shadow_queue_mb
    o["radiance_cache"], o["row_bands"] = radiance_cache, row_bands
    check(lib().slimSetRenderOptions(ptr(o)))


def stage_stats():
    """Per-stage launches, CUDA-event milliseconds and work counters."""
    out = np.zeros(16, L.STAGE_STATS)
    count = np.zeros(1, np.int32)
    check(lib().slimGetStageStats(ptr(out), len(out), ptr(count)))
    res = []
    for rec in out[:int(count[0])]:
        res.append({"name": rec["name"].decode(), "launches": int(rec["launches"]), "total_ms": float(rec["total_ms"]),
                    "work": {k: int(rec["work"][k]) for k in L.WORK_COUNTERS.names}})
    return res


def reset_stage_stats():
    check(lib().slimResetStageStats())


def work_counters():
    w = np.zeros((), L.WORK_COUNTERS)
    check(lib().slimGetWorkCounters(ptr(w)))
    return {k: int(w[k]) for k in L.WORK_COUNTERS.names}


def launch_count():
    """Kernels the library has launched since it was loaded."""
    n = np.zeros(1, np.uint64)
    check(lib().slimGetLaunchCount(ptr(n)))
    return int(n[0])


def pick(projection, x, y):
    """Selection::manipulate's pick behind pixel (x, y) (scene/selection.h:36-80)."""
    out = np.zeros((), L.PICK)
    check(lib().slimPick(ptr(projection), int(x), int(y), ptr(out)))
    return out
