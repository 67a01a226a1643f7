#!/usr/bin/env python3
"""Throughput of the B200 trace path on the 1080p mesh PBR workload.

Workload (config 2): 1920x1080, bounce depth 2, an icosphere (81,920
triangles) and a value-noise heightfield (130,050 triangles), 8 instances,
Cook-Torrance materials, 4 point lights, 1 emissive-quad area light,
synthetic seeded scene (no dataset).  A step is one frame: GPU refit of the
scene BVH + the full per-pixel path (primary, shadow and bounce rays, area
lights, glow, tone mapping, canvas write).

  value  Mrays/s with the scene resident in HBM (device buffers, CUDA events
         around each frame; L2 flushed between frames by writing 512 MiB).
  e2e    the same metric through the reference-facing C ABI with host
         buffers: per step slimUploadGeometries (H2D from pinned memory),
         slimRefitSceneBVH and slimRenderOnGPU into a pinned host canvas
         (D2H of pixels + depths).

Mrays/s counts every traced ray (primary + shadow + bounce), as counted by
the kernels' work counters on one untimed frame.

`--impl reference` times the reference's own CPU renderer (compiled from
its sources into oracle/_ref) on the host cores with the same scene.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s & ms/frame at 1080p: plain GPU vs radiance-cache at ≥40 dB PSNR"
UNIT = "Mrays/s"
L2_FLUSH_BYTES = 512 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--engine", default="auto", choices=["auto", "wavefront", "megakernel"],
                   help="auto (the library's default): the fused kernel for frames of mesh-free scenes whose "
                        "paths end at their first hit or that are small, the wavefront engine for the rest")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--config", default="config2", choices=["config1", "config2", "config3", "config4", "config5"],
                   help="workload (default: config2, the metric's 1080p mesh PBR scene)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--row-bands", type=int, default=0,
                   help="row bands of every wavefront frame (0: the library default; 1: whole frames, as for ncu "
                        "captures of whole-frame launches)")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    p.add_argument("--train-samples", type=int, default=65536,
                   help="radiance cache (config4): training paths per frame")
    p.add_argument("--train-suffix", type=int, default=0,
                   help="radiance cache (config4): 0 = training paths traced to full depth (as specified); k = "
                        "traced k bounces past the cache vertex into the cache's own answer")
    p.add_argument("--cache-scene", default="config2", choices=["config2", "config3"],
                   help="radiance cache (config4): the scene at depth 8 -- config 2's mesh PBR scene (as "
                        "specified) or config 3's glass/mirror/texture/IBL scene")
    p.add_argument("--no-cache-block", action="store_true",
                   help="default workload: skip the radiance-cache comparison block")
    p.add_argument("--no-batch-block", action="store_true",
                   help="default workload: skip the batched-requests (config 5) block")
    p.add_argument("--batch-requests", type=int, default=64,
                   help="config5: requests per batch (64 as specified; fewer for small profiling cases)")
    p.add_argument("--batch-small", action="store_true",
                   help="config5: resolutions drawn from 320x180 and 640x360 only (small profiling cases)")
    return p.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(values, device, world):
    """Every rank's timings reduced to the slowest rank's (the job ends when
    the last replica does): an all-reduce MAX over the process group."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def whole_job_rate(units_per_rank_step, steps, world, total_ms):
    """Units all ranks processed per second (replicas: every rank does the
    same per-step work), in millions."""
    return units_per_rank_step * steps * world / (total_ms / 1000.0) / 1e6


def device_uuid(dev):
    """NVML name of the CUDA device (CUDA_VISIBLE_DEVICES may renumber devices)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    NVML is polled from a thread every 2 ms (read-only queries), so even a
    timed region of a few milliseconds gets samples; nvidia-smi -lms 200 is
    the fallback when NVML cannot be loaded."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"
    REASONS = [("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4)]

    def __init__(self, index, uuid=None):
        self.index = index
        self.uuid = uuid
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []
        self.stop_flag = threading.Event()

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            if self.uuid:
                self.handle = pynvml.nvmlDeviceGetHandleByUUID(self.uuid)
            else:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _poll(self):
        p = self.nvml
        while not self.stop_flag.is_set():
            try:
                mhz = p.nvmlDeviceGetClockInfo(self.handle, p.NVML_CLOCK_SM)
                bits = p.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((float(mhz), int(bits)))
            except Exception:
                break
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            sms = [m for m, _ in self.samples]
            reasons = sorted({n for _, b in self.samples for n, bit in self.REASONS if b & bit})
            return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": float(self.max_mhz),
                    "reasons": reasons, "samples": len(sms), "source": "nvml, 2 ms polling"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = [n for n, _ in self.REASONS]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(sms), "source": "nvidia-smi -lms 200"}


def algorithmic_bytes(w, pixels=None):
    """Bytes the path must touch (memory-hierarchy roofline): 32 B per BVH
    node test, 64 B per triangle test, 64 B per mesh-hit attribute fetch,
    72 B per instance test, 16 B per texel-quad tap, plus 20 B per pixel of
    framebuffer written (a frame: one per primary ray; a stage: `pixels`)."""
    fb = w["primary_rays"] if pixels is None else pixels
    return (32 * (w["scene_node_tests"] + w["mesh_node_tests"]) + 64 * w["triangle_tests"] +
            64 * w["mesh_hit_fetches"] + 72 * w["geometry_tests"] + 16 * w["texel_taps"] + 20 * fb)


def reference_order_stage_bytes(w):
    """Algorithmic bytes of one frame split by wavefront stage, from the fused
    engine's counters (every ray walked in the reference's order, any-hit
    traversal work counted apart): extend = the closest-hit walks (scene and
    mesh nodes, triangles, instances, hit attribute fetches), shadow = the
    any-hit walks' scene nodes and instances, shadow_mesh = their mesh nodes
    and triangles."""
    if "shadow_scene_node_tests" not in w:
        return {}
    closest_nodes = w["scene_node_tests"] + w["mesh_node_tests"] - w["shadow_scene_node_tests"] - w["shadow_mesh_node_tests"]
    return {"extend": 32 * closest_nodes + 64 * (w["triangle_tests"] - w["shadow_triangle_tests"]) +
                      64 * w["mesh_hit_fetches"] + 72 * (w["geometry_tests"] - w["shadow_geometry_tests"]),
            "shadow": 32 * w["shadow_scene_node_tests"] + 72 * w["shadow_geometry_tests"],
            "shadow_mesh": 32 * w["shadow_mesh_node_tests"] + 64 * w["shadow_triangle_tests"]}


# Cache-level utilisation of the persistent mesh walks, from one
#   ncu --set full --clock-control none -k regex:<kernel> -s 2 -c 1
# launch each (config 2, 1920x1080, whole-frame passes; profiles/ holds the table): L1TEX and L2 (lts) throughput as
# a share of their hardware peaks.  The walks read nodes and triangles mostly from L1 (72-77 % hit rate) and wait on
# the latency of those dependent loads: L1 runs at half to three quarters of its peak, L2 at a tenth.
MEMORY_LEVELS = {
    "config2": {"k_extend_mesh": {"l1tex_throughput_pct": 50.9, "lts_throughput_pct": 10.4, "l1tex_hit_pct": 77.0,
                                  "warps_active_pct": 35.1, "threads_per_instruction": 16.3},
                "k_shadow_mesh": {"l1tex_throughput_pct": 72.8, "lts_throughput_pct": 15.1, "l1tex_hit_pct": 72.3,
                                  "warps_active_pct": 52.5, "threads_per_instruction": 18.6}},
}


# DRAM bytes (read + write) per launch of a stage, measured with
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum --clock-control none
# on the bench's own command (profiles/ holds the per-kernel table).  ncu flushes caches before every kernel, so
# these are cold-cache bytes.  A stage launch is all kernels of one round: extend = scene + mesh + resolve + overflow.
TRAFFIC_BYTES_PER_LAUNCH = {
    ("config2", "extend"): 180.0e6,       # rounds 1 and 2: 259 MB and 101 MB
    ("config2", "shadow_mesh"): 61.6e6,   # 93.0 MB and 30.2 MB
}
PIXEL_STAGES = ("shade", "tail", "fused")   # stages that write the framebuffer
CACHE_WARMUP_FRAMES = 32   # radiance-cache frames trained before the timed ones


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def frame_rays(workload):
    """Rays of one frame in the reference's order (primary + shadow +
    bounce), counted by the oracle on every host core."""
    from oracle import bindings as O
    from slimtracincpp_b200 import layout as L
    _, _, work = O.oracle_render(workload.scene, workload.projection(), workload.settings, workload.width,
                                 workload.height, layout=L, count=True, threads=0)
    return work["primary_rays"] + work["shadow_rays"] + work["bounce_rays"]


def reference_frames(workload, seconds, min_frames=5, max_frames=200, threads=None):
    """Whole frames of the reference's own CPU renderer (oracle/_ref, the
    timing build) on the host cores, one warm-up frame, then frames until
    `seconds` of wall time and at least `min_frames` are spent.  Returns the
    per-frame seconds, the thread count and the build description."""
    from oracle import bindings as O
    from slimtracincpp_b200 import layout as L
    threads = threads or os.cpu_count() or 1
    lib, build = O.reference_timed()
    proj = workload.projection()
    args = (workload.scene, proj, workload.settings, workload.width, workload.height)
    O.reference_render(*args, threads=threads, layout=L, lib=lib)
    times = []
    while len(times) < max_frames and (len(times) < min_frames or sum(times) < seconds):
        t0 = time.perf_counter()
        O.reference_render(*args, threads=threads, layout=L, lib=lib)
        times.append(time.perf_counter() - t0)
    return times, threads, build


def reference_one_core_frame(workload):
    """One frame of the reference's unmodified single-threaded
    RayTracingRenderer::renderOnCPU (renderer/renderer.h:87-100), timing
    build; seconds."""
    from oracle import bindings as O
    from slimtracincpp_b200 import layout as L
    lib, _ = O.reference_timed()
    t0 = time.perf_counter()
    O.reference_render_cpu(workload.scene, workload.projection(), workload.settings, workload.width, workload.height,
                           layout=L, lib=lib)
    return time.perf_counter() - t0


def cpu_baseline(workload, seconds, rays=None):
    """The reference's own CPU renderer (oracle/_ref) on all host cores:
    whole frames of the same workload for about `seconds`, plus one frame of
    its single-threaded renderOnCPU.  Ray counts come from the oracle."""
    from oracle import bindings as O
    kind = "reference" if O.reference_available() else "port"
    rays = rays if rays is not None else frame_rays(workload)
    if kind == "port":   # no reference build: the oracle itself, all cores
        from slimtracincpp_b200 import layout as L
        t0 = time.perf_counter()
        O.oracle_render(workload.scene, workload.projection(), workload.settings, workload.width, workload.height,
                        layout=L, threads=0)
        dt = time.perf_counter() - t0
        return {"value": rays / dt / 1e6, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": kind,
                "sample": f"1 frame of {workload.width}x{workload.height} by the oracle port", "ms_per_frame": dt * 1e3,
                "seconds": dt}
    times, threads, build = reference_frames(workload, seconds)
    med = statistics.median(times)
    one = reference_one_core_frame(workload)
    return {"value": rays / med / 1e6, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{len(times)} whole {workload.width}x{workload.height} frames ({rays} rays each) after 1 "
                      f"warm-up frame, median frame time, {threads} threads claiming 4-row chunks; reference built {build}",
            "ms_per_frame": med * 1e3, "frames": len(times),
            "one_core": {"value": rays / one / 1e6, "unit": UNIT, "cores": 1, "ms_per_frame": one * 1e3,
                         "sample": "1 frame of the unmodified single-threaded renderOnCPU (incremental directions)"},
            "seconds": sum(times)}


def native_libraries_loaded():
    """Shared objects of this repository mapped into this process."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            path = line.split()[-1] if line.strip() else ""
            if path.endswith(".so") and str(ROOT) in path:
                out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def run_reference(args):
    """The reference's own CPU path on the host cores: the scene is built by
    the reference's own code (mesh BVHs, scene BVH, camera projection from
    oracle/_ref), then whole frames are rendered by its renderPixel on every
    host thread; this process never loads libslimtracer_b200."""
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    from oracle import bindings as O
    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libslimref.so was not built"}))
        return 0
    if args.config == "config5":
        print(json.dumps({"impl": "reference", "unavailable": "config5: the reference has no batched renderer"}))
        return 0
    from slimtracincpp_b200 import layout as L
    from slimtracincpp_b200 import scenes
    from slimtracincpp_b200.scene import HOST_BUILDERS
    HOST_BUILDERS.update(O.reference_host_builders(L))
    w = scenes.CONFIGS[args.config](args.seed)
    rays = frame_rays(w)
    lib, build = O.reference_timed()
    threads = os.cpu_count() or 1
    proj = w.projection()
    fargs = (w.scene, proj, w.settings, w.width, w.height)
    for _ in range(max(1, min(args.warmup, 3))):
        O.reference_render(*fargs, threads=threads, layout=L, lib=lib)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.reference_render(*fargs, threads=threads, layout=L, lib=lib)
        times.append(time.perf_counter() - t0)
    one = reference_one_core_frame(w)
    total = sum(times)
    value = rays * args.steps / total / 1e6
    loaded = native_libraries_loaded()
    assert not any("libslimtracer_b200" in p for p in loaded), loaded
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {args.config} scene)",
            "config": {"workload": w.name, "width": w.width, "height": w.height,
                       "max_depth": int(w.settings["max_depth"]), "geometries": len(w.scene.geometries),
                       "triangles": sum(m.triangle_count for m in w.scene.meshes), "parallelism": "host threads",
                       "rays_per_frame": rays},
            "ms_per_frame": 1000.0 * statistics.median(times), "frame_ms": [1000.0 * t for t in times],
            "one_core": {"value": rays / one / 1e6, "unit": UNIT, "cores": 1, "ms_per_frame": one * 1e3,
                         "sample": "1 frame of the unmodified single-threaded renderOnCPU"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{args.steps} whole frames ({rays} rays each), {threads} threads claiming 4-row chunks, "
                                       f"scene built by the reference's own code; reference built {build}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "native_so_loaded": loaded}
    print(json.dumps(line))
    return 0


NRC_FLOPS_PER_QUERY = 2 * (96 * 64 + 3 * 64 * 64 + 64 * 16)   # tensor-core MACs x 2 (output padded to 16)


def nrc_roofline(torch, native, w, dev, frames=4):
    """Tensor-pipe roofline of the cache's query kernel (k_nrc_infer): the
    network's flops per launch over its CUDA-event time, a few cache frames
    with per-stage events (the cache keeps its trained weights)."""
    from slimtracincpp_b200 import layout as L
    from slimtracincpp_b200.radiance_cache import RadianceCache
    from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport
    r = RayTracingRenderer(w.scene, 8)
    vp = Viewport(w.camera, w.width, w.height)
    sp = torch.cuda.current_stream(dev).cuda_stream
    pix = torch.empty((w.samples, 4), dtype=torch.float32, device=dev)
    dep = torch.empty(w.samples, dtype=torch.float32, device=dev)
    RadianceCache.configure(cache_depth=2, train_samples=65536, batch=16384, seed=0)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON, profile_stages=True)
    for _ in range(2):
        r.render_to_device(vp, pix.data_ptr(), dep.data_ptr(), sp)
    torch.cuda.synchronize()
    native.reset_stage_stats()
    for _ in range(frames):
        r.render_to_device(vp, pix.data_ptr(), dep.data_ptr(), sp)
    RadianceCache().join(sp)
    torch.cuda.synchronize()
    stats = {s["name"]: s for s in native.stage_stats()}
    queries = RadianceCache().stats()["queries"]
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    q = stats.get("cache_query")
    if not q or not q["launches"]:
        return None
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak_tf = float(peaks.get("bf16_tflops", 1590.0))
    ms = q["total_ms"] / q["launches"]
    ach = queries * NRC_FLOPS_PER_QUERY / (ms / 1000.0) / 1e12
    return {"kernel": "k_nrc_infer", "bound": "tensor", "achieved": ach, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": ach / peak_tf, "flops_per_query": NRC_FLOPS_PER_QUERY, "queries": queries, "ms_per_launch": ms,
            "peak_source": "measured (MEASURED_PEAKS.json bf16_tflops)" if peaks else "fallback 1590 TFLOP/s"}


def timed_frames(torch, native, r, vp, sp, stream, outputs, flush):
    """One device-resident frame (scene refit + render) per entry of
    `outputs` (pixel, depth tensors), L2 flushed before each, timed with
    CUDA events on the launching stream."""
    lib = native.lib()
    starts = [torch.cuda.Event(enable_timing=True) for _ in outputs]
    ends = [torch.cuda.Event(enable_timing=True) for _ in outputs]
    for i, (pix, dep) in enumerate(outputs):
        flush.zero_()
        starts[i].record(stream)
        native.check(lib.slimRefitSceneBVH(sp))
        r.render_to_device(vp, pix.data_ptr(), dep.data_ptr(), sp)
        ends[i].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in zip(starts, ends)]


def pinned_scene_record(torch, w):
    """The scene record with its per-frame arrays (geometries, lights) in
    pinned host memory, as an app keeps them; returns (record, keep-alive
    tensors, bytes the per-frame uploads move)."""
    from slimtracincpp_b200 import layout as L
    sd = w.scene.data.copy()
    keep, nbytes = [], 0
    for field, arr, dtype in (("geometries", w.scene.geometries, L.GEOMETRY), ("lights", w.scene.lights, L.LIGHT)):
        if not len(arr):
            continue
        t = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
        t.numpy().view(dtype)[:] = arr
        sd[field] = t.data_ptr()
        keep.append(t)
        nbytes += arr.nbytes
    return sd, keep, nbytes


def per_frame_uploads(lib, native, sd):
    """renderer.h:72-77's per-frame uploads of render(update_scene=true):
    lights, cameras, geometries; the scene BVH is refit on the device
    instead of rebuilt on the host and uploaded."""
    native.check(lib.slimUploadLights(native.ptr(sd)))
    native.check(lib.slimUploadCameras(native.ptr(sd)))
    native.check(lib.slimUploadGeometries(native.ptr(sd)))
    native.check(lib.slimRefitSceneBVH(None))


def frame_quality(pix, ref_pix):
    """PSNR of the 8-bit canvas and max abs error of the stored colours
    against the reference frame (the plain depth-8 frame)."""
    ref8 = torch_floor8(ref_pix)
    p8 = torch_floor8(pix)
    mse = float(((p8 - ref8) ** 2).mean())
    psnr = 99.0 if mse == 0 else 10.0 * float(np.log10(255.0 ** 2 / mse))
    return psnr, float((pix[:, :3] - ref_pix[:, :3]).abs().max())


def torch_floor8(pix):
    import torch
    return torch.floor(255.0 * torch.sqrt(pix[:, :3].clamp(0, 1)))


def cache_comparison(torch, native, w, dev, steps, warmup, train_samples, suffixes, seed=0, row_bands=0,
                     overlap=True):
    """`suffixes`: training suffixes (with `train_samples` paths per frame),
    or (suffix, train samples) pairs."""
    """Config 4 (config 2's scene at bounce depth 8): plain wavefront
    frames against radiance-cache frames (paths stop at vertex 2; each frame
    trains on `train_samples` paths with four Adam steps of 16,384, then the
    cache answers every query).  For every training suffix in `suffixes` (0:
    full-depth training paths, as specified; k: self-training k bounces into
    the cache's own answers) the cache starts from fresh weights, learns
    online for max(warmup, 16) frames, then `steps` frames are timed back to
    back (the span from the first frame's start to the join of the last
    frame's overlapped training) and each is scored against the plain
    depth-8 frame."""
    from slimtracincpp_b200 import layout as L
    from slimtracincpp_b200.radiance_cache import RadianceCache
    from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport
    lib = native.lib()
    st = w.settings
    r = RayTracingRenderer(w.scene, 8, int(st["skybox_color_texture_id"]), int(st["skybox_radiance_texture_id"]),
                           int(st["skybox_irradiance_texture_id"]))
    vp = Viewport(w.camera, w.width, w.height)
    n = w.samples
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def buffers(k):
        return [(torch.empty((n, 4), dtype=torch.float32, device=dev), torch.empty(n, dtype=torch.float32, device=dev))
                for _ in range(k)]

    def counted(mode):
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, count_work=True, radiance_cache=mode)
        out = buffers(1)
        native.check(lib.slimRefitSceneBVH(sp))
        r.render_to_device(vp, out[0][0].data_ptr(), out[0][1].data_ptr(), sp)
        torch.cuda.synchronize()
        wk = native.work_counters()
        return wk["primary_rays"] + wk["shadow_rays"] + wk["bounce_rays"]

    plain_rays = counted(L.CACHE_OFF)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    ref = buffers(1)
    for _ in range(warmup):
        native.check(lib.slimRefitSceneBVH(sp))
        r.render_to_device(vp, ref[0][0].data_ptr(), ref[0][1].data_ptr(), sp)
    torch.cuda.synchronize()

    def span(frames_out, join=None):
        # the frames back to back, each after its L2 flush: the span from the
        # first frame's start to the last frame's end (and the join of its
        # overlapped training), so both arms pay the same flushes
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        events = timed_frames(torch, native, r, vp, sp, stream, frames_out, flush)
        if join:
            join(sp)
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / len(frames_out), events

    plain_span, plain_ms = span(ref * steps)
    out = {"plain_depth8": {"ms_per_frame": plain_span, "rays_per_frame": plain_rays,
                            "mrays_s": plain_rays / (plain_span / 1000.0) / 1e6,
                            "frame_event_ms_mean": sum(plain_ms) / steps}, "cache": [],
           "timing": "ms_per_frame of both arms: span of the back-to-back frames, each after a 512 MiB L2-flush "
                     "write, over the frame count (the cache arm's span ends at the join of the last frame's "
                     "overlapped training); frame_event_ms: each frame's own CUDA events, flush excluded"}
    # the ablation: the same frame with the paths cut at the cache vertex and nothing added
    RadianceCache.configure(cache_depth=2, train_samples=train_samples, batch=16384, seed=seed, train=False)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_TRUNCATE)
    trunc = buffers(1)
    native.check(lib.slimRefitSceneBVH(sp))
    r.render_to_device(vp, trunc[0][0].data_ptr(), trunc[0][1].data_ptr(), sp)
    torch.cuda.synchronize()
    tq = frame_quality(trunc[0][0], ref[0][0])
    out["truncated_at_cache_vertex"] = {"psnr_db": tq[0], "max_abs": tq[1]}
    cache_warmup = max(warmup, CACHE_WARMUP_FRAMES)
    for variant in suffixes:
        suffix, samples = variant if isinstance(variant, tuple) else (variant, train_samples)
        cache = RadianceCache.configure(cache_depth=2, train_samples=samples, batch=16384, seed=seed,
                                        train_suffix=suffix, overlap=overlap)
        native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON, row_bands=row_bands)
        outs = buffers(steps)
        for _ in range(cache_warmup):
            native.check(lib.slimRefitSceneBVH(sp))
            r.render_to_device(vp, outs[0][0].data_ptr(), outs[0][1].data_ptr(), sp)
        cache.join(sp)
        torch.cuda.synchronize()
        launches0 = native.launch_count()
        per_frame, frame_ms = span(outs, cache.join)
        launches = native.launch_count() - launches0
        quality = [frame_quality(p, ref[0][0]) for p, _ in outs]
        rays = counted(L.CACHE_ON)
        cst = cache.stats()
        out["cache"].append({
            "train_targets": "full-depth paths traced by the tracer (as specified)" if suffix == 0 else
                             f"self-training: {suffix} bounce(s) past the cache vertex, then the cache's own answer",
            "train_suffix": suffix, "train_samples_per_frame": samples, "ms_per_frame": per_frame,
            "rays_per_frame": rays,
            "speedup_vs_plain_depth8": plain_span / per_frame,
            "speedup_frame_events": (sum(plain_ms) / steps) / (sum(frame_ms) / len(frame_ms)),
            "psnr_db_per_frame": [q[0] for q in quality], "max_abs_per_frame": [q[1] for q in quality],
            "min_psnr_db": min(q[0] for q in quality), "frame_event_ms": frame_ms,
            "cache_warmup_frames": cache_warmup, "gpu_launches": launches,
            "queries": cst["queries"], "train_samples": cst["train_samples"], "loss": cst["loss"]})
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)
    return out


def run_cache_bench(args, torch, dist, dev, rank, world, local):
    """Config 4: the config-2 scene at bounce depth 8.  Plain wavefront frames
    against radiance-cache frames (paths stop at vertex 2, 65,536 training
    paths and four Adam steps of 16,384 per frame, then the cache answers
    every query); every timed cache frame is scored against the plain
    depth-8 frame (PSNR of the 8-bit canvas, max abs of the stored values).
    `--train-suffix k` trains on paths that end in the cache's own answer k
    bounces past the cache vertex instead of full-depth paths."""
    from slimtracincpp_b200 import layout as L
    from slimtracincpp_b200 import native, scenes
    from slimtracincpp_b200.radiance_cache import RadianceCache
    from slimtracincpp_b200.renderer import RayTracingRenderer, make_canvas
    if args.cache_scene == "config3":
        w = scenes.config3(args.seed, max_depth=8)
        w.name = f"config4_cache_on_config3_glass_mirror_ibl_{w.width}x{w.height}_d8_cache2"
    else:
        w = scenes.config4(args.seed)
    lib = native.lib()
    n = w.samples
    steps = args.steps
    clocks = ClockSampler(local, device_uuid(dev))
    clocks.start()
    if world > 1:
        dist.barrier()
    cmp = cache_comparison(torch, native, w, dev, steps, args.warmup, args.train_samples, [args.train_suffix],
                           args.seed)
    if world > 1:
        dist.barrier()
    clock_info = clocks.stop()
    c = cmp["cache"][0]

    # end to end through the C ABI with host buffers, cache on
    st = w.settings
    r = RayTracingRenderer(w.scene, 8, int(st["skybox_color_texture_id"]), int(st["skybox_radiance_texture_id"]),
                           int(st["skybox_irradiance_texture_id"]))
    RadianceCache.configure(cache_depth=2, train_samples=args.train_samples, batch=16384, seed=args.seed,
                            train_suffix=args.train_suffix)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT, radiance_cache=L.CACHE_ON)
    pin_pix = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    pin_dep = torch.empty(n, dtype=torch.float32, pin_memory=True)
    sd, _keep, h2d = pinned_scene_record(torch, w)
    cv, _, _ = make_canvas(w.width, w.height, L.AA_NONE)
    cv["pixels"], cv["depths"] = pin_pix.data_ptr(), pin_dep.data_ptr()
    proj = w.projection()
    for _ in range(max(args.warmup, CACHE_WARMUP_FRAMES)):
        per_frame_uploads(lib, native, sd)
        native.check(lib.slimRenderOnGPU(native.ptr(cv), native.ptr(proj), native.ptr(r.settings)))
    t0 = time.perf_counter()
    for _ in range(steps):
        per_frame_uploads(lib, native, sd)
        native.check(lib.slimRenderOnGPU(native.ptr(cv), native.ptr(proj), native.ptr(r.settings)))
    e2e_s = time.perf_counter() - t0
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)

    cache_total, plain_total, e2e_s = max_over_ranks([c["ms_per_frame"] * steps,
                                                      cmp["plain_depth8"]["ms_per_frame"] * steps, e2e_s], dev, world)
    value = whole_job_rate(c["rays_per_frame"], steps, world, cache_total)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
            "ms_per_step": cache_total / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 trace, bf16 MLP (f32 accumulate)", "data": f"synthetic (seeded {args.cache_scene} scene, depth 8)",
            "config": {"workload": w.name, "width": w.width, "height": w.height, "max_depth": 8, "cache_depth": 2,
                       "train_samples_per_frame": args.train_samples, "train_suffix": args.train_suffix,
                       "batch": 16384, "learning_rate": 1e-2, "cache_warmup_frames": c["cache_warmup_frames"],
                       "engine": "wavefront", "parallelism": f"replicas x{world}",
                       "l2": "flushed between steps (512 MiB write)", "rays_per_frame": c["rays_per_frame"]},
            "ms_per_frame": cache_total / steps,
            "plain_depth8": cmp["plain_depth8"],
            "speedup_vs_plain_depth8": plain_total / cache_total,
            "psnr_db_per_frame": c["psnr_db_per_frame"], "max_abs_per_frame": c["max_abs_per_frame"],
            "cache": {k: c[k] for k in ("queries", "train_samples", "loss", "train_targets")},
            "e2e": {"value": c["rays_per_frame"] * steps * world / e2e_s / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(pin_pix.numel() * 4 + pin_dep.numel() * 4),
                    "ms_per_step": 1000.0 * e2e_s / steps,
                    "per_step": "slimUploadLights/Cameras/Geometries (pinned), slimRefitSceneBVH, slimRenderOnGPU "
                                "into a pinned canvas"},
            "clocks": clock_info,
            "gpu_launches": c["gpu_launches"]}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def batch_comparison(torch, native, dev, steps, warmup, seed=0, meshes=None, count=64, resolutions=None):
    """Config 5: 64 requests (own seeded scenes, 320x180 ... 3840x2160, depth
    1-8, every other one with the radiance cache) rendered as one batch --
    captured in a CUDA graph, plan chosen by the project autotuner (waves over
    shared queues, or the plain requests in one persistent launch beside the
    cache requests' waves) -- against rendering them one at a time (a batch
    of one each, same plan, same graph replay).  Both plans are also timed
    on their own."""
    import numpy as np
    from slimtracincpp_b200 import layout as L
    from slimtracincpp_b200 import scenes
    from slimtracincpp_b200.batch import BatchRenderer
    from slimtracincpp_b200.radiance_cache import RadianceCache
    from slimtracincpp_b200.scene import Scene, geometry
    meshes = meshes if meshes is not None else scenes.config2_meshes()
    reqs = scenes.config5(seed, count=count, meshes=meshes, resolutions=resolutions)
    assets = Scene(np.array([geometry(L.GEOMETRY_SPHERE, 0)]), np.array([L.default_material()]), meshes=meshes)
    batch = BatchRenderer(assets)
    RadianceCache.configure(cache_depth=2, train_samples=65536, batch=16384, seed=seed)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    outs = [(torch.zeros((q.samples, 4), dtype=torch.float32, device=dev),
             torch.zeros(q.samples, dtype=torch.float32, device=dev)) for q in reqs]
    ptrs = [(p.data_ptr(), d.data_ptr()) for p, d in outs]
    pixels = sum(q.samples for q in reqs)

    # rays of one batch, counted by the kernels (untimed)
    native.set_render_options(engine=L.ENGINE_WAVEFRONT, count_work=True)
    batch.set_requests(reqs, ptrs)
    batch.render(sp)
    batch.synchronize(sp)
    wk = native.work_counters()
    rays = wk["primary_rays"] + wk["shadow_rays"] + wk["bounce_rays"]
    native.set_render_options(engine=L.ENGINE_WAVEFRONT)

    def timed(k):
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        for i in range(k):
            starts[i].record(stream)
            batch.render(sp)
            ends[i].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in zip(starts, ends)]

    batch.set_requests(reqs, ptrs)
    plan = batch.tune(sp)
    plans = {}
    for name, persistent in (("waves", False), ("persistent", True)):
        batch.set_plan(plan["queue_capacity"], plan["tile_pixels"], plan["block_size"], persistent)
        batch.render(sp)
        plans[name] = statistics.median(timed(3))
    batch.set_plan(plan["queue_capacity"], plan["tile_pixels"], plan["block_size"], plan["persistent"])
    for _ in range(warmup):
        batch.render(sp)
    batch.synchronize(sp)
    launches0 = native.launch_count()
    batch_ms = timed(steps)
    launches = native.launch_count() - launches0
    plan.update({k: v for k, v in batch.plan().items() if k in ("graph_nodes", "waves")})

    # end to end: the batch plus every canvas read back to pinned host memory
    pins = [(torch.empty_like(p, device="cpu").pin_memory(), torch.empty_like(d, device="cpu").pin_memory())
            for p, d in outs]
    e2e_steps = max(1, steps // 4)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        batch.render(sp)
        for (hp, hd), (p, d) in zip(pins, outs):
            hp.copy_(p, non_blocking=True)
            hd.copy_(d, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    d2h = sum(p.numel() * 4 + d.numel() * 4 for p, d in outs)

    # one at a time: each request as a batch of one, same plan, graph replay
    single_ms = []
    for q, ptr in zip(reqs, ptrs):
        batch.set_requests([q], [ptr])
        batch.set_plan(plan["queue_capacity"], plan["tile_pixels"], plan["block_size"], plan["persistent"])
        batch.render(sp)
        single_ms.append(sum(timed(3)) / 3)
    ms = sum(batch_ms) / steps
    return {"workload": f"config5_batch_{len(reqs)}_requests" + ("_small" if resolutions else ""),
            "requests": len(reqs), "pixels": pixels,
            "rays_per_batch": rays, "cache_requests": sum(q.radiance_cache != 0 for q in reqs),
            "resolutions": [f"{q.width}x{q.height}" for q in reqs],
            "max_depths": [int(q.settings["max_depth"]) for q in reqs],
            "batch_ms": ms, "batch_ms_total": sum(batch_ms), "mrays_s": rays / (ms / 1000.0) / 1e6,
            "plan": plan, "plans_ms": plans,
            "one_at_a_time": {"total_ms": sum(single_ms), "per_request_ms": single_ms,
                              "mrays_s": rays / (sum(single_ms) / 1000.0) / 1e6},
            "speedup_vs_one_at_a_time": sum(single_ms) / ms,
            "e2e": {"value": rays * e2e_steps / e2e_s / 1e6, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": 1000.0 * e2e_s / e2e_steps},
            "gpu_launches": launches, "steps": steps}


def run_batch_bench(args, torch, dist, dev, rank, world, local):
    """Config 5 as its own line (see batch_comparison)."""
    from slimtracincpp_b200 import native
    clocks = ClockSampler(local, device_uuid(dev))
    clocks.start()
    if world > 1:
        dist.barrier()
    b = batch_comparison(torch, native, dev, args.steps, args.warmup, args.seed, count=args.batch_requests,
                         resolutions=[(320, 180), (640, 360)] if args.batch_small else None)
    if world > 1:
        dist.barrier()
    clock_info = clocks.stop()
    total_ms, e2e_ms = max_over_ranks([b["batch_ms_total"], b["e2e"]["ms_per_step"]], dev, world)
    value = whole_job_rate(b["rays_per_batch"], args.steps, world, total_ms)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 trace, bf16 MLP (f32 accumulate)",
            "data": "synthetic (64 seeded request scenes)",
            "config": {"workload": b["workload"], "requests": b["requests"], "pixels": b["pixels"],
                       "rays_per_batch": b["rays_per_batch"], "cache_requests": b["cache_requests"],
                       "resolutions": b["resolutions"], "max_depths": b["max_depths"],
                       "parallelism": f"replicas x{world}",
                       "l2": "no flush: canvases and queues (> 3 GB) exceed L2"},
            "batch_ms": total_ms / args.steps, "plan": b["plan"], "plans_ms": b["plans_ms"],
            "one_at_a_time": b["one_at_a_time"], "speedup_vs_one_at_a_time": b["speedup_vs_one_at_a_time"],
            "e2e": dict(b["e2e"], value=b["rays_per_batch"] * world / (e2e_ms / 1000.0) / 1e6, ms_per_step=e2e_ms),
            "clocks": clock_info,
            "gpu_launches": b["gpu_launches"]}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_info()
    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.config == "config4":
        return run_cache_bench(args, torch, dist, dev, rank, world, local)
    if args.config == "config5":
        return run_batch_bench(args, torch, dist, dev, rank, world, local)

    from slimtracincpp_b200 import layout as L
    from slimtracincpp_b200 import native, scenes
    from slimtracincpp_b200.renderer import RayTracingRenderer, Viewport, make_canvas

    engine = {"auto": L.ENGINE_AUTO, "wavefront": L.ENGINE_WAVEFRONT, "megakernel": L.ENGINE_MEGAKERNEL}[args.engine]
    w = scenes.CONFIGS[args.config](args.seed)
    lib = native.lib()
    st = w.settings
    r = RayTracingRenderer(w.scene, int(st["max_depth"]), int(st["skybox_color_texture_id"]),
                           int(st["skybox_radiance_texture_id"]), int(st["skybox_irradiance_texture_id"]))
    vp = Viewport(w.camera, w.width, w.height)
    n = w.samples
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    # Counted frames (untimed).  The fused kernel walks every ray in the
    # reference's order: its counters are the reference algorithm's work for
    # the frame.  The timed engine's own counters give each stage's work.
    d_pix = torch.empty((n, 4), dtype=torch.float32, device=dev)
    d_dep = torch.empty(n, dtype=torch.float32, device=dev)
    native.set_render_options(engine=L.ENGINE_MEGAKERNEL, count_work=True)
    native.check(lib.slimRefitSceneBVH(sp))
    r.render_to_device(vp, d_pix.data_ptr(), d_dep.data_ptr(), sp)
    torch.cuda.synchronize()
    work = native.work_counters()
    native.set_render_options(engine=engine, count_work=True, profile_stages=True, row_bands=args.row_bands)
    native.reset_stage_stats()
    native.check(lib.slimRefitSceneBVH(sp))
    r.render_to_device(vp, d_pix.data_ptr(), d_dep.data_ptr(), sp)
    torch.cuda.synchronize()
    stage_work = {s["name"]: s["work"] for s in native.stage_stats()}
    rays_per_frame = work["primary_rays"] + work["shadow_rays"] + work["bounce_rays"]
    engine_work = native.work_counters()
    assert engine_work["primary_rays"] + engine_work["shadow_rays"] + engine_work["bounce_rays"] == rays_per_frame

    # timed device-resident frames: the library's default frame (row bands
    # in flight on two streams), no per-stage events in the way
    native.set_render_options(engine=engine, row_bands=args.row_bands)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        native.check(lib.slimRefitSceneBVH(sp))
        r.render_to_device(vp, d_pix.data_ptr(), d_dep.data_ptr(), sp)
    torch.cuda.synchronize()
    clocks = ClockSampler(local, device_uuid(dev))
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches0 = native.launch_count()
    for i in range(args.steps):
        flush.zero_()
        starts[i].record(stream)
        native.check(lib.slimRefitSceneBVH(sp))
        r.render_to_device(vp, d_pix.data_ptr(), d_dep.data_ptr(), sp)
        ends[i].record(stream)
    launches = native.launch_count() - launches0
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clock_info = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)

    # The same frames again with every stage launch bracketed by CUDA events,
    # as whole frames (one row band) so that each launch has the GPU to
    # itself: per-stage times and the dominant stage's roofline.
    native.set_render_options(engine=engine, profile_stages=True, row_bands=1)
    for _ in range(2):
        native.check(lib.slimRefitSceneBVH(sp))
        r.render_to_device(vp, d_pix.data_ptr(), d_dep.data_ptr(), sp)
    torch.cuda.synchronize()
    native.reset_stage_stats()
    prof_ms = sum(timed_frames(torch, native, r, vp, sp, stream, [(d_pix, d_dep)] * args.steps, flush))
    stats = {s["name"]: s for s in native.stage_stats()}
    engine_used = "megakernel" if stats.get("fused", {}).get("launches") else "wavefront"

    # end to end through the C ABI with host buffers
    native.set_render_options(engine=engine, row_bands=args.row_bands)
    pin_pix = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    pin_dep = torch.empty(n, dtype=torch.float32, pin_memory=True)
    sd, _keep, h2d = pinned_scene_record(torch, w)
    cv, _, _ = make_canvas(w.width, w.height, L.AA_NONE)
    cv["pixels"], cv["depths"] = pin_pix.data_ptr(), pin_dep.data_ptr()
    proj = w.projection()
    for _ in range(args.warmup):
        per_frame_uploads(lib, native, sd)
        native.check(lib.slimRenderOnGPU(native.ptr(cv), native.ptr(proj), native.ptr(r.settings)))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        per_frame_uploads(lib, native, sd)
        native.check(lib.slimRenderOnGPU(native.ptr(cv), native.ptr(proj), native.ptr(r.settings)))
    e2e_s = time.perf_counter() - t0
    d2h = int(pin_pix.numel() * 4 + pin_dep.numel() * 4)

    # max over ranks
    total_ms, e2e_s = max_over_ranks([total_ms, e2e_s], dev, world)
    value = whole_job_rate(rays_per_frame, args.steps, world, total_ms)
    e2e_value = whole_job_rate(rays_per_frame, args.steps, world, e2e_s * 1000.0)

    # roofline of the dominant kernel
    timed = {k: v for k, v in stats.items() if v["launches"]}
    dom_name = max(timed, key=lambda k: timed[k]["total_ms"]) if timed else None
    peak, peak_kind = measured_peaks()
    roofline = None
    if dom_name:
        d = timed[dom_name]
        per_launch_ms = d["total_ms"] / d["launches"]
        launches_per_frame = d["launches"] / args.steps
        ref_bytes = reference_order_stage_bytes(work)
        if dom_name in ref_bytes:
            alg_frame, alg_source = ref_bytes[dom_name], "reference-order counts (fused engine), this stage's part"
        else:
            px = work["primary_rays"] if dom_name in PIXEL_STAGES else 0
            alg_frame, alg_source = algorithmic_bytes(stage_work[dom_name], px), "the stage's own counters"
        alg = alg_frame / max(1.0, launches_per_frame)
        achieved = alg / (per_launch_ms / 1000.0) / 1e9
        roofline = {"kernel": dom_name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                    "traffic": TRAFFIC_BYTES_PER_LAUNCH.get((args.config, dom_name)),
                    "traffic_note": "ncu dram read+write per stage launch, cold caches",
                    "algorithmic_bytes_per_launch": alg, "algorithmic_bytes_source": alg_source,
                    "ms_per_launch": per_launch_ms,
                    "share_of_frame": d["total_ms"] / prof_ms,
                    "timing": "CUDA events around every launch of the stage, whole-frame passes (row_bands=1)",
                    "memory_levels": {"kernels": MEMORY_LEVELS.get(args.config),
                                      "source": "ncu --set full, one launch per kernel, cold caches",
                                      "note": "the scene's nodes and triangles (34 MB) stay in the 126 MB L2 and "
                                              "mostly hit L1: the walks are bound by dependent-load latency, "
                                              "with L1TEX at 51-73 % and L2 at 10-15 % of peak throughput"}}
    frame_bytes = algorithmic_bytes(work)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {args.config} scene)",
            "config": {"workload": w.name, "width": w.width, "height": w.height,
                       "max_depth": int(w.settings["max_depth"]), "geometries": len(w.scene.geometries),
                       "triangles": sum(m.triangle_count for m in w.scene.meshes),
                       "textures": len(w.scene.textures), "lights": len(w.scene.lights),
                       "engine": args.engine, "engine_used": engine_used, "parallelism": f"replicas x{world}",
                       "row_bands": (args.row_bands or (2 if n >= 1 << 18 else 1)) if engine_used == "wavefront" else 1,
                       "l2": "flushed between steps (512 MiB write)", "rays_per_frame": rays_per_frame,
                       "primary_rays": work["primary_rays"], "shadow_rays": work["shadow_rays"],
                       "bounce_rays": work["bounce_rays"]},
            "ms_per_frame": total_ms / args.steps,
            "frame_algorithmic_bytes": frame_bytes,
            "frame_achieved_gbs": frame_bytes / (total_ms / args.steps / 1000.0) / 1e9,
            "roofline": roofline,
            "stages_ms_per_frame": {k: v["total_ms"] / args.steps for k, v in timed.items()},
            "stage_profile": {"ms_per_frame": prof_ms / args.steps, "row_bands": 1,
                              "note": "stage times from a second timed loop with per-launch CUDA events"},
            "stage_work_per_frame": {k: v for k, v in stage_work.items() if any(v.values())},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": d2h,
                    "ms_per_step": 1000.0 * e2e_s / args.steps,
                    "per_step": "slimUploadLights/Cameras/Geometries (pinned), slimRefitSceneBVH, slimRenderOnGPU "
                                "into a pinned canvas"},
            "clocks": clock_info,
            "gpu_launches": launches}
    if args.config == "config2" and engine_used == "wavefront" and not args.no_cache_block:
        # the metric's second half, in the same process: config 4 (this scene at
        # bounce depth 8), plain frames against radiance-cache frames
        w4 = scenes.config4(args.seed, meshes=w.scene.meshes)
        cmp = cache_comparison(torch, native, w4, dev, args.steps, args.warmup, args.train_samples,
                               [0, 1, (1, args.train_samples // 2)],
                               args.seed)
        cmp["workload"] = w4.name
        cmp["nrc_roofline"] = nrc_roofline(torch, native, w4, dev)
        line["radiance_cache"] = cmp
    if args.config == "config2" and engine_used == "wavefront" and not args.no_batch_block:
        # config 5 (64 batched requests over config 2's meshes), same process
        line["batch"] = batch_comparison(torch, native, dev, min(args.steps, 5), min(args.warmup, 3), args.seed,
                                         meshes=w.scene.meshes)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = {k: v for k, v in cpu_baseline(w, args.cpu_seconds).items() if k != "seconds"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
