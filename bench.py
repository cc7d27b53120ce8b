#!/usr/bin/env python
"""Benchmark of the sm_100a path-tracing core on the config-2 workload.

Workload (one step): render the seeded 1,024,002-triangle icosphere scene
(800 icospheres x 1280 triangles + ground quad, 16 emissive spheres) at
1920x1080, 64 spp, max depth 12, NEE + MIS, FP32 RGB -- the reference's
offline SceneRenderer::Render call (core/scene.cu:276-306).  The metric is
Mrays/s: closest-hit plus any-hit BVH queries per second, whole job.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 is launched with torch.distributed.run: every rank renders the same
image with its own sample streams (frame offset rank * spp) and the FP64
accumulators are summed to rank 0 with one NCCL reduce per step (weak scaling).
The reference arm times the reference's own path loop on the host cores:
CalculateRadiance and everything under it, compiled for the host from a
build-time copy of the reference's sources (oracle/_ref/libref_path.so, made
by `make -C oracle ref-path`; kind "reference"), or the C restatement in
oracle/ (kind "port") where that library was not built.  It prints the same
JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

import scenes  # noqa: E402
from aperture_b200 import Camera, RadianceCache, RenderParams, RenderStats, Scene, make_params, nrc_config  # noqa: E402
from sharding import job_totals, partition_jobs, rank_frame_offset, reduce_accumulators  # noqa: E402

METRIC = "Mrays/s"
WIDTH, HEIGHT, SPP, DEPTH = 1920, 1080, 64, 12
WORKLOAD = ("config2: 800 icospheres x 1280 triangles + 2-triangle ground (1,024,002 triangles) + 16 emissive "
            "spheres, seed 0xA11CE+2, 1920x1080, 64 spp, max depth 12, NEE+MIS, RR from depth 3, FP32 RGB")


def config_block(n_gpus: int) -> dict:
    return {"workload": WORKLOAD, "triangles": 1024002, "width": WIDTH, "height": HEIGHT, "spp": SPP,
            "max_depth": DEPTH, "camera": "spheres_camera(): pos (0,30,-150), fov 60",
            "l2": "flushed between timed steps (256 MiB write); path state 470 MB > L2",
            "parallelism": f"replicas x{n_gpus}, FP64 accumulators reduced with NCCL" if n_gpus > 1 else "single GPU"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ("active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                if self.uuid and self.uuid not in parts[0]:
                    continue
                try:
                    sm.append(float(parts[1].split()[0]))
                    smax.append(float(parts[2].split()[0]))
                except ValueError:
                    continue
                for name, val in zip(names[1:], parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ----------------------------------------------------------------------------- CPU legs
def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_cpu_impl(prefer_reference: bool = True):
    """(scene factory, kind): the reference's own path loop built for the host
    (oracle/_ref/libref_path.so, host math library) when present and
    preferred, else the C restatement of oracle/oracle.c."""
    if ORACLE not in sys.path:
        sys.path.insert(0, ORACLE)
    if prefer_reference:
        import reference_path
        if reference_path.available(False):
            return (lambda objs: reference_path.RefPathScene(objs, detmath=False)), "reference"
    import oracle
    return oracle.OracleScene, "port"


def cpu_sample(objs, cam: Camera, params: RenderParams, target_s: float, threads: int, osc=None,
               prefer_reference: bool = True) -> dict:
    """Render a bounded, image-wide sample of pixels at 1 spp on the host cores
    (every step-th pixel; the step shrinks, then spp grows, until one sample
    takes about target_s / 2 or more)."""
    factory, kind = reference_cpu_impl(prefer_reference)
    if osc is None:
        osc = factory(objs)
    npix = cam.width * cam.height

    def run(step: int, spp: int):
        q = make_params(spp=spp, max_depth=params.max_depth, rr_depth=params.rr_depth, use_nee=params.use_nee,
                        sky=params.sky, seed=params.seed)
        t0 = time.perf_counter()
        _, e, s = osc.render_image(cam, q, 0, npix, step=step, threads=threads)
        return time.perf_counter() - t0, e, s

    step, spp = 16384, 1                     # start with ~127 pixels spread over the image
    while True:
        dt, e, s = run(step, spp)
        if dt >= 0.5 * target_s:
            break
        if step > 1:
            step = max(1, int(step * max(dt, 1e-3) / target_s))
        else:
            spp = max(spp + 1, int(spp * target_s / max(dt, 1e-3)))
    return {"osc": osc, "value": (e + s) / dt / 1e6, "seconds": dt, "pixels": (npix + step - 1) // step,
            "ext": e, "shadow": s, "kind": kind, "step": step, "spp": spp}


CPU_KIND_NOTE = {
    "reference": "the reference's CalculateRadiance (core/render/render.cuh:460-999) and all it calls, built for the "
                 "host from its sources (oracle/ref_path_patch.py edits), host math library; per path it scans every "
                 "object for Overlap (render.cuh:536, intersection.cuh:399-414) and traverses its own BuildBVH, whose "
                 "triangle proxies sit at the mesh centre",
    "port": "the C restatement (oracle/oracle.c) with its own binned-SAH BVH over triangle bounds and Overlap "
            "once per render",
}


def relmse(img, ref) -> float:
    """mean over pixels and channels of (I - I_ref)^2 / (I_ref^2 + 1e-2)"""
    return float(((img.double() - ref) ** 2 / (ref * ref + 1e-2)).mean())


def fp64_reference(torch, dev, scene: Scene, cam, params: RenderParams, spp: int, offset: int, stream,
                   chunk: int = 256):
    """Per-pixel FP64 mean of `spp` samples of the plain tracer (the per-path
    parity-tested CUDA core), rendered in chunks into an FP64 accumulator on
    the GPU; sample streams from frame `offset` on, disjoint from the timed
    renders'.  Returns (image, seconds)."""
    npix = cam.width * cam.height
    acc = torch.zeros(npix * 3, dtype=torch.float64, device=dev)
    out = torch.empty(npix * 3, dtype=torch.float32, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for k in range(0, spp, chunk):
        q = make_params(spp=min(chunk, spp - k), max_depth=params.max_depth, rr_depth=params.rr_depth,
                        use_nee=params.use_nee, sky=params.sky, spectral=params.spectral,
                        frame_offset=offset + k)
        scene.render_device(cam, q, out.data_ptr(), acc.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    return acc / spp, time.perf_counter() - t0


# ----------------------------------------------------------------------------- ours
NRC_SIZES = {"small": (480, 270, 16384, 4096), "full": (1920, 1080, 16384, 4096), "box": (480, 270, 16384, 4096),
             "config3": (1280, 720, 16384, 4096)}


def nrc_setup(torch, dev, scene: Scene, mode: str, stream) -> dict:
    """The scene, camera and judges of a time-to-relMSE measurement: an FP64
    oracle image of `ref` spp of the plain tracer (per-pixel FP64 sums on the
    GPU) and the plain tracer's relMSE after `target` spp with its device
    time.  mode "box": the config-3 scene (box, SDF tori, fBm medium, depth
    16) in RGB; otherwise the config-2 scene."""
    w, h, ref_spp, target = NRC_SIZES[mode]
    depth = DEPTH
    spectral = 0
    if mode in ("box", "config3"):
        objs, vols, med = scenes.medium_box_scene(precision=16, grid=256, medium_grid=128)
        scene = Scene(objs, volumes=vols, device=dev.index)
        scene.set_medium(**med)
        cam = scenes.box_camera(w, h)
        depth = 16
        if mode == "config3":
            scene.set_spectral(64)
            spectral = 4
    else:
        cam = scenes.spheres_camera(w, h)
    npix = w * h
    out = torch.empty(npix * 3, dtype=torch.float32, device=dev)

    def plain(spp_total: int, offset: int, acc):
        ms = 0.0
        chunk = 256
        for k in range(0, spp_total, chunk):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            scene.render_device(cam, make_params(spp=min(chunk, spp_total - k), max_depth=depth, frame_offset=offset + k,
                                                 spectral=spectral),
                                out.data_ptr(), acc.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        return ms

    with torch.cuda.stream(stream):
        acc_ref = torch.zeros(npix * 3, dtype=torch.float64, device=dev)
        ref_ms = plain(ref_spp, 10_000_000, acc_ref)
        ref = acc_ref / ref_spp
        acc_p = torch.zeros_like(acc_ref)
        plain_ms = plain(target, 20_000_000, acc_p)
        e_plain = relmse_sum(acc_p, target, ref)
    return {"scene": scene, "cam": cam, "depth": depth, "ref": ref, "ref_spp": ref_spp, "ref_ms": ref_ms,
            "target": target, "plain_ms": plain_ms, "e_plain": e_plain, "mode": mode, "w": w, "h": h,
            "spectral": spectral}


def relmse_sum(acc, n, ref) -> float:
    """relMSE of the mean of n samples whose FP64 sums are in acc"""
    img = acc / n
    return float(((img - ref) ** 2 / (ref * ref + 1e-2)).mean())


def nrc_curve(torch, dev, S: dict, stream, k: int = 1, spread_c: float = 0.01, steps: int = 4,
              max_factor: float = 3.0, seed: int = 1) -> dict:
    """Time-to-relMSE of the cache-terminated tracer against the plain one:
    frames of k samples per pixel (cache trained online: 65536 training paths
    and `steps` optimiser steps of 16384 samples per frame, paths terminated
    where the spread exceeds sqrt(spread_c) x the primary footprint), run until
    the relMSE reaches the plain tracer's at `target` spp or the device time
    reaches max_factor x the plain tracer's.  Device time (CUDA events on the
    launching stream) excludes the relMSE evaluations."""
    scene, cam, depth, ref = S["scene"], S["cam"], S["depth"], S["ref"]
    npix = S["w"] * S["h"]
    cache = RadianceCache(scene, nrc_config(spread_c=spread_c, train_steps=steps, seed=seed))
    if S["spectral"]:
        cache.set_spectral(S["spectral"])
    acc_n = torch.zeros(npix * 3, dtype=torch.float64, device=dev)
    t_ms, reached, curve = 0.0, None, []
    max_ms = max_factor * S["plain_ms"]
    f, samples = 0, 0
    check = max(1, 16 // k)
    with torch.cuda.stream(stream):
        while t_ms < max_ms and samples < 262144:
            evs = []
            for _ in range(check):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                cache.render_frame(cam, make_params(spp=k, max_depth=depth, frame_offset=30_000_000 + samples,
                                                    spectral=S["spectral"]), None,
                                   acc_n.data_ptr(), train=True, stream=stream.cuda_stream)
                e1.record(stream)
                evs.append((e0, e1))
                f += 1
                samples += k
            evs[-1][1].synchronize()
            t_ms += sum(a.elapsed_time(b) for a, b in evs)
            e = relmse_sum(acc_n, samples, ref)
            curve.append((samples, round(t_ms, 2), e))
            if e <= S["e_plain"]:
                reached = t_ms
                break
            check = min(check * 2, max(1, 256 // k))
    best = min(c[2] for c in curve)
    return {"spp_per_frame": k, "spread_c": spread_c, "train_steps": steps, "frames": f, "samples": samples,
            "cache_ms": round(t_ms, 2), "cache_relmse": curve[-1][2], "cache_best_relmse": best,
            "reached": reached is not None,
            "time_to_relmse_speedup": round(S["plain_ms"] / reached, 3) if reached else None,
            "ms_per_sample": round(t_ms / max(samples, 1), 4),
            "curve": [(a, b, round(c, 7)) for a, b, c in curve[:: max(1, len(curve) // 10)]]}


def measure_nrc(torch, dev, scene: Scene, mode: str, stream, k: int = 1, spread_c: float = 0.01, steps: int = 4) -> dict:
    """Config 4 on the config-2 scene (mode small/full) or the config-3 scene
    in RGB (mode box): the time-to-relMSE curve of nrc_curve for one setting;
    for the config-2 scene also the 300-frame seeded spline camera path at
    1920x1080 (ms per frame, per-stage times)."""
    S = nrc_setup(torch, dev, scene, mode, stream)
    what = {"box": "config-3 scene (box + SDF tori + fBm medium), RGB",
            "config3": "config 3: box + SDF tori (256^3 half grid) + 128^3 half fBm medium, four wavelengths per path "
                       "(four-wavelength cache, 16 spectral bins)"}.get(mode, "config4 static view: config-2 scene")
    res = {"workload": f"{what} {S['w']}x{S['h']}, max depth {S['depth']}, {k} spp per frame, cache trained online "
                       f"(65536 training paths, {steps} steps of 16384 per frame), spread constant {spread_c}",
           "oracle_spp": S["ref_spp"], "oracle_ms": round(S["ref_ms"], 1), "plain_spp": S["target"],
           "plain_ms": round(S["plain_ms"], 2), "plain_relmse": S["e_plain"]}
    res.update(nrc_curve(torch, dev, S, stream, k, spread_c, steps))
    if mode == "box":
        return res
    if mode == "config3":
        res["config4_spline"] = spline_path(torch, dev, Scene(scenes.spheres_scene(), device=dev.index), stream)
        return res
    res["spline_1920x1080"] = spline_path(torch, dev, S["scene"], stream)
    return res


def spline_path(torch, dev, scene: Scene, stream) -> dict:
    """Config 4's 300-frame seeded spline camera path at 1920x1080 on the
    config-2 scene, 1 spp per frame with the cache trained online: ms per frame
    and per stage (the first 10 frames untimed)."""
    cams = scenes.spline_cameras(frames=300)
    acc_s = torch.zeros(1920 * 1080 * 3, dtype=torch.float64, device=dev)
    cache2 = RadianceCache(scene, nrc_config(seed=2))
    tot = {"render": 0.0, "infer": 0.0, "train": 0.0, "total": 0.0, "q": 0, "rays": 0}
    for j, c in enumerate(cams):
        st = cache2.render_frame(c, make_params(spp=1, max_depth=DEPTH, frame_offset=40_000_000 + j), None,
                                 acc_s.data_ptr(), train=True, stats=True, stream=stream.cuda_stream)
        if j >= 10:
            tot["render"] += st.render_ms
            tot["infer"] += st.infer_ms
            tot["train"] += st.train_ms
            tot["total"] += st.total_ms
            tot["q"] += st.queries
            tot["rays"] += st.extension_rays + st.shadow_rays
    n = len(cams) - 10
    return {
        "frames": len(cams), "timed_frames": n, "ms_per_frame": round(tot["total"] / n, 3),
        "render_ms": round(tot["render"] / n, 3), "infer_ms": round(tot["infer"] / n, 3),
        "train_ms": round(tot["train"] / n, 3), "queries_per_frame": int(tot["q"] / n),
        "tracer_mrays_per_s": round(tot["rays"] / (tot["render"] / 1e3) / 1e6, 1),
        "last_loss": round(float(st.loss), 5)}


def sweep_nrc(torch, dev, stream, mode: str = "box") -> dict:
    """The cache's time-to-relMSE over spp per frame {1, 4, 16} ({16, 64} for
    the 1920x1080 mode "full") x spread constant {0.01, 0.1, 1} x optimiser
    steps per frame {1, 4}, against one oracle and one plain measurement."""
    S = nrc_setup(torch, dev, None if mode in ("box", "config3") else Scene(scenes.spheres_scene(), device=dev.index),
                  mode, stream)
    runs = []
    for k in ((16, 64) if mode == "full" else (1, 4, 16)):
        for c in (0.01, 0.1, 1.0):
            for steps in (1, 4):
                r = nrc_curve(torch, dev, S, stream, k, c, steps)
                r.pop("curve")
                runs.append(r)
                print(json.dumps({"sweep": r}), flush=True)
    return {"workload": f"{mode} {S['w']}x{S['h']} depth {S['depth']}", "plain_spp": S["target"],
            "plain_ms": round(S["plain_ms"], 2), "plain_relmse": S["e_plain"], "oracle_spp": S["ref_spp"],
            "runs": runs}


def _timed_render(torch, dev, scene: Scene, cam, params, out, stream, ref_spp: int = 4096) -> dict:
    """One warm-up render, one render timed by the library's CUDA events, then
    the relMSE of the timed render's image against an FP64 image of ref_spp
    samples of the same tracer (outside the timing)."""
    scene.render_device(cam, params, out.data_ptr(), None, stream.cuda_stream, RenderStats())   # warm-up
    st = RenderStats()
    scene.render_device(cam, params, out.data_ptr(), None, stream.cuda_stream, st)
    stream.synchronize()
    rays = st.extension_rays + st.shadow_rays
    res = {"ms": round(st.total_ms, 3), "mrays_per_s": round(rays / (st.total_ms / 1e3) / 1e6, 1),
           "msamples_per_s": round(st.paths / (st.total_ms / 1e3) / 1e6, 2), "paths": st.paths, "rays": rays}
    if ref_spp:
        npix = cam.width * cam.height
        ref, secs = fp64_reference(torch, dev, scene, cam, params, ref_spp, 50_000_000, stream)
        res["relmse"] = relmse(out[: npix * 3], ref)
        res["relmse_oracle"] = f"FP64 per-pixel mean of {ref_spp} spp of the same tracer, disjoint sample streams " \
                               f"({secs:.1f} s)"
    return res


def measure_denoise(torch, dev, stream, scene: Scene, frames: int = 8, reps: int = 10) -> dict:
    """The denoiser on the headline scene at 1920x1080: `frames` interactive
    frames (spp 1) that record the guide buffers, then the bilateral filter
    (15 x 15 window) over their mean, timed with CUDA events on the launching
    stream after two warm-up launches."""
    from aperture_b200 import denoise_bilateral, render_frame_denoise
    w, h = WIDTH, HEIGHT
    n = w * h
    cam = scenes.spheres_camera(w, h)
    gbuf = torch.zeros(n * 48, dtype=torch.uint8, device=dev)
    stats = torch.zeros(n * 48, dtype=torch.uint8, device=dev)
    acc = torch.zeros(n * 3, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)  # the zero fills run on the default stream
    s = stream.cuda_stream
    for f in range(frames):
        render_frame_denoise(scene, cam, make_params(spp=1, max_depth=DEPTH, frame_offset=f), None, acc, gbuf,
                             stats, s)
    with torch.cuda.stream(stream):
        hdr = (acc / frames).float()
        out = torch.empty_like(hdr)
    for _ in range(2):
        denoise_bilateral(hdr, out, gbuf, stats, w, h, s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        denoise_bilateral(hdr, out, gbuf, stats, w, h, s)
    e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / reps
    per_px = 48 + 48 + 12 + 12
    return {"workload": f"bilateral filter (radius 7, t-test gated) of the config-2 scene at {w}x{h} after "
                        f"{frames} recorded frames",
            "ms": round(ms, 4), "mpixels_per_s": round(n / ms / 1e3, 1),
            "pair_weights_per_s_g": round(n * 225 / ms / 1e6, 2),
            "algorithmic_bytes_per_pixel": per_px,
            "achieved_gbs": round(n * per_px / ms / 1e6, 1),
            "bound": "compute (225 pair weights per pixel from shared memory)"}


def measure_config5(torch, dev, stream, njobs: int = 64) -> dict:
    """Config 5: njobs seeded render jobs -- resolutions log-uniform in
    128-1024 per axis, spp uniform in {4, 16, 64, 256}, scenes from the
    config-2 generator with triangle counts log-uniform in 10K-2M and their own
    seeds, every second job four wavelengths per path, every other pair of jobs
    with a radiance cache of its own.  The jobs without a cache run in one
    launch of the batch graph (device-side loop) after the autotuner; each
    cache job renders its samples as cache frames of up to 16 samples with online
    training (four-wavelength cache for the spectral ones).  Per job: paths,
    rays, Mrays/s of its part; relMSE against a 4096-spp FP64 image of the
    plain tracer for every eighth job."""
    import concurrent.futures as cf

    import spectral_tables
    from aperture_b200 import autotune_batch, render_batch
    from sharding import job_cost
    spectral_ok = spectral_tables.available()
    rng = np.random.default_rng(0xA11CE + 5)
    specs = []
    for j in range(njobs):
        tris = float(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        nsph = max(8, int(round(tris / 1280)))
        w = int(np.exp(rng.uniform(np.log(128), np.log(1024))))
        h = int(np.exp(rng.uniform(np.log(128), np.log(1024))))
        spp = int(rng.choice([4, 16, 64, 256]))
        specs.append({"job": j, "triangles": nsph * 1280 + 2, "spheres": nsph, "width": w, "height": h, "spp": spp,
                      "spectral": 4 if (spectral_ok and j % 2 == 1) else 0, "cache": (j // 2) % 2 == 1})
    t0 = time.perf_counter()

    def build(sp):
        sc = Scene(scenes.spheres_scene(seed=0xA11CE + 100 + sp["job"], n_spheres=sp["spheres"]), device=dev.index)
        if sp["spectral"]:
            sc.set_spectral(32)
        return sc

    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        built = list(ex.map(build, specs))
    build_s = time.perf_counter() - t0
    outs = [torch.empty(sp["width"] * sp["height"] * 3, dtype=torch.float32, device=dev) for sp in specs]
    torch.cuda.synchronize(dev)
    plain = [k for k, sp in enumerate(specs) if not sp["cache"]]
    jobs = [(built[k], scenes.spheres_camera(specs[k]["width"], specs[k]["height"]),
             make_params(spp=specs[k]["spp"], max_depth=DEPTH, spectral=specs[k]["spectral"]), outs[k].data_ptr(), None)
            for k in plain]
    tune = autotune_batch(jobs, probe_spp=4, stream=stream.cuda_stream)
    render_batch(jobs, stream=stream.cuda_stream)          # warm-up with the tuned knobs
    st = render_batch(jobs, stream=stream.cuda_stream)
    batch_rays = st.extension_rays + st.shadow_rays
    # cache jobs: frames of up to 16 samples per pixel, cache trained online
    cache_ms, cache_rays, cache_paths = 0.0, 0, 0
    for k, sp in enumerate(specs):
        if not sp["cache"]:
            continue
        cam = scenes.spheres_camera(sp["width"], sp["height"])
        c = RadianceCache(built[k], nrc_config(seed=k + 1))
        if sp["spectral"]:
            c.set_spectral(4)
        acc = torch.zeros(sp["width"] * sp["height"] * 3, dtype=torch.float64, device=dev)
        ms = 0.0
        for f in range(0, sp["spp"], 16):   # frames of 16 spp (the best frame size of the cache sweep)
            fs = c.render_frame(cam, make_params(spp=min(16, sp["spp"] - f), max_depth=DEPTH, spectral=sp["spectral"],
                                                 frame_offset=f),
                                None, acc.data_ptr(), train=True, stats=True, stream=stream.cuda_stream)
            ms += fs.total_ms
            cache_rays += fs.extension_rays + fs.shadow_rays
        cache_paths += sp["width"] * sp["height"] * sp["spp"]
        cache_ms += ms
        sp["cache_ms"] = round(ms, 3)
        outs[k].copy_((acc / sp["spp"]).float())
    # relMSE of every eighth job against a 4096-spp FP64 image of the plain tracer
    for k in range(0, njobs, 8):
        sp = specs[k]
        cam = scenes.spheres_camera(sp["width"], sp["height"])
        ref, _ = fp64_reference(torch, dev, built[k], cam,
                                make_params(spp=4096, max_depth=DEPTH, spectral=sp["spectral"]), 4096, 60_000_000,
                                stream)
        sp["relmse"] = relmse(outs[k], ref)
    costs = [job_cost(sp["width"], sp["height"], sp["spp"], sp["triangles"], sp["spectral"], sp["cache"])
             for sp in specs]
    total_ms = st.total_ms + cache_ms
    return {"workload": f"{njobs} seeded jobs: config-2 generator with 10K-2M triangles (log-uniform), resolutions "
                        "log-uniform 128-1024 per axis, spp in {4,16,64,256}, every second job four wavelengths, "
                        "half the jobs with their own radiance cache (frames of up to 16 spp, trained online); jobs "
                        "without a cache in one launch of the batch graph (device-side loop), autotuned",
            "jobs": njobs, "ms": round(total_ms, 3),
            "mrays_per_s": round((batch_rays + cache_rays) / (total_ms / 1e3) / 1e6, 1),
            "batch": {"jobs": len(plain), "ms": round(st.total_ms, 3),
                      "mrays_per_s": round(batch_rays / (st.total_ms / 1e3) / 1e6, 1),
                      "msamples_per_s": round(st.paths / (st.total_ms / 1e3) / 1e6, 2), "paths": st.paths,
                      "graph_launches": st.graph_launches, "loop_passes": st.loop_passes,
                      "autotuned": {"iterations_per_graph": tune.iterations_per_graph, "path_budget": tune.path_budget,
                                  "trace_blocks_per_sm": tune.trace_blocks_per_sm,
                                  "shade_blocks_per_sm": tune.shade_blocks_per_sm, "candidates": tune.candidates,
                                    "probe_ms_best": round(tune.best_ms, 3),
                                    "probe_ms_default": round(tune.default_ms, 3)}},
            "cache_jobs": {"jobs": njobs - len(plain), "ms": round(cache_ms, 3), "paths": cache_paths,
                           "mrays_per_s": round(cache_rays / max(cache_ms / 1e3, 1e-9) / 1e6, 1)},
            "scene_build_s": round(build_s, 1),
            "lpt_2gpu_makespan_share": round(max(sum(costs[j] for j in p) for p in partition_jobs(costs, 2))
                                             / sum(costs), 4),
            "per_job": specs}


def measure_configs(torch, dev, stream, c5_jobs: int) -> dict:
    """The other benchmark configurations, one timed render each after one
    warm-up (device time from the library's CUDA events): config 1 (box,
    256x256, 16 spp), config 3 (box + SDF torus on a 256^3 half grid + 128^3
    half fBm medium, 1280x720, 256 spp, depth 16, four wavelengths when the
    spectral tables are present) and config 5 (measure_config5, c5_jobs jobs)."""
    import spectral_tables
    res = {}
    out = torch.empty(1280 * 720 * 3, dtype=torch.float32, device=dev)
    sc1 = Scene(scenes.box_scene(), device=dev.index)
    r = _timed_render(torch, dev, sc1, scenes.box_camera(256, 256), make_params(spp=16, max_depth=8), out, stream)
    res["config1"] = dict(workload="box scene (34 triangles + cube light), 256x256, 16 spp, depth 8, RGB", **r)
    spectral = spectral_tables.available()
    objs, vols, med = scenes.medium_box_scene(precision=16, grid=256, medium_grid=128)
    sc3 = Scene(objs, volumes=vols, device=dev.index)
    sc3.set_medium(**med)
    if spectral:
        sc3.set_spectral(64)
    r = _timed_render(torch, dev, sc3, scenes.box_camera(1280, 720),
                      make_params(spp=256, max_depth=16, spectral=4 if spectral else 0), out, stream)
    res["config3"] = dict(workload="box + glass analytic torus + GGX torus on a 256^3 half SDF grid + 128^3 half fBm "
                                   "medium (sigma_t 2, albedo 0.8, g 0.3), 1280x720, 256 spp, depth 16, "
                                   + ("4 hero wavelengths, RGB LUT 64^3" if spectral else "RGB (spectral tables absent)"),
                          **r)
    if spectral:
        res["spectral_lut_512"] = measure_spectral_lut(torch)
    if c5_jobs > 0:
        res["config5"] = measure_config5(torch, dev, stream, c5_jobs)
    return res


def measure_spectral_lut(torch, res: int = 512) -> dict:
    """The reference-size RGB lookup table (512^3 entries of 4 floats, 2 GiB;
    PrecomputeRGBLUTKernel, spectrum_lut.cuh:12-38) built by the SIMT kernel
    and on the tensor cores, each timed by CUDA events after one warm-up build,
    and the largest difference between the two tables."""
    from aperture_b200 import LUT_SIMT, LUT_TENSOR, spectral_rgb_lut
    a, _ = spectral_rgb_lut(res, LUT_SIMT)
    a, ms_simt = spectral_rgb_lut(res, LUT_SIMT, out=a)
    b, _ = spectral_rgb_lut(res, LUT_TENSOR)
    b, ms_tc = spectral_rgb_lut(res, LUT_TENSOR, out=b)
    big = float(a.abs().max())
    diff = float((a - b).abs().max())
    entries = res ** 3
    flop = entries * (2 * 8 * 32 * 32 + 2 * 4 * 32)   # input layer, 7 blocks, output
    out = {"entries": entries, "simt_ms": round(ms_simt, 2), "tensor_ms": round(ms_tc, 2),
           "speedup": round(ms_simt / ms_tc, 2), "max_abs_diff_rel_to_max": diff / big,
           "network_tflops_simt": round(flop / (ms_simt / 1e3) / 1e12, 2),
           "network_tflops_tensor": round(flop / (ms_tc / 1e3) / 1e12, 2),
           "note": "tensor path: 6 bf16 products per fp32 product (three-term splits), so the MMA work is 6x the "
                   "network's fp32 FLOPs"}
    del a, b
    torch.cuda.empty_cache()
    return out


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != world:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}; launch N>1 with torch.distributed.run")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    props = torch.cuda.get_device_properties(local)
    uuid = str(getattr(props, "uuid", "") or "") or None

    objs = scenes.spheres_scene()
    scene = Scene(objs, device=local)
    cam = scenes.spheres_camera(WIDTH, HEIGHT)
    params = make_params(spp=SPP, max_depth=DEPTH, frame_offset=rank_frame_offset(rank, SPP))
    npix = WIDTH * HEIGHT
    stream = torch.cuda.Stream(device=dev)
    out = torch.empty(npix * 3, dtype=torch.float32, device=dev)
    accum = torch.zeros(npix * 3, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(stats: RenderStats | None):
        scene.render_device(cam, params, out.data_ptr(), accum.data_ptr(), stream.cuda_stream, stats)
        if world > 1:
            with torch.cuda.stream(stream):
                reduce_accumulators(accum, dist)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(RenderStats())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    sampler = ClockSampler(uuid) if rank == 0 else None
    if sampler:
        sampler.start()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    tot = {"ext": 0, "sh": 0, "paths": 0, "launches": 0, "ext_ms": 0.0, "sh_ms": 0.0, "ext_launch": 0,
           "sh_launch": 0}
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            st = RenderStats()
            ev[k][0].record(stream)
            step(st)
            ev[k][1].record(stream)
            tot["ext"] += st.extension_rays
            tot["sh"] += st.shadow_rays
            tot["paths"] += st.paths
            tot["launches"] += st.kernel_launches
            tot["ext_ms"] += st.extend_ms
            tot["sh_ms"] += st.shadow_ms
            tot["ext_launch"] += st.extend_launches
            tot["sh_launch"] += st.shadow_launches
            tot["ev"] = tot.get("ev", 0) + st.extend_node_visits
            tot["et"] = tot.get("et", 0) + st.extend_prim_tests
            tot["sv"] = tot.get("sv", 0) + st.shadow_node_visits
            tot["stt"] = tot.get("stt", 0) + st.shadow_prim_tests
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    total_ms, (all_rays, all_paths) = job_totals(total_ms, [tot["ext"] + tot["sh"], tot["paths"]],
                                                 dist if world > 1 else None, dev)
    value = all_rays / (total_ms / 1e3) / 1e6

    # end to end through the C ABI with host buffers (image copied back every step
    # into a page-locked host array; camera and parameters copied in by the call)
    e2e_s = []
    e2e_rays = 0
    host_img = torch.empty(npix * 3, dtype=torch.float32, pin_memory=True).numpy()
    for k in range(args.steps):
        t0 = time.perf_counter()
        img, st = scene.render(cam, params, out=host_img)
        e2e_s.append(time.perf_counter() - t0)
        e2e_rays += st.extension_rays + st.shadow_rays
    e2e_t, (e2e_r,) = job_totals(sum(e2e_s), [e2e_rays], dist if world > 1 else None, dev)
    e2e_value = e2e_r / e2e_t / 1e6

    if rank == 0:
        with open(os.path.join(ROOT, "tests", "golden", "algorithmic_bytes.json")) as f:
            ab = json.load(f)
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except Exception:
            pass
        hbm = peaks.get("hbm_gbs")
        peak_src = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        kernels = {
            "extend (closest hit)": (tot["ext_ms"], tot["ext_launch"], tot["ext"] * ab["extension"]["bytes_per_query"]),
            "shadow (any hit)": (tot["sh_ms"], tot["sh_launch"], tot["sh"] * ab["shadow"]["bytes_per_query"]),
        }
        dom = max(kernels, key=lambda k: kernels[k][0])
        ms, nl, byts = kernels[dom]
        per_launch_bytes = byts / max(nl, 1)
        per_launch_s = ms / 1e3 / max(nl, 1)
        achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else None
        l2 = measure_l2(torch, dev)
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tj = json.load(f)
            tk = "extend" if dom.startswith("extend") else "shadow"
            if tk in tj and "dram_bytes_per_query" in tj[tk]:
                traffic = tj[tk]["dram_bytes_per_query"] * (tot["ext"] if tk == "extend" else tot["sh"]) / max(nl, 1)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": config_block(world),
            "samples_per_s": round(all_paths / (total_ms / 1e3), 1),
            "rays": {"extension": tot["ext"], "shadow": tot["sh"], "per_path": round((tot["ext"] + tot["sh"]) / max(tot["paths"], 1), 4)},
            "kernel_ms": {"extend": round(tot["ext_ms"], 3), "shadow": round(tot["sh_ms"], 3), "total": round(total_ms, 3)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1) if achieved else None,
                         "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4) if achieved else None,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback",
                         "traffic": traffic,
                         "algorithmic_bytes_per_query": ab["extension" if dom.startswith("extend") else "shadow"]["bytes_per_query"],
                         "l2_copy_gbs_measured": round(l2, 1),
                         "frac_of_l2_copy": round(achieved / l2, 4) if achieved and l2 else None},
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": ctypes.sizeof(Camera) + ctypes.sizeof(RenderParams),
                    "d2h_bytes_per_step": npix * 3 * 4},
            "gpu_launches": int(tot["launches"]),
            "clocks": clocks,
        }
        if not args.no_relmse:
            ref_img, ref_s = fp64_reference(torch, dev, scene, cam, params, 4096, 50_000_000, stream)
            line["relmse"] = relmse(out, ref_img)
            line["relmse_oracle"] = (f"FP64 per-pixel mean of 4096 spp of the same tracer (sample streams disjoint "
                                     f"from the timed renders', {ref_s:.1f} s); relMSE of one timed step's 64-spp image")
            del ref_img
        if world == 1 and args.nrc != "off":
            line["nrc"] = measure_nrc(torch, dev, scene, args.nrc, stream, args.nrc_spp, args.nrc_c, args.nrc_steps)
        if world == 1 and args.configs > 0:
            line["other_configs"] = measure_configs(torch, dev, stream, args.configs)
        if world == 1 and not args.no_denoise:
            line["denoise"] = measure_denoise(torch, dev, stream, scene)
        if world == 1 and not args.no_cpu:
            cs = cpu_sample(objs, cam, params, args.cpu_seconds, cpu_threads())
            line["cpu_baseline"] = {"value": round(cs["value"], 6), "unit": "Mrays/s", "cores": cpu_threads(),
                                    "kind": cs["kind"], "what": CPU_KIND_NOTE[cs["kind"]],
                                    "sample": f"{cs['pixels']} pixels spread over the image (every {cs['step']}. pixel) at {cs['spp']} spp, "
                                              f"{cs['ext'] + cs['shadow']} queries in {cs['seconds']:.1f} s"}
            if cs["kind"] == "reference":
                cp = cpu_sample(objs, cam, params, min(args.cpu_seconds, 6.0), cpu_threads(), prefer_reference=False)
                line["cpu_baseline_port"] = {"value": round(cp["value"], 4), "unit": "Mrays/s", "cores": cpu_threads(),
                                             "kind": "port", "what": CPU_KIND_NOTE["port"],
                                             "sample": f"{cp['pixels']} pixels at {cp['spp']} spp, "
                                                       f"{cp['ext'] + cp['shadow']} queries in {cp['seconds']:.1f} s"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def measure_l2(torch, dev) -> float:
    """Copy bandwidth of an L2-resident 32 MiB buffer (read + write bytes)."""
    a = torch.empty(8 << 20, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    for _ in range(5):
        b.copy_(a)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(200):
        b.copy_(a)
    e.record()
    torch.cuda.synchronize()
    return 2 * a.numel() * 4 * 200 / (s.elapsed_time(e) / 1e3) / 1e9


# ----------------------------------------------------------------------------- reference arm
def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    objs = scenes.spheres_scene()
    cam = scenes.spheres_camera(WIDTH, HEIGHT)
    params = make_params(spp=SPP, max_depth=DEPTH)
    threads = cpu_threads()
    osc = None
    vals, secs, qs = [], [], 0
    sample = None
    for k in range(args.warmup + args.steps):
        cs = cpu_sample(objs, cam, params, args.cpu_seconds, threads, osc=osc)
        osc = cs["osc"]
        if k >= args.warmup:
            vals.append(cs["value"])
            secs.append(cs["seconds"])
            qs += cs["ext"] + cs["shadow"]
            sample = cs
    value = qs / sum(secs) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 6), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * sum(secs) / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": config_block(world), "impl": "reference",
        "cpu_baseline": {"value": round(value, 6), "unit": "Mrays/s", "cores": threads, "kind": sample["kind"],
                         "what": CPU_KIND_NOTE[sample["kind"]],
                         "sample": f"per step every {sample['step']}th pixel ({sample['pixels']} pixels) at {sample['spp']} spp "
                                   f"on {threads} host threads (OpenMP)"},
        "e2e": {"value": round(value, 6), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profile_queues() -> None:
    """One 8-spp render of the benchmark scene for ncu captures (-k/-s/-c select
    a launch of the steady state, where the path pool is full), then the mean
    extension and shadow queries per traversal launch of that render."""
    objs = scenes.spheres_scene()
    scene = Scene(objs)
    cam = scenes.spheres_camera(WIDTH, HEIGHT)
    params = make_params(spp=8, max_depth=DEPTH)
    img, st = scene.render(cam, params)
    print(json.dumps({"profile": "config2 at 8 spp", "iterations": st.extend_launches,
                      "extension_rays": st.extension_rays, "shadow_rays": st.shadow_rays,
                      "extension_per_launch": st.extension_rays / max(st.extend_launches, 1),
                      "shadow_per_launch": st.shadow_rays / max(st.shadow_launches, 1)}), flush=True)


def profile_denoise() -> None:
    """Two recorded frames of the headline scene at 1920x1080, then three
    bilateral-filter calls (for ncu captures of k_dn_ttest and k_dn_filter)."""
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    r = measure_denoise(torch, dev, stream, Scene(scenes.spheres_scene()), frames=2, reps=1)
    print(json.dumps({"profile": "denoise", **r}), flush=True)


def profile_nrc(width: int = 480, height: int = 270) -> None:
    """Six radiance-cache frames (config-2 scene, training on) for ncu
    captures of the cache kernels; prints the frame statistics."""
    objs = scenes.spheres_scene()
    scene = Scene(objs)
    cam = scenes.spheres_camera(width, height)
    import torch
    acc = torch.zeros(width * height * 3, dtype=torch.float64, device="cuda")
    cache = RadianceCache(scene, nrc_config())
    for f in range(6):
        st = cache.render_frame(cam, make_params(spp=1, max_depth=DEPTH, frame_offset=f), None, acc.data_ptr(),
                                train=True, stats=True)
        print(json.dumps({"frame": f, "ms": round(st.total_ms, 3), "render_ms": round(st.render_ms, 3),
                          "infer_ms": round(st.infer_ms, 3), "train_ms": round(st.train_ms, 3),
                          "queries": st.queries, "train_samples": st.train_samples, "loss": st.loss}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU sample length per measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-denoise", action="store_true", help="skip the denoiser measurement")
    ap.add_argument("--no-relmse", action="store_true",
                    help="skip the headline's relMSE (its 4096-spp FP64 image; for ncu launch lists)")
    ap.add_argument("--profile-denoise", action="store_true",
                    help="record two frames and run the bilateral filter three times (for ncu captures)")
    ap.add_argument("--configs", type=int, default=64,
                    help="also time configs 1, 3 and 5 (this many batch jobs); 0 skips")
    ap.add_argument("--nrc", choices=("off", "small", "full", "box", "config3"), default="config3",
                    help="radiance-cache time-to-relMSE measurement (config3: the config-3 scene with four "
                         "wavelengths at 1280x720, plus config 4's spline path; small / full: the config-2 scene "
                         "at 480x270 / 1920x1080; box: the config-3 scene in RGB at 480x270)")
    # defaults: the best of the 18 settings of the config-3 sweep (--nrc-sweep config3)
    ap.add_argument("--nrc-spp", type=int, default=16, help="samples per pixel of a cache frame")
    ap.add_argument("--nrc-c", type=float, default=1.0, help="spread constant of the cache's termination rule")
    ap.add_argument("--nrc-steps", type=int, default=4, help="optimiser steps per cache frame")
    ap.add_argument("--nrc-sweep", choices=("box", "small", "full", "config3"), default=None,
                    help="time-to-relMSE over spp per frame x spread constant x optimiser steps, then exit")
    ap.add_argument("--profile-nrc", action="store_true",
                    help="six radiance-cache frames (for ncu captures of the cache kernels)")
    ap.add_argument("--profile-size", default="480x270", help="frame size of --profile-nrc")
    ap.add_argument("--profile-lut", type=int, default=0,
                    help="build the spectral RGB lookup table of this resolution by both methods (for ncu captures)")
    ap.add_argument("--profile-queues", action="store_true",
                    help="render the workload once at 1 spp (for ncu captures) and print the per-depth queue sizes")
    args = ap.parse_args()
    if args.profile_queues:
        profile_queues()
        return
    if args.profile_lut:
        import torch
        from aperture_b200 import LUT_SIMT, LUT_TENSOR, spectral_rgb_lut
        a, ms_a = spectral_rgb_lut(args.profile_lut, LUT_SIMT)
        b, ms_b = spectral_rgb_lut(args.profile_lut, LUT_TENSOR)
        print(json.dumps({"profile": "spectral lut", "res": args.profile_lut, "simt_ms": ms_a, "tensor_ms": ms_b,
                          "max_abs_diff": float((a - b).abs().max())}), flush=True)
        return
    if args.nrc_sweep:
        import torch
        dev = torch.device("cuda", 0)
        r = sweep_nrc(torch, dev, torch.cuda.Stream(device=dev), args.nrc_sweep)
        print(json.dumps({"nrc_sweep": r}), flush=True)
        return
    if args.profile_denoise:
        profile_denoise()
        return
    if args.profile_nrc:
        w, h = (int(x) for x in args.profile_size.split("x"))
        profile_nrc(w, h)
        return
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up steps
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
