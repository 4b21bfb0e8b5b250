#!/usr/bin/env python
"""Throughput benchmark of the CUDA forward path tracer (Mpaths/s on one B200).

A step renders one full frame of the mesh-heavy workload: a seeded 1024x1024-vertex fBm
terrain (2,093,058 triangles) with 32 tessellated spheres of 20,480 triangles each
(40 % Lambert, 30 % Beckmann metal, 30 % glass IOR 1.5), lit by a 2048x1024 float32 sky
map plus a 0.53 degree sun, 1920x1080 pixels at 64 samples per pixel, max depth 16.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank renders the full frame with its own sample streams
(weak scaling) and the linear framebuffers are summed with one NCCL all-reduce per step.
The reference arm (--impl reference) times the CPU restatement of the reference tracer
(oracle/) on this machine's host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
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

METRIC = "Mpaths/s at 1 B200"
UNIT = "Mpaths/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def workload(args):
    from naivetrace_b200 import scenes
    if args.small:
        return scenes.terrain_spheres(xres=480, yres=270, terrain_n=256, sphere_level=4, num_spheres=32,
                                      env_w=512, env_h=256), 16, 16, "terrain_spheres_small"
    return scenes.terrain_spheres(), args.spp, 16, "terrain_spheres"


def workload_config(scene, spp, depth, name):
    cam = scene.camera
    return {
        "workload": f"{name}: fBm terrain + 32 spheres, {scene.num_triangles} triangles, sky map + sun, "
                    f"{cam.xres}x{cam.yres} at {spp} spp, max depth {depth}",
        "triangles": scene.num_triangles,
        "resolution": [cam.xres, cam.yres],
        "spp": spp,
        "max_depth": depth,
        "paths_per_step": cam.xres * cam.yres * spp,
        "l2_policy": "inputs larger than L2: BVH + triangles ~0.3 GB and ~30 GB of path state per wave of 2^27 paths",
    }


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, power, reasons = [], [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(names[1:], parts[5:9]):
                if val.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "power_w_max": max(power),
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        peaks = json.loads(PEAKS_FILE.read_text())
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def cpu_reference(scene, spp, depth, budget_s=20.0, chunk_pixels=16384, seed=1):
    """Times the oracle (CPU restatement of the reference pt) on all host cores over a
    bounded sample of the frame at 1 sample per pixel: chunks of consecutive pixels spread
    uniformly over the frame (chunk k starts at chunk slot (k * 61) mod slots, so the first
    `slots` chunks visit every part of the frame once; later rounds use the next sample
    index), until about budget_s of CPU time.  Returns (Mpaths/s, cores, description)."""
    from oracle.oracle import OracleScene
    from naivetrace_b200.scene import make_params
    cores = os.cpu_count() or 1
    o = OracleScene(scene, make_params(max_ray_depth=depth))
    npix = o.npix
    chunk_pixels = max(1, min(chunk_pixels, npix))
    slots = max(1, npix // chunk_pixels)
    stride = 61 if np.gcd(61, slots) == 1 else 1
    acc = np.zeros(3 * npix)
    light = np.zeros(3 * npix)
    done_paths = 0
    t0 = time.perf_counter()
    k = 0
    while True:
        pb = ((k * stride) % slots) * chunk_pixels
        pe = npix if (k * stride) % slots == slots - 1 else pb + chunk_pixels
        o.render(1, seed=seed, sample_offset=k // slots, pixel_begin=pb, pixel_end=pe, nthreads=cores,
                 accum=acc, light_accum=light)
        done_paths += pe - pb
        k += 1
        el = time.perf_counter() - t0
        if el >= budget_s or k >= 100000:
            break
    mpaths = done_paths / el / 1e6
    desc = (f"{k} chunks of {chunk_pixels} consecutive pixels spread uniformly over the "
            f"{scene.camera.xres}x{scene.camera.yres} frame at 1 sample each ({done_paths} paths, "
            f"{min(k, slots)} of {slots} chunk slots, {el:.1f} s, depth {depth}) on {cores} threads")
    return mpaths, cores, desc


def config_figures(device, cpu_budget=5.0, frames=2):
    """Throughput of the plain tracer on the other configurations of the workload family,
    each with the CPU restatement timed beside it on a bounded sample:
    cfg 0 the Cornell box 256x256 at 16 spp (depth 10), cfg 2A the Cornell box filled with a
    homogeneous chromatic medium and cfg 2B the planet's atmosphere under a fisheye camera,
    both 1024x1024 at 128 spp (depth 32).  One untimed frame (allocation, warm-up), then
    `frames` frames timed with CUDA events on the library's stream; the same again with the
    hits shaded in traversal order instead of material-sorted order."""
    import torch

    from naivetrace_b200 import scenes
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    cfgs = [("cfg0_cornell_box", scenes.cornell_box(256, 256), 16, 10),
            ("cfg2a_cornell_box_medium", scenes.cornell_box_medium(1024, 1024), 128, 32),
            ("cfg2b_planet_atmosphere", scenes.planet_atmosphere(1024, 1024), 128, 32)]
    def frame_ms(scene, spp, depth, sort):
        g = GpuContext(scene, make_params(max_ray_depth=depth, device=device, sort_shading=sort))
        g.render(spp, 1)
        g.clear()
        g.reset_stats()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for k in range(frames):
            g.render(spp, 2 + k)
        b.record()
        torch.cuda.synchronize()
        st = g.stats()
        g.close()
        return a.elapsed_time(b) / frames, st

    out = {}
    for name, scene, spp, depth in cfgs:
        ms, st = frame_ms(scene, spp, depth, None)
        ms_unsorted, _ = frame_ms(scene, spp, depth, False)
        paths = scene.camera.xres * scene.camera.yres * spp
        v, cores, desc = cpu_reference(scene, spp, depth, budget_s=cpu_budget, chunk_pixels=4096)
        out[name] = {
            "workload": f"{scene.camera.xres}x{scene.camera.yres} at {spp} spp, max depth {depth}, "
                        f"{scene.num_triangles} triangles, {len(scene.media)} media",
            "ms_per_frame": ms,
            "ms_per_frame_traversal_order": ms_unsorted,
            "mpaths_per_s": paths / (ms * 1e-3) / 1e6,
            "mrays_per_s": (st["extension_rays"] + st["shadow_rays"]) / frames / (ms * 1e-3) / 1e6,
            "rays_per_path": (st["extension_rays"] + st["shadow_rays"]) / frames / paths,
            "error_flags": st["error_flags"],
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
            "gpu_over_cpu": (paths / (ms * 1e-3) / 1e6) / v if v > 0 else None,
        }
    return out


class GuidingWorkload:
    """The guiding workload (a room lit through a 0.3 x 0.3 gap, 1280x720, depth 12) with its
    converged reference: a 4096-spp plain render (16 passes of 256 spp)."""

    def __init__(self, xres=1280, yres=720, depth=12):
        from naivetrace_b200 import scenes
        from naivetrace_b200.algo import GpuContext
        from naivetrace_b200.scene import make_params
        self.xres, self.yres, self.depth = xres, yres, depth
        self.scene = scenes.guiding_room(xres, yres)
        self.params = make_params(max_ray_depth=depth)
        ref = GpuContext(self.scene, self.params)
        for k in range(16):
            ref.render(256, seed=1_000_000 + k)
        self.R = ref.framebuffer().astype(np.float64)
        ref.close()
        # Warm-up context: kernels loaded, memory pool filled.
        w = GpuContext(self.scene, self.params)
        w.render(4, 1)
        w.set_guiding(True, 1, seed=7)
        w.render(1, 2)
        w.close()

    def relmse(self, g):
        I = g.framebuffer().astype(np.float64)
        return float(np.mean((I - self.R) ** 2 / (self.R * self.R + 1e-2)))

    def curve(self, guided=False, tree=False, train_passes=8, budget_ms=1000.0, discard_training=False,
              **guide_kw):
        """relMSE after every pass against the wall time of the render calls so far (training
        included).  Plain runs double their spp per pass (1, 2, 4, ...); guided runs first
        render `train_passes` one-sample passes that train the guide after each pass, then
        freeze it and double.  With discard_training the training passes' samples are
        dropped from the image when the guide freezes (as the reference's guided tracer
        does), else every sample stays in the image (each is unbiased).  Returns the curve
        [(ms, spp in the image, relMSE)] and the context's stats."""
        from naivetrace_b200 import abi
        from naivetrace_b200.algo import GpuContext
        g = GpuContext(self.scene, self.params)
        kw = dict(seed=7)
        kw.update(guide_kw)
        if tree:
            kw.update(method=abi.GUIDE_TREE)
        # One untimed pass at the largest wave size (2^27 paths) allocates the path state
        # (with the guiding arrays for the guided run); the guide is not trained by it.
        if guided:
            g.set_guiding(True, 0, **kw)
        g.render(-(-(1 << 27) // (self.xres * self.yres)), 3)
        g.clear()
        g.reset_stats()

        def timed(spp, seed):
            t = time.perf_counter()
            g.render(spp, seed)
            return (time.perf_counter() - t) * 1e3

        pts, el, spp_total, seed = [], 0.0, 0, 10
        if guided and train_passes > 0:
            g.set_guiding(True, 1, **kw)
            for k in range(train_passes):
                el += timed(1, seed)
                seed += 1
                spp_total += 1
                if not discard_training:
                    pts.append((el, spp_total, self.relmse(g)))
            g.set_guiding(True, 0, **kw)
            if discard_training:
                g.clear()
                spp_total = 0
        spp = 1
        while el < budget_ms and spp_total < 1 << 14:
            el += timed(spp, seed)
            seed += 1
            spp_total += spp
            pts.append((el, spp_total, self.relmse(g)))
            spp *= 2
        st = g.stats()
        g.close()
        return pts, st


def time_to(pts, tgt):
    """Time at which a relMSE curve first reaches tgt (log-log interpolation between passes)."""
    prev = None
    for t, s, e in pts:
        if e <= tgt:
            if prev is None or prev[2] <= e:
                return t
            a = (np.log(prev[2]) - np.log(tgt)) / (np.log(prev[2]) - np.log(e))
            return float(np.exp(np.log(prev[0]) + a * (np.log(t) - np.log(prev[0]))))
        prev = (t, s, e)
    return None


def at_time(pts, t0):
    ts = np.log([x[0] for x in pts])
    es = np.log([x[2] for x in pts])
    return float(np.exp(np.interp(np.log(t0), ts, es)))


GUIDE_SETTINGS = dict(train_passes=2, discard_training=False, learning_rate=1e-3, record_pool=1 << 16,
                      batch=8192, steps_per_pass=64, max_depth=2)
# The guided configuration's own training settings: 2^18 records per step at lr 1e-2.
CONFIG_GUIDE_SETTINGS = dict(GUIDE_SETTINGS, batch=1 << 18, record_pool=1 << 18, learning_rate=1e-2)


def guiding_comparison(target=0.01, budget_ms=1000.0, settings=None):
    """Learned-guided against plain GPU tracing on the guiding workload: relMSE against a
    4096-spp plain render after every pass, with the wall time of the render calls
    (training included) summed.  Reports the time to reach relMSE `target`, their ratio and
    the relMSE of both at equal time; the tree guider runs the same schedule."""
    st_kw = dict(GUIDE_SETTINGS if settings is None else settings)
    wl = GuidingWorkload()
    plain, _ = wl.curve(False, budget_ms=budget_ms)
    guided, gst = wl.curve(True, budget_ms=budget_ms, **st_kw)
    cfg_guided, cst = wl.curve(True, budget_ms=budget_ms, **CONFIG_GUIDE_SETTINGS)
    tree_kw = dict(st_kw)
    tree_kw.update(tree_subdivision=200, tree_em_iters=4)
    tree, tst = wl.curve(True, tree=True, budget_ms=budget_ms, **tree_kw)
    quad_kw = dict(st_kw)
    quad_kw.update(tree_subdivision=200, tree_distribution=1)
    quad, qst = wl.curve(True, tree=True, budget_ms=budget_ms, **quad_kw)
    t_eq = min(plain[-1][0], guided[-1][0])
    tp, tg = time_to(plain, target), time_to(guided, target)
    ep, eg = at_time(plain, t_eq), at_time(guided, t_eq)
    return {
        "workload": f"guiding_room: 4x3x4 room lit through a 0.3x0.3 gap, {wl.xres}x{wl.yres}, max depth {wl.depth}, "
                    f"relMSE = mean((I-R)^2/(R^2+1e-2)) against a 4096-spp plain render",
        "target_relmse": target,
        "time_to_target_ms": {"plain": tp, "guided": tg},
        "time_ratio_guided_over_plain": (tg / tp) if (tp and tg) else None,
        "equal_time_ms": t_eq,
        "relmse_at_equal_time": {"plain": ep, "guided": eg},
        "gain_equal_time": ep / eg if eg > 0 else None,
        "settings": st_kw,
        "training": {"adam_steps": int(gst["guide_steps"]), "records": int(gst["guide_records"]),
                     "train_kernel_ms": gst["guide_train_ms"]},
        "config_training_settings": {
            "what": "the learned guider with the configuration's training settings (2^18 records per Adam "
                    "step, lr 1e-2) on the same schedule",
            "settings": CONFIG_GUIDE_SETTINGS,
            "time_to_target_ms": time_to(cfg_guided, target),
            "time_ratio_guided_over_plain": (time_to(cfg_guided, target) / tp) if (tp and time_to(cfg_guided, target))
            else None,
            "relmse_at_equal_time": at_time(cfg_guided, min(t_eq, cfg_guided[-1][0])),
            "training": {"adam_steps": int(cst["guide_steps"]), "records": int(cst["guide_records"]),
                         "train_kernel_ms": cst["guide_train_ms"]},
        },
        "tree_guider": {
            "what": "kd-tree cells (200 records per initial cell) with 8-lobe vMF mixtures, batch EM (4 "
                    "iterations per round), the same schedule of training passes",
            "time_to_target_ms": time_to(tree, target),
            "relmse_at_equal_time": at_time(tree, min(t_eq, tree[-1][0])),
            "gain_equal_time": ep / at_time(tree, t_eq) if tree[-1][0] >= t_eq else None,
            "rounds": int(tst["guide_steps"]), "records": int(tst["guide_records"]),
            "round_ms_total": tst["guide_train_ms"],
            "curve": [[round(t, 2), s, round(e, 6)] for t, s, e in tree],
        },
        "tree_guider_quadtree": {
            "what": "kd-tree cells (200 records per initial cell) with the reference's quadtree radiance "
                    "distributions and the stochastic record filter, the same schedule of training passes",
            "time_to_target_ms": time_to(quad, target),
            "relmse_at_equal_time": at_time(quad, min(t_eq, quad[-1][0])),
            "gain_equal_time": ep / at_time(quad, t_eq) if quad[-1][0] >= t_eq else None,
            "rounds": int(qst["guide_steps"]), "records": int(qst["guide_records"]),
            "round_ms_total": qst["guide_train_ms"],
            "curve": [[round(t, 2), s, round(e, 6)] for t, s, e in quad],
        },
        "curve_plain": [[round(t, 2), s, round(e, 6)] for t, s, e in plain],
        "curve_guided": [[round(t, 2), s, round(e, 6)] for t, s, e in guided],
    }


def multiview_comparison(g, n_views=96, seed=4):
    """The multi-view workload on the already uploaded terrain scene: n seeded views, square
    sides from {128, 256, 512, 768, 1024}, 4-64 spp, max depth of the context.  The batch
    runs as one wavefront after the autotuner picked the queue capacity, launch width, block
    size and BVH layout: plain, and with learned guiding on (the network trained first by
    four one-sample passes of the batch, then frozen); the same views are then rendered one
    call per view by the plain tracer.  Per-view completion times: for a batch the device
    time at which the wave holding the view's last path ended (CUDA events), for one call per
    view the time at which the view's call returned; p50 and p99 over the views."""
    import torch
    from naivetrace_b200 import scenes
    views = scenes.terrain_views(n_views, seed=seed)
    paths = sum(c.xres * c.yres * s for c, s in views)
    tune = g.autotune_views(views)
    g.render_views(views, seed=1)  # warm-up at the tuned configuration (allocates the path state)

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3

    def pct(x):
        x = np.asarray(x, np.float64)
        return {"p50_ms": float(np.percentile(x, 50)), "p99_ms": float(np.percentile(x, 99))}

    batch_ms = timed(lambda: g.render_views(views, seed=seed))
    batch_done = g.views_completion_ms(len(views))
    # Learned guiding on: train on the batch itself, then time a frozen guided batch.
    probe = [(c, 1) for c, _ in views]
    g.set_guiding(True, 1, seed=7)
    for k in range(4):
        g.render_views(probe, seed=100 + k)
    g.set_guiding(True, 0, seed=7)
    g.render_views(views, seed=2)  # allocates the guided path state
    guided_ms = timed(lambda: g.render_views(views, seed=seed))
    guided_done = g.views_completion_ms(len(views))
    g.set_guiding(False)
    seq_done, t = [], 0.0
    for k, v in enumerate(views):
        t += timed(lambda: g.render_views([v], seed=seed + k))
        seq_done.append(t)
    seq_ms = t
    return {
        "workload": f"terrain_views: {n_views} seeded views of the terrain_spheres scene, sides "
                    f"{{128..1024}}, 4-64 spp, {sum(c.xres * c.yres for c, _ in views)} pixels, {paths} paths",
        "paths": paths,
        "batched": {"ms": batch_ms, "mpaths_per_s": paths / (batch_ms * 1e-3) / 1e6, **pct(batch_done)},
        "batched_guided": {"ms": guided_ms, "mpaths_per_s": paths / (guided_ms * 1e-3) / 1e6, **pct(guided_done),
                           "what": "learned guiding on (2 guided bounces), network trained by 4 one-sample "
                                   "passes of the batch and frozen"},
        "one_call_per_view": {"ms": seq_ms, "mpaths_per_s": paths / (seq_ms * 1e-3) / 1e6, **pct(seq_done)},
        "speedup": seq_ms / batch_ms,
        "autotune": tune,
        "timing": "wall clock around synchronised calls (host-side view upload and image read-back included); "
                  "per-view completion from device events (batches) or call returns (one call per view)",
    }


def pt2_comparison(scene, spp, depth, device):
    """The null-path tracer (--algo pt2) on the bench workload, with pseudo-random and with
    quasi-random (Sobol) sampling: one untimed 4-spp pass, then one timed frame each (CUDA
    events around the render call)."""
    import torch
    from naivetrace_b200 import abi
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    out = {"workload": "the bench frame rendered by pt2 (no Russian roulette: every path runs to the depth cap "
                       "unless it escapes or its weight vanishes)"}
    paths = scene.camera.xres * scene.camera.yres * spp
    for qmc in (False, True):
        g = GpuContext(scene, make_params(max_ray_depth=depth, device=device, algo=abi.ALGO_PT2, qmc=qmc))
        g.render(spp, 1)  # allocates the path state of the timed frame
        g.clear()
        g.reset_stats()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        g.render(spp, 2)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        st = g.stats()
        out["qmc" if qmc else "pcg"] = {
            "ms": ms, "mpaths_per_s": paths / (ms * 1e-3) / 1e6,
            "mrays_per_s": (st["extension_rays"] + st["shadow_rays"]) / (ms * 1e-3) / 1e6,
            "rays_per_path": (st["extension_rays"] + st["shadow_rays"]) / paths,
            "error_flags": st["error_flags"]}
        g.close()
    return out


def sort_comparison(scene, spp, depth, device, frames=2):
    """The bench frame with the hit queue shaded in traversal order and in material-sorted
    order (tt_params.sort_shading): CUDA-event time per frame of each, after one untimed
    frame that allocates the path state."""
    import torch

    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    out = {"workload": "the bench frame, shaded in traversal order and in material-sorted order"}
    for key, sort in (("traversal_order", False), ("material_sorted", True)):
        g = GpuContext(scene, make_params(max_ray_depth=depth, device=device, sort_shading=sort))
        g.render(spp, 1)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for k in range(frames):
            g.render(spp, 2 + k)
        b.record()
        torch.cuda.synchronize()
        out[key] = {"ms_per_frame": a.elapsed_time(b) / frames, "error_flags": g.stats()["error_flags"]}
        g.close()
    out["speedup_sorted"] = out["traversal_order"]["ms_per_frame"] / out["material_sorted"]["ms_per_frame"]
    return out


def run_reference_arm(args):
    from naivetrace_b200 import dist as nd
    r = nd.init_from_env()
    world, rank = r.world, r.rank
    if rank != 0:
        nd.shutdown(r)
        return 0
    scene, spp, depth, name = workload(args)
    vals = []
    desc = ""
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference(scene, spp, depth, budget_s=2.0)
    for _ in range(args.steps):
        v, cores, desc = cpu_reference(scene, spp, depth, budget_s=args.cpu_budget)
        vals.append(v)
    value = float(np.mean(vals))
    paths = scene.camera.xres * scene.camera.yres * spp
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": paths / (value * 1e6) * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded procedural scene)",
        "config": dict(workload_config(scene, spp, depth, name), parallelism=f"replicas{world}, framebuffer all-reduce"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": desc + "; the reference itself cannot be built here (Embree, Eigen, TBB, "
                                          "Boost, yaml-cpp, pcg32 are absent), so this is the CPU restatement"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    nd.shutdown(r)
    return 0


def scene_bytes(scene):
    v, n, t, m = scene.arrays()
    b = v.nbytes + (n.nbytes if n is not None else 0) + t.nbytes + m.nbytes
    for e in scene.env_lights:
        if e.texture is not None:
            b += e.texture.nbytes
    return int(b)


def run_ours(args):
    import torch

    from naivetrace_b200 import abi
    from naivetrace_b200 import dist as nd
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params

    r = nd.init_from_env()
    world, rank, local = r.world, r.rank, r.local
    device = local if torch.cuda.is_available() else 0
    torch.cuda.set_device(device)
    scene, spp, depth, name = workload(args)
    params = make_params(max_ray_depth=depth, wave_paths=args.wave, device=device)
    seed = nd.rank_seed(1, rank)
    g = GpuContext(scene, params)
    npix = g.npix
    paths_per_step = npix * spp

    # Bytes-per-ray model: a counting pass (1 spp, seed 1) records BVH nodes visited and
    # triangles tested by the closest-hit kernel.
    g.set_profiling(2)
    g.render(1, seed=1)
    cst = g.stats()
    ext_rays = max(cst["extension_rays"], 1)
    nodes_per_ray = cst["node_visits"] / ext_rays
    tris_per_ray = cst["tri_tests"] / ext_rays
    bytes_per_ray = 48.0 + cst["bvh_node_bytes"] * nodes_per_ray + cst["tri_bytes"] * tris_per_ray
    g.set_profiling(0)
    g.clear()
    g.reset_stats()

    fb_tensors = None
    if r.distributed:
        fb_tensors = (torch.zeros(3 * npix, dtype=torch.float64, device="cuda"),
                      torch.zeros(3 * npix, dtype=torch.float64, device="cuda"))

    def step():
        g.render(spp, seed)
        if r.distributed:
            s = torch.cuda.current_stream().cuda_stream
            st = g.lib.tt_read_accumulators_device(g.h, C.c_void_p(fb_tensors[0].data_ptr()),
                                                   C.c_void_p(fb_tensors[1].data_ptr()), C.c_void_p(s))
            abi.check(g.lib, g.h, st, "tt_read_accumulators_device")
            nd.allreduce_sum_(fb_tensors, r)

    for _ in range(args.warmup):
        step()
    g.clear()
    g.reset_stats()
    g.set_profiling(1)
    clocks = ClockSampler(device)
    nd.barrier(r)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    nd.barrier(r)
    clk = clocks.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    st = g.stats()
    g.set_profiling(0)
    elapsed_ms = nd.max_over_ranks(elapsed_ms, r)
    ms_per_step = elapsed_ms / args.steps
    value = nd.weak_scaling_value(paths_per_step, world, ms_per_step)
    mrays = world * (st["extension_rays"] + st["shadow_rays"]) / args.steps / (ms_per_step * 1e-3) / 1e6
    # Roofline of the dominant kernel (closest-hit traversal).
    ext_launch_ms = st["extend_ms"] / max(st["extend_launches"], 1)
    achieved_gbs = st["extension_rays"] * bytes_per_ray / (st["extend_ms"] * 1e-3) / 1e9 if st["extend_ms"] > 0 else 0.0
    peak, peak_kind = hbm_peak()
    rays_per_launch = st["extension_rays"] / max(st["extend_launches"], 1)
    traffic = None
    tfile = ROOT / "profiles" / "extend_traffic.json"
    if tfile.exists():
        try:
            td = json.loads(tfile.read_text())
            traffic = td.get("bytes_per_ray", 0) * rays_per_launch
        except Exception:
            traffic = None

    # End to end through the C ABI from host buffers: create + upload (BVH build and the
    # scene's host-to-device copies) + render + framebuffer read-back + destroy.
    e2e_ms = []
    d2h = 3 * npix * 4
    h2d = scene_bytes(scene)
    # The frame is read back into page-locked host memory (a pageable destination halves the
    # device-to-host rate).
    rgb = torch.zeros(3 * npix, dtype=torch.float32, pin_memory=True).numpy()
    e2e_phases = []
    for k in range(1 + args.e2e_steps):  # the first call is an untimed warm-up
        nd.barrier(r)
        t0 = time.perf_counter()
        ge = GpuContext(scene, params, upload=False)
        t1 = time.perf_counter()
        ge.upload()
        t2 = time.perf_counter()
        ge.render(spp, seed)
        t3 = time.perf_counter()
        ge.lib.tt_read_framebuffer(ge.h, rgb.ctypes.data_as(C.POINTER(C.c_float)), None)
        t4 = time.perf_counter()
        ge.close()
        t5 = time.perf_counter()
        if k > 0:
            e2e_ms.append((t5 - t0) * 1e3)
            e2e_phases.append([round((b - a) * 1e3, 1) for a, b in ((t0, t1), (t1, t2), (t2, t3), (t3, t4), (t4, t5))])
    e2e_step = float(np.median(e2e_ms)) if e2e_ms else float("nan")
    e2e_step = nd.max_over_ranks(e2e_step, r)
    e2e_value = nd.weak_scaling_value(paths_per_step, world, e2e_step)

    guiding = None
    if rank == 0 and world == 1 and not args.no_guiding:
        guiding = guiding_comparison()
    multiview = None
    if rank == 0 and world == 1 and not args.no_multiview and not args.small:
        multiview = multiview_comparison(g)
    pt2 = None
    if rank == 0 and world == 1 and not args.no_pt2:
        pt2 = pt2_comparison(scene, spp, depth, device)
    sorted_shading = None
    if rank == 0 and world == 1 and not args.no_sort:
        sorted_shading = sort_comparison(scene, spp, depth, device)
    configs = None
    if rank == 0 and world == 1 and not args.no_configs and not args.small:
        configs = config_figures(device, cpu_budget=min(5.0, args.cpu_budget))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, desc = cpu_reference(scene, spp, depth, budget_s=args.cpu_budget)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded procedural scene, no dataset)",
            "config": dict(workload_config(scene, spp, depth, name), parallelism=f"replicas{world}, framebuffer all-reduce"),
            "mrays_per_s": mrays,
            "roofline": {
                "kernel": "k_extend (closest-hit BVH traversal)",
                "bound": "hbm",
                "achieved": achieved_gbs,
                "peak": peak,
                "peak_source": peak_kind,
                "unit": "GB/s",
                "frac": achieved_gbs / peak if peak else None,
                "traffic": traffic,
                "bytes_per_ray": bytes_per_ray,
                "nodes_per_ray": nodes_per_ray,
                "tris_per_ray": tris_per_ray,
                "avg_launch_ms": ext_launch_ms,
                "rays_per_launch": rays_per_launch,
            },
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_step, "ms_each": [round(x, 1) for x in e2e_ms],
                    "phases_ms_each": {"order": ["create", "upload", "render", "read", "destroy"],
                                       "calls": e2e_phases},
                    "what": "tt_create + tt_upload_scene (scene H2D, device BVH build) + tt_render_pass + "
                            "tt_read_framebuffer + tt_destroy"},
            "guiding": guiding,
            "multiview": multiview,
            "pt2": pt2,
            "configs": configs,
            "sorted_shading": sorted_shading,
            "gpu_launches": int(st["kernel_launches"]),
            "clocks": clk,
            "stats": {k: st[k] for k in ("extension_rays", "shadow_rays", "extend_launches", "extend_ms",
                                         "shadow_launches", "shadow_ms", "pass_ms", "bvh_nodes", "bvh_depth",
                                         "error_flags")},
        }
        print(json.dumps(line))
    g.close()
    nd.shutdown(r)
    return 0


def profile_run(args):
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    from naivetrace_b200 import abi
    if args.profile_scene == "medium":
        from naivetrace_b200 import scenes
        scene, spp, depth, name = scenes.cornell_box_medium(1024, 1024), args.spp, 32, "cornell_box_medium"
    elif args.profile_scene == "room":
        from naivetrace_b200 import scenes
        scene, spp, depth, name = scenes.guiding_room(1280, 720), args.spp, 12, "guiding_room"
    else:
        scene, spp, depth, name = workload(args)
    algo = abi.ALGO_PT2 if args.algo == "pt2" else abi.ALGO_PT
    g = GpuContext(scene, make_params(max_ray_depth=depth, wave_paths=args.wave, algo=algo,
                                      sort_shading=True if args.sort else (False if args.unsorted else None)))
    g.render(spp, 1)
    st = g.stats()
    q = g.queue_lengths(depth + 1)
    print(json.dumps({"profile_run": name, "spp": spp, "extension_rays": st["extension_rays"],
                      "shadow_rays": st["shadow_rays"], "kernel_launches": st["kernel_launches"],
                      "last_wave_extension_rays_per_bounce": q[:, 0].tolist(),
                      "last_wave_shadow_rays_per_bounce": q[:, 1].tolist(),
                      "error_flags": st["error_flags"]}))
    g.close()
    return 0 if st["error_flags"] == 0 else 1


def profile_views(args):
    """No timing: 24 seeded views (sides 128-256, 4-16 spp) of the scaled-down terrain scene
    in one batch (first wave eager, later waves replayed from the captured graph)."""
    from naivetrace_b200 import scenes
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    args.small = True
    scene, _, depth, _ = workload(args)
    g = GpuContext(scene, make_params(max_ray_depth=depth, wave_paths=1 << 20))
    views = scenes.terrain_views(24, seed=4, spp_range=(4, 16), resolutions=(128, 256))
    imgs = g.render_views(views, seed=1)
    st = g.stats()
    print(json.dumps({"profile_views": len(views), "paths": sum(c.xres * c.yres * s for c, s in views),
                      "finite": bool(all(np.isfinite(i).all() for i in imgs)), "error_flags": st["error_flags"]}))
    g.close()
    return 0 if st["error_flags"] == 0 else 1


def profile_guiding(args):
    """No timing: the guiding workload at 640x360 (depth 12), four one-sample training passes
    (16 Adam steps each) and one frozen four-sample pass; for ncu captures of the guider's
    kernels."""
    from naivetrace_b200 import scenes
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    from naivetrace_b200 import abi
    net = abi.GUIDE_NET_MMA if args.guide_net == "mma" else abi.GUIDE_NET_TCGEN05
    g = GpuContext(scenes.guiding_room(640, 360), make_params(max_ray_depth=12))
    g.set_guiding(True, 1, seed=7, network=net)
    for k in range(4):
        g.render(1, seed=100 + k)
    g.set_guiding(True, 0, seed=7, network=net)
    g.render(4, seed=3)
    st = g.stats()
    print(json.dumps({"profile_guiding": "guiding_room 640x360", "guide_steps": st["guide_steps"],
                      "guide_records": st["guide_records"], "error_flags": st["error_flags"]}))
    g.close()
    return 0 if st["error_flags"] == 0 else 1


def profile_training(args):
    """No timing: four Adam steps of the guiding network on 2^18 synthetic training records
    (the configuration's records per step), each step the tcgen05 gradient kernel and the
    fused reduction and Adam step (for ncu captures)."""
    from naivetrace_b200 import scenes
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    n = 1 << 18
    rng = np.random.default_rng(5)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    rec = np.zeros((n, 14), np.float32)
    rec[:, 0:3] = rng.random((n, 3))
    rec[:, 3:6] = unit(n)
    rec[:, 6:9] = unit(n)
    rec[:, 9:12] = unit(n)
    rec[:, 12] = 1.0 / (4.0 * np.pi)
    rec[:, 13] = rng.exponential(1.0, n)
    g = GpuContext(scenes.guiding_room(16, 16), make_params(max_ray_depth=12))
    g.set_guiding(True, 1, seed=7, batch=n, record_pool=n)
    loss = g.guide_train(rec, steps=4, learning_rate=1e-3)
    st = g.stats()
    print(json.dumps({"profile_training": "2^18 records, 4 Adam steps", "loss": loss, "error_flags": st["error_flags"]}))
    g.close()
    return 0 if (np.isfinite(loss) and st["error_flags"] == 0) else 1


def profile_network(args):
    """No timing: the guiding network's forward pass on 2^20 feature rows, three times through
    the tcgen05 kernel and three times through the mma.sync kernel (for ncu launch lists)."""
    from naivetrace_b200 import scenes
    from naivetrace_b200.algo import GpuContext
    from naivetrace_b200.scene import make_params
    g = GpuContext(scenes.guiding_room(16, 16), make_params(max_ray_depth=12))
    g.set_guiding(True, 1, seed=7)
    x = np.random.default_rng(1).uniform(-1.0, 1.0, (1 << 20, 96)).astype(np.float32)
    outs = []
    for _ in range(3):
        outs.append(g.guide_forward(x, tcgen05=True))
        outs.append(g.guide_forward(x))
    same = all(np.array_equal(outs[0], o) for o in outs)
    finite = all(np.isfinite(o).all() for o in outs)
    print(json.dumps({"profile_network": "2^20 rows", "tcgen05_equals_mma": bool(same), "finite": bool(finite)}))
    g.close()
    return 0 if finite else 1


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--wave", type=int, default=0, help="paths per wavefront wave (0 = library default)")
    ap.add_argument("--e2e-steps", type=int, default=7)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for the CPU baseline")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-guiding", action="store_true", help="skip the learned-guided vs plain comparison")
    ap.add_argument("--no-multiview", action="store_true", help="skip the multi-view batch comparison")
    ap.add_argument("--no-pt2", action="store_true", help="skip the null-path tracer (pt2) frames")
    ap.add_argument("--no-sort", action="store_true", help="skip the material-sorted shading frames")
    ap.add_argument("--sort", action="store_true", help="--profile-run: shade in material-sorted order (the default)")
    ap.add_argument("--unsorted", action="store_true", help="--profile-run: shade in traversal order")
    ap.add_argument("--profile-scene", choices=["terrain", "medium", "room"], default="terrain",
                    help="--profile-run: the bench's terrain workload, the medium-filled Cornell box (1024^2) "
                         "or the gap-lit room of the guiding workload (1280x720)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the Cornell box, medium and atmosphere configurations")
    ap.add_argument("--algo", choices=["pt", "pt2"], default="pt", help="tracer of --profile-run")
    ap.add_argument("--profile-views", action="store_true",
                    help="no timing: a batch of 24 small views of the scaled-down scene (for ncu captures)")
    ap.add_argument("--small", action="store_true", help="scaled-down scene (for profiling captures)")
    ap.add_argument("--profile-guiding", action="store_true",
                    help="no timing: training and frozen passes of the guiding workload (for ncu captures)")
    ap.add_argument("--guide-net", choices=["tcgen05", "mma"], default="tcgen05",
                    help="network kernel of --profile-guiding")
    ap.add_argument("--profile-network", action="store_true",
                    help="no timing: the guiding network's forward pass through both kernels (for ncu launch lists)")
    ap.add_argument("--profile-training", action="store_true",
                    help="no timing: Adam steps of the guiding network on 2^18 synthetic records (for ncu captures)")
    ap.add_argument("--profile-run", action="store_true",
                    help="no timing: upload the workload and render one pass of --spp samples (for ncu captures)")
    args = ap.parse_args(argv)
    if args.profile_run:
        return profile_run(args)
    if args.profile_guiding:
        return profile_guiding(args)
    if args.profile_network:
        return profile_network(args)
    if args.profile_training:
        return profile_training(args)
    if args.profile_views:
        return profile_views(args)
    if args.warmup < 3 and not args.small:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
