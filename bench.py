#!/usr/bin/env python
"""Traversal microbenchmark: closest-hit + any-hit rays/s on a 1M-triangle soup.

Workload (one step): a 1,048,576-triangle soup in the unit cube (centroids
uniform, edge lengths log-normal(ln 0.004, 0.5), uniform orientations), BVH
built once on the GPU (binned SAH, 32 bins, 8-wide); 4,194,304 closest-hit
rays (2,097,152 primary rays of a 2048x1024 pinhole camera at (0.5,0.5,-1),
60 deg FOV + 2,097,152 incoherent rays: origins uniform in the cube,
directions uniform on the sphere) and the same 4,194,304 rays as any-hit
shadow rays with tmax uniform in (0, 1]. A step traces all 8,388,608 queries.

`value` is device throughput with rays resident in HBM; `e2e` goes through
the C ABI with pinned host buffers (host->device copy of the rays and
device->host copy of the results inside the timed region).

`room` (rank 0, one GPU): the small procedural room of the reference's own
CPU-runnable configuration, GPU samples/s next to the reference renderer's
on the host cores.

`many_lights` (rank 0, one GPU): the many-light city, samples/s and relMSE
per light sampler (uniform, power, light BVH).

`batch` (rank 0, one GPU): frames/s and samples/s of 48 animated scenes
rendered together (morph + BVH rebuild + render per scene per frame), with
the device-driven rebuild and with the host-driven one.

`guiding` (rank 0, one GPU): time to relMSE 0.01, guided vs plain MIS, on the
glossy interior (20 x 4 x 12 m room, 2.0M triangles, 70% GGX with roughness
in [0.02, 0.4], sky of radiance 5 through two 1 x 2 m window openings, depth
12) at 1920 x 1080, against a 2,048-spp image rendered in the same run by the
trained, frozen guided estimator in two independent halves, whose own error is
removed from every relMSE (see guiding_benchmark). relMSE = mean over pixels and channels of
(x - r)^2 / (r^2 + 0.01 mean(r)^2). Time is the wall time of the render calls
(synchronous), guided training included; the time to the target is
interpolated in log-log between the curve points that bracket it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --collapse-sweep   # traversal under each wide-BVH collapse rule
    python bench.py --e2e-breakdown    # where the end-to-end step's time goes
Multi-GPU: one process per GPU under torchrun; each rank is an independent
replica of the workload (weak scaling), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "traversal Mrays/s (closest+any hit) vs CPU host"
UNIT = "Mrays/s"
WORKLOAD = "traversal microbenchmark: 1,048,576-tri soup, 4,194,304 closest + 4,194,304 any-hit rays"
NODE_BYTES = 80
TRI_BYTES = 48
RAY_BYTES = 32
HIT_BYTES = 16


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-guiding", action="store_true", help="skip the guided vs plain time-to-relMSE measurement")
    p.add_argument("--guiding-ref-spp", type=int, default=2048)
    p.add_argument("--guiding-res", type=str, default="1920x1080", help="WxH of the guided vs plain measurement")
    p.add_argument("--batch-frames", type=int, default=2,
                   help="frames of the 48-scene animated batch to time (0 = skip)")
    p.add_argument("--no-many-lights", action="store_true", help="skip the many-light city measurement")
    p.add_argument("--no-room", action="store_true", help="skip the small-room render measurement")
    p.add_argument("--profile", action="store_true",
                   help="profiling run: one build, one warm-up and one timed step, no e2e / CPU baseline")
    p.add_argument("--collapse-sweep", action="store_true",
                   help="traversal workload under each wide-BVH collapse rule and SAH triangle cost (one JSON line each)")
    p.add_argument("--e2e-breakdown", action="store_true",
                   help="where the end-to-end traversal step's time goes (device, chunked, copies, each host call)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


def traffic_from_profile():
    """DRAM bytes per closest-hit launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "trace_closest_soup1M.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_full_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML every 100 ms."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, device_index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self._h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._nv = pynvml
        except Exception:
            self._h = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._nv.nvmlDeviceGetClockInfo(self._h, self._nv.NVML_CLOCK_SM))
                self.reasons |= self._nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        names = [n for b, n in self.REASONS.items() if self.reasons & b and n != "gpu_idle"]
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples)}


def ref_build_label():
    """Which build of the reference the timed CPU arms use."""
    import oracle

    name = os.path.basename(oracle.timing_build())
    flags = {"libalpine_ref_fast_v4.so": "-O3 -march=x86-64-v4 (AVX-512) -ffp-contract=off",
             "libalpine_ref_fast_v3.so": "-O3 -march=x86-64-v3 (AVX2) -ffp-contract=off",
             "libalpine_ref.so": "-O3 -march=x86-64-v3 -ffp-contract=off (parity build)"}
    return f"{name}: {flags.get(name, '?')}"


def cpu_baseline(verts, idx, closest, shadow, budget_s):
    """The reference's own WideBvh (oracle/_ref: src/accelerators/wide_bvh.cpp
    with the ISPC kernels restated in C++) on all host cores, on a bounded
    sample of the same rays (interleaved closest / any-hit chunks)."""
    import oracle

    if not oracle.ref_available():
        return None
    ncores = os.cpu_count() or 1
    acc = oracle.RefAccel(oracle.RefAccel.WIDE_BVH, verts, idx, timing=True)
    rng = np.random.default_rng(7)
    order = rng.permutation(closest.shape[0])
    chunk = 16384
    done, t_total, k = 0, 0.0, 0
    while t_total < budget_s and (k + 1) * chunk <= order.size:
        sel = np.sort(order[k * chunk:(k + 1) * chunk])
        rc, rs = closest[sel], shadow[sel]
        t0 = time.perf_counter()
        acc.intersect(rc, nthreads=ncores)
        acc.occluded(rs, nthreads=ncores)
        t_total += time.perf_counter() - t0
        done += 2 * chunk
        k += 1
    return {"value": done / t_total / 1e6, "unit": UNIT, "cores": ncores, "kind": "reference",
            "build": ref_build_label(),
            "sample": f"{done // 2} random rays of the workload (primary+incoherent mix), closest + any hit each; "
                      f"reference WideBvh build {acc.build_ms:.0f} ms (not in the rate)",
            "seconds": t_total}


GUIDING_RES = (1920, 1080)
GUIDING_DEPTH = 12
# training schedule measured best on B200 (waves of 8 spp, up to 32 Adam
# steps of about 16,384 samples after each, 4,096 steps in all)
GUIDE_OPTIONS = dict(guide=True, guide_fraction=0.5, guide_spp_per_wave=8, guide_batch=16384, guide_steps_per_wave=32,
                     guide_lr=1e-2, guide_min_roughness=0.2, guide_train_steps=4096)


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2 * ref.mean() ** 2)))


def guiding_benchmark(device, ref_spp, target=0.01, res=GUIDING_RES, guided_repeats=3):
    """Time to relMSE `target` of plain and guided rendering on the glossy
    interior at res (see the module docstring), and the reference CPU
    renderer's projected time for the plain estimator (its measured
    samples/s on the same scene x the spp the plain estimator needs).

    The reference image r is ref_spp samples of the guided estimator (its
    guide trained, then frozen: an unbiased estimator for that fixed guide,
    with far less variance per second than plain MIS) in two independent
    halves h1, h2 (different seeds). Its own error is removed from every
    relMSE: for unbiased x and r, E[(x - r)^2] = Var x + Var r, and
    (h1 - h2)^2 / 4 is an unbiased per-pixel estimate of Var r, so
    relMSE(x) = mean(((x - r)^2 - (h1 - h2)^2 / 4) / (r^2 + 0.01 mean(r)^2)).
    (A plain 1,024-spp reference at this resolution has about 8x the target
    error itself; its noise then correlates with the denominator enough that
    the subtraction leaves a bias near the target.) A curve that has not
    reached the target after max_s seconds reports the 1/spp extrapolation
    of its last point, marked as such.
    A curve is sampled at growing spp (doubling, then a step aimed just past
    the target from the measured 1/spp trend) and the time to the target is
    interpolated in log-log between the two points that bracket it."""
    import math

    from alpine_b200 import gpu, scenes

    W, H = res
    scene = scenes.glossy_interior_scene()

    def context(**opts):
        c = gpu.Context(device, W, H, GUIDING_DEPTH)
        scenes.load_scene(c, scene, W, H)
        c.set_render_options(sampler=gpu.RNG_COUNTER, accumulate_fp64=True, **opts)
        c.reset_accumulation()
        return c

    def mean(c):
        a, n = c.read_accumulation(W, H, fp64=True)
        return a[..., :3].astype(np.float64) / n

    t0 = time.perf_counter()
    # the reference: the guided estimator, trained and then frozen, in two
    # halves of independent samples (for a fixed guide the estimator is
    # unbiased; per unit time it has far less variance than plain MIS)
    c = context(seed=999, **GUIDE_OPTIONS)
    c.render(128)  # trains the guide (16 waves, 512 Adam steps) and warms up
    halves = []
    for seed in (1000, 2000):
        c.set_render_options(sampler=gpu.RNG_COUNTER, accumulate_fp64=True, seed=seed,
                             **dict(GUIDE_OPTIONS, guide_train=False))
        c.reset_accumulation()
        c.render(ref_spp // 2)
        halves.append(mean(c))
    c.close()
    ref = 0.5 * (halves[0] + halves[1])
    ref_var = (halves[0] - halves[1]) ** 2 / 4.0
    ref_s = time.perf_counter() - t0
    denom = ref ** 2 + 1e-2 * ref.mean() ** 2
    ref_err = float(np.mean(ref_var / denom))  # the reference's own relMSE, removed below
    del halves

    def err(x):
        return float(np.mean(((x - ref) ** 2 - ref_var) / denom))

    def curve(opts, max_spp=1 << 15, max_s=240.0):
        c = context(**opts)
        done, elapsed, pts = 0, 0.0, []
        spp = 4
        while done < max_spp and elapsed < max_s:
            t1 = time.perf_counter()
            c.render(spp)
            elapsed += time.perf_counter() - t1
            done += spp
            e = err(mean(c))
            pts.append((done, elapsed, e))
            print(f"guiding curve {'guided' if opts.get('guide') else 'plain'}: {done} spp {elapsed:.2f} s "
                  f"relMSE {e:.5f}", file=sys.stderr, flush=True)
            if e < target:
                break
            # double, or jump to just past the target when the 1/spp trend says it is near
            want = int(done * e / (0.9 * target)) if e > 0 else 2 * done
            spp = max(4, min(done, want - done) if want < 2 * done else done)
        steps = c.guide_steps()[0] if opts.get("guide") else 0
        c.close()
        at = None
        for i in range(1, len(pts)):
            (s0, t_0, e0), (s1, t_1, e1) = pts[i - 1], pts[i]
            if e1 <= target < e0 and e0 > 0 and e1 > 0:
                f = (math.log(target) - math.log(e0)) / (math.log(e1) - math.log(e0))
                at = (t_0 + f * (t_1 - t_0), math.exp(math.log(s0) + f * (math.log(s1) - math.log(s0))))
                break
        if at is None and pts and pts[-1][2] > 0:
            # not reached within the time cap: the 1/spp trend of the last
            # point, marked as extrapolated
            s_, t_, e_ = pts[-1]
            at = (t_ * e_ / target, s_ * e_ / target, "extrapolated")
        return at, pts, steps

    warm = context(seed=5, **GUIDE_OPTIONS)  # module loading, allocations
    warm.render(2)
    warm.close()
    # each arm with its measured-best shading order: grouping the queue by
    # material costs the plain interior 10% and gains the guided one 2%
    plain_at, plain_pts, _ = curve(dict(seed=1, shade_order=gpu.SHADE_ORDER_QUEUE))
    # the guided arm learns online (its gradient sums are unordered), so its
    # time to the target varies from run to run: three runs with different
    # seeds, the median reported and all listed. The plain estimator is
    # stationary (relMSE x spp constant along its curve): one run.
    guided_runs = [curve(dict(seed=2 + 100 * k, shade_order=gpu.SHADE_ORDER_BY_MATERIAL, **GUIDE_OPTIONS))
                   for k in range(guided_repeats)]
    timed = sorted((r for r in guided_runs if r[0] is not None), key=lambda r: r[0][0])
    guided_at, guided_pts, steps = timed[len(timed) // 2] if timed else guided_runs[0]
    out = {
        "metric": "time to relMSE 0.01, guided vs plain MIS", "unit": "s", "target_relmse": target,
        "scene": "glossy interior, 2.0M triangles, sky 5 through two 1x2 m windows, depth 12, no lights",
        "resolution": [W, H], "reference_spp": ref_spp, "reference_s": ref_s,
        "reference_relmse_removed": ref_err,
        "relmse": "mean(((x - r)^2 - (h1 - h2)^2 / 4) / (r^2 + 0.01 mean(r)^2)), r = (h1 + h2) / 2",
        "reference": "the guided estimator after 512 training steps, frozen, in two independent halves",
        "plain_extrapolated": bool(plain_at and len(plain_at) > 2),
        "guided_extrapolated": bool(guided_at and len(guided_at) > 2),
        "plain_s": plain_at[0] if plain_at else None, "plain_spp": plain_at[1] if plain_at else None,
        "guided_s": guided_at[0] if guided_at else None, "guided_spp": guided_at[1] if guided_at else None,
        "speedup": (plain_at[0] / guided_at[0]) if plain_at and guided_at else None,
        "guided_repeats_s": [r[0][0] if r[0] else None for r in guided_runs],
        "guided_repeats_spp": [r[0][1] if r[0] else None for r in guided_runs],
        "guide": {k: v for k, v in GUIDE_OPTIONS.items() if k != "guide"} | {"adam_steps": steps},
        "shade_order": {"plain": "queue", "guided": "by material"},
        "plain_curve": [[s, round(t, 4), round(e, 5)] for s, t, e in plain_pts],
        "guided_curve": [[s, round(t, 4), round(e, 5)] for s, t, e in guided_pts],
    }
    out["cpu_reference"] = cpu_render_baseline(scene, 320, 180, out["plain_spp"], W * H)
    return out


def cpu_render_baseline(scene, W, H, plain_spp, pixels, spp=2):
    """The reference renderer (oracle/_ref: class Alpine with its WideBvh) on
    all host cores: samples/s on the same scene at W x H, and the time the
    plain estimator (the same algorithm) would need for plain_spp samples of
    `pixels` pixels at that rate."""
    import oracle

    from alpine_b200 import scenes

    if not oracle.ref_available():
        return None
    r = oracle.RefRenderer(W, H, GUIDING_DEPTH, accelerator=oracle.RefRenderer.ACC_WIDE_BVH, timing=True)
    t0 = time.perf_counter()
    scenes.load_scene(r, scene, W, H)
    load_s = time.perf_counter() - t0
    r.reset_accumulation()
    r.render(1)
    t0 = time.perf_counter()
    r.render(spp)
    dt = time.perf_counter() - t0
    r.close()
    rate = spp * W * H / dt
    return {"samples_per_s": rate, "cores": os.cpu_count() or 1, "kind": "reference", "build": ref_build_label(),
            "sample": f"{spp} spp at {W}x{H} after 1 warm-up spp; scene load + BVH build {load_s:.1f} s",
            "projected_time_to_target_s": (plain_spp * pixels / rate) if plain_spp else None}


def batch_benchmark(device, frames):
    """48 independent animated scenes (BASELINE cfg4 shapes; alpine_b200.batch):
    every frame morphs and rebuilds every BVH and renders every scene at its
    resolution and spp, the renders of all scenes in flight together, each a
    replayed CUDA graph. Timed with the device-driven rebuild (one host
    thread, no host wait within a frame) and with the host-driven rebuild
    (one host thread, and a pool of host threads). Warm-up frames (graph
    captures) are not timed."""
    from alpine_b200 import batch

    cfgs = batch.batch_configs()
    t0 = time.perf_counter()
    br = batch.BatchRenderer(cfgs, device=device, cuda_graph=True)
    setup = time.perf_counter() - t0
    keys = ("seconds", "frames_per_s", "samples_per_s", "build_ms_per_frame")
    br.run(1, start=0, rebuild="sync")
    serial = br.run(frames, start=1, threads=1, rebuild="sync")
    threaded = br.run(frames, start=1 + frames, rebuild="sync")
    br.run(1, start=1 + 2 * frames)  # warm-up of the device-driven rebuild (graph capture)
    r = br.run(frames, start=2 + 2 * frames)
    r["rebuild"] = "device-driven (alpine_gpu_update_scene_async, a replayed graph), one host thread, no host wait"
    r["sync_rebuild_one_host_thread"] = {k: serial[k] for k in keys}
    r["sync_rebuild_host_threads"] = {**{k: threaded[k] for k in keys}, "host_threads": br.threads}
    r["build_ms_per_frame_note"] = ("sum over scenes of each rebuild's device time; the rebuilds overlap one another "
                                    "and the renders, so the sum exceeds the wall time")
    # the rebuilds alone (morph + BVH build of all 48 scenes, no rendering), wall clock
    rb, rba = [], []
    for f in range(frames):
        t1 = time.perf_counter()
        list(br._pool.map(lambda c: c.update_scene(float(100 + f)), br.ctxs))
        rb.append(1e3 * (time.perf_counter() - t1))
        t1 = time.perf_counter()
        for c in br.ctxs:
            c.update_scene_async(float(200 + f))
        for c in br.ctxs:
            c.synchronize()
        rba.append(1e3 * (time.perf_counter() - t1))
    r["rebuild_only_wall_ms_per_frame"] = statistics.mean(rba)
    r["rebuild_only_wall_ms_per_frame_sync_threads"] = statistics.mean(rb)
    r.update({"scenes": len(cfgs), "triangles": br.triangles, "setup_s": setup,
              "samples_per_frame": sum(c["width"] * c["height"] * c["spp"] for c in cfgs),
              "workload": "48 scenes, tris log-uniform 1k-500k, res 128^2-1024^2, spp 4/16/64, 1-64 quad lights, "
                          "0.02-amplitude sinusoid morph, BVH rebuilt per frame, depth 8, light-BVH sampler"})
    br.close()
    return r


def room_benchmark(device, W=256, H=256, spp=16, depth=8, repeats=5):
    """The small procedural room (4,036 triangles, 0.5 x
    0.5 quad ceiling light of radiance 15, power sampler, depth 8, 256 x 256,
    16 spp) rendered by the GPU and by the reference's own renderer
    (oracle/_ref: class Alpine with its binary BVH) on all host cores. Both
    run the reference's estimator (no Russian roulette); the GPU is also
    timed with roulette from depth 3 as configs[0] asks. Samples per second;
    the GPU's best of `repeats` renders; the image means are compared."""
    from alpine_b200 import gpu, scenes
    import oracle

    scene = scenes.room_scene(light="quad")
    out = {"workload": f"room, {W}x{H}, {spp} spp, depth {depth}, power sampler, quad light", "gpu": {}}

    def gpu_rate(rr):
        c = gpu.Context(device, W, H, depth)
        scenes.load_scene(c, scene, W, H)
        c.build_light_sampler(gpu.SAMPLER_POWER)
        c.set_render_options(sampler=gpu.RNG_COUNTER, russian_roulette_depth=rr, seed=3)
        c.reset_accumulation()
        c.render(spp)
        best = float("inf")
        for _ in range(repeats):
            c.reset_accumulation()
            t0 = time.perf_counter()
            c.render(spp)
            best = min(best, time.perf_counter() - t0)
        a, n = c.read_accumulation(W, H)
        c.close()
        return W * H * spp / best, float(a[..., :3].mean() / n)

    rate, gmean = gpu_rate(0)
    out["gpu"]["samples_per_s"] = rate
    out["gpu"]["samples_per_s_rr3"] = gpu_rate(3)[0]
    if oracle.ref_available():
        r = oracle.RefRenderer(W, H, depth, accelerator=oracle.RefRenderer.ACC_BVH, timing=True)
        scenes.load_scene(r, scene, W, H)
        r.build_light_sampler(gpu.SAMPLER_POWER)
        r.reset_accumulation()
        t0 = time.perf_counter()
        r.render(spp)
        dt = time.perf_counter() - t0
        a, n = r.read_accumulation()
        r.close()
        rmean = float(a[..., :3].mean() / n)
        out["cpu_reference"] = {"samples_per_s": W * H * spp / dt, "cores": os.cpu_count() or 1, "kind": "reference",
                                "build": ref_build_label(),
                                "sample": f"one render of {spp} spp (binary BVH, quad light as a harness Light)"}
        out["speedup_vs_cpu_reference"] = rate / out["cpu_reference"]["samples_per_s"]
        out["image_mean"] = {"gpu": gmean, "reference": rmean, "rel_diff": abs(gmean - rmean) / rmean}
    return out


def many_lights_benchmark(device, spp=4, cmp_res=(480, 270), cmp_spp=64, ref_spp=4096):
    """Many-light city (BASELINE cfg3 shapes; alpine_b200.scenes.city_scene:
    2,000 buildings, ~1.2M triangles, 131,072 window quad lights): samples/s
    of each light sampler at 1920x1080, depth 8 (`spp` samples per pixel after
    a warm-up); and at cmp_res the relMSE of each sampler at cmp_spp against a
    ref_spp light-BVH image, with the equal-time efficiency 1 / (relMSE x
    time)."""
    from alpine_b200 import gpu, scenes

    t0 = time.perf_counter()
    scene = scenes.city_scene()
    gen_s = time.perf_counter() - t0
    names = {gpu.SAMPLER_UNIFORM: "uniform", gpu.SAMPLER_POWER: "power", gpu.SAMPLER_BVH: "light_bvh"}
    out = {"triangles": int(sum(m["idx"].shape[0] for m in scene["meshes"])), "lights": len(scene["lights"]),
           "scene_generation_s": gen_s, "resolution": [1920, 1080], "depth": 8, "spp": spp, "samplers": {}}

    def context(w, h, kind, seed):
        c = gpu.Context(device, w, h, 8)
        scenes.load_scene(c, scene, w, h)
        t1 = time.perf_counter()
        c.build_light_sampler(kind)
        build = time.perf_counter() - t1
        c.set_render_options(sampler=gpu.RNG_COUNTER, seed=seed)
        c.reset_accumulation()
        return c, build

    for kind, name in names.items():
        c, build = context(1920, 1080, kind, 1)
        c.render(1)
        t1 = time.perf_counter()
        c.render(spp)
        dt = time.perf_counter() - t1
        c.close()
        out["samplers"][name] = {"samples_per_s": 1920 * 1080 * spp / dt, "sampler_build_s": build}
    W, H = cmp_res
    c, _ = context(W, H, gpu.SAMPLER_BVH, 99)
    c.render(ref_spp)
    a, n = c.read_accumulation(W, H, fp64=True)
    ref = a[..., :3].astype(np.float64) / n
    c.close()
    for kind, name in names.items():
        c, _ = context(W, H, kind, 3)
        c.render(1)
        c.reset_accumulation()
        t1 = time.perf_counter()
        c.render(cmp_spp)
        dt = time.perf_counter() - t1
        a, n = c.read_accumulation(W, H, fp64=True)
        c.close()
        e = relmse(a[..., :3].astype(np.float64) / n, ref)
        out["samplers"][name].update({"relmse_at_cmp_spp": e, "cmp_seconds": dt, "efficiency": 1.0 / (e * dt)})
    out["comparison"] = f"{W}x{H}, {cmp_spp} spp vs a {ref_spp}-spp light-BVH image"
    return out


def traversal_split(ctx, d_closest, d_shadow, d_hits, d_occ, stream, half, reps=5):
    """Device Mrays/s of each half of the workload on its own: the 2,097,152
    coherent primary rays and the 2,097,152 incoherent rays, closest hit and
    any hit, each timed with CUDA events on the launching stream (mean of
    `reps` launches after one warm-up)."""
    import torch

    sp = stream.cuda_stream
    out = {}
    for name, off in (("coherent", 0), ("incoherent", half)):
        for kind in ("closest", "any"):
            src = (d_closest if kind == "closest" else d_shadow).data_ptr() + off * 32
            if kind == "closest":
                dst = d_hits.data_ptr() + off * 16

                def launch():
                    ctx.trace_device(src, half, dst, sp)
            else:
                dst = d_occ.data_ptr() + off

                def launch():
                    ctx.occluded_device(src, half, dst, sp)
            launch()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            for _ in range(reps):
                launch()
            ev[1].record(stream)
            torch.cuda.synchronize()
            out[f"{name}_{kind}"] = half * reps / (ev[0].elapsed_time(ev[1]) / 1e3) / 1e6
    ctx.synchronize()
    return out


def host_link_bandwidth(h_rays, d_rays, h_hits, d_hits, stream, h2d_bytes_per_step, reps=5):
    """GB/s of plain pinned-host copies over the host link, timed with CUDA
    events on the stream: the ray buffer host -> device and the hit buffer
    device -> host, each alone. `h2d_ms_per_step` is the time the link needs
    for one step's ray bytes, the floor under the end-to-end step."""
    import torch

    src = torch.from_numpy(h_rays)
    back = torch.from_numpy(h_hits.view(np.uint8)).view(-1)
    dh = d_hits.view(torch.uint8).view(-1)
    assert src.is_pinned() and back.is_pinned()
    out = {}
    for name, dst, s_ in (("h2d_gbs", d_rays, src), ("d2h_gbs", back, dh)):
        dst.copy_(s_, non_blocking=True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(reps):
            dst.copy_(s_, non_blocking=True)
        ev[1].record(stream)
        torch.cuda.synchronize()
        out[name] = s_.numel() * s_.element_size() * reps / (ev[0].elapsed_time(ev[1]) / 1e3) / 1e9
    out["h2d_ms_per_step"] = h2d_bytes_per_step / (out["h2d_gbs"] * 1e9) * 1e3
    return out


def l2_copy_bandwidth(stream, sizes_mib=(4, 8, 16, 24), reps=400):
    """GB/s (read + write bytes) of a device copy whose source and
    destination stay resident in the 126 MB L2 (best over a few sizes): the
    denominator for kernels whose working set is served from L2."""
    import torch

    best = 0.0
    for mib in sizes_mib:
        n = mib * (1 << 20) // 4
        a = torch.ones(n, dtype=torch.float32, device="cuda")
        b = torch.empty_like(a)
        for _ in range(10):
            b.copy_(a)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(reps):
            b.copy_(a)
        ev[1].record(stream)
        torch.cuda.synchronize()
        best = max(best, 2 * a.numel() * 4 * reps / (ev[0].elapsed_time(ev[1]) / 1e3) / 1e9)
    return best


def run_reference(args):
    """--impl reference: the reference's CPU WideBvh on the host cores, same
    metric; each step is a 131,072-query sample of the workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from alpine_b200 import scenes
    import oracle

    verts, idx, closest, shadow = scenes.traversal_workload()
    ncores = os.cpu_count() or 1
    acc = oracle.RefAccel(oracle.RefAccel.WIDE_BVH, verts, idx, timing=True)
    rng = np.random.default_rng(11)
    per = 65536
    times = []
    for s in range(args.warmup + args.steps):
        sel = np.sort(rng.choice(closest.shape[0], per, replace=False))
        rc, rs = closest[sel], shadow[sel]
        t0 = time.perf_counter()
        acc.intersect(rc, nthreads=ncores)
        acc.occluded(rs, nthreads=ncores)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    ms = 1e3 * sum(times) / len(times)
    value = 2 * per / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_per_step": f"{per} closest + {per} any-hit queries",
                   "accelerator": "reference WideBvh (8-wide, ISPC kernels restated in C++), CPU"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "reference",
                         "build": ref_build_label(),
                         "sample": f"{per} closest + {per} any-hit random rays of the workload per step",
                         "build_ms": acc.build_ms},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    from alpine_b200 import gpu, scenes

    from alpine_b200 import replicas

    world, rank, local = replicas.world_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, "cuda")

    verts, idx, closest, shadow = scenes.traversal_workload()
    n = closest.shape[0]
    ctx = gpu.Context(local)
    ctx.add_mesh(verts, idx)
    stats = ctx.build()
    build_times = []
    if args.profile:
        args.warmup, args.steps, args.no_cpu_baseline = 1, 1, True
    else:
        for _ in range(3):  # rebuild timings (device time of the whole build)
            build_times.append(ctx.build()["build_ms"])

    d_closest = torch.from_numpy(closest).cuda()
    d_shadow = torch.from_numpy(shadow).cuda()
    d_hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    d_occ = torch.empty(n, dtype=torch.uint8, device="cuda")
    # a dedicated stream: the kernels and the CUDA events must share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    assert sp != 0

    if args.profile:
        nv_c = tv_c = nv_s = tv_s = 0
    else:
        nv_c, tv_c = ctx.traversal_stats(d_closest.data_ptr(), n, False)
        nv_s, tv_s = ctx.traversal_stats(d_shadow.data_ptr(), n, True)

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        ctx.trace_device(d_closest.data_ptr(), n, d_hits.data_ptr(), sp)
        if ev is not None:
            ev[1].record(stream)
        ctx.occluded_device(d_shadow.data_ptr(), n, d_occ.data_ptr(), sp)
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for k in range(args.steps):
            step(evs[k])
        end.record(stream)
        torch.cuda.synchronize()
    ctx.synchronize()
    barrier()
    total_ms = start.elapsed_time(end)
    value, ms_step = replicas.job_rate(2 * n, total_ms / args.steps, world, dist, "cuda")
    closest_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    any_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    value /= 1e6  # Mrays/s

    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "closest_ms": closest_ms, "any_ms": any_ms}), flush=True)
        ctx.close()
        return
    split = traversal_split(ctx, d_closest, d_shadow, d_hits, d_occ, stream, n // 2)
    l2_gbs = l2_copy_bandwidth(stream)
    # end to end through the C ABI with pinned host buffers
    h_closest = torch.from_numpy(closest).pin_memory().numpy()
    h_shadow = torch.from_numpy(shadow).pin_memory().numpy()
    h_hits = torch.empty(n * 16, dtype=torch.uint8).pin_memory().numpy().view(gpu.HIT_DTYPE)
    h_occ = torch.empty(n, dtype=torch.uint8).pin_memory().numpy()
    for _ in range(max(1, args.warmup)):
        ctx.trace(h_closest, h_hits)
        ctx.occluded(h_shadow, h_occ)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.trace(h_closest, h_hits)
        ctx.occluded(h_shadow, h_occ)
    e2e_value, e2e_ms = replicas.job_rate(2 * n, 1e3 * (time.perf_counter() - t0) / args.steps, world, dist, "cuda")
    barrier()
    e2e_value /= 1e6
    link = host_link_bandwidth(h_closest, d_closest, h_hits, d_hits, stream, 2 * n * RAY_BYTES)

    peak, peak_kind = peaks()
    bytes_closest = n * (RAY_BYTES + HIT_BYTES) + nv_c * NODE_BYTES + tv_c * TRI_BYTES
    bytes_any = n * (RAY_BYTES + 1) + nv_s * NODE_BYTES + tv_s * TRI_BYTES
    achieved = bytes_closest / (closest_ms / 1e3) / 1e9
    roofline = {
        "bound": "hbm", "kernel": "k_trace<closest>", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic_from_profile(),
        "traffic_source": "DRAM bytes of one full-size launch from the committed ncu summary of this workload "
                          "(profiles/trace_closest_soup1M.md); not captured in this run",
        "limiter": "instruction issue and SIMD divergence: the BVH (about 65 MB) is served from L2, so DRAM "
                   "traffic is a small fraction of the algorithmic bytes",
        "l2": {"achieved": achieved, "peak": l2_gbs, "frac": achieved / l2_gbs if l2_gbs else None,
               "peak_source": "L2-resident device copy (best of 4-24 MiB buffers) measured in this run"},
        "algorithmic_bytes_per_launch": bytes_closest,
        "per_ray": {"node_visits": nv_c / n, "tri_tests": tv_c / n, "bytes": bytes_closest / n},
        "any_hit": {"ms": any_ms, "achieved_gbs": bytes_any / (any_ms / 1e3) / 1e9,
                    "node_visits": nv_s / n, "tri_tests": tv_s / n},
        "closest_ms": closest_ms,
    }
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(verts, idx, closest, shadow, args.cpu_seconds)
    guiding = batched = many = room = ginfer = None
    if rank == 0 and world == 1 and (not args.no_guiding or args.batch_frames or not args.no_many_lights
                                     or not args.no_room):
        ctx.close()
        ctx = None
    if rank == 0 and world == 1 and not args.no_guiding:
        ginfer = guide_inference_benchmark(local, l2_gbs)
    if rank == 0 and world == 1 and not args.no_room:
        room = room_benchmark(local)
    if rank == 0 and world == 1 and not args.no_many_lights:
        many = many_lights_benchmark(local)
    if rank == 0 and world == 1 and not args.no_guiding:
        gw, gh = (int(x) for x in args.guiding_res.split("x"))
        guiding = guiding_benchmark(local, args.guiding_ref_spp, res=(gw, gh))
    if rank == 0 and world == 1 and args.batch_frames:
        batched = batch_benchmark(local, args.batch_frames)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": WORKLOAD, "triangles": int(idx.shape[0]), "rays_per_step": 2 * n,
                "bvh": "GPU binned SAH (32 bins) -> 8-wide quantised BVH",
                "build_ms": stats["build_ms"], "rebuild_ms": build_times, "wide_nodes": stats["wide_nodes"],
                "wide_depth": stats["wide_depth"], "sah_cost": stats["sah_cost"],
                "l2": "inputs larger than L2 (rays 2 x 128 MiB + hits 64 MiB per step); BVH resident",
                "parallelism": f"replicas x{world}",
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * n * RAY_BYTES,
                    "d2h_bytes_per_step": n * (HIT_BYTES + 1), "ms_per_step": e2e_ms,
                    "host_link": {**link, "link_bound_mrays_s": 2 * n / (link["h2d_ms_per_step"] / 1e3) / 1e6}},
            "roofline": roofline,
            "traversal_split_mrays_s": split,
            "cpu_baseline": base,
            "gpu_launches": 2 * args.steps,
            "clocks": clocks.summary(),
            "guiding": guiding,
            "batch": batched,
            "many_lights": many,
            "room": room,
            "guide_inference": ginfer,
        }
        print(json.dumps(line), flush=True)
    if ctx is not None:
        ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def guide_inference_benchmark(device, l2_gbs, n=1 << 21, reps=10):
    """Device throughput of the guide's inference (`alpine_gpu_guide_infer_device`,
    the render's k_infer with raw outputs) on n queries, both inference
    kernels, CUDA events on the launching stream (mean of `reps` launches
    after 3 warm-ups). Queries are uniform in the unit scene box with random
    directions and normals: a harsher gather pattern than a render's, whose
    queries lie on surfaces. The model is freshly initialised (the time does
    not depend on the parameter values).
    Roofline quantities per query: MLP FLOPs 2 x (4 x 64 x 64 + 64 x 48)
    (inputs padded to 64, outputs to 48), against the measured BF16 GEMM peak;
    bytes: the hash-grid corner gathers (levels x 8 corners x features x 2 B
    of FP16) plus 48 B of query in and 160 B of outputs, against the L2 copy
    bandwidth measured in this run (the grid is L2-resident)."""
    import torch

    from alpine_b200 import gpu

    ctx = gpu.Context(device)
    ctx.guide_reset(1, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    dims = ctx.guide_dims()
    levels = len(dims["res"])
    features = dims["grid_params"] // (levels * dims["table_size"])
    g = torch.Generator(device="cuda").manual_seed(7)
    q = torch.zeros((n, 12), dtype=torch.float32, device="cuda")
    q[:, 0:3] = torch.rand((n, 3), generator=g, device="cuda")
    q[:, 3] = 0.02 + 0.98 * torch.rand(n, generator=g, device="cuda")
    for a, b in ((4, 7), (8, 11)):
        v = torch.randn((n, 3), generator=g, device="cuda")
        q[:, a:b] = v / v.norm(dim=1, keepdim=True)
    raw = torch.empty((n, 40), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    flops = 2.0 * (4 * 64 * 64 + 64 * 48)
    gather = levels * 8 * features * 2
    io = 48 + 160
    bf16_peak = None
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        bf16_peak = float(json.load(open(path))["bf16_tflops"])
    out = {"queries": n, "levels": levels, "features_per_level": features,
           "flops_per_query": flops, "gather_bytes_per_query": gather, "io_bytes_per_query": io}
    for name, kernel in (("warp_mma", gpu.GUIDE_KERNEL_WARP_MMA), ("tensor_memory", gpu.GUIDE_KERNEL_TENSOR_MEMORY)):
        ctx.guide_set_kernel(kernel)
        for _ in range(3):
            ctx.guide_infer_device(q.data_ptr(), n, raw.data_ptr(), sp)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(reps):
            ctx.guide_infer_device(q.data_ptr(), n, raw.data_ptr(), sp)
        ev[1].record(stream)
        torch.cuda.synchronize()
        ctx.synchronize()
        s = ev[0].elapsed_time(ev[1]) / 1e3 / reps
        tflops = n * flops / s / 1e12
        gbs = n * (gather + io) / s / 1e9
        out[name] = {"ms": s * 1e3, "gqueries_per_s": n / s / 1e9, "tflops": tflops,
                     "tflops_frac": tflops / bf16_peak if bf16_peak else None, "gbs": gbs,
                     "l2_frac": gbs / l2_gbs if l2_gbs else None}
    ctx.guide_set_kernel(gpu.GUIDE_KERNEL_WARP_MMA)
    out["peaks"] = {"bf16_tflops": bf16_peak, "bf16_source": "of measured (burst)" if bf16_peak else None,
                    "l2_gbs": l2_gbs}
    out["bound"] = "gathers (L1/L2 latency and throughput), not the tensor cores"
    ctx.close()
    return out


def collapse_sweep(device=0):
    """The traversal workload's BVH built with the reference's greedy collapse
    and with the SAH-optimal one at several triangle costs: filled slots per
    wide node, node visits and triangle tests per closest-hit ray, and the
    device Mrays/s of each half of the workload (traversal_split). Hits are
    compared with the greedy build's (they differ only on exact ties)."""
    import torch

    from alpine_b200 import gpu, scenes

    verts, idx, closest, shadow = scenes.traversal_workload()
    n = closest.shape[0]
    half = n // 2
    ctx = gpu.Context(device)
    ctx.add_mesh(verts, idx)
    d_closest = torch.from_numpy(closest).cuda()
    d_shadow = torch.from_numpy(shadow).cuda()
    d_hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    d_occ = torch.empty(n, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    first = None
    for name, rule, cost in [("greedy", gpu.COLLAPSE_GREEDY, 0.0)] + [
            (f"sah_{c}", gpu.COLLAPSE_SAH, c) for c in (0.3, 0.5, 1.0, 2.0)]:
        ctx.set_build_options(rule, cost)
        st = ctx.build()
        r = {"collapse": name, "wide_nodes": st["wide_nodes"], "children_per_node": st["child_slots"] / st["wide_nodes"],
             "wide_depth": st["wide_depth"], "build_ms": min(ctx.build()["build_ms"] for _ in range(2))}
        for hn, off in (("coherent", 0), ("incoherent", half)):
            nv, tv = ctx.traversal_stats(d_closest.data_ptr() + off * RAY_BYTES, half, False)
            r[f"{hn}_closest_nodes_per_ray"] = nv / half
            r[f"{hn}_closest_tris_per_ray"] = tv / half
        r["mrays_s"] = traversal_split(ctx, d_closest, d_shadow, d_hits, d_occ, stream, half, reps=10)
        ctx.trace_device(d_closest.data_ptr(), n, d_hits.data_ptr(), stream.cuda_stream)
        ctx.synchronize()
        h = d_hits.cpu().numpy()
        first = h.copy() if first is None else first
        r["prims_differing_from_greedy"] = int((h[:, 0] != first[:, 0]).sum())
        r["t_differing_from_greedy"] = int((h[:, 1] != first[:, 1]).sum())
        print(json.dumps(r), flush=True)
    ctx.set_build_options()
    ctx.close()


def e2e_breakdown(device=0, reps=8):
    """Where the end-to-end traversal step's time goes, all on one GPU: the
    device-resident step as two full launches and as 32 chunks on 6
    streams, the same with the step's host->device copies running beside
    it, the copies alone, and each host-buffer call of the library (ms per
    step; wall time around synchronised repetitions)."""
    import torch

    from alpine_b200 import gpu, scenes

    verts, idx, closest, shadow = scenes.traversal_workload()
    n = closest.shape[0]
    ctx = gpu.Context(device)
    ctx.add_mesh(verts, idx)
    ctx.build()
    dc, ds = torch.from_numpy(closest).cuda(), torch.from_numpy(shadow).cuda()
    dc2, ds2 = torch.empty_like(dc), torch.empty_like(ds)
    dh = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    do = torch.empty(n, dtype=torch.uint8, device="cuda")
    hc, hs = torch.from_numpy(closest).pin_memory(), torch.from_numpy(shadow).pin_memory()
    hh = torch.empty((n, 4), dtype=torch.int32).pin_memory()
    ho = torch.empty(n, dtype=torch.uint8).pin_memory()
    streams = [torch.cuda.Stream() for _ in range(6)]
    main, cp, back = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.set_stream(main)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return 1e3 * (time.perf_counter() - t0) / reps

    def full():
        ctx.trace_device(dc.data_ptr(), n, dh.data_ptr(), main.cuda_stream)
        ctx.occluded_device(ds.data_ptr(), n, do.data_ptr(), main.cuda_stream)

    def chunked(k_total=32):
        c = n // k_total
        for k in range(k_total):
            ctx.trace_device(dc.data_ptr() + k * c * RAY_BYTES, c, dh.data_ptr() + k * c * HIT_BYTES,
                             streams[k % 6].cuda_stream)
        for k in range(k_total):
            ctx.occluded_device(ds.data_ptr() + k * c * RAY_BYTES, c, do.data_ptr() + k * c,
                                streams[k % 6].cuda_stream)

    def copies():
        with torch.cuda.stream(cp):
            dc2.copy_(hc, non_blocking=True)
            ds2.copy_(hs, non_blocking=True)
        with torch.cuda.stream(back):
            hh.copy_(dh, non_blocking=True)
            ho.copy_(do, non_blocking=True)

    def beside():
        with torch.cuda.stream(cp):
            dc2.copy_(hc, non_blocking=True)
            ds2.copy_(hs, non_blocking=True)
        full()

    h_hits = torch.empty(n * HIT_BYTES, dtype=torch.uint8).pin_memory().numpy().view(gpu.HIT_DTYPE)
    h_occ = ho.numpy()
    out = {"device_full_ms": timed(full), "device_chunked32_ms": timed(chunked),
           "device_full_with_h2d_beside_ms": timed(beside), "copies_only_ms": timed(copies),
           "e2e_ms": timed(lambda: (ctx.trace(hc.numpy(), h_hits), ctx.occluded(hs.numpy(), h_occ))),
           "e2e_trace_ms": timed(lambda: ctx.trace(hc.numpy(), h_hits)),
           "e2e_occluded_ms": timed(lambda: ctx.occluded(hs.numpy(), h_occ))}
    print(json.dumps(out), flush=True)
    ctx.close()


def main():
    args = parse_args()
    if args.collapse_sweep:
        collapse_sweep()
        return
    if args.e2e_breakdown:
        e2e_breakdown()
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
