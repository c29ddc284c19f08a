"""Small fixed rendering workloads for profiling (ncu launch lists and
captures) and quick timing. Each renders twice, so a capture can skip the
first render's launches (or, with AG_NVTX=1, select the second render's by
its NVTX range "measure").

    python -m alpine_b200.workloads room     # 256x256, 2 x 16 spp, depth 8, RR from depth 3,
                                             # power sampler, quad ceiling light (the small room)
    python -m alpine_b200.workloads room_queue  # the same, shading in queue order (not grouped by material)
    python -m alpine_b200.workloads guided   # glossy interior 320x180, depth 12, guided:
                                             # 16 Adam steps, then 2 x 32 spp
    python -m alpine_b200.workloads guided_tc  # the same with the tcgen05 inference kernel
    python -m alpine_b200.workloads guided_dwmma  # the same with the mma.sync weight-gradient kernel
    python -m alpine_b200.workloads city     # many-light city 960x540, 1 + 2 spp, depth 8, light BVH
    python -m alpine_b200.workloads interior        # glossy interior 320x180, depth 12, plain MIS, 2 x 64 spp
    python -m alpine_b200.workloads interior_guided # the same guided with the time-to-relMSE schedule
                                                    # (8 spp waves, 32 Adam steps per wave, 512 steps):
                                                    # 256 spp while training, then 64 spp
    python -m alpine_b200.workloads interior_guided_1080  # the same schedule at 1920x1080: 32 spp
                                                          # (training ends within them), then 8 spp
"""
from __future__ import annotations

import os
import sys
import time

from . import gpu, scenes


def run(mode: str, device: int = 0) -> float:
    """Runs one workload; returns the wall time of its second render (s)."""
    if mode in ("room", "room_queue"):
        sc, (W, H), depth = scenes.room_scene(light="quad"), (256, 256), 8
        opts, sampler, spp = dict(russian_roulette_depth=3), gpu.SAMPLER_POWER, (16, 16)
        if mode == "room_queue":  # shading in traversal-queue order
            opts["shade_order"] = gpu.SHADE_ORDER_QUEUE
    elif mode in ("guided", "guided_tc", "guided_dwmma"):
        sc, (W, H), depth = scenes.glossy_interior_scene(), (320, 180), 12
        opts = dict(accumulate_fp64=True, guide=True, guide_spp_per_wave=2, guide_batch=65536, guide_steps_per_wave=4,
                    guide_min_roughness=0.2, guide_train_steps=16)
        sampler, spp = None, (32, 32)
    elif mode in ("interior", "interior_guided", "interior_guided_1080"):
        big = mode == "interior_guided_1080"
        sc, (W, H), depth = scenes.glossy_interior_scene(), ((1920, 1080) if big else (320, 180)), 12
        opts, sampler, spp = dict(accumulate_fp64=True), None, (64, 64)
        if big:
            opts.update(guide=True, guide_spp_per_wave=8, guide_batch=16384, guide_steps_per_wave=32, guide_lr=1e-2,
                        guide_min_roughness=0.2, guide_train_steps=512, shade_order=gpu.SHADE_ORDER_BY_MATERIAL)
            spp = (32, 8)
        elif mode == "interior_guided":
            opts.update(guide=True, guide_spp_per_wave=8, guide_batch=16384, guide_steps_per_wave=32, guide_lr=1e-2,
                        guide_min_roughness=0.2, guide_train_steps=512)
            spp = (256, 64)
    elif mode == "city":
        sc, (W, H), depth = scenes.city_scene(), (960, 540), 8
        opts, sampler, spp = {}, gpu.SAMPLER_BVH, (1, 2)
    else:
        raise ValueError(f"unknown workload {mode!r}")
    c = gpu.Context(device, W, H, depth)
    if mode == "guided_tc":
        c.guide_set_kernel(gpu.GUIDE_KERNEL_TENSOR_MEMORY)
    if mode == "guided_dwmma":  # training's weight gradients on mma.sync instead of tcgen05
        c.guide_set_gradient_kernel(gpu.GUIDE_KERNEL_WARP_MMA)
    scenes.load_scene(c, sc, W, H)
    if sampler is not None:
        c.build_light_sampler(sampler)
    c.set_render_options(sampler=gpu.RNG_COUNTER, **opts)
    c.reset_accumulation()
    c.render(spp[0])
    # an NVTX range "measure" around the second render when AG_NVTX=1, so a
    # profiler can capture its launches alone (ncu --nvtx --nvtx-include measure/)
    nvtx = None
    if os.environ.get("AG_NVTX") == "1":
        import torch

        nvtx = torch.cuda.nvtx
        nvtx.range_push("measure")
    t0 = time.perf_counter()
    c.render(spp[1])
    dt = time.perf_counter() - t0
    if nvtx is not None:
        nvtx.range_pop()
    c.close()
    return dt


if __name__ == "__main__":
    for m in sys.argv[1:] or ["room"]:
        print(f"{m}: second render {run(m) * 1e3:.1f} ms", flush=True)
