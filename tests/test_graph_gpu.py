"""GPU tests of CUDA-graph replay, asynchronous multi-context rendering and
the autotuner.

With the counter RNG every (pixel, sample) draws its own numbers and samples
are accumulated in sample order, so the image does not depend on how the
work is launched: replayed graphs, concurrent contexts and every wave size /
traversal block size the autotuner may pick give bit-identical sums.
"""
import numpy as np
import pytest

from alpine_b200 import gpu, scenes

pytestmark = pytest.mark.gpu

W, H = 48, 40


def _ctx(scene, **opts):
    c = gpu.Context(0, W, H, 6)
    scenes.load_scene(c, scene, W, H)
    c.build_light_sampler(gpu.SAMPLER_BVH)
    c.set_render_options(sampler=gpu.RNG_COUNTER, seed=5, russian_roulette_depth=3, **opts)
    c.reset_accumulation()
    return c


def _sums(c):
    return c.read_accumulation(W, H)[0].tobytes()


def test_graph_replay_is_identical():
    scene = scenes.add_random_lights(scenes.room_scene(seed=2), 12, seed=3)
    eager = _ctx(scene)
    graph = _ctx(scene, cuda_graph=True)
    for _ in range(3):
        eager.render(8)
        graph.render(8)
    assert _sums(eager) == _sums(graph)
    captures, launches = graph.graph_stats()
    assert captures == 1 and launches == 3
    eager.close()
    graph.close()


def test_graph_replays_across_rebuilds():
    scene = scenes.room_scene(seed=3)
    sphere = scene["meshes"][-1]
    sphere["morph"] = scenes.sinusoid_morph(sphere["verts"], sphere["normals"], amplitude=0.04, with_normals=True)
    eager = _ctx(scene)
    graph = _ctx(scene, cuda_graph=True)
    for frame in range(4):
        for c in (eager, graph):
            c.update_scene(float(frame))
            c.render(4)
    assert _sums(eager) == _sums(graph)
    captures, launches = graph.graph_stats()
    assert captures == 1 and launches == 4
    eager.close()
    graph.close()


def test_async_contexts_match_sync():
    scene = scenes.room_scene(seed=4)
    ref = _ctx(scene)
    ref.render(16)
    want = _sums(ref)
    ref.close()
    ctxs = [_ctx(scene, cuda_graph=(i % 2 == 1)) for i in range(4)]
    for c in ctxs:
        c.render_async(8)
    for c in ctxs:
        c.render_async(8)
    for c in ctxs:
        c.render_wait()
        assert _sums(c) == want
        c.close()


def test_autotune_keeps_the_image():
    scene = scenes.room_scene(seed=6)
    base = _ctx(scene)
    base.render(8)
    want = _sums(base)
    base.close()
    tuned = _ctx(scene)
    t = tuned.autotune(probe_spp=4)
    print("autotune:", t)
    assert t["trace_block"] in (64, 128, 256)
    assert t["max_paths_per_wave"] >= 1 << 18 and t["samples_per_second"] > 0
    tuned.render(8)
    assert _sums(tuned) == want
    tuned.close()


def test_autotune_guided_picks_an_inference_kernel_and_keeps_the_model():
    scene = scenes.room_scene(seed=6)
    c = _ctx(scene, guide=True, guide_spp_per_wave=4, guide_steps_per_wave=4, guide_batch=4096)
    try:
        c.render(8)  # trains the guide a little
        steps = c.guide_steps()[0]
        weights = c.guide_get_weights()
        assert steps > 0
        t = c.autotune(probe_spp=4)
        print("autotune (guided):", t)
        assert t["guide_kernel"] in (gpu.GUIDE_KERNEL_WARP_MMA, gpu.GUIDE_KERNEL_TENSOR_MEMORY)
        assert t["trace_block"] in (64, 128, 256)
        assert c.guide_steps()[0] == steps
        assert c.guide_get_weights().tobytes() == weights.tobytes()
    finally:
        c.close()


def test_batch_host_threads_give_identical_frames():
    """The batch renderer's ways of enqueueing a frame render the same
    images, scene by scene: the host-driven rebuild from one host thread and
    from per-scene host threads (concurrent morph + rebuild + graph-replayed
    render enqueue), and the device-driven rebuild from one thread with no
    host wait."""
    from alpine_b200 import batch

    cfgs = batch.batch_configs(n=6, seed=5, max_tris=20000, resolutions=(64, 96), spps=(4,))
    outs = []
    for threads, rebuild in ((1, "sync"), (6, "sync"), (1, "async")):
        br = batch.BatchRenderer(cfgs, threads=threads)
        try:
            br.run(3, rebuild=rebuild)
            outs.append([c.read_accumulation(cfg["width"], cfg["height"])[0].tobytes()
                         for c, cfg in zip(br.ctxs, cfgs)])
        finally:
            br.close()
    assert outs[0] == outs[1] == outs[2]
