"""GPU tests of the rebuild without host round trips (alpine_gpu_build_async /
alpine_gpu_update_scene_async), called through the C ABI.

The device-driven build runs the same kernels on the same data as the
host-driven alpine_gpu_build; only where the per-level counts live differs
(device memory instead of host variables). The build is deterministic, so
the bar is the identical tree: the same node, level and slot counts, the same
node visits and triangle tests per ray (the reference's BvhStats counters,
src/accelerators/bvh_common.h:19-61), and bit-identical closest / any hits,
primitive ids of exact ties included. Checked for both collapse rules, on
degenerate inputs, with spheres, across animation frames (against the
synchronous update_scene, renders included), through the captured graph's
replays, and for the level cap's error path.
"""
import numpy as np
import pytest

import oracle
from alpine_b200 import batch, gpu, scenes
from parity import compare_closest

pytestmark = pytest.mark.gpu

TREE_KEYS = ("binary_nodes", "binary_levels", "wide_nodes", "wide_depth", "child_slots")


def _traces(ctx, rays):
    return ctx.trace(rays), ctx.occluded(rays)


def _visits(ctx, rays):
    import torch

    d = torch.from_numpy(rays).cuda()
    out = ctx.traversal_stats(d.data_ptr(), rays.shape[0], False)
    torch.cuda.synchronize()
    return out


def _same_tree(ctx, rays):
    """Builds synchronously, then asynchronously; returns both sets of answers."""
    sync = ctx.build()
    h1, o1 = _traces(ctx, rays)
    v1 = _visits(ctx, rays)
    ctx.build_async()
    ctx.synchronize()
    st = ctx.read_build_stats()
    for k in TREE_KEYS:
        assert st[k] == sync[k], k
    assert st["sah_cost"] == pytest.approx(sync["sah_cost"], rel=1e-5)  # float atomics: summation order
    h2, o2 = _traces(ctx, rays)
    assert h2.tobytes() == h1.tobytes()
    assert o2.tobytes() == o1.tobytes()
    assert _visits(ctx, rays) == v1
    return sync, st, h2


@pytest.mark.parametrize("collapse", [gpu.COLLAPSE_SAH, gpu.COLLAPSE_GREEDY])
@pytest.mark.parametrize("n,mu,seed", [(1, -1.0, 1), (7, -2.0, 2), (600, -3.0, 3), (30000, -4.5, 4),
                                       (250000, -5.0, 5)])
def test_async_build_is_the_same_tree(n, mu, seed, collapse):
    verts, idx = scenes.triangle_soup(n, seed=seed, mu=mu)
    ctx = gpu.Context(0)
    try:
        ctx.set_build_options(collapse)
        ctx.add_mesh(verts, idx)
        rays = np.concatenate([scenes.primary_rays(96, 48), scenes.incoherent_rays(6000, seed=seed + 50)])
        _, st, hits = _same_tree(ctx, rays)
        if n <= 600:
            tris = oracle.make_tris(verts, idx)
            compare_closest(rays, tris, hits, *oracle.closest_brute(rays, tris)[:4])
        assert st["graph_captures"] == 1 and st["graph_launches"] == 1
    finally:
        ctx.close()


def test_async_build_degenerate_inputs_and_spheres():
    """1200 coincident triangles (the median split path, exact ties), zero-area
    and NaN triangles, and analytic spheres beside them."""
    good_v, _ = scenes.triangle_soup(1500, seed=10, mu=np.log(0.05))
    same = np.tile(np.array([[0.4, 0.4, 0.5], [0.6, 0.4, 0.5], [0.5, 0.6, 0.5]], np.float32), (1200, 1))
    line = np.array([[0.1, 0.1, 0.1], [0.2, 0.2, 0.2], [0.3, 0.3, 0.3]], np.float32)
    nanv = np.array([[np.nan, 0.5, 0.5], [0.5, 0.5, 0.5], [0.5, 0.6, 0.5]], np.float32)
    verts = np.concatenate([good_v, same, line, nanv])
    idx = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
    rng = np.random.default_rng(32)
    sph = np.concatenate([rng.random((200, 3)), rng.uniform(0.005, 0.05, (200, 1))], axis=1).astype(np.float32)
    ctx = gpu.Context(0)
    try:
        ctx.add_mesh(verts, idx)
        ctx.add_spheres(sph)
        aim = np.zeros((300, 8), np.float32)
        aim[:, 0:3] = [0.5, 0.47, 0.0]
        aim[:, 4:7] = [0.0, 0.0, 1.0]
        aim[:, 0] += rng.normal(0, 0.02, 300)
        aim[:, 7] = np.float32(3.4e38)
        rays = np.concatenate([scenes.incoherent_rays(5000, seed=11), aim])
        _, _, hits = _same_tree(ctx, rays)
        assert (hits["prim"] >= 0x80000000).sum() > 10
    finally:
        ctx.close()


def test_async_build_graph_replays_and_full_size():
    """The 1M-triangle soup: the graph captured once and replayed; every
    replay gives the synchronous build's tree."""
    verts, idx, closest, _ = scenes.traversal_workload()
    rays = closest[:: 16].copy()
    ctx = gpu.Context(0)
    try:
        ctx.add_mesh(verts, idx)
        sync, _, hits = _same_tree(ctx, rays)
        for _ in range(2):
            ctx.build_async()
        ctx.synchronize()
        st = ctx.read_build_stats()
        assert st["graph_captures"] == 1 and st["graph_launches"] == 3
        for k in TREE_KEYS:
            assert st[k] == sync[k], k
        assert ctx.trace(rays).tobytes() == hits.tobytes()
    finally:
        ctx.close()


def test_async_level_cap_reports_and_keeps_the_tree():
    verts, idx = scenes.triangle_soup(30000, seed=21)
    rays = scenes.incoherent_rays(4000, seed=22)
    ctx = gpu.Context(0)
    try:
        ctx.add_mesh(verts, idx)
        ctx.build()
        before = ctx.trace(rays)
        ctx.build_async(max_binary_levels=2, max_wide_levels=8)
        with pytest.raises(gpu.GpuError) as e:
            ctx.synchronize()
        assert e.value.code == gpu.ERR_LIMIT and "level cap" in str(e.value)
        assert ctx.trace(rays).tobytes() == before.tobytes()  # the previous tree stayed in place
        ctx.build_async(max_binary_levels=64, max_wide_levels=1)
        with pytest.raises(gpu.GpuError) as e:
            ctx.synchronize()
        assert e.value.code == gpu.ERR_LIMIT
        ctx.build()  # a synchronous build recovers
        assert ctx.trace(rays).tobytes() == before.tobytes()
    finally:
        ctx.close()


def _peeled_soup(n=4096, seed=23):
    """n small triangles at x = 1e-6 * 1.01^i: every binned-SAH split cuts
    off the sparse far end (about 350 triangles), so nodes of more than 512
    triangles reach down about ten levels."""
    verts, idx = scenes.triangle_soup(n, seed=seed, mu=np.log(0.001))
    v = verts.reshape(n, 3, 3) * np.float32(1e-3)
    v[:, :, 0] += (1e-6 * 1.01 ** np.arange(n))[:, None].astype(np.float32)
    return v.reshape(-1, 3).astype(np.float32), idx


def test_async_reports_big_nodes_below_the_first_builds_levels():
    """The block-wide kernels for nodes of more than 512 triangles run on the
    levels where the last synchronous build had such nodes (plus two): a
    frame whose geometry has them deeper is reported, and a synchronous
    build of that geometry lets the next rebuilds follow it."""
    verts, idx = scenes.triangle_soup(4096, seed=24)
    peeled, _ = _peeled_soup()
    rays = scenes.incoherent_rays(3000, seed=25)
    ref = gpu.Context(0)
    ctx = gpu.Context(0)
    try:
        ref.add_mesh(peeled, idx)
        deep = ref.build()
        ctx.add_mesh(verts, idx)
        shallow = ctx.build()
        assert deep["big_levels"] >= shallow["big_levels"] + 3
        ctx.update_vertices(0, peeled)
        ctx.build_async(max_binary_levels=deep["binary_levels"] + 4, max_wide_levels=24)
        with pytest.raises(gpu.GpuError) as e:
            ctx.synchronize()
        assert e.value.code == gpu.ERR_LIMIT and "level cap" in str(e.value)
        ctx.build()
        ctx.build_async()
        ctx.synchronize()
        assert ctx.trace(rays).tobytes() == ref.trace(rays).tobytes()
    finally:
        ref.close()
        ctx.close()


def test_async_needs_a_synchronous_build_first():
    ctx = gpu.Context(0)
    try:
        ctx.add_mesh(*scenes.triangle_soup(100, seed=3))
        with pytest.raises(gpu.GpuError) as e:
            ctx.build_async()
        assert e.value.code == gpu.ERR_INVALID_STATE
    finally:
        ctx.close()


@pytest.mark.parametrize("seed,tris", [(7, 20000), (8, 3000)])
def test_async_animation_matches_update_scene(seed, tris):
    """Animated batch scenes over several frames: morph + async rebuild +
    render enqueued without host waits gives the synchronous update_scene's
    hits and accumulation bit for bit."""
    scene = batch.batch_scene(seed, tris)
    w = h = 48
    rays = scenes.incoherent_rays(3000, seed=seed)
    rays[:, 0:3] = rays[:, 0:3] * 8.0 - 4.0
    ctxs = []
    try:
        for _ in range(2):
            c = gpu.Context(0, w, h, 6)
            scenes.load_scene(c, scene, w, h)
            c.build_light_sampler(gpu.SAMPLER_POWER)
            c.set_render_options(sampler=gpu.RNG_COUNTER, seed=seed, russian_roulette_depth=3)
            c.reset_accumulation()
            ctxs.append(c)
        a, b = ctxs
        for frame in range(4):
            t = float(frame) * 1.7
            a.update_scene(t)
            a.render(4)
            b.update_scene_async(t)
            b.render_async(4)
            b.render_wait()
            assert b.trace(rays).tobytes() == a.trace(rays).tobytes()
        acc_a = a.read_accumulation(w, h)[0]
        acc_b = b.read_accumulation(w, h)[0]
        assert acc_a[..., :3].sum() > 0
        assert acc_b.tobytes() == acc_a.tobytes()
        st = b.read_build_stats()
        assert st["graph_captures"] == 1 and st["graph_launches"] == 4
    finally:
        for c in ctxs:
            c.close()
