"""GPU parity tests of the traversal path, called through the C ABI.

Compared against the reference's own answers (golden fixtures made by
oracle/_ref) and the oracle's canonical queries; the bar is bit-exact
(see tests/parity.py).
"""
import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes
from parity import MISS, check_hits_valid, compare_closest

pytestmark = pytest.mark.gpu

FLT_MAX = np.float32(3.4028234663852886e38)


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.close()


def _load(ctx, verts, idx):
    ctx.reset_scene()
    ctx.add_mesh(verts, idx)
    return ctx.build()


def test_golden_reference_wide_bvh(ctx, golden):
    _load(ctx, golden["verts"], golden["idx"])
    tris = oracle.make_tris(golden["verts"], golden["idx"])
    hits = ctx.trace(golden["rays"])
    rep = compare_closest(golden["rays"], tris, hits, golden["wide_prim"], golden["wide_t"], golden["wide_b1"],
                          golden["wide_b2"])
    assert rep["hits"] > 1000
    occ = ctx.occluded(golden["shadow"])
    assert (occ == golden["wide_occluded"]).all()


@pytest.mark.parametrize("n,mu,sigma,seed", [(1, -1.0, 0.1, 1), (2, -1.5, 0.2, 2), (3, -2.0, 0.3, 3),
                                             (7, -2.0, 0.3, 4), (100, -2.5, 0.5, 5), (513, -3.0, 0.5, 6),
                                             (5000, -3.5, 0.8, 7), (20000, -4.5, 0.5, 8)])
def test_random_soups_vs_bruteforce(ctx, n, mu, sigma, seed):
    verts, idx = scenes.triangle_soup(n, seed=seed, mu=mu, sigma=sigma)
    stats = _load(ctx, verts, idx)
    assert stats["triangles"] == n
    tris = oracle.make_tris(verts, idx)
    rays = np.concatenate([scenes.primary_rays(64, 32), scenes.incoherent_rays(3000, seed=seed + 100)])
    rays[1::5, 3] = 0.02  # tmin > 0 on some rays
    rays[2::5, 7] = 0.3   # finite tmax on some rays
    hits = ctx.trace(rays)
    ref = oracle.closest_brute(rays, tris)
    compare_closest(rays, tris, hits, *ref[:4])
    sh = rays.copy()
    sh[:, 7] = scenes.shadow_tmax(len(rays), seed=seed + 200)
    assert (ctx.occluded(sh) == oracle.any_brute(sh, tris)).all()


def test_empty_scene(ctx):
    ctx.reset_scene()
    st = ctx.build()
    assert st["triangles"] == 0
    rays = scenes.incoherent_rays(100, seed=1)
    hits = ctx.trace(rays)
    assert (hits["prim"] == MISS).all() and (hits["t"] == FLT_MAX).all()
    assert (ctx.occluded(rays) == 0).all()


def test_degenerate_inputs(ctx):
    """Zero-area triangles, coincident triangles (median split path with more
    than one warp task of references), NaN vertices, axis-aligned rays."""
    rng = np.random.default_rng(9)
    good_v, good_i = scenes.triangle_soup(1500, seed=10, mu=np.log(0.05))
    # 1200 identical triangles: all centroids coincide
    same = np.tile(np.array([[0.4, 0.4, 0.5], [0.6, 0.4, 0.5], [0.5, 0.6, 0.5]], np.float32), (1200, 1))
    # zero-area triangles (collinear and point)
    line = np.array([[0.1, 0.1, 0.1], [0.2, 0.2, 0.2], [0.3, 0.3, 0.3]], np.float32)
    point = np.array([[0.7, 0.7, 0.7]] * 3, np.float32)
    nanv = np.array([[np.nan, 0.5, 0.5], [0.5, 0.5, 0.5], [0.5, 0.6, 0.5]], np.float32)
    verts = np.concatenate([good_v, same, line, point, nanv])
    idx = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
    _load(ctx, verts, idx)
    tris = oracle.make_tris(verts, idx)
    rays = scenes.incoherent_rays(4000, seed=11)
    # axis-aligned directions, including zero components and -0.0
    ax = np.zeros((600, 8), np.float32)
    ax[:, 0:3] = rng.random((600, 3))
    for k in range(600):
        ax[k, 4 + (k % 3)] = 1.0 if (k // 3) % 2 == 0 else -1.0
    sub = ax[::4, 4:7]
    ax[::4, 4:7] = np.where(sub == 0, np.float32(-0.0), sub)  # negative zeros
    ax[:, 7] = FLT_MAX
    # rays aimed exactly at the coincident stack
    aim = np.zeros((200, 8), np.float32)
    aim[:, 0:3] = [0.5, 0.47, 0.0]
    aim[:, 4:7] = [0.0, 0.0, 1.0]
    aim[:, 0] += rng.normal(0, 0.02, 200)
    aim[:, 7] = FLT_MAX
    rays = np.concatenate([rays, ax, aim])
    hits = ctx.trace(rays)
    ref = oracle.closest_brute(rays, tris)
    rep = compare_closest(rays, tris, hits, *ref[:4])
    assert rep["ties"] > 0  # the coincident stack produces exact ties
    assert (ctx.occluded(rays) == oracle.any_brute(rays, tris)).all()


def test_multiple_meshes_and_update(ctx):
    v1, i1 = scenes.triangle_soup(800, seed=41, mu=np.log(0.05))
    v2, i2 = scenes.triangle_soup(1200, seed=42, mu=np.log(0.05))
    ctx.reset_scene()
    assert ctx.add_mesh(v1, i1) == 0
    assert ctx.add_mesh(v2, i2) == 1
    ctx.build()
    verts = np.concatenate([v1, v2])
    idx = np.concatenate([i1, i2 + v1.shape[0]])
    tris = oracle.make_tris(verts, idx)
    rays = scenes.incoherent_rays(3000, seed=43)
    compare_closest(rays, tris, ctx.trace(rays), *oracle.closest_brute(rays, tris)[:4])
    # move the second mesh and rebuild (Accelerator::updateShape + updateScene)
    v2b = v2 + np.float32(0.01) * np.sin(np.arange(v2.shape[0], dtype=np.float32))[:, None]
    ctx.update_vertices(1, v2b)
    with pytest.raises(gpu.GpuError):
        ctx.trace(rays)  # stale BVH must be rejected
    ctx.build()
    tris = oracle.make_tris(np.concatenate([v1, v2b]), idx)
    compare_closest(rays, tris, ctx.trace(rays), *oracle.closest_brute(rays, tris)[:4])


def test_build_is_deterministic(ctx):
    verts, idx = scenes.triangle_soup(30000, seed=51)
    s1 = _load(ctx, verts, idx)
    rays = scenes.incoherent_rays(20000, seed=52)
    h1 = ctx.trace(rays)
    s2 = _load(ctx, verts, idx)
    h2 = ctx.trace(rays)
    for k in ("binary_nodes", "binary_levels", "wide_nodes", "wide_depth"):
        assert s1[k] == s2[k]
    assert h1.tobytes() == h2.tobytes()


@pytest.mark.parametrize("rule", [gpu.COLLAPSE_GREEDY, gpu.COLLAPSE_SAH])
@pytest.mark.parametrize("n,seed,cost", [(2, 71, 0.0), (5, 72, 0.0), (300, 73, 0.0), (20000, 74, 0.0),
                                         (20000, 75, 0.05), (20000, 76, 4.0)])
def test_collapse_rules_vs_bruteforce(ctx, rule, n, seed, cost):
    """Both collapse rules (and SAH triangle costs from very low to very
    high) give the exact closest and any hits."""
    ctx.set_build_options(rule, cost)
    try:
        verts, idx = scenes.triangle_soup(n, seed=seed, mu=-3.0, sigma=0.5)
        st = _load(ctx, verts, idx)
        assert st["wide_nodes"] <= st["child_slots"] <= 8 * st["wide_nodes"]
        tris = oracle.make_tris(verts, idx)
        rays = np.concatenate([scenes.primary_rays(32, 32), scenes.incoherent_rays(3000, seed=seed + 100)])
        compare_closest(rays, tris, ctx.trace(rays), *oracle.closest_brute(rays, tris)[:4])
        sh = rays.copy()
        sh[:, 7] = scenes.shadow_tmax(len(rays), seed=seed + 200)
        assert (ctx.occluded(sh) == oracle.any_brute(sh, tris)).all()
    finally:
        ctx.set_build_options()


def test_sah_collapse_fills_nodes(ctx):
    """The SAH-optimal collapse fills more slots per wide node than the
    greedy rule, and lowers what it minimises: node visits plus triangle
    tests (at the default triangle cost of 1 node visit) per ray."""
    import torch

    verts, idx = scenes.triangle_soup(100000, seed=81, mu=-4.0, sigma=0.5)
    rays = torch.from_numpy(scenes.incoherent_rays(20000, seed=82)).cuda()
    res = {}
    for rule in (gpu.COLLAPSE_GREEDY, gpu.COLLAPSE_SAH):
        ctx.set_build_options(rule)
        st = _load(ctx, verts, idx)
        nodes, tris = ctx.traversal_stats(rays.data_ptr(), rays.shape[0], False)
        res[rule] = (st["child_slots"] / st["wide_nodes"], nodes / rays.shape[0], tris / rays.shape[0])
    ctx.set_build_options()
    print("children per node, nodes and triangles per ray: greedy %s, SAH %s" % (res[1], res[0]))
    assert res[gpu.COLLAPSE_SAH][0] > res[gpu.COLLAPSE_GREEDY][0]
    cost = {k: v[1] + 1.0 * v[2] for k, v in res.items()}
    assert cost[gpu.COLLAPSE_SAH] < 0.95 * cost[gpu.COLLAPSE_GREEDY]


def test_build_options_rejected(ctx):
    with pytest.raises(gpu.GpuError):
        ctx.set_build_options(7)
    with pytest.raises(gpu.GpuError):
        ctx.set_build_options(gpu.COLLAPSE_SAH, -1.0)
    ctx.set_build_options()


def _pinned(a):
    """A copy of a in page-locked host memory."""
    import torch

    a = np.ascontiguousarray(a)
    out = torch.empty(a.nbytes, dtype=torch.uint8).pin_memory().numpy().view(a.dtype).reshape(a.shape)
    out[...] = a
    return out


def test_pinned_host_buffers_pipeline(ctx):
    """Pinned host buffers go through the chunked pipeline (rays copied in on
    one stream, traversals on six, results copied out on another): the
    answers equal the pageable path's bit for bit, below one chunk, over a
    few chunks and over all 32. A query right after an asynchronous rebuild
    of moved geometry waits for that rebuild."""
    verts, idx = scenes.triangle_soup(50000, seed=81, mu=np.log(0.01))
    _load(ctx, verts, idx)
    for n in (1000, 200000, 2500000):
        rays = np.concatenate([scenes.primary_rays(256, 128), scenes.incoherent_rays(n, seed=n)])[:n]
        rays[1::3, 7] = scenes.shadow_tmax(rays[1::3].shape[0], seed=n + 1)
        want_h, want_o = ctx.trace(rays), ctx.occluded(rays)
        pr = _pinned(rays)
        ph = _pinned(np.zeros(n, gpu.HIT_DTYPE))
        po = _pinned(np.zeros(n, np.uint8))
        ctx.trace(pr, ph)
        ctx.occluded(pr, po)
        assert ph.tobytes() == want_h.tobytes()
        assert po.tobytes() == want_o.tobytes()
    # ordering after an asynchronous rebuild of moved geometry
    moved = verts + np.float32(0.02) * np.cos(np.arange(verts.shape[0], dtype=np.float32))[:, None]
    ref = gpu.Context(0)
    try:
        ref.add_mesh(moved, idx)
        ref.build()
        rays = scenes.incoherent_rays(300000, seed=84)
        want = ref.trace(rays)
        ctx.update_vertices(0, moved)
        ctx.build_async()
        pr, ph = _pinned(rays), _pinned(np.zeros(rays.shape[0], gpu.HIT_DTYPE))
        ctx.trace(pr, ph)
        assert ph.tobytes() == want.tobytes()
    finally:
        ref.close()


def test_device_pointer_api(ctx):
    import torch

    verts, idx = scenes.triangle_soup(4000, seed=61, mu=np.log(0.02))
    _load(ctx, verts, idx)
    rays = scenes.incoherent_rays(10000, seed=62)
    dr = torch.from_numpy(rays).cuda()
    dh = torch.empty((rays.shape[0], 4), dtype=torch.int32, device="cuda")
    do = torch.empty(rays.shape[0], dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    ctx.trace_device(dr.data_ptr(), rays.shape[0], dh.data_ptr(), s.cuda_stream)
    ctx.occluded_device(dr.data_ptr(), rays.shape[0], do.data_ptr(), s.cuda_stream)
    ctx.synchronize()
    s.synchronize()
    host = ctx.trace(rays)
    assert dh.cpu().numpy().tobytes() == host.tobytes()
    assert (do.cpu().numpy() == ctx.occluded(rays)).all()


@pytest.mark.slow
def test_full_size_traversal_workload(ctx):
    """The 1M-triangle / 4M-ray microbenchmark: every reported hit re-evaluates
    exactly; any-hit equals (closest t < tmax) on all rays; a 65,536-ray sample
    matches the oracle's canonical closest hit."""
    verts, idx, closest, shadow = scenes.traversal_workload()
    st = _load(ctx, verts, idx)
    assert st["triangles"] == 1 << 20
    tris = oracle.make_tris(verts, idx)
    hits = ctx.trace(closest)
    nh = check_hits_valid(closest, tris, hits)
    assert nh > 1 << 20
    occ = ctx.occluded(shadow)
    expect = (hits["prim"] != MISS) & (hits["t"] < shadow[:, 7])
    assert (occ.astype(bool) == expect).all()
    rng = np.random.default_rng(0)
    sample = np.sort(rng.choice(closest.shape[0], 65536, replace=False))
    ob = oracle.OracleBvh(tris)
    ref = ob.closest(closest[sample])
    compare_closest(closest[sample], tris, hits[sample], *ref[:4])
