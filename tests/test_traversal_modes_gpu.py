"""GPU tests of the traversal options, called through the C ABI.

* The binary-BVH triangle rule (the reference's Primitive::intersect,
  src/accelerators/bvh_common.cpp:66-103: |det| >= FLT_EPSILON, divisions,
  b1 <= 1, b2 <= 1 - b1) against the reference binary BVH's own answers
  (golden fixtures made by oracle/_ref) and the oracle's canonical queries
  under the same rule. The bar is bit-exact (tests/parity.py).
* Device-side limits: a visit cap or stack limit set far below what the BVH
  needs makes rays run out; they end as misses, the call reports
  ALPINE_GPU_ERR_LIMIT with a message naming the limit, nothing traps, and the
  context keeps working once the limit is lifted. The reference's traversals
  only assert here (src/accelerators/bvh.cpp:231, wide_bvh.cpp:604).
"""
import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes
from parity import MISS, check_hits_valid, compare_closest

pytestmark = pytest.mark.gpu

BIN = oracle.TRI_PRIM


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.close()


def _load(ctx, verts, idx, triangle_test=gpu.TRIANGLE_TEST_BINARY_BVH, **limits):
    ctx.set_traversal_options(triangle_test, **limits)
    ctx.reset_scene()
    ctx.add_mesh(verts, idx)
    return ctx.build()


def test_golden_reference_binary_bvh(ctx, golden):
    _load(ctx, golden["verts"], golden["idx"])
    tris = oracle.make_tris(golden["verts"], golden["idx"])
    hits = ctx.trace(golden["rays"])
    rep = compare_closest(golden["rays"], tris, hits, golden["bvh_prim"], golden["bvh_t"], golden["bvh_b1"],
                          golden["bvh_b2"], sem=BIN)
    assert rep["hits"] > 1000
    assert (ctx.occluded(golden["shadow"]) == golden["bvh_occluded"]).all()


def test_binary_and_wide_rules_differ_where_the_reference_does(ctx, golden):
    """The two accelerators of the reference disagree on some rays; the GPU
    reproduces each one's answer in its own mode."""
    tris = oracle.make_tris(golden["verts"], golden["idx"])
    out = {}
    for mode in (gpu.TRIANGLE_TEST_WIDE_BVH, gpu.TRIANGLE_TEST_BINARY_BVH):
        _load(ctx, golden["verts"], golden["idx"], mode)
        out[mode] = ctx.trace(golden["rays"])
    ref_differs = (golden["bvh_t"].view(np.uint32) != golden["wide_t"].view(np.uint32))
    gpu_differs = (out[0]["t"].view(np.uint32) != out[1]["t"].view(np.uint32))
    assert (ref_differs == gpu_differs).all()
    check_hits_valid(golden["rays"], tris, out[1], sem=BIN)


@pytest.mark.parametrize("n,mu,sigma,seed", [(1, -1.0, 0.1, 1), (7, -2.0, 0.3, 4), (513, -3.0, 0.5, 6),
                                             (5000, -3.5, 0.8, 7), (20000, -4.5, 0.5, 8)])
def test_binary_rule_random_soups_vs_bruteforce(ctx, n, mu, sigma, seed):
    verts, idx = scenes.triangle_soup(n, seed=seed, mu=mu, sigma=sigma)
    _load(ctx, verts, idx)
    tris = oracle.make_tris(verts, idx)
    rays = np.concatenate([scenes.primary_rays(64, 32), scenes.incoherent_rays(3000, seed=seed + 100)])
    rays[1::5, 3] = 0.02
    rays[2::5, 7] = 0.3
    compare_closest(rays, tris, ctx.trace(rays), *oracle.closest_brute(rays, tris, BIN)[:4], sem=BIN)
    sh = rays.copy()
    sh[:, 7] = scenes.shadow_tmax(len(rays), seed=seed + 200)
    assert (ctx.occluded(sh) == oracle.any_brute(sh, tris, BIN)).all()


def test_binary_rule_degenerate_inputs(ctx):
    """Near-degenerate slivers (|det| between 1e-6 and FLT_EPSILON), zero-area
    triangles and NaN vertices under the binary rule."""
    good_v, _ = scenes.triangle_soup(1500, seed=10, mu=np.log(0.05))
    rng = np.random.default_rng(12)
    base = rng.random((400, 3)).astype(np.float32)
    sliver = np.stack([base, base + [1e-3, 0, 0], base + [0.5e-3, 2e-4, 0]], 1).astype(np.float32)
    line = np.array([[0.1, 0.1, 0.1], [0.2, 0.2, 0.2], [0.3, 0.3, 0.3]], np.float32)
    nanv = np.array([[np.nan, 0.5, 0.5], [0.5, 0.5, 0.5], [0.5, 0.6, 0.5]], np.float32)
    verts = np.concatenate([good_v, sliver.reshape(-1, 3), line, nanv])
    idx = np.arange(verts.shape[0], dtype=np.uint32).reshape(-1, 3)
    _load(ctx, verts, idx)
    tris = oracle.make_tris(verts, idx)
    rays = scenes.incoherent_rays(4000, seed=13)
    aim = np.zeros((400, 8), np.float32)  # rays straight down onto the slivers
    aim[:, 0:3] = base + [4e-4, 5e-5, 1.0]
    aim[:, 4:7] = [0.0, 0.0, -1.0]
    aim[:, 7] = 3.4e38
    rays = np.concatenate([rays, aim])
    compare_closest(rays, tris, ctx.trace(rays), *oracle.closest_brute(rays, tris, BIN)[:4], sem=BIN)
    assert (ctx.occluded(rays) == oracle.any_brute(rays, tris, BIN)).all()


@pytest.mark.parametrize("limit,word", [("max_visits", "visit cap"), ("stack_limit", "stack overflow")])
def test_device_limit_runs_out_and_reports(ctx, limit, word):
    verts, idx = scenes.triangle_soup(20000, seed=21, mu=np.log(0.01))
    tris = oracle.make_tris(verts, idx)
    rays = scenes.incoherent_rays(4000, seed=22)
    _load(ctx, verts, idx, gpu.TRIANGLE_TEST_WIDE_BVH)
    full = ctx.trace(rays)
    ctx.set_traversal_options(gpu.TRIANGLE_TEST_WIDE_BVH, **{limit: 2 if limit == "max_visits" else 1})
    out = np.empty(len(rays), gpu.HIT_DTYPE)
    with pytest.raises(gpu.GpuError) as e:
        ctx.trace(rays, out=out)
    assert e.value.code == gpu.ERR_LIMIT and word in str(e.value)
    # rays that finished within the limit agree with the full traversal (a
    # ray can only end early as a miss)
    cut = out["prim"] == MISS
    ran_out = cut & (full["prim"] != MISS)
    assert ran_out.sum() > 0
    same = ~cut
    assert out[same].tobytes() == full[same].tobytes()
    with pytest.raises(gpu.GpuError) as e:
        ctx.occluded(rays)
    assert e.value.code == gpu.ERR_LIMIT
    # the limit lifted: the context still works and the status word is clear
    ctx.set_traversal_options(gpu.TRIANGLE_TEST_WIDE_BVH)
    again = ctx.trace(rays)
    assert again.tobytes() == full.tobytes()
    compare_closest(rays, tris, again, *oracle.closest_brute(rays, tris)[:4])


def test_render_reports_device_limit():
    scene = scenes.room_scene(seed=3)
    w = h = 16
    ctx = gpu.Context(0, w, h, 4)
    try:
        scenes.load_scene(ctx, scene, w, h)
        ctx.build_light_sampler(gpu.SAMPLER_POWER)
        ctx.set_render_options(sampler=gpu.RNG_COUNTER)
        ctx.set_traversal_options(gpu.TRIANGLE_TEST_WIDE_BVH, max_visits=1)
        ctx.reset_accumulation()
        with pytest.raises(gpu.GpuError) as e:
            ctx.render(2)
        assert e.value.code == gpu.ERR_LIMIT and "visit cap" in str(e.value)
        ctx.set_traversal_options(gpu.TRIANGLE_TEST_WIDE_BVH)
        ctx.reset_accumulation()
        ctx.render(2)
        acc, n = ctx.read_accumulation(w, h)
        assert n == 2 and np.isfinite(acc).all() and acc[..., :3].sum() > 0
    finally:
        ctx.close()


def test_invalid_traversal_options(ctx):
    for kw in ({"triangle_test": 2}, {"stack_limit": 25}):
        with pytest.raises(gpu.GpuError) as e:
            ctx.set_traversal_options(**kw)
        assert e.value.code == gpu.ERR_INVALID_ARGUMENT
