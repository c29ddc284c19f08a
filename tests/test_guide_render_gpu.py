"""GPU tests of rendering with the learned guide.

Guided rendering draws each continuation direction from the guide's vMF
mixture (probability 1/2) or from the material's own procedure and weights it
by the one-sample MIS estimator f / (p_guide / 2 + p_mat / 2). Its per-pixel
means must agree with plain rendering (counter RNG) within the statistical
error measured from both sides' batches, and training must make the guide
useful: lower per-pixel error than plain rendering at equal samples on a
scene lit indirectly.
"""
import math

import numpy as np
import pytest

from alpine_b200 import gpu, scenes

pytestmark = pytest.mark.gpu


def _ctx(scene, w, h, depth, **opts):
    ctx = gpu.Context(0, w, h, depth)
    scenes.load_scene(ctx, scene, w, h)
    ctx.build_light_sampler(gpu.SAMPLER_POWER)
    ctx.set_render_options(sampler=gpu.RNG_COUNTER, **opts)
    ctx.reset_accumulation()
    return ctx


def _batches(ctx, w, h, batches, per):
    means, prev = [], np.zeros((h, w, 3), np.float64)
    for _ in range(batches):
        ctx.render(per)
        a, _ = ctx.read_accumulation(w, h)
        cur = a[..., :3].astype(np.float64)
        means.append((cur - prev) / per)
        prev = cur
    return np.array(means)


def _z_compare(a, b, label):
    ma, mb = a.mean(0), b.mean(0)
    se = np.sqrt(a.var(0, ddof=1) / a.shape[0] + b.var(0, ddof=1) / b.shape[0])
    ok = se > 1e-7
    z = (ma - mb)[ok] / se[ok]
    rel = abs(ma.mean() - mb.mean()) / mb.mean()
    print(f"{label}: |z|>5 fraction {(np.abs(z) > 5).mean():.4f}, mean z {z.mean():.3f}, "
          f"image mean {ma.mean():.5f} vs {mb.mean():.5f} (rel {rel:.2e})")
    return z, rel


GUIDE = dict(guide=True, guide_spp_per_wave=32, guide_batch=4096, guide_steps_per_wave=4)


def test_guided_room_unbiased():
    scene = scenes.room_scene(seed=4)
    w = h = 24
    plain = _ctx(scene, w, h, 8, seed=1)
    pb = _batches(plain, w, h, 16, 512)
    plain.close()
    g = _ctx(scene, w, h, 8, seed=2, **GUIDE)
    gb = _batches(g, w, h, 16, 512)
    steps, waves = g.guide_steps()
    g.close()
    assert steps > 0 and waves > 0
    z, rel = _z_compare(gb, pb, "guided vs plain (room)")
    assert (np.abs(z) > 5).mean() < 0.02
    assert abs(z.mean()) < 0.25
    assert rel < 0.02


def test_guided_interior_unbiased_and_trained():
    """Small glossy interior (20k triangles, windows as the only lights,
    depth 12): unbiased against plain rendering, and the trained guide lowers
    the per-pixel variance at equal samples."""
    scene = scenes.glossy_interior_scene(seed=3, target_tris=20000, n_boxes=30, n_spheres=6)
    w, h = 48, 32
    plain = _ctx(scene, w, h, 12, seed=1)
    pb = _batches(plain, w, h, 16, 256)
    plain.close()
    g = _ctx(scene, w, h, 12, seed=2, **GUIDE)
    g.render(1024)  # training
    g.reset_accumulation()
    gb = _batches(g, w, h, 16, 256)
    steps, _ = g.guide_steps()
    g.close()
    z, rel = _z_compare(gb, pb, "guided vs plain (interior)")
    assert (np.abs(z) > 5).mean() < 0.02
    assert abs(z.mean()) < 0.3
    assert rel < 0.03
    # variance at equal spp, over pixels with signal
    vp, vg = pb.var(0, ddof=1).sum(-1), gb.var(0, ddof=1).sum(-1)
    m = pb.mean(0).sum(-1) > 1e-3
    ratio = vg[m].sum() / vp[m].sum()
    print(f"interior: {steps} Adam steps, guided / plain variance at equal spp {ratio:.3f}")
    assert ratio < 1.0


def test_guided_deterministic_without_training():
    """With training off, the guide is fixed and guided rendering is
    deterministic (counter RNG, sample-ordered accumulation)."""
    scene = scenes.room_scene(seed=5)
    out = []
    for _ in range(2):
        g = _ctx(scene, 16, 16, 4, seed=9, guide=True, guide_train=False, guide_spp_per_wave=8)
        g.render(32)
        out.append(g.read_accumulation(16, 16)[0].tobytes())
        g.close()
    assert out[0] == out[1]
