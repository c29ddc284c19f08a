"""GPU tests of analytic spheres (Sphere::Data, src/shapes/sphere.h; in the
reference only Embree intersects them, src/accelerators/embree.cpp:107-122,
which is not vendored: the oracle is the project's FP64 ray / sphere
intersection, oracle.sphere_hits_fp64, so sphere parity is unpinned against
the reference by construction).

Bar: hit / miss agrees with the FP64 oracle except for near-tangent rays
(tangency margin < 1e-4); t within 4e-6 relative (plus 1e-6 absolute) of the
FP64 t; the reported sphere is the FP64-closest one unless the two nearest
hits are within that tolerance; mixed scenes take the nearer of the exact
FP32 triangle hit and the sphere hit; any-hit agrees with closest t < tmax.
A rendered analytic sphere matches a finely tessellated one.
"""
import math

import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes
from parity import MISS, check_hits_valid

pytestmark = pytest.mark.gpu

SPH = 0x80000000


def _spheres(n, seed, rmin=0.01, rmax=0.08):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.random((n, 3)), rng.uniform(rmin, rmax, (n, 1))], 1).astype(np.float32)


def _check_spheres(rays, sph, hits, tri_t=None, tri_prim=None):
    t64, margin = oracle.sphere_hits_fp64(rays, sph)
    best = np.argmin(t64, 1)
    bt = t64[np.arange(len(rays)), best]
    srt = np.sort(t64, 1)
    second = srt[:, 1] if sph.shape[0] > 1 else np.full(len(rays), np.inf)
    near_tangent = (margin < 1e-4).any(1)
    g_t = hits["t"].astype(np.float64)
    g_prim = hits["prim"]
    if tri_t is None:
        tri_t = np.full(len(rays), np.inf)
    tri_t = np.where(np.isfinite(tri_t) & (tri_t < 3.0e38), tri_t, np.inf)
    exp_t = np.minimum(bt, tri_t)
    tol = 4e-6 * np.abs(exp_t) + 1e-6
    exp_hit = np.isfinite(exp_t)
    got_hit = g_prim != MISS
    ok = near_tangent | (exp_hit == got_hit)
    assert ok.all(), f"{(~ok).sum()} rays disagree on hit / miss"
    both = exp_hit & got_hit & ~near_tangent
    assert (np.abs(g_t[both] - exp_t[both]) <= tol[both]).all(), "t outside the FP64 tolerance"
    with np.errstate(invalid="ignore"):  # inf - inf where no triangle or second sphere is hit
        sphere_expected = both & (bt < tri_t - tol) & (second > bt + 2 * tol)
    assert (g_prim[sphere_expected] == (SPH | best[sphere_expected])).all(), "wrong sphere reported"
    tri_expected = both & (tri_t < bt - tol)
    if tri_prim is not None:
        assert (g_prim[tri_expected] == tri_prim[tri_expected]).all()
    return int(got_hit.sum()), int((got_hit & ((g_prim & SPH) != 0)).sum())


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("n,seed", [(1, 1), (7, 2), (300, 3), (5000, 4)])
def test_spheres_vs_fp64(ctx, n, seed):
    sph = _spheres(n, seed, 0.05 if n < 10 else 0.01, 0.4 if n < 10 else 0.06)
    ctx.reset_scene()
    first = ctx.add_spheres(sph)
    assert first == 0
    st = ctx.build()
    assert st["spheres"] == n and st["triangles"] == 0
    rays = np.concatenate([scenes.primary_rays(64, 32), scenes.incoherent_rays(4000, seed=seed + 10)])
    rays[1::5, 3] = 0.02
    rays[2::5, 7] = 0.3
    hits = ctx.trace(rays)
    nh, ns = _check_spheres(rays, sph, hits)
    assert nh > 100 and ns == nh
    sh = rays.copy()
    sh[:, 7] = scenes.shadow_tmax(len(rays), seed=seed + 20)
    t64, margin = oracle.sphere_hits_fp64(sh, sph)
    exp = np.isfinite(t64).any(1)
    occ = ctx.occluded(sh).astype(bool)
    tangent = (margin < 1e-4).any(1) | (np.abs(t64.min(1) - sh[:, 7]) < 1e-5 * np.maximum(sh[:, 7], 1))
    assert ((occ == exp) | tangent).all()


def test_mixed_triangles_and_spheres(ctx):
    verts, idx = scenes.triangle_soup(20000, seed=31, mu=np.log(0.01))
    sph = _spheres(2000, 32)
    ctx.reset_scene()
    ctx.add_mesh(verts, idx)
    with pytest.raises(gpu.GpuError):  # geometry changed: stale BVH rejected after adding spheres
        ctx.build()
        ctx.add_spheres(sph)
        ctx.trace(scenes.incoherent_rays(10, seed=1))
    ctx.build()
    rays = scenes.incoherent_rays(6000, seed=33)
    hits = ctx.trace(rays)
    tris = oracle.make_tris(verts, idx)
    tp, tt, _, _ = oracle.closest_brute(rays, tris)[:4]
    tri_t = np.where(tp != MISS, tt.astype(np.float64), np.inf)
    nh, ns = _check_spheres(rays, sph, hits, tri_t, tp)
    assert ns > 100 and nh - ns > 100
    # triangle hits re-evaluate exactly
    tri_hits = hits.copy()
    tri_hits["prim"][(hits["prim"] & SPH) != 0] = MISS
    sel = tri_hits["prim"] != MISS
    check_hits_valid(rays[sel], tris, tri_hits[sel])
    occ = ctx.occluded(rays)
    assert (occ.astype(bool) == (hits["prim"] != MISS)).all()


def test_analytic_sphere_renders_like_a_tessellated_one():
    """The room with its GGX sphere as an analytic sphere against the same
    sphere tessellated finely (512 x 256 with smooth normals): the image means
    agree closely and the analytic one's normal AOV is the outward normal."""
    base = scenes.room_scene(seed=4, light="quad", sphere_segments=512, sphere_bands=256)
    w = h = 48
    means = []
    for analytic in (False, True):
        sc = dict(base, meshes=list(base["meshes"]))
        sphere_mesh = sc["meshes"].pop()  # the UV sphere is the last mesh
        c = gpu.Context(0, w, h, 6)
        try:
            scenes.load_scene(c, sc, w, h) if analytic else scenes.load_scene(c, base, w, h)
            if analytic:
                v = sphere_mesh["verts"]
                ctr = 0.5 * (v.min(0) + v.max(0))
                rad = float(np.linalg.norm(v - ctr, axis=1).max())
                mat = int(sphere_mesh["tri_material"][0])
                c.add_spheres(np.array([[*ctr, rad]], np.float32), np.array([mat], np.uint32))
                c.build()
            c.build_light_sampler(gpu.SAMPLER_POWER)
            c.set_render_options(sampler=gpu.RNG_COUNTER, seed=5)
            c.reset_accumulation()
            c.render(2048)
            a, n = c.read_accumulation(w, h)
            means.append(a[..., :3].mean() / n)
        finally:
            c.close()
    rel = abs(means[1] - means[0]) / means[0]
    print(f"analytic vs tessellated sphere: image means {means[0]:.5f} {means[1]:.5f} (rel {rel:.2e})")
    assert rel < 0.01
