"""CPU tests: the oracle restatement is pinned to the reference's own answers."""
import numpy as np
import pytest

import oracle
from alpine_b200 import scenes

MISS = 0xFFFFFFFF


def _closest_matches(g, name, sem):
    tris = oracle.make_tris(g["verts"], g["idx"])
    p, t, b1, b2, ntie = oracle.closest_brute(g["rays"], tris, sem)
    rp = g[f"{name}_prim"]
    assert ((p == MISS) == (rp == MISS)).all()
    h = p != MISS
    assert (t[h].view(np.uint32) == g[f"{name}_t"][h].view(np.uint32)).all()
    # unique closest hits: identical primitive and barycentrics
    u = h & (ntie == 1)
    assert (p[u] == rp[u]).all()
    assert (b1[u] == g[f"{name}_b1"][u]).all() and (b2[u] == g[f"{name}_b2"][u]).all()
    return int(h.sum())


def test_oracle_matches_reference_wide_bvh(golden):
    assert _closest_matches(golden, "wide", oracle.TRI_ISPC) > 1000


def test_oracle_matches_reference_binary_bvh(golden):
    assert _closest_matches(golden, "bvh", oracle.TRI_PRIM) > 1000


@pytest.mark.parametrize("name,sem", [("wide", oracle.TRI_ISPC), ("bvh", oracle.TRI_PRIM)])
def test_oracle_any_hit_matches_reference(golden, name, sem):
    tris = oracle.make_tris(golden["verts"], golden["idx"])
    occ = oracle.any_brute(golden["shadow"], tris, sem)
    assert (occ == golden[f"{name}_occluded"]).all()
    assert 0.05 < occ.mean() < 0.95


def test_oracle_bvh_equals_brute_force():
    verts, idx = scenes.triangle_soup(3000, seed=21, mu=np.log(0.05))
    tris = oracle.make_tris(verts, idx)
    rays = np.concatenate([scenes.primary_rays(48, 24), scenes.incoherent_rays(2000, seed=22)])
    rays[::7, 3] = 0.05  # some rays with tmin > 0
    ob = oracle.OracleBvh(tris)
    a = oracle.closest_brute(rays, tris)
    b = ob.closest(rays, nthreads=2)
    for x, y in zip(a, b):
        assert (np.asarray(x).view(np.uint32) == np.asarray(y).view(np.uint32)).all()
    sh = rays.copy()
    sh[:, 7] = scenes.shadow_tmax(len(rays), seed=23)
    assert (oracle.any_brute(sh, tris) == ob.any(sh, nthreads=2)).all()


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_oracle_matches_reference_fresh_case():
    verts, idx = scenes.triangle_soup(5000, seed=31, mu=np.log(0.03), sigma=0.8)
    tris = oracle.make_tris(verts, idx)
    rays = scenes.incoherent_rays(4000, seed=32)
    acc = oracle.RefAccel(oracle.RefAccel.WIDE_BVH, verts, idx)
    rp, rt, rb1, rb2 = acc.intersect(rays, nthreads=2)
    p, t, b1, b2, ntie = oracle.closest_brute(rays, tris)
    assert (t.view(np.uint32) == rt.view(np.uint32)).all()
    u = ntie <= 1
    assert (p[u] == rp[u]).all()


def test_fp64_error_bound(golden):
    """FP32 hits lie within ORC_ULP_BOUND * eps * cond of the FP64 oracle."""
    tris = oracle.make_tris(golden["verts"], golden["idx"])
    eps = np.finfo(np.float32).eps
    hits = np.nonzero(golden["wide_prim"] != MISS)[0]
    worst = 0.0
    for i in hits:
        ray = golden["rays"][i]
        ok, t, b1, b2, cond = oracle.tri_fp64(ray, tris[golden["wide_prim"][i]])
        assert ok
        errs = np.abs(np.array([golden["wide_t"][i] - t, golden["wide_b1"][i] - b1, golden["wide_b2"][i] - b2]))
        ratio = errs / (eps * np.maximum(cond, 1e-30))
        worst = max(worst, float(ratio.max()))
    assert worst <= 16.0, worst


def test_box_tests_conservative():
    """Both reference slab tests accept every ray that hits a triangle inside the box."""
    rng = np.random.default_rng(5)
    for _ in range(2000):
        v = rng.random((3, 3)).astype(np.float32)
        tri = np.concatenate([v[0], v[1] - v[0], v[2] - v[0]]).astype(np.float32)
        box = np.concatenate([v.min(0), v.max(0)]).astype(np.float32)
        b = rng.random(3)
        b /= b.sum()
        target = (b[0] * v[0] + b[1] * v[1] + b[2] * v[2])
        o = rng.random(3) * 4 - 2
        d = target - o
        d /= np.linalg.norm(d)
        ray = np.array([*o, 0.0, *d, np.finfo(np.float32).max], np.float32)
        hit, t, _, _ = oracle.tri_test(ray, tri)
        if not hit:
            continue
        inv = (1.0 / ray[4:7]).astype(np.float32)
        assert oracle.lib().orc_box_ispc(ray[:3].copy(), inv, np.float32(3e38), box) == 1
        assert oracle.lib().orc_box_ref(ray[:3].copy(), inv, np.float32(3e38), box) == 1
