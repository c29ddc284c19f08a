"""The drop-in boundary exercised from the reference's side.

oracle/_ref/libalpine_ref_plugin.so is the reference (its unmodified sources)
with the GPU plug-in a maintainer adds to it (alpine_b200/plugin), compiled
against the reference's own headers:

* GpuAccelerator implements the reference's Accelerator interface
  (src/accelerators/accelerator.h:13-39). Driven through that interface from
  16 threads at once, as Alpine::render's per-tile tasks drive it
  (src/alpine.cpp:276-285, 316), its Intersection records (shape pointer,
  primId, t, barycentrics and the geometric normal ng) equal those of the
  reference accelerator whose triangle rule it runs, bit for bit, apart from
  exact ties.
* The reference's own Alpine::render with the GpuAccelerator installed (the
  new `case AcceleratorType::Gpu` of Alpine::resetScene) renders the same
  image as with the reference's accelerator: the reference integrator and
  sampler streams are unchanged, only the traversal moved to the GPU.
* With the GpuBackend render branch on, the Alpine methods forward to the GPU
  integrator; its image passes the per-pixel z-test against the reference's
  own render, and the reference's postProcess reads the GPU accumulation.
"""
import numpy as np
import pytest

import oracle
from alpine_b200 import gpu, scenes
from parity import MISS

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.plugin_available(), reason="plug-in library not built")]


def _compare(ref, got, rays, tris, sem):
    rp, rt, rb1, rb2, rng, rok = ref
    gp, gt, gb1, gb2, gng, gok = got
    assert ((rp == MISS) == (gp == MISS)).all()
    h = rp != MISS
    assert (rt.view(np.uint32)[h] == gt.view(np.uint32)[h]).all()
    same = h & (rp == gp)
    ties = h & (rp != gp)
    if ties.any():  # a different primitive must be an exact tie
        ok, t2, _, _ = oracle.tri_test_batch(rays[ties], tris, gp[ties], sem)
        assert ok.all() and (t2.view(np.uint32) == rt[ties].view(np.uint32)).all()
    for a, b in ((rb1, gb1), (rb2, gb2)):
        assert (a.view(np.uint32)[same] == b.view(np.uint32)[same]).all()
    assert (rng.view(np.uint32)[same] == gng.view(np.uint32)[same]).all(), "ng differs"
    assert gok[h].all() and rok[h].all()
    return int(h.sum()), int(ties.sum())


@pytest.mark.parametrize("rule", ["wide", "binary"])
def test_gpu_accelerator_through_accelerator_interface(rule):
    ref_kind, gpu_kind, sem = ((oracle.RefAccel.WIDE_BVH, oracle.RefAccel.GPU, oracle.TRI_ISPC) if rule == "wide"
                               else (oracle.RefAccel.BVH, oracle.RefAccel.GPU_BINARY, oracle.TRI_PRIM))
    verts, idx = scenes.triangle_soup(20000, seed=81, mu=np.log(0.01))
    rays = np.concatenate([scenes.primary_rays(48, 32), scenes.incoherent_rays(3000, seed=82)])
    shadow = rays.copy()
    shadow[:, 7] = scenes.shadow_tmax(len(rays), seed=83)
    ref = oracle.RefAccel(ref_kind, verts, idx)
    acc = oracle.RefAccel(gpu_kind, verts, idx)
    tris = oracle.make_tris(verts, idx)
    hits, ties = _compare(ref.intersect_ng(rays, 1), acc.intersect_ng(rays, 16), rays, tris, sem)
    assert hits > 1000
    assert (ref.occluded(shadow, 1) == acc.occluded(shadow, 16)).all()
    # Mesh::update's path: new positions through getVertexBuffer, updateShape,
    # updateScene; ng follows the moved vertices
    moved = verts + np.float32(0.003) * np.cos(np.arange(verts.shape[0], dtype=np.float32))[:, None]
    ref.update_vertices(0, moved)
    acc.update_vertices(0, moved)
    tris = oracle.make_tris(moved, idx)
    _compare(ref.intersect_ng(rays, 1), acc.intersect_ng(rays, 16), rays, tris, sem)
    assert (ref.occluded(shadow, 1) == acc.occluded(shadow, 16)).all()


@pytest.mark.parametrize("binary", [False, True])
def test_alpine_render_with_gpu_accelerator(binary):
    """Alpine::render (reference integrator, reference sampler streams, one
    std::async task per tile) with the GpuAccelerator against the same render
    with the reference's own accelerator: identical sums on every pixel whose
    paths met no exact tie."""
    w = h = 24
    scene = scenes.room_scene(seed=8, light="quad")
    R = oracle.RefRenderer
    out = {}
    for plugin, acc in ((False, R.ACC_BVH if binary else R.ACC_WIDE_BVH),
                        (True, R.ACC_GPU_BINARY if binary else R.ACC_GPU)):
        r = R(w, h, 8, accelerator=acc, plugin=plugin)
        scenes.load_scene(r, scene, w, h)
        r.build_light_sampler(gpu.SAMPLER_POWER)
        r.reset_accumulation()
        r.render(2)
        out[plugin] = r.read_accumulation()
        r.close()
    (a, na), (b, nb) = out[False], out[True]
    assert na == nb == 2
    same = (a == b).all(-1).mean()
    print(f"GpuAccelerator render: {same:.4f} of pixels bit-identical to the reference accelerator's")
    assert same > 0.995


@pytest.mark.parametrize("which", ["room", "textured"])
def test_alpine_render_through_gpu_branch(which):
    """The GpuBackend render branch: Alpine's render state forwarded to the GPU
    integrator (counter RNG). z-test of the reference's own render (256 spp)
    against the branch's batches (16 x 1024 spp), both read back through the
    Alpine's accumulation; the reference's postProcess runs on the GPU sums.
    The textured scene adds textures, tangents and the environment map."""
    w = h = 24
    scene = scenes.room_scene(seed=4, light="quad") if which == "room" else scenes.textured_scene(seed=3)
    R = oracle.RefRenderer
    r = R(w, h, 8, accelerator=R.ACC_WIDE_BVH)
    scenes.load_scene(r, scene, w, h)
    r.build_light_sampler(gpu.SAMPLER_POWER)
    r.reset_accumulation()
    r.render(256)
    a, n = r.read_accumulation()
    r.close()
    rmean = a[..., :3].astype(np.float64) / n
    g = R(w, h, 8, accelerator=R.ACC_WIDE_BVH, gpu_branch=True, seed=9)
    scenes.load_scene(g, scene, w, h)
    g.build_light_sampler(gpu.SAMPLER_POWER)
    g.reset_accumulation()
    batches, prev = [], np.zeros((h, w, 3), np.float64)
    for k in range(16):
        g.render(1024)
        s, total = g.read_accumulation()
        assert total == 1024 * (k + 1)
        cur = s[..., :3].astype(np.float64)
        batches.append((cur - prev) / 1024)
        prev = cur
    ldr = g.post_process(True)
    g.close()
    gb = np.array(batches)
    gmean = gb.mean(0)
    var1 = gb.var(0, ddof=1) * 1024
    se = np.sqrt(var1 / 256 + var1 / (16 * 1024))
    ok = se > 1e-7
    z = (rmean - gmean)[ok] / se[ok]
    print(f"GPU render branch z-test ({which}): |z|>5 fraction {(np.abs(z) > 5).mean():.4f}, mean z {z.mean():.3f}")
    assert np.allclose(rmean[~ok], gmean[~ok], rtol=1e-4, atol=1e-6)
    assert (np.abs(z) > 5).mean() < 0.02 and abs(z.mean()) < 0.25
    assert ldr.shape == (h, w, 3) and ldr.max() > 0
