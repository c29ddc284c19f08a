"""Parity checks of GPU traversal results against the oracle.

Bar (integer / index work is bit-exact; FP32 t and barycentrics are computed
by the same rounded formula as the reference, so they are bit-exact too):
  * hit / miss agree for every ray;
  * t is bit-identical to the oracle's canonical closest t;
  * the primitive id equals the oracle's, or the GPU's primitive evaluates to
    exactly the same t (an exact tie: the reference keeps whichever it finds
    first, so ties are reported, not failed);
  * b1, b2 are bit-identical whenever the primitive ids agree;
  * any-hit flags are identical.
"""
from __future__ import annotations

import numpy as np

import oracle

MISS = 0xFFFFFFFF


def compare_closest(rays, tris, hits, ref_prim, ref_t, ref_b1, ref_b2, sem=oracle.TRI_ISPC):
    """Returns a report dict; raises AssertionError on a parity failure."""
    gp = hits["prim"]
    gt = hits["t"]
    hit_r = ref_prim != MISS
    hit_g = gp != MISS
    bad_hit = np.nonzero(hit_r != hit_g)[0]
    assert bad_hit.size == 0, f"hit/miss disagree on {bad_hit.size} rays, first {bad_hit[:8]}"
    h = hit_r
    bad_t = np.nonzero(h & (gt.view(np.uint32) != ref_t.view(np.uint32)))[0]
    assert bad_t.size == 0, (f"t differs on {bad_t.size} rays, first {bad_t[:8]}: gpu {gt[bad_t[:4]]} "
                             f"ref {ref_t[bad_t[:4]]}")
    diff = np.nonzero(h & (gp != ref_prim))[0]
    ties = 0
    if diff.size:
        ok, t2, _, _ = oracle.tri_test_batch(rays[diff], tris, gp[diff], sem)
        exact = ok & (t2.view(np.uint32) == ref_t[diff].view(np.uint32))
        assert exact.all(), f"{(~exact).sum()} rays report a different primitive that is not an exact tie"
        ties = int(diff.size)
    same = h & (gp == ref_prim)
    bad_b = np.nonzero(same & ((hits["b1"].view(np.uint32) != ref_b1.view(np.uint32)) |
                               (hits["b2"].view(np.uint32) != ref_b2.view(np.uint32))))[0]
    assert bad_b.size == 0, f"barycentrics differ on {bad_b.size} rays"
    return {"rays": int(len(gp)), "hits": int(h.sum()), "ties": ties}


def check_hits_valid(rays, tris, hits, sem=oracle.TRI_ISPC):
    """Every reported hit re-evaluates to exactly the reported t, b1, b2."""
    gp = hits["prim"]
    h = gp != MISS
    ok, t, b1, b2 = oracle.tri_test_batch(rays, tris, np.where(h, gp, MISS).astype(np.uint32), sem)
    assert (ok == h).all(), f"{int((ok != h).sum())} reported hits do not re-evaluate as hits"
    assert (t[h].view(np.uint32) == hits["t"][h].view(np.uint32)).all()
    assert (b1[h].view(np.uint32) == hits["b1"][h].view(np.uint32)).all()
    assert (b2[h].view(np.uint32) == hits["b2"][h].view(np.uint32)).all()
    return int(h.sum())
