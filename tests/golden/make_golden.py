"""Generates the golden traversal fixtures from the compiled reference.

Run from the repository root after `make -C oracle` (needs oracle/_ref, i.e.
the reference tree at build time):

    python tests/golden/make_golden.py

Writes tests/golden/traversal_small.npz: a seeded 2,048-triangle soup, 4,096
rays (1,024 primary + 3,072 incoherent), and the reference's own answers --
WideBvh (src/accelerators/wide_bvh.cpp with the ISPC kernels restated) and the
binary Bvh (src/accelerators/bvh.cpp) -- for closest hit (prim, t, b1, b2) and
for any hit with tmax uniform in (0, 1].
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from alpine_b200 import scenes  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "traversal_small.npz")


def main():
    verts, idx = scenes.triangle_soup(2048, seed=11, mu=np.log(0.04))
    rays = np.concatenate([scenes.primary_rays(32, 32), scenes.incoherent_rays(3072, seed=12)])
    shadow = rays.copy()
    shadow[:, 7] = scenes.shadow_tmax(rays.shape[0], seed=13)
    out = {"verts": verts, "idx": idx, "rays": rays, "shadow": shadow}
    for kind, name in ((oracle.RefAccel.WIDE_BVH, "wide"), (oracle.RefAccel.BVH, "bvh")):
        acc = oracle.RefAccel(kind, verts, idx)
        p, t, b1, b2 = acc.intersect(rays, nthreads=1)
        out[f"{name}_prim"], out[f"{name}_t"], out[f"{name}_b1"], out[f"{name}_b2"] = p, t, b1, b2
        out[f"{name}_occluded"] = acc.occluded(shadow, nthreads=1)
    np.savez_compressed(OUT, **out)
    print(OUT, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
