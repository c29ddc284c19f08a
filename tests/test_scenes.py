"""CPU tests of the scene generators and host-side helpers: geometry
invariants the parity tests and the bench rely on (closed, outward-facing
meshes, window openings, light orientation, triangle budgets, deterministic
batch configurations)."""
import math

import numpy as np
import pytest

from alpine_b200 import batch, scenes


def _normals(v, t):
    v = v.astype(np.float64)
    return np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])


def _edge_counts(t, v=None):
    """Triangles sharing each edge; with v, coincident vertices are welded
    first (the UV sphere repeats its pole vertex once per segment)."""
    if v is not None:
        _, weld = np.unique(np.round(np.asarray(v, np.float64), 5), axis=0, return_inverse=True)
        t = weld.reshape(-1)[t]
        t = t[(t[:, 0] != t[:, 1]) & (t[:, 1] != t[:, 2]) & (t[:, 2] != t[:, 0])]
    e = np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return counts


def test_uv_sphere_is_closed_and_outward():
    c = np.array([0.3, -0.2, 0.1])
    v, t, n = scenes.uv_sphere(tuple(c), 0.5, 32, 16)
    assert t.shape[0] == 2 * 32 * (16 - 1)
    nrm = _normals(v, t)
    cent = v[t].mean(1) - c
    assert ((nrm * cent).sum(1) > 0).all()
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-6)
    assert (_edge_counts(t, v) == 2).all()  # closed: every edge shared by two triangles


@pytest.mark.parametrize("s", [0, 1, 3])
def test_icosphere(s):
    v, f = batch.icosphere(s)
    assert f.shape[0] == 20 * 4 ** s
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
    assert ((_normals(v, f) * v[f].mean(1)).sum(1) > 0).all()
    assert (_edge_counts(f) == 2).all()


def test_box_mesh_winding():
    v, t = scenes.box_mesh((0, 0, 0), (1, 2, 3))
    c = np.array([0.5, 1.0, 1.5])
    out = (_normals(v, t) * (v[t].mean(1) - c)).sum(1)
    assert (out > 0).all()
    v, t = scenes.box_mesh((0, 0, 0), (1, 2, 3), inward=True)
    assert ((_normals(v, t) * (v[t].mean(1) - c)).sum(1) < 0).all()


def test_glossy_interior_openings_and_budget():
    sc = scenes.glossy_interior_scene(target_tris=40000, n_boxes=20, n_spheres=4)
    tris = sum(m["idx"].shape[0] for m in sc["meshes"])
    assert 0.8 * 40000 < tris < 1.2 * 40000
    assert sc["lights"] == [] and sc["background"] == (5.0, 5.0, 5.0)
    # the window wall: 4 x 12 m minus two 1 x 2 m openings, facing +x
    wall = sc["meshes"][1]
    n = _normals(wall["verts"], wall["idx"])
    assert (n[:, 0] > 0).all()
    assert abs(0.5 * np.linalg.norm(n, axis=1).sum() - (48.0 - 4.0)) < 1e-3
    # GGX share of the objects (furniture and spheres) is about 70 %
    kinds = [sc["materials"][m["tri_material"][0]][0] for m in sc["meshes"][2:]]
    assert 0.4 < np.mean(kinds) < 1.0


def test_city_facades_and_lights_face_outwards():
    sc = scenes.city_scene(seed=3, buildings=1, lights=40, extent=200.0)
    m = sc["meshes"][0]
    v, t = m["verts"].astype(np.float64), m["idx"]
    n = _normals(v, t)
    assert n[0, 1] > 0  # ground faces up
    c = v[4:].mean(0)
    assert (((v[t[2:]].mean(1) - c) * n[2:]).sum(1) > 0).all()
    for light in sc["lights"]:
        kind, L, corner, eu, ev = light
        assert kind == "quad" and min(L) > 0
        ln = np.cross(eu, ev)
        horiz = (np.array(corner) - c) * np.array([1.0, 0.0, 1.0])
        assert np.dot(ln, horiz) > 0


def test_city_budget():
    sc = scenes.city_scene(seed=1, buildings=100, lights=2000, extent=300.0)
    assert len(sc["lights"]) > 1900
    assert sc["meshes"][0]["idx"].shape[0] > 100 * 12


def test_blackbody_colour_order():
    warm, cold = scenes.blackbody_rgb(2700.0), scenes.blackbody_rgb(6500.0)
    assert warm.max() == pytest.approx(1.0) and cold.max() == pytest.approx(1.0)
    assert warm[2] < cold[2] and warm[0] >= cold[0]


def test_sinusoid_morph():
    v, t, n = scenes.uv_sphere((0, 0, 0), 1.0, 8, 4)
    mo = scenes.sinusoid_morph(v, n, amplitude=0.02, phase=0.5, frames=60, period=60.0, with_normals=True)
    assert mo["deltas"].shape == (1, v.shape[0], 3)
    assert np.allclose(np.linalg.norm(mo["deltas"][0], axis=1), 0.02, atol=1e-6)
    assert mo["times"].shape == (60,) and mo["weights"].shape == (60, 1)
    assert mo["weights"][0, 0] == pytest.approx(math.sin(0.5), abs=1e-6)
    assert mo["normal_deltas"].shape == (1, v.shape[0], 3)


def test_batch_configs_are_deterministic_and_in_range():
    a, b = batch.batch_configs(seed=3), batch.batch_configs(seed=3)
    assert a == b and len(a) == 48
    for c in a:
        assert 1000 <= c["tris"] <= 500_000
        assert c["width"] == c["height"] and c["width"] in batch.RESOLUTIONS
        assert c["spp"] in batch.SPPS
    sc = batch.batch_scene(a[0]["seed"], 5000)
    tris = sum(m["idx"].shape[0] for m in sc["meshes"])
    assert 5000 <= tris < 5000 + 20 * 4 ** 7
    assert 1 <= len(sc["lights"]) <= 64
    assert all("morph" in m for m in sc["meshes"][1:])
