"""CPU tests of the GLB reader (alpine_b200/csrc/glb_parse.h) and of the
reference's own loader running on it.

The test scene is written by tests/glb_writer.py with the Python standard
library. The reference's GltfLoader (src/loaders/gltf_loader.cpp, compiled
unchanged into oracle/_ref against the tinygltf stand-in) loads it; its
Mesh::Data must equal what an independent numpy reading of the same file
gives after the loader's own FP32 transform arithmetic (getMatrix and
mul(float4x4, float4), src/math/matrix.h), bit for bit. The product's
alpine_gpu_glb_inspect (no GPU needed) reports the file's contents.
"""
import json
import math
import struct

import numpy as np
import pytest

import oracle
from alpine_b200 import gpu

import glb_writer

f32 = np.float32


def read_glb(path):
    """Independent reader: JSON chunk and accessors via numpy."""
    data = open(path, "rb").read()
    magic, ver, total = struct.unpack_from("<4sII", data, 0)
    assert magic == b"glTF" and ver == 2
    jl, jt = struct.unpack_from("<II", data, 12)
    doc = json.loads(data[20:20 + jl])
    bl, bt = struct.unpack_from("<II", data, 20 + jl)
    binb = data[28 + jl:28 + jl + bl]

    def acc(i):
        a = doc["accessors"][i]
        n = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4}[a["type"]]
        dt = {5126: np.float32, 5125: np.uint32, 5123: np.uint16}[a["componentType"]]
        if "sparse" in a:
            out = np.zeros((a["count"], n), np.float32)
            s = a["sparse"]
            iv, vv = doc["bufferViews"][s["indices"]["bufferView"]], doc["bufferViews"][s["values"]["bufferView"]]
            it = {5123: np.uint16, 5125: np.uint32}[s["indices"]["componentType"]]
            idx = np.frombuffer(binb, it, s["count"], iv["byteOffset"])
            out[idx] = np.frombuffer(binb, np.float32, s["count"] * n, vv["byteOffset"]).reshape(-1, n)
            return out
        v = doc["bufferViews"][a["bufferView"]]
        arr = np.frombuffer(binb, dt, a["count"] * n, v["byteOffset"] + a.get("byteOffset", 0))
        return arr.reshape(-1, n) if n > 1 else arr

    return doc, acc


def node_matrix(n):
    """getMatrix (gltf_loader.cpp:120-180) in float32, the reference's order."""
    if "matrix" in n:
        return np.array(n["matrix"], np.float32)
    qx, qy, qz, qw = (f32(x) for x in n.get("rotation", [0, 0, 0, 1]))
    sx, sy, sz = (f32(x) for x in n.get("scale", [1, 1, 1]))
    tx, ty, tz = (f32(x) for x in n.get("translation", [0, 0, 0]))
    one, two = f32(1), f32(2)
    m = [(one - two * qy * qy - two * qz * qz) * sx, (two * qx * qy + two * qz * qw) * sx,
         (two * qx * qz - two * qy * qw) * sx, f32(0),
         (two * qx * qy - two * qz * qw) * sy, (one - two * qx * qx - two * qz * qz) * sy,
         (two * qy * qz + two * qx * qw) * sy, f32(0),
         (two * qx * qz + two * qy * qw) * sz, (two * qy * qz - two * qx * qw) * sz,
         (one - two * qx * qx - two * qy * qy) * sz, f32(0), tx, ty, tz, f32(1)]
    return np.array(m, np.float32)


def mulv(m, v):
    """mul(float4x4, float4): columns scaled and summed in order; v [N, 4]."""
    c = m.reshape(4, 4)
    acc = c[0][None] * v[:, 0:1]
    for k in (1, 2, 3):
        acc = acc + c[k][None] * v[:, k:k + 1]
    return acc


def mulm(a, b):
    return np.concatenate([mulv(a, b.reshape(4, 4)[k][None])[0] for k in range(4)]).astype(np.float32)


def expected_meshes(path):
    doc, acc = read_glb(path)
    mats = {}

    def walk(i, parent):
        n = doc["nodes"][i]
        m = mulm(parent, node_matrix(n))
        if "mesh" in n:
            mats[n["mesh"]] = m
        for ch in n.get("children", []):
            walk(ch, m)

    ident = np.eye(4, dtype=np.float32).reshape(-1)
    for r in doc["scenes"][0]["nodes"]:
        walk(r, ident)
    out = []
    for mi, mesh in enumerate(doc["meshes"]):
        pos, nrm = [], []
        for p in mesh["primitives"]:
            pos.append(acc(p["attributes"]["POSITION"]))
            nrm.append(acc(p["attributes"]["NORMAL"]))
        pos, nrm = np.concatenate(pos), np.concatenate(nrm)
        one = np.ones((pos.shape[0], 1), np.float32)
        P = mulv(mats[mi], np.concatenate([pos, one], 1))[:, :3]
        N = mulv(mats[mi], np.concatenate([nrm, 0 * one], 1))[:, :3]
        out.append((P, N))
    return doc, out


@pytest.fixture(scope="module")
def scene_path(tmp_path_factory):
    p = tmp_path_factory.mktemp("glb") / "scene.glb"
    glb_writer.make_scene(p)
    return p


def test_inspect_counts(scene_path):
    info = gpu.glb_inspect(scene_path)
    doc, _ = read_glb(scene_path)
    tris = sum(doc["accessors"][p["indices"]]["count"] // 3 for m in doc["meshes"] for p in m["primitives"])
    assert info["shapes"] == 4 and info["materials"] == 4 and info["images"] == 2
    assert info["lights"] == 2 and info["channels"] == 4 and info["triangles"] == tris


def test_inspect_rejects_bad_files(tmp_path):
    bad = tmp_path / "bad.glb"
    bad.write_bytes(b"glTF\x02\x00\x00\x00\x10\x00\x00\x00garbage")
    with pytest.raises(gpu.GpuError):
        gpu.glb_inspect(bad)
    with pytest.raises(gpu.GpuError):
        gpu.glb_inspect(tmp_path / "missing.glb")


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build missing")
def test_reference_loader_on_project_reader(scene_path):
    doc, exp = expected_meshes(scene_path)
    r = oracle.RefRenderer(16, 16, 4, accelerator=oracle.RefRenderer.ACC_WIDE_BVH)
    try:
        r.load_glb(scene_path)
        meshes = r.meshes()
        lights = r.lights()
    finally:
        r.close()
    assert len(meshes) == 4
    for (P, N), m in zip(exp, meshes):
        assert m["pos"].tobytes() == P.astype(np.float32).tobytes()
        assert m["nrm"].tobytes() == N.astype(np.float32).tobytes()
    # the mesh referenced twice carries the later node's translation
    ctr = 0.5 * (meshes[3]["pos"].min(0) + meshes[3]["pos"].max(0))
    assert np.allclose(ctr, [2.0, 0.3, -1.0], atol=1e-5)
    # lights, in node traversal order (node 3 carries light 1, node 4 light
    # 0): point lights of power colour * intensity * 4 pi at the node origin
    assert len(lights) == 2
    power1 = np.array([1.0, 1.0, 1.0], np.float32) * f32(8.0) * f32(4.0) * f32(math.pi)
    power0 = np.array([1.0, 0.9, 0.8], np.float32) * f32(30.0) * f32(4.0) * f32(math.pi)
    assert np.allclose(lights[0][0], power1, rtol=1e-6) and np.allclose(lights[1][0], power0, rtol=1e-6)
    assert np.allclose(lights[1][1], [0.0, 3.0, -1.0]) and np.allclose(lights[0][1], [-1.5, 0.5, 0.5])
