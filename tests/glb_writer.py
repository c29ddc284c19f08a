"""Writes binary glTF 2.0 (.glb) test scenes with the Python standard library
and numpy only (json, struct, zlib), independently of the C++ reader under
test. PNG images are written with every scanline filter type (none, sub,
up, average, Paeth) in turn and zlib-compressed, so the reader's inflate and
unfiltering paths are all exercised.

make_scene(path) writes the loader test scene: a two-primitive mesh (16- and
32-bit indices, two materials, normals, texture coordinates, two morph
targets with position and normal deltas), a textured floor with tangents and
a normal map, a box with a sparse morph target, a mesh referenced by two nodes
(the later node's transform wins in the reference loader), node transforms
given as TRS and as a matrix under a parent, two punctual lights, and
animations with LINEAR "weights" channels plus channels the loader skips
(STEP interpolation, a "translation" path).
"""
from __future__ import annotations

import json
import math
import struct
import zlib

import numpy as np


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def png_bytes(pixels: np.ndarray) -> bytes:
    """8-bit RGB or RGBA PNG of pixels [H, W, C]; row y uses filter y % 5."""
    h, w, c = pixels.shape
    ctype = {3: 2, 4: 6}[c]
    rows = []
    px = pixels.astype(np.int32).reshape(h, w * c)
    for y in range(h):
        raw = px[y]
        prev = px[y - 1] if y else np.zeros_like(raw)
        a = np.concatenate([np.zeros(c, np.int32), raw[:-c]])
        cc = np.concatenate([np.zeros(c, np.int32), prev[:-c]])
        f = y % 5
        pred = [np.zeros_like(raw), a, prev, (a + prev) >> 1, _paeth(a, prev, cc)][f]
        rows.append(bytes([f]) + ((raw - pred) & 0xFF).astype(np.uint8).tobytes())

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    ihdr = struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", ihdr) + chunk(b"IDAT", zlib.compress(b"".join(rows), 9)) +
            chunk(b"IEND", b""))


class GlbBuilder:
    def __init__(self):
        self.bin = bytearray()
        self.doc = {"asset": {"version": "2.0"}, "buffers": [], "bufferViews": [], "accessors": []}

    def view(self, data: bytes) -> int:
        while len(self.bin) % 4:
            self.bin += b"\0"
        self.doc["bufferViews"].append({"buffer": 0, "byteOffset": len(self.bin), "byteLength": len(data)})
        self.bin += data
        return len(self.doc["bufferViews"]) - 1

    def accessor(self, arr: np.ndarray, type_: str) -> int:
        comp = {np.dtype(np.float32): 5126, np.dtype(np.uint32): 5125, np.dtype(np.uint16): 5123}[arr.dtype]
        count = arr.shape[0] if arr.ndim > 1 or type_ == "SCALAR" else arr.size
        if type_ == "SCALAR":
            count = arr.size
        v = self.view(np.ascontiguousarray(arr).tobytes())
        self.doc["accessors"].append({"bufferView": v, "componentType": comp, "count": int(count), "type": type_})
        return len(self.doc["accessors"]) - 1

    def sparse_accessor(self, count: int, indices: np.ndarray, values: np.ndarray) -> int:
        iv = self.view(np.ascontiguousarray(indices).tobytes())
        vv = self.view(np.ascontiguousarray(values, np.float32).tobytes())
        ictype = {np.dtype(np.uint16): 5123, np.dtype(np.uint32): 5125}[indices.dtype]
        self.doc["accessors"].append({"componentType": 5126, "count": int(count), "type": "VEC3",
                                      "sparse": {"count": int(indices.size),
                                                 "indices": {"bufferView": iv, "componentType": ictype},
                                                 "values": {"bufferView": vv}}})
        return len(self.doc["accessors"]) - 1

    def image(self, pixels: np.ndarray) -> int:
        v = self.view(png_bytes(pixels))
        self.doc.setdefault("images", []).append({"bufferView": v, "mimeType": "image/png"})
        return len(self.doc["images"]) - 1

    def write(self, path):
        self.doc["buffers"] = [{"byteLength": len(self.bin)}]
        js = json.dumps(self.doc).encode()
        js += b" " * ((4 - len(js) % 4) % 4)
        binb = bytes(self.bin) + b"\0" * ((4 - len(self.bin) % 4) % 4)
        total = 12 + 8 + len(js) + 8 + len(binb)
        with open(path, "wb") as f:
            f.write(struct.pack("<4sII", b"glTF", 2, total))
            f.write(struct.pack("<II", len(js), 0x4E4F534A) + js)
            f.write(struct.pack("<II", len(binb), 0x004E4942) + binb)


def _sphere(seg=24, bands=12, radius=0.5):
    th = math.pi * np.arange(bands + 1) / bands
    ph = 2 * math.pi * np.arange(seg + 1) / seg  # a seam column, so uvs do not wrap inside a triangle
    T, P = np.meshgrid(th, ph, indexing="ij")
    n = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    uv = np.stack([P / (2 * math.pi), T / math.pi], -1).reshape(-1, 2)
    tan = np.stack([-np.sin(P), np.zeros_like(P), np.cos(P), np.ones_like(P)], -1).reshape(-1, 4)
    J, I = np.meshgrid(np.arange(bands), np.arange(seg), indexing="ij")
    a, b = J * (seg + 1) + I, J * (seg + 1) + I + 1
    c, d = (J + 1) * (seg + 1) + I + 1, (J + 1) * (seg + 1) + I
    tris = np.concatenate([np.stack([a, c, b], -1).reshape(-1, 3), np.stack([a, d, c], -1).reshape(-1, 3)])
    return (radius * n).astype(np.float32), n.astype(np.float32), uv.astype(np.float32), tan.astype(np.float32), tris


def _compact(pos, nrm, uv, tan, tris):
    used = np.unique(tris)
    remap = np.full(pos.shape[0], -1, np.int64)
    remap[used] = np.arange(used.size)
    return pos[used], nrm[used], uv[used], tan[used], remap[tris]


def make_scene(path, seed=1):
    rng = np.random.default_rng(seed)
    g = GlbBuilder()
    d = g.doc
    # images and textures
    yy, xx = np.mgrid[0:32, 0:32]
    chk = (((xx // 4) + (yy // 4)) % 2)[..., None]
    img0 = np.where(chk, [220, 180, 60], [40, 90, 200]).astype(np.uint8) + rng.integers(0, 20, (32, 32, 3)).astype(np.uint8)
    u = (np.mgrid[0:16, 0:16][1] + 0.5) / 16
    v = (np.mgrid[0:16, 0:16][0] + 0.5) / 16
    nm = np.stack([0.3 * np.sin(4 * math.pi * u), 0.3 * np.cos(4 * math.pi * v), np.ones_like(u)], -1)
    nm /= np.linalg.norm(nm, axis=-1, keepdims=True)
    img1 = np.concatenate([np.round((nm * 0.5 + 0.5) * 255), np.full((16, 16, 1), 255)], -1).astype(np.uint8)
    g.image(img0)
    g.image(img1)
    d["textures"] = [{"source": 0}, {"source": 1}]
    d["materials"] = [
        {"pbrMetallicRoughness": {"baseColorFactor": [0.8, 0.3, 0.2, 1.0], "metallicFactor": 1.0,
                                  "roughnessFactor": 0.35}},
        {"pbrMetallicRoughness": {"baseColorFactor": [1.0, 1.0, 1.0, 1.0], "metallicFactor": 0.0,
                                  "roughnessFactor": 0.6, "baseColorTexture": {"index": 0}},
         "normalTexture": {"index": 1}},
        {},  # glTF defaults: metallic 1, roughness 1 -> a Conductor
        {"pbrMetallicRoughness": {"baseColorFactor": [0.5, 0.6, 0.7, 1.0], "metallicFactor": 0.0,
                                  "roughnessFactor": 1.0}},
    ]
    meshes = []
    # mesh 0: a sphere split into two primitives, two morph targets
    pos, nrm, uv, tan, tris = _sphere()
    half = tris.shape[0] // 2
    prims = []
    for k, (sel, itype, mat) in enumerate(((tris[:half], np.uint16, 0), (tris[half:], np.uint32, 1))):
        p, n, t_uv, t_tan, t = _compact(pos, nrm, uv, tan, sel)
        V = p.shape[0]
        d0 = (0.15 * n * np.sin(3 * p[:, :1] + k)).astype(np.float32)
        dn0 = (0.1 * np.roll(n, 1, axis=1)).astype(np.float32)
        d1 = (0.1 * rng.normal(size=(V, 3))).astype(np.float32)
        prims.append({
            # no TANGENT here: with morph targets the reference's shading morphs the
            # tangents too (src/shapes/mesh.cpp:104-144) and reads per-target
            # tangent deltas, which a target without TANGENT lacks
            "attributes": {"POSITION": g.accessor(p, "VEC3"), "NORMAL": g.accessor(n, "VEC3"),
                           "TEXCOORD_0": g.accessor(t_uv, "VEC2")},
            "indices": g.accessor(t.astype(itype).reshape(-1), "SCALAR"), "material": mat,
            "targets": [{"POSITION": g.accessor(d0, "VEC3"), "NORMAL": g.accessor(dn0, "VEC3")},
                        {"POSITION": g.accessor(d1, "VEC3"), "NORMAL": g.accessor(np.zeros_like(d1), "VEC3")}],
        })
    meshes.append({"primitives": prims, "weights": [0.0, 0.0]})
    # mesh 1: a floor with texture coordinates beyond 1 and tangents
    fp = np.array([[-3, 0, -3], [3, 0, -3], [3, 0, 3], [-3, 0, 3]], np.float32)
    fn = np.tile(np.array([[0, 1, 0]], np.float32), (4, 1))
    fuv = np.array([[0, 0], [3, 0], [3, 3], [0, 3]], np.float32)
    ft = np.tile(np.array([[1, 0, 0, 1]], np.float32), (4, 1))
    meshes.append({"primitives": [{"attributes": {"POSITION": g.accessor(fp, "VEC3"), "NORMAL": g.accessor(fn, "VEC3"),
                                                  "TEXCOORD_0": g.accessor(fuv, "VEC2"),
                                                  "TANGENT": g.accessor(ft, "VEC4")},
                                   "indices": g.accessor(np.array([0, 2, 1, 0, 3, 2], np.uint16), "SCALAR"),
                                   "material": 1}]})
    # mesh 2: a box (per-face vertices) with one sparse morph target
    c = np.array([[x, y, z] for x in (-0.4, 0.4) for y in (-0.4, 0.4) for z in (-0.4, 0.4)], np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    bp, bn, bi = [], [], []
    for q in quads:
        p4 = c[list(q)]
        nn = np.cross(p4[1] - p4[0], p4[2] - p4[0])
        nn /= np.linalg.norm(nn)
        base = len(bp)
        bp += list(p4)
        bn += [nn] * 4
        bi += [base, base + 1, base + 2, base, base + 2, base + 3]
    bp, bn = np.array(bp, np.float32), np.array(bn, np.float32)
    sidx = np.array([0, 5, 9, 14, 22], np.uint16)
    sval = (0.2 * rng.normal(size=(sidx.size, 3))).astype(np.float32)
    meshes.append({"primitives": [{"attributes": {"POSITION": g.accessor(bp, "VEC3"), "NORMAL": g.accessor(bn, "VEC3")},
                                   "indices": g.accessor(np.array(bi, np.uint32), "SCALAR"), "material": 3,
                                   # the reference's shading reads every target's
                                   # normal deltas, so the target carries (zero) ones
                                   "targets": [{"POSITION": g.sparse_accessor(bp.shape[0], sidx, sval),
                                                "NORMAL": g.accessor(np.zeros_like(bn), "VEC3")}]}],
                   "weights": [0.0]})
    # mesh 3: a small sphere (default material) referenced by two nodes
    p3, n3, _, _, t3 = _sphere(12, 6, 0.3)
    meshes.append({"primitives": [{"attributes": {"POSITION": g.accessor(p3, "VEC3"), "NORMAL": g.accessor(n3, "VEC3")},
                                   "indices": g.accessor(t3.astype(np.uint16).reshape(-1), "SCALAR"),
                                   "material": 2}]})
    d["meshes"] = meshes
    ang = math.radians(20.0)
    q = [0.0, math.sin(ang / 2), 0.0, math.cos(ang / 2)]
    mat = [1.1, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.9, 0.0, 0.0, -0.5, 0.0, 1.0]  # column-major
    q2 = [0.2, 0.1, 0.0, 1.0]
    n2 = math.sqrt(sum(x * x for x in q2))
    q2 = [x / n2 for x in q2]
    d["nodes"] = [
        {"rotation": q, "scale": [1.2, 1.2, 1.2], "translation": [0.0, 0.5, 0.0], "children": [1, 2, 5]},
        {"mesh": 0, "translation": [0.3, 0.8, 0.0]},
        {"mesh": 1, "matrix": mat},
        {"mesh": 2, "translation": [-1.5, 0.5, 0.5], "rotation": q2,
         "extensions": {"KHR_lights_punctual": {"light": 1}}},
        {"translation": [0.0, 3.0, -1.0], "extensions": {"KHR_lights_punctual": {"light": 0}}},
        {"mesh": 3, "translation": [1.0, 0.0, 1.0]},
        {"mesh": 3, "translation": [2.0, 0.3, -1.0]},
    ]
    d["extensions"] = {"KHR_lights_punctual": {"lights": [
        {"type": "point", "color": [1.0, 0.9, 0.8], "intensity": 30.0},
        {"type": "spot", "intensity": 8.0, "spot": {}},
    ]}}
    d["extensionsUsed"] = ["KHR_lights_punctual"]
    d["scenes"] = [{"nodes": [0, 3, 4, 6]}]
    d["scene"] = 0
    t0 = g.accessor(np.array([0.0, 1.0, 2.5], np.float32), "SCALAR")
    w0 = g.accessor(np.array([0.0, 0.0, 1.0, 0.3, 0.2, 1.0], np.float32), "SCALAR")
    t1 = g.accessor(np.array([0.5, 2.0], np.float32), "SCALAR")
    w1 = g.accessor(np.array([0.0, 1.0], np.float32), "SCALAR")
    tr = g.accessor(np.array([[0, 0, 0], [0, 1, 0]], np.float32), "VEC3")
    d["animations"] = [{"samplers": [{"input": t0, "output": w0},  # LINEAR by default
                                     {"input": t1, "output": w1, "interpolation": "LINEAR"},
                                     {"input": t1, "output": tr, "interpolation": "LINEAR"},
                                     {"input": t1, "output": w1, "interpolation": "STEP"}],
                        "channels": [{"sampler": 0, "target": {"node": 1, "path": "weights"}},
                                     {"sampler": 1, "target": {"node": 3, "path": "weights"}},
                                     {"sampler": 2, "target": {"node": 1, "path": "translation"}},
                                     {"sampler": 3, "target": {"node": 3, "path": "weights"}}]}]
    g.write(path)
    return d
