"""Batched, animated rendering of many independent scenes on one GPU.

The workload: scenes of seeded displaced icospheres and boxes with
Lambertian or GGX materials and 1-64 quad lights. Triangle counts are
log-uniform between 1k and 500k; resolutions are one of 128^2, 256^2, 512^2
and 1024^2; spp is one of 4, 16 and 64. Every object is animated by one morph
target: the vertices move along their normals by a 0.02-amplitude sinusoid
with a per-object phase, keyed at 60 frames. The BVH is rebuilt every frame.

`BatchRenderer` keeps one context (stream, buffers, BVH, captured render
graph) per scene. A frame morphs and rebuilds every scene, enqueues every
render without waiting, then waits for all. Contexts are independent, so the
GPU runs the renders of different scenes concurrently, overlapping them with
the rebuilds of other scenes. Two ways to rebuild:
* "async" (the default): the device-driven rebuild (alpine_gpu_build_async,
  a captured graph replayed every frame). A frame's morph, rebuild and
  render of every scene are enqueued from one host thread with no host wait
  until the end of the frame;
* "sync": the host-driven rebuild, which waits on the host once per BVH
  level; the scenes' morph + rebuild + enqueue then run on a pool of host
  threads, so that those waits overlap.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import gpu, scenes

RESOLUTIONS = (128, 256, 512, 1024)
SPPS = (4, 16, 64)
FRAMES = 60


def icosphere(subdivisions):
    """Unit icosphere: 20 * 4^subdivisions triangles, outward winding."""
    p = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                  [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
                  [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdivisions):
        edges = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
        uniq, inv = np.unique(edges, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid])
        m = inv.reshape(3, -1).T + base  # midpoints of edges (0,1), (1,2), (2,0)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        f = np.concatenate([np.stack([a, m[:, 0], m[:, 2]], 1), np.stack([b, m[:, 1], m[:, 0]], 1),
                            np.stack([c, m[:, 2], m[:, 1]], 1), np.stack([m[:, 0], m[:, 1], m[:, 2]], 1)])
    # orient faces outwards
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    flip = (n * v[f].mean(1)).sum(1) < 0
    f[flip] = f[flip][:, [0, 2, 1]]
    return v, f


def displaced_icosphere(rng, center, radius, subdivisions, amplitude=0.15):
    """An icosphere displaced along its normals by a seeded sum of sinusoids;
    returns (verts, idx, normals) with normals of the undisplaced sphere."""
    v, f = icosphere(subdivisions)
    k = rng.normal(0, 3.0, (4, 3))
    ph = rng.uniform(0, 2 * math.pi, 4)
    disp = sum(np.sin(v @ k[i] + ph[i]) for i in range(4)) / 4
    p = np.asarray(center) + v * (radius * (1 + amplitude * disp))[:, None]
    return p.astype(np.float32), f.astype(np.uint32), v.astype(np.float32)


def batch_scene(seed, target_tris):
    """One scene of the batch (see the module docstring)."""
    rng = np.random.default_rng(seed)
    meshes, materials, lights = [], [], []

    def material():
        if rng.random() < 0.5:
            return (0, tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), 1.0)
        return (int(rng.random() < 0.5), tuple(float(x) for x in rng.uniform(0.4, 0.95, 3)), float(rng.uniform(0.05, 0.6)))

    gv, gi = scenes.box_mesh((-6.0, -0.2, -6.0), (6.0, 0.0, 6.0))
    materials.append((0, (0.6, 0.6, 0.6), 1.0))
    meshes.append({"verts": gv, "idx": gi, "normals": None, "tri_material": np.zeros(gi.shape[0], np.uint32)})
    used = gi.shape[0]
    obj = 0
    while used < target_tris:
        left = target_tris - used
        if rng.random() < 0.25 or left < 320:
            lo = rng.uniform(-4.5, 3.5, 3) * np.array([1, 0, 1])
            size = rng.uniform(0.3, 1.5, 3)
            bv, bi = scenes.box_mesh(tuple(lo), tuple(lo + size))
            bv = scenes.rotate_y(bv, float(rng.uniform(0, math.pi)), lo + size / 2)
            v, idx, nrm = bv, bi, None
        else:
            s = int(np.clip(math.floor(math.log(max(left, 80) / 20, 4)), 1, 7))
            s = int(rng.integers(1, s + 1))
            r = float(rng.uniform(0.3, 1.2))
            c = (float(rng.uniform(-4.5, 4.5)), r + float(rng.uniform(0.0, 1.0)), float(rng.uniform(-4.5, 4.5)))
            v, idx, nrm = displaced_icosphere(rng, c, r, s)
        materials.append(material())
        mesh = {"verts": v, "idx": idx, "normals": nrm,
                "tri_material": np.full(idx.shape[0], len(materials) - 1, np.uint32)}
        mesh["morph"] = scenes.sinusoid_morph(v, nrm, amplitude=0.02, phase=float(rng.uniform(0, 2 * math.pi)),
                                              frames=FRAMES, period=float(FRAMES))
        meshes.append(mesh)
        used += idx.shape[0]
        obj += 1
    for _ in range(int(rng.integers(1, 65))):
        w, d = rng.uniform(0.2, 1.0, 2)
        x, z = rng.uniform(-4.5, 4.5, 2)
        y = float(rng.uniform(3.0, 5.0))
        L = float(rng.uniform(2.0, 12.0))
        # edges (0, 0, d) x (w, 0, 0): cross points down (-y)
        lights.append(("quad", (L, L * 0.9, L * 0.8), (float(x), y, float(z)), (0.0, 0.0, float(d)), (float(w), 0.0, 0.0)))
    camera = ((0.0, 4.5, 9.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), math.radians(55.0))
    return {"meshes": meshes, "materials": materials, "lights": lights, "camera": camera,
            "background": (0.05, 0.05, 0.07)}


def batch_configs(n=48, seed=11, max_tris=500_000, resolutions=RESOLUTIONS, spps=SPPS):
    """n scene configurations: triangle count log-uniform in [1k, max_tris],
    resolution and spp drawn from the given sets."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        tris = int(math.exp(rng.uniform(math.log(1000), math.log(max_tris))))
        res = int(rng.choice(resolutions))
        out.append({"seed": seed * 1000 + i, "tris": tris, "width": res, "height": res, "spp": int(rng.choice(spps))})
    return out


class BatchRenderer:
    """One context per scene; frames are rendered concurrently (see the
    module docstring)."""

    def __init__(self, configs, device=0, depth=8, cuda_graph=True, sampler=gpu.SAMPLER_BVH, autotune=False,
                 threads=16):
        import concurrent.futures as cf

        self.configs = configs
        self.ctxs = []
        self.triangles = 0
        self.threads = threads
        self._pool = cf.ThreadPoolExecutor(max_workers=max(1, threads))
        for cfg in configs:
            scene = batch_scene(cfg["seed"], cfg["tris"])
            c = gpu.Context(device, cfg["width"], cfg["height"], depth)
            scenes.load_scene(c, scene, cfg["width"], cfg["height"])
            c.build_light_sampler(sampler)
            c.set_render_options(sampler=gpu.RNG_COUNTER, seed=cfg["seed"], russian_roulette_depth=3,
                                 cuda_graph=cuda_graph)
            if autotune:
                cfg["tuning"] = c.autotune(probe_spp=min(4, cfg["spp"]))
            c.update_scene(0.0)  # a synchronous build sizes the buffers of the device-driven rebuild
            c.reset_accumulation()
            self.triangles += sum(m["idx"].shape[0] for m in scene["meshes"])
            self.ctxs.append(c)

    def frame(self, t, threads=None, rebuild="async"):
        """Morph + rebuild + render every scene at time t; returns the summed
        device build time (ms).

        rebuild="async": every scene's morph, device-driven rebuild and
        render are enqueued from this thread, then all are waited for.
        rebuild="sync": a scene's rebuild waits on the host once per BVH
        level; with threads > 1 the scenes' morph + rebuild + render enqueue
        run on a pool of host threads (each context is used by one thread at
        a time; the C calls release the GIL), so those waits overlap instead
        of adding up."""
        threads = self.threads if threads is None else threads
        if rebuild == "async":
            for c, cfg in zip(self.ctxs, self.configs):
                c.update_scene_async(t)
                c.render_async(cfg["spp"])
            for c in self.ctxs:
                c.render_wait()
            return sum(c.read_build_stats()["build_ms"] for c in self.ctxs)

        def one(i):
            c, cfg = self.ctxs[i], self.configs[i]
            ms = c.update_scene(t)["build_ms"]
            c.render_async(cfg["spp"])
            return ms

        if threads > 1:
            build_ms = sum(self._pool.map(one, range(len(self.ctxs))))
        else:
            build_ms = sum(one(i) for i in range(len(self.ctxs)))
        for c in self.ctxs:
            c.render_wait()
        return build_ms

    def run(self, frames, start=0, threads=None, rebuild="async"):
        """Renders `frames` frames; returns wall time, build time and rates."""
        t0 = time.perf_counter()
        build = 0.0
        for f in range(start, start + frames):
            build += self.frame(float(f), threads, rebuild)
        dt = time.perf_counter() - t0
        samples = frames * sum(c["width"] * c["height"] * c["spp"] for c in self.configs)
        return {"frames": frames, "seconds": dt, "frames_per_s": frames / dt, "samples_per_s": samples / dt,
                "build_ms_per_frame": build / frames}

    def close(self):
        for c in self.ctxs:
            c.close()
        self.ctxs = []
        self._pool.shutdown()
