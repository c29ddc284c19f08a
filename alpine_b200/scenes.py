"""Seeded synthetic scenes and ray sets.

All generators are deterministic functions of their seed. Geometry is returned
as (vertices float32[V,3], indices uint32[T,3]); rays as float32[N,8] with the
layout {ox, oy, oz, tmin, dx, dy, dz, tmax} used by the C-ABI.
"""
from __future__ import annotations

import math

import numpy as np

FLT_MAX = np.float32(3.4028234663852886e38)


def _random_rotations(rng, n):
    """Uniform random rotation matrices (n, 3, 3) from uniform unit quaternions."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    qx = a * np.sin(2 * np.pi * u2)
    qy = a * np.cos(2 * np.pi * u2)
    qz = b * np.sin(2 * np.pi * u3)
    qw = b * np.cos(2 * np.pi * u3)
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (qy * qy + qz * qz)
    R[:, 0, 1] = 2 * (qx * qy - qz * qw)
    R[:, 0, 2] = 2 * (qx * qz + qy * qw)
    R[:, 1, 0] = 2 * (qx * qy + qz * qw)
    R[:, 1, 1] = 1 - 2 * (qx * qx + qz * qz)
    R[:, 1, 2] = 2 * (qy * qz - qx * qw)
    R[:, 2, 0] = 2 * (qx * qz - qy * qw)
    R[:, 2, 1] = 2 * (qy * qz + qx * qw)
    R[:, 2, 2] = 1 - 2 * (qx * qx + qy * qy)
    return R


def triangle_soup(n_tris: int = 1 << 20, seed: int = 2, mu: float = math.log(0.004), sigma: float = 0.5):
    """Triangle soup in the unit cube: centroids uniform in [0,1]^3, edge
    lengths log-normal(mu, sigma), orientations uniform on the sphere.

    Each triangle has its three corners at angles 0/120/240 degrees (plus a
    common random phase) around its centre, at radii r_k = l_k / sqrt(3) with
    l_k ~ log-normal(mu, sigma), then rotated by a uniform random rotation.
    """
    rng = np.random.default_rng(seed)
    c = rng.random((n_tris, 3))
    lengths = np.exp(rng.normal(mu, sigma, (n_tris, 3)))
    r = lengths / math.sqrt(3.0)
    phase = rng.random(n_tris)[:, None] * 2 * np.pi
    ang = phase + np.array([0.0, 2 * np.pi / 3, 4 * np.pi / 3])[None, :]
    local = np.stack([r * np.cos(ang), r * np.sin(ang), np.zeros_like(r)], axis=-1)  # (n,3,3)
    R = _random_rotations(rng, n_tris)
    world = np.einsum("nij,nkj->nki", R, local) + c[:, None, :]
    verts = world.reshape(-1, 3).astype(np.float32)
    idx = np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3)
    return verts, idx


def look_at_basis(eye, target, up):
    """Camera basis of the reference (src/camera.cpp:87-96): columns viewX,
    viewY, viewZ with viewZ = normalize(target - eye),
    viewX = normalize(cross(viewZ, up)), viewY = cross(viewX, viewZ)."""
    eye = np.asarray(eye, np.float64)
    z = np.asarray(target, np.float64) - eye
    z /= np.linalg.norm(z)
    x = np.cross(z, np.asarray(up, np.float64))
    x /= np.linalg.norm(x)
    y = np.cross(x, z)
    return x, y, z


def primary_rays(width=2048, height=1024, eye=(0.5, 0.5, -1.0), target=(0.5, 0.5, 0.0), up=(0.0, 1.0, 0.0),
                 fovy_deg=60.0, tmax=None):
    """Pinhole rays through pixel centres, as Camera::generateRay
    (src/camera.cpp:73-85) with film at distance 1, film height tan(fovy/2),
    film width = height * aspect."""
    x, y, z = look_at_basis(eye, target, up)
    fh = math.tan(0.5 * math.radians(fovy_deg))
    fw = fh * (width / height)
    px = (np.arange(width) + 0.5) / width
    py = (np.arange(height) + 0.5) / height
    fx = (px[None, :] - 0.5) * fw
    fy = (0.5 - py[:, None]) * fh
    d = fx[..., None] * x + fy[..., None] * y + z  # (h, w, 3)
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    n = width * height
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = np.asarray(eye, np.float32)
    rays[:, 4:7] = d.reshape(-1, 3)
    rays[:, 7] = FLT_MAX if tmax is None else tmax
    return rays


def incoherent_rays(n, seed=3, tmax=None):
    """Origins uniform in [0,1]^3, directions uniform on the sphere."""
    rng = np.random.default_rng(seed)
    o = rng.random((n, 3))
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = v
    rays[:, 7] = FLT_MAX if tmax is None else tmax
    return rays


def shadow_tmax(n, seed=4):
    """tmax uniform in (0, 1]."""
    rng = np.random.default_rng(seed)
    return (1.0 - rng.random(n)).astype(np.float32)


def traversal_workload(n_tris=1 << 20, n_primary=(2048, 1024), n_incoherent=1 << 21, seed=2):
    """The traversal microbenchmark: a triangle soup, closest-hit rays
    (primary then incoherent, tmax = FLT_MAX) and the same rays as any-hit
    shadow rays with tmax uniform in (0, 1]."""
    verts, idx = triangle_soup(n_tris, seed=seed)
    prim = primary_rays(*n_primary)
    inc = incoherent_rays(n_incoherent, seed=seed + 1)
    closest = np.concatenate([prim, inc])
    shadow = closest.copy()
    shadow[:, 7] = shadow_tmax(closest.shape[0], seed=seed + 2)
    return verts, idx, closest, shadow
