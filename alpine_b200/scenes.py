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


# ---------------------------------------------------------------------------
# Rendering scenes. A scene is a dict:
#   meshes:    list of {verts, idx, normals (or None), tri_material}
#   materials: list of (kind, (r, g, b), roughness), kind 0 = dielectric, 1 = conductor
#   lights:    list of ("disk", power, color, position, target, radius) |
#                      ("point", power, color, position) |
#                      ("quad", radiance, corner, edge_u, edge_v)
#   camera:    (eye, target, up, fovy_radians)
#   background (r, g, b)

def box_mesh(lo, hi, inward=False):
    """12-triangle axis-aligned box; normals (cross(e0, e1)) point outwards,
    or inwards when inward=True."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 4, 7, 3), (1, 2, 6, 5), (0, 1, 5, 4), (3, 7, 6, 2)]  # outward CCW
    tris = []
    for a, b, c, d in quads:
        t1, t2 = (a, b, c), (a, c, d)
        if inward:
            t1, t2 = (a, c, b), (a, d, c)
        tris += [t1, t2]
    return v, np.array(tris, np.uint32)


def rotate_y(v, angle, center):
    c, s = math.cos(angle), math.sin(angle)
    R = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], np.float64)
    return ((v - center) @ R.T + center).astype(np.float32)


def uv_sphere(center, radius, segments=64, bands=32):
    """UV sphere with smooth per-vertex normals; pole bands are triangle fans.
    Vertex (band j, segment i) is number j * segments + i."""
    th = math.pi * np.arange(bands + 1, dtype=np.float64) / bands
    ph = 2 * math.pi * np.arange(segments, dtype=np.float64) / segments
    T, P = np.meshgrid(th, ph, indexing="ij")
    n = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    verts = (np.asarray(center, np.float64) + radius * n).astype(np.float32)
    J, I = np.meshgrid(np.arange(bands), np.arange(segments), indexing="ij")
    a, b = J * segments + I, J * segments + (I + 1) % segments
    c, d = (J + 1) * segments + (I + 1) % segments, (J + 1) * segments + I
    t1 = np.stack([a, b, c], -1)
    t2 = np.stack([a, c, d], -1)
    keep = np.stack([J != 0, J != bands - 1], -1)        # per (j, i): first, second triangle
    tris = np.stack([t1, t2], 2)[keep]                   # row-major: (j, i, k) order
    return verts, tris.astype(np.uint32), n.astype(np.float32)


def room_scene(seed=1, light="disk", sphere_segments=64, sphere_bands=32):
    """The small procedural room: a closed 2x2x2 box (inward normals), two
    boxes rotated by a seeded angle in [0, pi/2), a UV sphere with smooth
    normals, a 0.5 x 0.5 ceiling light of radiance 15. Walls and boxes are
    Lambertian with albedo uniform in [0.2, 0.8]^3 (one box is a GGX
    dielectric with roughness 0.3); the sphere is a GGX conductor with
    roughness 0.3. light='disk' uses a disk light of equal area and power (the
    reference has no quad light), light='quad' the quad itself."""
    rng = np.random.default_rng(seed)
    meshes, materials = [], []

    def albedo():
        return tuple(float(x) for x in rng.uniform(0.2, 0.8, 3))

    rv, ri = box_mesh((-1, -1, -1), (1, 1, 1), inward=True)
    wall_mats = []
    for _ in range(6):
        materials.append((0, albedo(), 1.0))
        wall_mats.append(len(materials) - 1)
    meshes.append({"verts": rv, "idx": ri, "normals": None,
                   "tri_material": np.repeat(np.array(wall_mats, np.uint32), 2)})
    for k, (lo, hi, rough) in enumerate([((-0.7, -1.0, -0.2), (-0.2, -0.2, 0.3), 1.0),
                                         ((0.15, -1.0, 0.2), (0.65, -0.55, 0.7), 0.3)]):
        bv, bi = box_mesh(lo, hi)
        ang = float(rng.uniform(0, math.pi / 2))
        ctr = (np.array(lo) + np.array(hi)) / 2
        bv = rotate_y(bv, ang, ctr)
        materials.append((0, albedo(), rough))
        meshes.append({"verts": bv, "idx": bi, "normals": None,
                       "tri_material": np.full(bi.shape[0], len(materials) - 1, np.uint32)})
    sv, si, sn = uv_sphere((0.35, -0.25, -0.35), 0.3, sphere_segments, sphere_bands)
    materials.append((1, (0.95, 0.75, 0.45), 0.3))
    meshes.append({"verts": sv, "idx": si, "normals": sn,
                   "tri_material": np.full(si.shape[0], len(materials) - 1, np.uint32)})
    L, side = 15.0, 0.5
    y = 0.999
    if light == "quad":
        # edges (side, 0, 0) x (0, 0, side): cross points down (-y), into the room
        lights = [("quad", (L, L, L), (-0.25, y, -0.25), (side, 0.0, 0.0), (0.0, 0.0, side))]
    else:
        area = side * side
        lights = [("disk", L * area * math.pi, (1.0, 1.0, 1.0), (0.0, y, 0.0), (0.0, 0.0, 0.0),
                   math.sqrt(area / math.pi))]
    camera = ((0.0, 0.0, -0.95), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), math.radians(70.0))
    return {"meshes": meshes, "materials": materials, "lights": lights, "camera": camera,
            "background": (0.0, 0.0, 0.0)}


def wall_with_openings(x, z_range, y_range, openings):
    """Quads of the plane x = const over z_range x y_range minus the
    rectangular openings [(z0, z1, y0, y1), ...]; normals cross(e0, e1)
    point to +x."""
    zs = sorted({z_range[0], z_range[1], *[o[0] for o in openings], *[o[1] for o in openings]})
    ys = sorted({y_range[0], y_range[1], *[o[2] for o in openings], *[o[3] for o in openings]})
    verts, tris = [], []
    for i in range(len(zs) - 1):
        for j in range(len(ys) - 1):
            zc, yc = 0.5 * (zs[i] + zs[i + 1]), 0.5 * (ys[j] + ys[j + 1])
            if any(o[0] < zc < o[1] and o[2] < yc < o[3] for o in openings):
                continue
            b = len(verts)
            verts += [(x, ys[j], zs[i]), (x, ys[j], zs[i + 1]), (x, ys[j + 1], zs[i + 1]), (x, ys[j + 1], zs[i])]
            tris += [(b, b + 2, b + 1), (b, b + 3, b + 2)]
    return np.array(verts, np.float32), np.array(tris, np.uint32)


def glossy_interior_scene(seed=1, target_tris=2_000_000, n_boxes=80, n_spheres=24, glossy_fraction=0.7,
                          sky=5.0, roughness=(0.02, 0.4), glossy_floor=True):
    """Glossy interior: a closed 20 x 4 x 12 m room (x in [-10, 10], y in
    [0, 4], z in [-6, 6]) of about `target_tris` triangles made of seeded
    furniture boxes and subdivided UV spheres (`roughness`: the GGX range,
    `glossy_floor`: whether the floor is GGX). Light comes only through two
    1 x 2 m window openings in the x = -10 wall, from a constant sky of
    radiance `sky` (the background radiance of rays that escape, added at any
    depth; there are no light sources, so next-event estimation finds none of
    it). A `glossy_fraction` of the objects, and the floor, are GGX conductors
    with roughness uniform in [0.02, 0.4]; the rest, walls and ceiling are
    Lambertian."""
    rng = np.random.default_rng(seed)
    meshes, materials = [], []

    def surface():
        if rng.random() < glossy_fraction:
            return (1, tuple(float(x) for x in rng.uniform(0.5, 0.95, 3)), float(rng.uniform(*roughness)))
        return (0, tuple(float(x) for x in rng.uniform(0.3, 0.8, 3)), 1.0)

    rv, ri = box_mesh((-10.0, 0.0, -6.0), (10.0, 4.0, 6.0), inward=True)
    # box_mesh face order: z0, z1, x0, x1, y0 (floor), y1 (ceiling); x0 is
    # replaced by the wall with the window openings
    keep = [0, 1, 3, 4, 5]
    face_mats = {}
    for f in keep:
        if f == 4 and glossy_floor:
            materials.append((1, (0.8, 0.8, 0.8), float(rng.uniform(*roughness))))
        else:
            materials.append((0, tuple(float(x) for x in rng.uniform(0.5, 0.8, 3)), 1.0))
        face_mats[f] = len(materials) - 1
    sel = np.concatenate([[2 * f, 2 * f + 1] for f in keep])
    meshes.append({"verts": rv, "idx": ri[sel], "normals": None,
                   "tri_material": np.repeat(np.array([face_mats[f] for f in keep], np.uint32), 2)})
    openings = [(zc - 0.5, zc + 0.5, 1.0, 3.0) for zc in (-3.0, 2.0)]
    wv, wi = wall_with_openings(-10.0, (-6.0, 6.0), (0.0, 4.0), openings)
    materials.append((0, tuple(float(x) for x in rng.uniform(0.5, 0.8, 3)), 1.0))
    meshes.append({"verts": wv, "idx": wi, "normals": None,
                   "tri_material": np.full(wi.shape[0], len(materials) - 1, np.uint32)})
    eye = (9.6, 3.5, 5.6)

    def placed(lo_x, hi_x, lo_z, hi_z):  # a centre at least 3 m (x-z) from the camera
        while True:
            x, z = rng.uniform(lo_x, hi_x), rng.uniform(lo_z, hi_z)
            if (x - eye[0]) ** 2 + (z - eye[2]) ** 2 > 9.0:
                return x, z

    for _ in range(n_boxes):
        w, dpt = rng.uniform(0.4, 2.5, 2)
        h = rng.uniform(0.3, 2.2)
        cx, cz = placed(-8.5, 9.0, -5.0, 5.0)
        lo, hi = (cx - w / 2, 0.0, cz - dpt / 2), (cx + w / 2, h, cz + dpt / 2)
        bv, bi = box_mesh(lo, hi)
        bv = rotate_y(bv, float(rng.uniform(0, math.pi / 2)), np.array([cx, 0.0, cz]))
        materials.append(surface())
        meshes.append({"verts": bv, "idx": bi, "normals": None,
                       "tri_material": np.full(bi.shape[0], len(materials) - 1, np.uint32)})
    used = sum(m["idx"].shape[0] for m in meshes)
    per = max(64, (target_tris - used) // max(1, n_spheres))
    bands = max(4, int(round(math.sqrt(per / 4.0))))
    for _ in range(n_spheres):
        r = float(rng.uniform(0.2, 0.9))
        x, z = placed(-8.5, 9.0, -5.0, 5.0)
        ctr = (float(x), r + float(rng.uniform(0.0, 1.5)), float(z))
        sv, si, sn = uv_sphere(ctr, r, 2 * bands, bands)
        materials.append(surface())
        meshes.append({"verts": sv, "idx": si, "normals": sn,
                       "tri_material": np.full(si.shape[0], len(materials) - 1, np.uint32)})
    camera = (eye, (-10.0, 1.0, -1.0), (0.0, 1.0, 0.0), math.radians(60.0))
    return {"meshes": meshes, "materials": materials, "lights": [], "camera": camera,
            "background": (sky, sky, sky)}


def sinusoid_morph(verts, normals, amplitude=0.02, phase=0.0, frames=60, period=60.0, with_normals=False):
    """One morph target moving every vertex by `amplitude` along its normal
    (the radial direction when there are no normals), driven by the weight
    sin(2 pi t / period + phase) sampled at `frames` keyframes t = 0, 1, ...
    (glTF-style keyframed morph weights)."""
    v = np.asarray(verts, np.float32)
    if normals is not None:
        d = np.asarray(normals, np.float32)
    else:
        c = v.mean(0)
        d = v - c
        d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-12)
    deltas = (amplitude * d)[None].astype(np.float32)
    times = np.arange(frames, dtype=np.float32)
    weights = np.sin(2 * np.pi * times / period + phase).astype(np.float32)[:, None]
    out = {"deltas": deltas, "times": times, "weights": weights}
    if with_normals and normals is not None:
        # a small tilt of the normals, so that normal morphing is exercised
        out["normal_deltas"] = (0.3 * np.roll(np.asarray(normals, np.float32), 1, axis=1))[None]
    return out


def blackbody_rgb(kelvin):
    """Relative linear RGB of a blackbody: Planck's law sampled at 610, 550
    and 465 nm, normalised to a maximum of 1."""
    h, c, k = 6.62607015e-34, 2.99792458e8, 1.380649e-23
    lam = np.array([610e-9, 550e-9, 465e-9])
    b = 1.0 / (lam ** 5 * (np.exp(h * c / (lam * k * kelvin)) - 1.0))
    return b / b.max()


def city_scene(seed=1, buildings=2000, lights=131072, extent=1000.0, panel=2.5, window=(1.2, 1.5)):
    """Many-light city: `buildings` extruded boxes (footprints uniform in
    [5, 40] m, heights log-normal(ln 20, 0.6)) on a ground plane of
    `extent` m, facades tessellated into `panel`-metre panels, and `lights`
    emissive window quads on the facades, facing outwards (power log-normal
    with sigma 1.5, colour temperature uniform in [2700, 6500] K). Materials:
    GGX with roughness uniform in [0.05, 1], metallic (conductor) with
    probability 0.2, else a dielectric (F0 0.04 coat over a diffuse base)."""
    rng = np.random.default_rng(seed)
    half = extent / 2
    verts, idx, tmat, materials = [], [], [], []
    nv = 0

    def add_quads(corners):  # corners [n, 4, 3] counter-clockwise seen from the front
        nonlocal nv
        n = corners.shape[0]
        verts.append(corners.reshape(-1, 3))
        b = nv + 4 * np.arange(n, dtype=np.int64)[:, None]
        idx.append(np.concatenate([b + [0, 1, 2], b + [0, 2, 3]]).reshape(2, n, 3).transpose(1, 0, 2).reshape(-1, 3))
        nv += 4 * n
        return 2 * n

    materials.append((0, (0.35, 0.35, 0.35), 1.0))  # ground
    g = np.array([[[-half, 0, -half], [-half, 0, half], [half, 0, half], [half, 0, -half]]], np.float64)
    tmat.append(np.zeros(add_quads(g), np.uint32))
    facades = []  # (origin, u axis, v axis, width, height) per facade
    for b in range(buildings):
        w, d = rng.uniform(5.0, 40.0, 2)
        hgt = float(np.exp(rng.normal(math.log(20.0), 0.6)))
        cx, cz = rng.uniform(-half + 40, half - 40, 2)
        ang = rng.uniform(0, math.pi / 2)
        ca, sa = math.cos(ang), math.sin(ang)
        ex, ez = np.array([ca, 0, -sa]), np.array([sa, 0, ca])
        c0 = np.array([cx, 0.0, cz]) - ex * w / 2 - ez * d / 2
        base = [c0, c0 + ex * w, c0 + ex * w + ez * d, c0 + ez * d]
        kind = 1 if rng.random() < 0.2 else 0
        materials.append((kind, tuple(float(x) for x in rng.uniform(0.3, 0.9, 3)), float(rng.uniform(0.05, 1.0))))
        mid = len(materials) - 1
        quads = []
        for k in range(4):
            p0, p1 = base[k], base[(k + 1) % 4]
            length = float(np.linalg.norm(p1 - p0))
            u = (p1 - p0) / length
            nu, nh = max(1, int(length / panel)), max(1, int(hgt / panel))
            us = np.linspace(0, length, nu + 1)
            hs = np.linspace(0, hgt, nh + 1)
            U0, H0 = np.meshgrid(us[:-1], hs[:-1], indexing="ij")
            U1, H1 = np.meshgrid(us[1:], hs[1:], indexing="ij")
            a = p0 + U0.reshape(-1, 1) * u + H0.reshape(-1, 1) * np.array([0, 1, 0])
            bb = p0 + U1.reshape(-1, 1) * u + H0.reshape(-1, 1) * np.array([0, 1, 0])
            cc = p0 + U1.reshape(-1, 1) * u + H1.reshape(-1, 1) * np.array([0, 1, 0])
            dd = p0 + U0.reshape(-1, 1) * u + H1.reshape(-1, 1) * np.array([0, 1, 0])
            # walls go counter-clockwise around the footprint seen from above,
            # so (a, d, c, b) faces outwards
            quads.append(np.stack([a, dd, cc, bb], 1))
            facades.append((p0, u, length, hgt))
        top = np.array([[base[0] + [0, hgt, 0], base[3] + [0, hgt, 0], base[2] + [0, hgt, 0], base[1] + [0, hgt, 0]]])
        quads.append(top)
        q = np.concatenate(quads)
        tmat.append(np.full(add_quads(q), mid, np.uint32))
    v = np.concatenate(verts).astype(np.float32)
    t = np.concatenate(idx).astype(np.uint32)
    # orient every triangle so that its normal points away from its building's centre line or up
    meshes = [{"verts": v, "idx": t, "normals": None, "tri_material": np.concatenate(tmat)}]
    light_list = []
    fa = rng.integers(0, len(facades), lights)
    temps = rng.uniform(2700.0, 6500.0, lights)
    powers = np.exp(rng.normal(0.0, 1.5, lights)) * 20.0
    ww, wh = window
    for i in range(lights):
        p0, u, length, hgt = facades[fa[i]]
        if length < ww + 0.2 or hgt < wh + 1.0:
            continue
        s_ = rng.uniform(0.1, length - ww - 0.1)
        y = rng.uniform(0.5, hgt - wh - 0.2)
        outward = np.cross(np.array([0.0, 1.0, 0.0]), u)  # facing away from the footprint
        corner = p0 + u * s_ + np.array([0.0, y, 0.0]) + outward * 0.05
        area = ww * wh
        L = powers[i] / (area * math.pi) * blackbody_rgb(temps[i])
        # edges (0, wh, 0) x (ww u): cross points along `outward`
        light_list.append(("quad", tuple(float(x) for x in L), tuple(float(x) for x in corner),
                           (0.0, float(wh), 0.0), tuple(float(x) for x in u * ww)))
    camera = ((0.0, 180.0, -half * 0.9), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), math.radians(50.0))
    return {"meshes": meshes, "materials": materials, "lights": light_list, "camera": camera,
            "background": (0.01, 0.01, 0.02)}


def add_random_lights(scene, n, seed=5, kinds=("disk", "point")):
    """Adds n seeded disk / point lights spread over the room's ceiling half
    (many-light sampler tests)."""
    rng = np.random.default_rng(seed)
    for i in range(n):
        kind = kinds[i % len(kinds)]
        pos = (float(rng.uniform(-0.9, 0.9)), float(rng.uniform(0.2, 0.95)), float(rng.uniform(-0.9, 0.9)))
        color = tuple(float(x) for x in rng.uniform(0.3, 1.0, 3))
        power = float(np.exp(rng.normal(0.0, 1.5)))
        if kind == "disk":
            tgt = (pos[0] + float(rng.normal(0, 0.3)), -1.0, pos[2] + float(rng.normal(0, 0.3)))
            scene["lights"].append(("disk", power, color, pos, tgt, float(rng.uniform(0.02, 0.1))))
        else:
            scene["lights"].append(("point", power * 0.2, color, pos))
    return scene


def textured_scene(seed=1, tex=64, env=(128, 64)):
    """An open scene for the texture paths: a floor with a repeating
    checkerboard base-colour texture (texture coordinates up to 4, so the
    lookup wraps), a UV sphere with vertex normals, tangents and a bumpy
    normal map on a GGX conductor, a box with a base-colour texture on every
    face, under a lat-long environment map (sky gradient and a bright sun
    patch) that escaping rays read, plus one disk light."""
    rng = np.random.default_rng(seed)
    textures = []
    # checkerboard (linear colours)
    yy, xx = np.mgrid[0:tex, 0:tex]
    chk = ((xx // 8 + yy // 8) % 2).astype(np.float32)
    a, b = rng.uniform(0.1, 0.4, 3), rng.uniform(0.5, 0.9, 3)
    t0 = np.concatenate([a[None, None] * (1 - chk[..., None]) + b[None, None] * chk[..., None],
                         np.ones((tex, tex, 1))], -1).astype(np.float32)
    textures.append(t0)
    # normal map in [-1, 1]: a bump pattern in tangent space
    u = (xx + 0.5) / tex
    v = (yy + 0.5) / tex
    n = np.stack([0.35 * np.sin(6 * math.pi * u), 0.35 * np.cos(4 * math.pi * v), np.ones_like(u)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    textures.append(np.concatenate([n, np.ones((tex, tex, 1))], -1).astype(np.float32))
    # noise colours
    textures.append(np.concatenate([rng.uniform(0.05, 0.95, (tex, tex, 3)), np.ones((tex, tex, 1))], -1)
                    .astype(np.float32))
    materials = [(0, (0.5, 0.5, 0.5), 1.0, 0, None),        # floor: checkerboard Lambertian
                 (1, (0.9, 0.7, 0.4), 0.25, None, 1),       # sphere: normal-mapped conductor
                 (0, (0.5, 0.5, 0.5), 0.3, 2, None)]        # box: textured two-lobe dielectric
    meshes = []
    fv = np.array([[-4, 0, -4], [4, 0, -4], [4, 0, 4], [-4, 0, 4]], np.float32)
    fi = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)  # normal +y
    fuv = np.array([[0, 0], [4, 0], [4, 4], [0, 4]], np.float32)
    meshes.append({"verts": fv, "idx": fi, "normals": None, "tri_material": np.zeros(2, np.uint32), "uvs": fuv})
    seg, bands = 48, 24
    sv, si, sn = uv_sphere((0.0, 1.0, 0.0), 1.0, seg, bands)
    th = math.pi * np.arange(bands + 1) / bands
    ph = 2 * math.pi * np.arange(seg) / seg
    T, P = np.meshgrid(th, ph, indexing="ij")
    suv = np.stack([P / (2 * math.pi), T / math.pi], -1).reshape(-1, 2).astype(np.float32)
    tang = np.stack([-np.sin(P), np.zeros_like(P), np.cos(P), np.ones_like(P)], -1).reshape(-1, 4).astype(np.float32)
    meshes.append({"verts": sv, "idx": si, "normals": sn, "tri_material": np.ones(si.shape[0], np.uint32),
                   "uvs": suv, "tangents": tang})
    # box with per-face vertices (24) so every face has its own coordinates
    lo, hi = np.array([1.3, 0.0, -0.8]), np.array([2.3, 1.0, 0.2])
    bv, bi = box_mesh(lo, hi)
    verts, idx, uvs = [], [], []
    for t in bi:
        base = len(verts)
        for k in t:
            verts.append(bv[k])
        p0, p1, p2 = bv[t[0]], bv[t[1]], bv[t[2]]
        nrm = np.cross(p1 - p0, p2 - p0)
        ax = int(np.argmax(np.abs(nrm)))
        o = [d for d in range(3) if d != ax]
        for k in t:
            uvs.append([(bv[k][o[0]] - lo[o[0]]) / (hi[o[0]] - lo[o[0]]),
                        (bv[k][o[1]] - lo[o[1]]) / (hi[o[1]] - lo[o[1]])])
        idx.append([base, base + 1, base + 2])
    meshes.append({"verts": np.array(verts, np.float32), "idx": np.array(idx, np.uint32), "normals": None,
                   "tri_material": np.full(len(idx), 2, np.uint32), "uvs": np.array(uvs, np.float32)})
    ew, eh = env
    ey, ex = np.mgrid[0:eh, 0:ew]
    vv = (ey + 0.5) / eh
    sky = np.stack([0.3 + 0.7 * (1 - vv), 0.5 + 0.5 * (1 - vv), np.ones_like(vv)], -1) * 0.8
    sun = (np.abs(ex - ew * 0.3) < ew / 32) & (np.abs(ey - eh * 0.25) < eh / 16)
    sky[sun] = (40.0, 36.0, 30.0)
    lights = [("disk", 60.0, (1.0, 0.9, 0.8), (-2.0, 4.0, -1.0), (0.0, 0.0, 0.0), 0.4)]
    camera = ((0.5, 2.2, -5.5), (0.5, 0.8, 0.0), (0.0, 1.0, 0.0), math.radians(55.0))
    return {"meshes": meshes, "materials": materials, "lights": lights, "camera": camera,
            "background": (0.0, 0.0, 0.0), "textures": textures, "environment": sky.astype(np.float32)}


def load_scene(target, scene, width, height):
    """Loads a scene description into an alpine_b200 gpu.Context or an
    oracle RefRenderer (same method names)."""
    is_gpu = hasattr(target, "set_triangle_attributes")
    for t in scene.get("textures", ()):  # ids 0, 1, ... in order on both sides
        target.add_texture(t)
    if is_gpu:
        target.reset_scene()
        target.set_materials(scene["materials"])
    animated = False
    for m in scene["meshes"]:
        mo = m.get("morph")
        animated |= mo is not None
        if is_gpu:
            sid = target.add_mesh(m["verts"], m["idx"])
            target.set_triangle_attributes(sid, m["normals"], m["tri_material"])
            if m.get("uvs") is not None:
                target.set_triangle_uvs(sid, m["uvs"], m.get("tangents"))
            if mo is not None:
                target.set_morph_targets(sid, mo["deltas"], mo.get("normal_deltas"))
                target.add_animation_channel(sid, mo["times"], mo["weights"])
        elif mo is not None:
            target.add_morph_mesh(m["verts"], m["idx"], m["normals"], m["tri_material"], scene["materials"],
                                  mo["deltas"], mo.get("normal_deltas"), mo["times"], mo["weights"])
        else:
            target.add_mesh(m["verts"], m["idx"], m["normals"], m["tri_material"], scene["materials"],
                            uvs=m.get("uvs"), tangents=m.get("tangents"))
    if scene.get("environment") is not None:
        target.set_environment_map(scene["environment"])
    for l in scene["lights"]:
        if l[0] == "disk":
            target.add_disk_light(*l[1:])
        elif l[0] == "point":
            target.add_point_light(*l[1:])
        else:
            target.add_quad_light(*l[1:])
    eye, tgt, up, fovy = scene["camera"]
    target.set_camera(eye, tgt, up, fovy, width / height)
    target.set_background(*scene["background"])
    if animated:
        target.update_scene(scene.get("time", 0.0))  # Alpine::updateScene: animation, then the rebuild
    else:
        target.build()
