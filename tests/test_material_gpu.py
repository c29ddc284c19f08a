"""GPU tests of the materials against the reference's Material classes.

* Material::sample, computeBsdf and computePdf on fixed (wo, u) and (wo, wi)
  grids against the reference (oracle/_ref: src/materials/*.cpp compiled with
  FP contraction off; the GPU probes are compiled the same way). Differences
  come only from libm vs CUDA ulp differences in cos, sin and pow.
* The true density p and effective integrand f of Material::sample's output
  direction (used for one-sample MIS with the learned guide) are checked with
  the two identities unbiasedness rests on, for samples drawn by the GPU's own
  Material::sample:
      E_{wi ~ sample}[h(wi) / p(wi)]  = integral of h over {p > 0}
      E_{wi ~ sample}[estimator h(wi)] = integral of f h
  with the right sides estimated by uniform hemisphere sampling.
"""
import math

import numpy as np
import pytest

import oracle
from alpine_b200 import gpu

pytestmark = pytest.mark.gpu

MATERIALS = [
    (1, (0.95, 0.75, 0.45), 0.3),   # GGX conductor
    (1, (0.9, 0.9, 0.9), 0.05),     # glossy conductor
    (1, (0.6, 0.8, 0.9), 0.6),      # rough conductor
    (0, (0.7, 0.4, 0.2), 0.3),      # dielectric: Lambertian + GGX (F0 0.04)
    (0, (0.5, 0.6, 0.7), 0.02),     # dielectric, near-specular coat
    (0, (0.5, 0.5, 0.5), 1.0),      # dielectric: Lambertian only
]


@pytest.fixture(scope="module")
def ctx():
    c = gpu.Context(0, 16, 16, 4)
    yield c
    c.close()


def _wo_grid(n_theta=9, n_phi=8):
    out = []
    for i in range(n_theta):
        ct = 0.02 + 0.98 * (i + 0.5) / n_theta
        st = math.sqrt(1 - ct * ct)
        for j in range(n_phi):
            ph = 2 * math.pi * (j + 0.25) / n_phi
            out.append((st * math.cos(ph), st * math.sin(ph), ct))
    out.append((0.3, 0.2, -0.5))  # below the surface: every sample is rejected or reflected
    return np.array(out, np.float32)


def _u_grid(n=48):
    g = (np.arange(n, dtype=np.float32) + 0.5) / n
    u0, u1 = np.meshgrid(g, g, indexing="ij")
    return np.stack([u0.ravel(), u1.ravel()], -1)


@pytest.mark.parametrize("mat", MATERIALS)
def test_sample_matches_reference(ctx, mat):
    wo = _wo_grid()
    u = _u_grid()
    W = np.repeat(wo, u.shape[0], 0)
    U = np.tile(u, (wo.shape[0], 1))
    gwi, gest, gpdf, gok = ctx.material_sample(mat, W, U)
    rwi, rest, rpdf, rok = oracle.ref_material_sample(mat, W, U)
    same_ok = (gok == rok).mean()
    both = gok & rok
    dwi = np.abs(gwi[both] - rwi[both]).max()
    rel_est = (np.abs(gest[both] - rest[both]) / np.maximum(np.abs(rest[both]), 1e-6)).max(-1)
    rel_pdf = np.abs(gpdf[both] - rpdf[both]) / np.maximum(rpdf[both], 1e-6)
    print(f"{mat}: ok agree {same_ok:.6f}, max |dwi| {dwi:.2e}, est rel p99.9 {np.quantile(rel_est, 0.999):.2e}, "
          f"pdf rel p99.9 {np.quantile(rel_pdf, 0.999):.2e}")
    assert same_ok > 0.999
    assert dwi < 1e-4
    assert np.quantile(rel_est, 0.999) < 1e-3 and np.quantile(rel_pdf, 0.999) < 1e-3
    assert (rel_est < 1e-5).mean() > 0.99 and (rel_pdf < 1e-5).mean() > 0.99


@pytest.mark.parametrize("mat", MATERIALS)
def test_eval_matches_reference(ctx, mat):
    rng = np.random.default_rng(3)
    n = 1 << 15
    wo = rng.normal(size=(n, 3)).astype(np.float32)
    wi = rng.normal(size=(n, 3)).astype(np.float32)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    wo[: n // 2, 2] = np.abs(wo[: n // 2, 2])
    wi[: n // 2, 2] = np.abs(wi[: n // 2, 2])
    gb, gp, _, _ = ctx.material_eval(mat, wo, wi)
    rb, rp = oracle.ref_material_eval(mat, wo, wi)
    rel_b = (np.abs(gb - rb) / np.maximum(np.abs(rb), 1e-6)).max(-1)
    rel_p = np.abs(gp - rp) / np.maximum(np.abs(rp), 1e-6)
    print(f"{mat}: bsdf rel max {rel_b.max():.2e}, pdf rel max {rel_p.max():.2e}")
    assert np.quantile(rel_b, 0.999) < 1e-4 and np.quantile(rel_p, 0.999) < 1e-4


def _uniform_hemisphere(n, rng):
    z = rng.random(n)
    ph = 2 * math.pi * rng.random(n)
    s = np.sqrt(np.maximum(0.0, 1 - z * z))
    return np.stack([s * np.cos(ph), s * np.sin(ph), z], -1).astype(np.float32)


def _mean_se(x):
    x = np.asarray(x, np.float64)
    return x.mean(0), x.std(0, ddof=1) / math.sqrt(x.shape[0])


@pytest.mark.parametrize("mat", MATERIALS[:1] + MATERIALS[2:4] + MATERIALS[5:])
@pytest.mark.parametrize("wo", [(0.0, 0.0, 1.0), (0.6, 0.3, 0.5), (-0.2, 0.9, 0.25), (0.95, 0.0, 0.12)])
def test_sampling_density_and_integrand(ctx, mat, wo):
    rng = np.random.default_rng(11)
    n = 1 << 21
    wo = np.array(wo, np.float32)
    wo /= np.linalg.norm(wo)
    W = np.repeat(wo[None], n, 0)
    wi, est, _, ok = ctx.material_sample(mat, W, rng.random((n, 2), dtype=np.float32))
    _, _, dens, _ = ctx.material_eval(mat, W[ok], wi[ok])
    assert (dens > 0).all(), "a sampled direction has zero density"
    h = lambda d: 1.0 + 2.0 * d[:, 2] ** 2 + d[:, 0]  # positive test function
    # importance-sampling side
    lhs_a = np.zeros(n)
    lhs_a[ok] = h(wi[ok]) / dens
    lhs_f = np.zeros((n, 3))
    lhs_f[ok] = est[ok] * h(wi[ok])[:, None]
    # uniform hemisphere side
    m = 1 << 22
    du = _uniform_hemisphere(m, rng)
    _, _, pu, fu = ctx.material_eval(mat, np.repeat(wo[None], m, 0), du)
    rhs_a = 2 * math.pi * h(du) * (pu > 0)
    rhs_f = 2 * math.pi * fu * h(du)[:, None]
    for name, l, r in (("support", lhs_a, rhs_a), ("integrand", lhs_f, rhs_f)):
        ml, sl = _mean_se(l)
        mr, sr = _mean_se(r)
        z = np.abs(ml - mr) / np.sqrt(sl ** 2 + sr ** 2 + 1e-30)
        print(f"{mat} wo={wo}: {name} sampled {ml} uniform {mr} z {z}")
        assert np.all(z < 5.0), name
