"""Test infrastructure (oracle): FP64 numpy restatement of the learned guide
(hash-grid encoding, MLP, 8-lobe vMF mixture, the KL training loss and its
analytic gradient), used to check the GPU's BF16 tensor-core inference and
training kernels. No counterpart in the reference. Published methods
restated: hash-grid encoding (Mueller et al., Instant NGP, SIGGRAPH 2022),
vMF mixture density, and the KL-divergence gradient -(L/p) grad log q of
Neural Importance Sampling (Mueller et al., TOG 2019).
"""
from __future__ import annotations

import numpy as np

LEVELS, FEAT, T_LOG2 = 8, 4, 19
T = 1 << T_LOG2
GRID_DIMS = LEVELS * FEAT
IN, HID, OUT, LOBES, LAYERS = 64, 64, 48, 8, 5
MIN_RES, MAX_RES = 16, 2048
LOGK_MIN, LOGK_MAX = -2.0, 8.0


def layer_in(l):
    return IN if l == 0 else HID


def layer_out(l):
    return OUT if l == LAYERS - 1 else HID


def layer_offset(l):
    return sum(layer_out(i) * layer_in(i) for i in range(l))


WEIGHT_COUNT = layer_offset(LAYERS)


def resolutions():
    b = np.exp((np.log(float(MAX_RES)) - np.log(float(MIN_RES))) / (LEVELS - 1))
    return [int(np.floor(MIN_RES * b ** l)) for l in range(LEVELS)]


def unpack(w):
    return [np.asarray(w[layer_offset(l):layer_offset(l + 1)], np.float64).reshape(layer_out(l), layer_in(l))
            for l in range(LAYERS)]


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.ascontiguousarray(x, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def normalise(pos, lo, hi):
    lo = np.asarray(lo, np.float32)
    e = np.asarray(hi, np.float32) - lo
    m = np.float32(max(float(e.max()), 0.0)) * np.float32(1.0001) if e.max() > 0 else np.float32(1.0)
    inv = np.float32(1.0) / m
    q = (np.asarray(pos, np.float32) - lo) * inv
    return np.clip(q, np.float32(0.0), np.float32(0.99999)).astype(np.float32)


def grid_index(res, x, y, z):
    dense = (res + 1) ** 3
    if dense <= T:
        return (x + (res + 1) * (y + (res + 1) * z)).astype(np.uint64)
    h = (x.astype(np.uint64) * np.uint64(1)) ^ ((y.astype(np.uint64) * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) \
        ^ ((z.astype(np.uint64) * np.uint64(805459861)) & np.uint64(0xFFFFFFFF))
    return h & np.uint64(T - 1)


def corners(p32, res):
    """(indices (n, 8), weights (n, 8)) of the grid cell at one level, in the
    GPU's FP32 arithmetic."""
    f = p32 * np.float32(res)
    i = np.floor(f)
    t = (f - i).astype(np.float32)
    i = i.astype(np.int64)
    idx = np.empty((p32.shape[0], 8), np.uint64)
    w = np.empty((p32.shape[0], 8), np.float64)
    for c in range(8):
        ox, oy, oz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        idx[:, c] = grid_index(res, i[:, 0] + ox, i[:, 1] + oy, i[:, 2] + oz)
        wx = t[:, 0] if ox else np.float32(1) - t[:, 0]
        wy = t[:, 1] if oy else np.float32(1) - t[:, 1]
        wz = t[:, 2] if oz else np.float32(1) - t[:, 2]
        w[:, c] = (wx * wy * wz).astype(np.float32)
    return idx, w


def grid_flat_indices(queries, lo, hi, res):
    """Flat parameter indices ((level*T + entry)*2 + feature) touched by the queries."""
    p = normalise(np.asarray(queries)[:, 0:3], lo, hi)
    out = []
    for l in range(LEVELS):
        idx, _ = corners(p, res[l])
        base = (np.uint64(l) * np.uint64(T) + idx) * np.uint64(FEAT)
        out += [(base + np.uint64(f)).reshape(-1) for f in range(FEAT)]
    return np.unique(np.concatenate(out))


def fma32(a, b, c):
    """FP32 fused multiply-add of FP32 arrays, through FP64: a * b is exact
    there for the encoding's operands (a 24-bit weight times an 11-bit FP16
    value), and the sum is rounded once to FP32 (twice only when the
    exponents of the product and c differ by more than 18)."""
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64) + np.asarray(c, np.float64)).astype(np.float32)


def encode(queries, lo, hi, res, grid_lookup, half=True):
    """Inputs (n, 64). grid_lookup(flat_indices) -> fp32 parameter values.
    half=True reproduces the GPU's encoding: FP16 grid values, each feature
    summed over the 8 corners in corner order by FP32 fused multiply-adds
    (src: alpine_b200/csrc/guide.cu, encode_row), so that the BF16 rounding
    of an input that lands near a rounding boundary goes the same way.
    half=False sums the FP32 values in FP64."""
    q = np.asarray(queries, np.float64)
    p = normalise(q[:, 0:3], lo, hi)
    n = q.shape[0]
    X = np.zeros((n, IN))
    for l in range(LEVELS):
        idx, w = corners(p, res[l])
        base = (np.uint64(l) * np.uint64(T) + idx) * np.uint64(FEAT)
        for f in range(FEAT):
            v = np.asarray(grid_lookup((base + np.uint64(f)).reshape(-1)), np.float64).reshape(n, 8)
            if half:
                v = v.astype(np.float16).astype(np.float32)
                acc = np.zeros(n, np.float32)
                for c in range(8):
                    acc = fma32(w[:, c], v[:, c], acc)
                X[:, FEAT * l + f] = acc
            else:
                X[:, FEAT * l + f] = (w * v).sum(1)
    nrm = q[:, 8:11]
    nl = np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = np.where(nl > 0, nrm / np.maximum(nl, 1e-30), np.array([0, 0, 1.0]))
    X[:, 32:35] = q[:, 4:7]
    X[:, 35:38] = nrm
    X[:, 38] = q[:, 3]
    X[:, 39] = 1.0
    return X


def forward(X, Ws, emulate_bf16=False):
    """Returns (raw outputs (n, 48), list of layer inputs)."""
    acts = []
    h = bf16(X) if emulate_bf16 else X
    Wq = [bf16(W) for W in Ws] if emulate_bf16 else Ws
    for l in range(LAYERS):
        acts.append(h)
        y = h @ Wq[l].T
        if l < LAYERS - 1:
            h = np.maximum(y, 0.0)
            if emulate_bf16:
                h = bf16(h)
        else:
            return y, acts


def decode(raw):
    r = np.asarray(raw, np.float64)[:, :40].reshape(-1, LOBES, 5)
    d = r[..., 0:3]
    l = np.linalg.norm(d, axis=-1, keepdims=True)
    mu = np.where(l > 1e-12, d / np.maximum(l, 1e-300), np.array([0, 0, 1.0]))
    s = np.clip(r[..., 3], LOGK_MIN, LOGK_MAX)
    kappa = np.exp(s)
    a = r[..., 4]
    lam = np.exp(a - a.max(-1, keepdims=True))
    lam /= lam.sum(-1, keepdims=True)
    return mu, kappa, lam


def vmf(mu, kappa, w):
    return kappa / (2 * np.pi * -np.expm1(-2 * kappa)) * np.exp(kappa * ((mu * w[:, None, :]).sum(-1) - 1))


def mixture_pdf(raw, w):
    mu, kappa, lam = decode(raw)
    return (lam * vmf(mu, kappa, np.asarray(w, np.float64))).sum(-1)


def loss(raw, w, weight):
    return float(-(np.asarray(weight) * np.log(np.maximum(mixture_pdf(raw, w), 1e-300))).sum())


def output_grad(raw, w, weight):
    """d loss / d raw (n, 48) for loss = -sum_i weight_i log q(w_i)."""
    raw = np.asarray(raw, np.float64)
    w = np.asarray(w, np.float64)
    mu, kappa, lam = decode(raw)
    v = vmf(mu, kappa, w)
    q = np.maximum((lam * v).sum(-1, keepdims=True), 1e-300)
    resp = lam * v / q
    wt = np.asarray(weight, np.float64)[:, None]
    g = np.zeros((raw.shape[0], OUT))
    gl = g[:, :40].reshape(-1, LOBES, 5)
    gl[..., 4] = -wt * (resp - lam)
    s = raw[:, :40].reshape(-1, LOBES, 5)[..., 3]
    dk = 1 / kappa - 2 / np.expm1(2 * kappa) + ((mu * w[:, None, :]).sum(-1) - 1)
    inside = (s > LOGK_MIN) & (s < LOGK_MAX)
    gl[..., 3] = np.where(inside, -wt * resp * dk * kappa, 0.0)
    d = raw[:, :40].reshape(-1, LOBES, 5)[..., 0:3]
    l = np.linalg.norm(d, axis=-1, keepdims=True)
    mw = (mu * w[:, None, :]).sum(-1, keepdims=True)
    gd = (w[:, None, :] - mw * mu) * (kappa[..., None] / np.maximum(l, 1e-300))
    gl[..., 0:3] = -wt[..., None] * resp[..., None] * gd
    g[:, :40] = gl.reshape(-1, 40)
    return g


def backward(acts, Ws, gout):
    """dW per layer and d loss / d input (n, 64)."""
    dWs = [None] * LAYERS
    dy = gout
    for l in range(LAYERS - 1, -1, -1):
        dWs[l] = dy.T @ acts[l]
        dx = dy @ Ws[l]
        if l > 0:
            dy = dx * (acts[l] > 0)
        else:
            return dWs, dx
