"""CPU test pinning the morph-animation semantics the GPU restates
(csrc/animation.cu): a float32 numpy restatement of Animation::update
(src/animation.cpp:10-39: clamp the time to the keyframe range, find the
segment, std::lerp the weights) and Mesh::update (src/shapes/mesh.cpp:29-55:
v = base, then v += target_j * w_j in order) equals the reference's own code
(oracle/_ref) bit for bit."""
import numpy as np
import pytest

import oracle
from alpine_b200 import scenes

f32 = np.float32


def lerp_c20(a, b, t):
    """std::lerp (C++20, P0811R3) in the form the GNU C++ library evaluates it."""
    a, b, t = f32(a), f32(b), f32(t)
    if (a <= 0 and b >= 0) or (a >= 0 and b <= 0):
        return f32(f32(t * b) + f32(f32(f32(1) - t) * a))
    if t == f32(1):
        return b
    x = f32(a + f32(t * f32(b - a)))
    if (t > 1) == (b > a):
        return x if b < x else b
    return x if b > x else b


def channel_weights(times, weights, time):
    times = np.asarray(times, f32)
    ct = f32(min(max(f32(time), times[0]), times[-1]))
    k = len(times)
    index = k - 2
    for i in range(k - 1):
        if ct <= times[i + 1]:
            index = i
            break
    t = f32(f32(ct - times[index]) / f32(times[index + 1] - times[index]))
    return np.array([lerp_c20(weights[index][j], weights[index + 1][j], t) for j in range(len(weights[0]))], f32)


def morph(base, deltas, w):
    v = np.array(base, f32)
    for j in range(deltas.shape[0]):
        v = (v + (deltas[j] * w[j]).astype(f32)).astype(f32)
    return v


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("offset", [-1.0, 0.0, 0.37, 1.0, 2.5, 100.0])
def test_restated_morph_matches_reference(offset):
    v, t, _ = scenes.uv_sphere((0.1, -0.2, 0.3), 0.7, 16, 8)
    rng = np.random.default_rng(5)
    deltas = rng.normal(0, 0.05, (3, v.shape[0], 3)).astype(f32)
    times = np.cumsum(rng.uniform(0.2, 1.0, 5)).astype(f32)
    weights = rng.uniform(-1.5, 1.5, (5, 3)).astype(f32)
    weights[1, 0] = 0.0
    weights[2, 1] = weights[3, 1]  # a flat segment
    time = f32(times[1] + offset * (times[2] - times[1]))
    ref = oracle.ref_morph_vertices(v, t, deltas, times, weights, time)
    mine = morph(v, deltas, channel_weights(times, weights, time))
    assert mine.view(np.uint32).tolist() == ref.view(np.uint32).tolist()
