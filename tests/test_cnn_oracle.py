"""Pins the network oracle (oracle/cnn.py): float64 gradients against central finite
differences of its own loss, the adjoint identity of its transposed convolution, and the
coarse-grid transfer operators.  CPU only."""
import numpy as np
import pytest

import cnn


def _params64(seed):
    P = cnn.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    return [(W.astype(np.float64), (rng.standard_normal(b.shape) * 0.1)) for W, b in P]


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], np.float32)
    r = cnn.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # tie -> even mantissa (down)
    assert r[2] == 1.0 + 4 * 2 ** -8         # tie -> even mantissa (up)
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert (cnn.bf16(r) == r).all()


def test_transpose_is_adjoint():
    rng = np.random.default_rng(3)
    a = rng.standard_normal((2, 4, 5, 3, 7))
    g = rng.standard_normal((2, 4, 5, 3, 6))
    W = rng.standard_normal((27, 7, 6))
    lhs = (cnn.conv3(a, W) * g).sum()
    rhs = (a * cnn.conv3_transpose(g, W)).sum()
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_wgrad_matches_directional_derivative():
    rng = np.random.default_rng(4)
    a = rng.standard_normal((1, 3, 4, 5, 3))
    g = rng.standard_normal((1, 3, 4, 5, 2))
    dW = rng.standard_normal((27, 3, 2))
    lhs = (cnn.conv3(a, dW) * g).sum()
    assert abs(lhs - (cnn.wgrad(a, g) * dW).sum()) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("layer", [0, 2, 5])
def test_gradients_against_finite_differences(layer):
    P = _params64(11)
    rng = np.random.default_rng(12)
    u = rng.standard_normal((2, 3, 4, 5, cnn.CIN))
    target = rng.standard_normal((2, 3, 4, 5))
    L0, grads = cnn.loss_and_grads(P, u, target, emulate_bf16=False)
    dW, db = grads[layer]
    h = 1e-6
    idx = [tuple(int(rng.integers(0, s)) for s in P[layer][0].shape) for _ in range(6)]
    for ix in idx:
        Wp = [(W.copy(), b.copy()) for W, b in P]
        Wm = [(W.copy(), b.copy()) for W, b in P]
        Wp[layer][0][ix] += h
        Wm[layer][0][ix] -= h
        fd = (cnn.loss_and_grads(Wp, u, target, False)[0] - cnn.loss_and_grads(Wm, u, target, False)[0]) / (2 * h)
        assert abs(fd - dW[ix]) <= 1e-6 * max(abs(fd), 1e-8) + 1e-10, (ix, fd, dW[ix])
    j = int(rng.integers(0, P[layer][1].shape[0]))
    Bp = [(W.copy(), b.copy()) for W, b in P]
    Bm = [(W.copy(), b.copy()) for W, b in P]
    Bp[layer][1][j] += h
    Bm[layer][1][j] -= h
    fd = (cnn.loss_and_grads(Bp, u, target, False)[0] - cnn.loss_and_grads(Bm, u, target, False)[0]) / (2 * h)
    assert abs(fd - db[j]) <= 1e-6 * max(abs(fd), 1e-8) + 1e-10


def test_bf16_emulation_close_to_float64():
    P = cnn.init_params(5)
    rng = np.random.default_rng(6)
    u = rng.standard_normal((1, 6, 6, 6, cnn.CIN)).astype(np.float32)
    y64, _ = cnn.forward(P, u, emulate_bf16=False)
    y16, _ = cnn.forward(P, u, emulate_bf16=True)
    assert np.linalg.norm(y16 - y64) <= 3e-2 * np.linalg.norm(y64)


def test_restrict_prolong():
    rng = np.random.default_rng(7)
    f = rng.standard_normal((8, 12, 4))
    r = cnn.restrict(f, 4)
    assert r.shape == (2, 3, 1)
    assert np.isclose(r[1, 2, 0], f[4:8, 8:12, 0:4].mean())
    # trilinear prolongation reproduces fields linear in the (clamped) cell centres
    zc, yc, xc = np.meshgrid(np.arange(3), np.arange(4), np.arange(5), indexing="ij")
    lin = 1.0 + 0.5 * zc - 0.25 * yc + 2.0 * xc
    p = cnn.prolong(lin, 2)
    zf, yf, xf = np.meshgrid(*(np.clip((np.arange(2 * G) + 0.5) / 2 - 0.5, 0, G - 1) for G in (3, 4, 5)),
                             indexing="ij")
    assert np.allclose(p, 1.0 + 0.5 * zf - 0.25 * yf + 2.0 * xf)
    assert np.allclose(cnn.prolong(np.ones((2, 2, 2)), 4), 1.0)
