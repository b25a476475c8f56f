"""CPU oracle of the learned coarse-grid preconditioner stage (TEST INFRASTRUCTURE ONLY).

Imported by tests/ as the checker of the GPU network kernels, never by the product.

The reference has no learned component, so nothing in PARCEL pins this code; it is pinned
instead by central finite differences of its own loss in float64 (tests/test_cnn_oracle.py).
With ``emulate_bf16=True`` it rounds to bfloat16 (round to nearest even) exactly where the
GPU kernels store bfloat16: the network input, the weights of every layer, the hidden
activations after ReLU, and the activation gradients between layers.  Sums are float64
here and float32 on the GPU, so the comparison is made with a stated tolerance.

Network (channels last, arrays [B, Z, Y, X, C]; zero padding at the grid boundary):
    a0 = [t/sigma, dhat]                          2 input channels
    a1 = relu(conv3(a0, W1) + b1)                 2 -> 32
    a2..a5 = relu(conv3(a_{l-1}, W_l) + b_l)      32 -> 32 (four layers)
    y  = conv3(a5, W6) + b6                       32 -> 1
W_l has shape [27, C_in, C_out] with tap index t = 9 (dz+1) + 3 (dy+1) + (dx+1):
    conv3(a, W)[z, y, x, co] = sum_t sum_ci a[z+dz, y+dy, x+dx, ci] W[t, ci, co].
Loss: L = 1/(2M) sum (y - y*)^2 over the M = B Z Y X output voxels.

Coarse-grid transfer of the preconditioner stage: restrict() is the mean over each
c x c x c block of fine cells; prolong() is cell-centred trilinear interpolation with
clamping at the boundary.
"""
from __future__ import annotations

import numpy as np

CIN = 2
CH = 32
NLAYER = 6


def layer_shapes():
    """(C_in, C_out) of the six layers."""
    return [(CIN, CH)] + [(CH, CH)] * 4 + [(CH, 1)]


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def init_params(seed: int = 0):
    """He-normal weights (float32), zero biases."""
    rng = np.random.default_rng(seed)
    P = []
    for ci, co in layer_shapes():
        W = (rng.standard_normal((27, ci, co)) * np.sqrt(2.0 / (27 * ci))).astype(np.float32)
        P.append((W, np.zeros(co, np.float32)))
    return P


def _taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def conv3(a, W):
    """conv3(a, W) without bias; float64 sums."""
    B, Z, Y, X, _ = a.shape
    ap = np.pad(a.astype(np.float64), ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, Z, Y, X, W.shape[2]))
    for t, dz, dy, dx in _taps():
        out += ap[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X, :] @ W[t].astype(np.float64)
    return out


def conv3_transpose(g, W):
    """Adjoint of conv3 in its input: out[u, ci] = sum_t sum_co W[t, ci, co] g[u - d_t, co]."""
    Wt = np.ascontiguousarray(W[::-1].transpose(0, 2, 1))
    return conv3(g, Wt)


def wgrad(a, g):
    """dW[t, ci, co] = sum_v a[v + d_t, ci] g[v, co]; float64."""
    B, Z, Y, X, Ci = a.shape
    ap = np.pad(a.astype(np.float64), ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    g2 = g.astype(np.float64).reshape(-1, g.shape[-1])
    dW = np.zeros((27, Ci, g.shape[-1]))
    for t, dz, dy, dx in _taps():
        sh = ap[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X, :].reshape(-1, Ci)
        dW[t] = sh.T @ g2
    return dW


def forward(params, u, emulate_bf16=True):
    """Returns (y [B,Z,Y,X], activations [a0..a5])."""
    if emulate_bf16:
        a = bf16(np.asarray(u, np.float32))
    else:
        a = np.asarray(u, np.float64)
    acts = [a]
    y = None
    for l, (W, b) in enumerate(params):
        z = conv3(a, bf16(W) if emulate_bf16 else W) + b
        if l < NLAYER - 1:
            a = bf16(np.maximum(z, 0.0).astype(np.float32)) if emulate_bf16 else np.maximum(z, 0.0)
            acts.append(a)
        else:
            y = z[..., 0]
    return y, acts


def loss_and_grads(params, u, target, emulate_bf16=True):
    """Loss and gradients [(dW, db)] of L = 1/(2M) sum (y - target)^2."""
    y, acts = forward(params, u, emulate_bf16)
    M = y.size
    diff = y - target
    L = 0.5 * float((diff.astype(np.float64) ** 2).sum()) / M
    g = (diff / M)[..., None]
    if emulate_bf16:
        g = g.astype(np.float32)
    grads = [None] * NLAYER
    for l in range(NLAYER - 1, -1, -1):
        W = params[l][0]
        Wq = bf16(W) if emulate_bf16 else W
        a_in = acts[l]
        grads[l] = (wgrad(a_in, g), g.astype(np.float64).sum(axis=(0, 1, 2, 3)))
        if l > 0:
            gi = conv3_transpose(g, Wq) * (a_in > 0)
            g = bf16(gi.astype(np.float32)) if emulate_bf16 else gi
    return L, grads


def adam_state(params):
    z = []
    for W, b in params:
        z += [np.zeros_like(W), np.zeros_like(b)]
    return {"t": 0, "m": [x.copy() for x in z], "v": [x.copy() for x in z]}


def adam_step(params, grads, state, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step on float32 master weights (state from adam_state)."""
    state["t"] += 1
    t = state["t"]
    c1 = np.float32(1.0 - beta1 ** t)
    c2 = np.float32(1.0 - beta2 ** t)
    b1, b2 = np.float32(beta1), np.float32(beta2)
    out = []
    for i, ((W, b), (dW, db)) in enumerate(zip(params, grads)):
        newp = []
        for j, (p, g) in enumerate(((W, dW), (b, db))):
            k = 2 * i + j
            g = np.asarray(g, np.float32)
            state["m"][k] = b1 * state["m"][k] + (np.float32(1) - b1) * g
            state["v"][k] = b2 * state["v"][k] + (np.float32(1) - b2) * g * g
            mh = state["m"][k] / c1
            vh = state["v"][k] / c2
            newp.append((p - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))).astype(np.float32))
        out.append(tuple(newp))
    return out


def restrict(f, c):
    """Mean over c^3 blocks of a fine field f[Z, Y, X] (dims divisible by c)."""
    Z, Y, X = f.shape
    return f.reshape(Z // c, c, Y // c, c, X // c, c).mean(axis=(1, 3, 5))


def prolong(yc, c):
    """Cell-centred trilinear interpolation of a coarse field yc[Gz, Gy, Gx] to the fine
    grid (c Gz, c Gy, c Gx), clamping the stencil at the boundary."""
    out = yc.astype(np.float64)
    for axis in range(3):
        G = out.shape[axis]
        i = np.arange(G * c)
        xi = (i + 0.5) / c - 0.5
        i0 = np.floor(xi).astype(int)
        w = xi - i0
        lo = np.clip(i0, 0, G - 1)
        hi = np.clip(i0 + 1, 0, G - 1)
        a = np.take(out, lo, axis=axis)
        b = np.take(out, hi, axis=axis)
        shape = [1, 1, 1]
        shape[axis] = G * c
        w = w.reshape(shape)
        out = a * (1 - w) + b * w
    return out
