"""The learned coarse-grid stage on the GPU against the network oracle (oracle/cnn.py),
through the C-ABI, plus flexible GMRES with and without the stage.

Tolerances: the GPU sums in FP32 in a different order than the oracle's float64 sums, and
a different last bit before a BF16 rounding moves that activation by up to 2^-8, so
network outputs and gradients are compared in relative L2 norm: 1e-2 for outputs and
loss, 3e-2 per layer for gradients.  The Adam update is element-wise FP32 arithmetic and
is compared at 1e-5 relative.
"""
import ctypes as C

import numpy as np
import pytest

import cnn
import oracle
from parcel_b import _lib, api, problems

pytestmark = pytest.mark.gpu


def _params_flat(P):
    return np.concatenate([np.concatenate([W.reshape(-1), b.reshape(-1)]) for W, b in P]).astype(np.float32)


def _unflat(flat):
    out, o = [], 0
    for ci, co in cnn.layer_shapes():
        W = flat[o:o + 27 * ci * co].reshape(27, ci, co)
        o += 27 * ci * co
        b = flat[o:o + co]
        o += co
        out.append((W, b))
    return out


def _rand_params(seed):
    P = cnn.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    return [(W, (rng.standard_normal(b.shape) * 0.05).astype(np.float32)) for W, b in P]


class Net:
    """Thin test wrapper over the network entry points (coarsen = 1: u lives on the grid)."""

    def __init__(self, nx, ny, nz):
        self.L = _lib.load()
        h = C.c_void_p()
        assert self.L.parcel_b_learned_create(nx, ny, nz, 1, 0, C.byref(h)) == 0, _lib.last_error()
        self.h = h
        self.g = (nz, ny, nx)

    def set(self, P):
        flat = _params_flat(P)
        assert self.L.parcel_b_learned_set_params(self.h, flat.ctypes.data_as(C.c_void_p), 0.0) == 0

    def get(self):
        flat = np.zeros(self.L.parcel_b_learned_num_params(), np.float32)
        s = C.c_double()
        assert self.L.parcel_b_learned_get_params(self.h, flat.ctypes.data_as(C.c_void_p), C.byref(s)) == 0
        return flat

    def forward(self, u):
        B = u.shape[0]
        y = np.zeros((B,) + self.g, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        rc = self.L.parcel_b_learned_forward(self.h, B, u.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p))
        assert rc == 0, _lib.last_error()
        return y

    def grad(self, u, t):
        B = u.shape[0]
        u = np.ascontiguousarray(u, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.L.parcel_b_learned_num_params(), np.float32)
        loss = C.c_double()
        rc = self.L.parcel_b_learned_grad(self.h, B, u.ctypes.data_as(C.c_void_p), t.ctypes.data_as(C.c_void_p),
                                          C.byref(loss), g.ctypes.data_as(C.c_void_p))
        assert rc == 0, _lib.last_error()
        return loss.value, g

    def __del__(self):
        try:
            self.L.parcel_b_learned_destroy(self.h)
        except Exception:
            pass


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("grid,batch", [((12, 10, 9), 2), ((40, 9, 5), 1), ((64, 8, 4), 3)])
def test_forward_matches_oracle(grid, batch):
    nx, ny, nz = grid
    net = Net(nx, ny, nz)
    P = _rand_params(1)
    net.set(P)
    rng = np.random.default_rng(2)
    u = rng.standard_normal((batch, nz, ny, nx, 2)).astype(np.float32)
    y = net.forward(u)
    yo, _ = cnn.forward(P, u, emulate_bf16=True)
    assert _rel(y, yo) < 1e-2


def test_gradients_match_oracle():
    nx, ny, nz = 36, 6, 5
    net = Net(nx, ny, nz)
    P = _rand_params(3)
    net.set(P)
    rng = np.random.default_rng(4)
    u = rng.standard_normal((2, nz, ny, nx, 2)).astype(np.float32)
    t = rng.standard_normal((2, nz, ny, nx)).astype(np.float32)
    loss, g = net.grad(u, t)
    lo, go = cnn.loss_and_grads(P, u, t, emulate_bf16=True)
    assert abs(loss - lo) <= 1e-2 * lo
    for l, ((dW, db), (dWo, dbo)) in enumerate(zip(_unflat(g), go)):
        assert _rel(dW, dWo) < 3e-2, (l, _rel(dW, dWo))
        assert _rel(db, dbo) < 3e-2, (l, _rel(db, dbo))


def test_adam_step_matches_oracle():
    nx, ny, nz = 16, 6, 4
    net = Net(nx, ny, nz)
    P = _rand_params(5)
    net.set(P)
    rng = np.random.default_rng(6)
    u = rng.standard_normal((1, nz, ny, nx, 2)).astype(np.float32)
    t = rng.standard_normal((1, nz, ny, nx)).astype(np.float32)
    state = cnn.adam_state(P)
    cur = P
    for _ in range(3):
        _, g = net.grad(u, t)
        assert net.L.parcel_b_learned_adam(net.h, 1e-3) == 0
        cur = cnn.adam_step(cur, _unflat(g), state, 1e-3)
        assert _rel(net.get(), _params_flat(cur)) < 1e-5


def _vardiff(N, seed):
    g = problems.gaussian_random_field(N, corr_len=N / 8.0, variance=2.0, seed=seed)
    return problems.vardiff3d(N, np.exp(g))


def _prm(**kw):
    d = dict(solver=3, ipreflag=2, ILU_method=0, precon_thblock=8, GMRES_m=30, itrmax=3000, rtolmax=1e-10)
    d.update(kw)
    return d


def test_fgmres_without_stage_matches_gmres_oracle():
    """Flexible GMRES with a fixed preconditioner is right-preconditioned GMRES."""
    A = _vardiff(16, 7)
    b = problems.rhs_normal(A.n, 8)
    res = api.solve_learned(A, b, None, **_prm())
    xo, ho, no, io = oracle.solve(A, b, **_prm())
    assert res["iret"] == 0 and io == 0
    assert abs(res["niter"] - no) <= 2
    k = min(len(ho), len(res["reshistory"]))
    m = ho[:k] > 1e-8
    assert np.max(np.abs(res["reshistory"][:k][m] - ho[:k][m]) / ho[:k][m]) < 1e-6
    assert oracle.true_relres(A, b, res["x"]) < 1e-10


def _vardiff8(N, seed):
    """The learned-stage benchmark's coefficient field (correlation length 8 cells)."""
    g = problems.gaussian_random_field(N, corr_len=8.0, variance=2.0, seed=seed)
    return problems.vardiff3d(N, np.exp(g))


def test_two_level_stage_and_network_ablation():
    """Ablation on the 128^3 variable-coefficient problem (coarse grid 16^3), FP32 FGMRES(40)
    inside FP64 refinement, BJ-ILU(0) 64 blocks, to an FP64 true residual of 1e-10:
      (a) no stage;  (b) Galerkin coarse stage, k coarse PCG steps from zero;
      (c) the same stage started from the trained network's guess.
    The coarse stage must cut the iterations at least fivefold; with one coarse PCG step
    the network's guess must save at least 10 % of the stage's iterations, with two steps
    it must not cost any (the network is trained on residual / coarse-error pairs from
    plain solves with other right-hand sides)."""
    N, c = 128, 8
    A = _vardiff8(N, 5)
    prm = _prm(precon_thblock=64, GMRES_m=40, itrmax=20000, inner_precision=1, inner_rtol=1e-4, max_refine=80)
    net = api.Learned(N, N, N, c, seed=1)
    for s in (100, 101):
        net.collect(A, problems.rhs_normal(A.n, s), max_pairs=64, **_prm(precon_thblock=64, GMRES_m=40,
                                                                        itrmax=20000))
    assert net.num_pairs() >= 16
    first, last = net.train(steps=400, batch=4, lr=2e-3, seed=3)
    assert last < 0.1 * first, (first, last)
    b = problems.rhs_normal(A.n, 1000)
    runs = {}
    base = api.solve_learned(A, b, None, **prm)
    for k in (1, 2):
        for use_net in (0, 1):
            net.set_stage(k, use_net)
            runs[k, use_net] = api.solve_learned(A, b, net, **prm)
    for r in [base] + list(runs.values()):
        assert r["iret"] == 0 and r["stats"]["fallback"] == 0, r["stats"]
        assert oracle.true_relres(A, b, r["x"]) < 1e-10
    its = {key: r["niter"] for key, r in runs.items()}
    assert its[2, 0] * 5 <= base["niter"], (its, base["niter"])
    assert its[1, 1] <= 0.9 * its[1, 0], its
    assert its[2, 1] <= its[2, 0], its


def test_learned_mixed_precision_reaches_tolerance():
    N, c = 32, 4
    A = _vardiff(N, 9)
    net = api.Learned(N, N, N, c, seed=2)
    net.collect(A, problems.rhs_normal(A.n, 31), max_pairs=16, **_prm())
    net.train(steps=100, batch=4, lr=2e-3, seed=4)
    b = problems.rhs_normal(A.n, 32)
    res = api.solve_learned(A, b, net, inner_precision=1, inner_rtol=1e-4, max_refine=40, **_prm())
    assert res["iret"] == 0, res["stats"]
    assert oracle.true_relres(A, b, res["x"]) < 1e-10
