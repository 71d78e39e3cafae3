"""Host logic of the friction assimilation front-end (no GPU): control transforms, the
penalties' gradients, zonation, the minimisers and the descent log, on a stand-in model whose J
is a known quadratic of the friction map (its gradient is exact)."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from tests.conftest import load_pkg

pkg = load_pkg()
A = pkg.assimilation


class QuadraticModel:
    """J(k) = sum w (k1 - k*)^2 + sum w (k2 - k*)^2, with the SpModel methods the problem uses."""

    def __init__(self, n=40, seed=0):
        rng = np.random.default_rng(seed)
        self.n = n
        self.w = rng.uniform(0.5, 2.0, n)
        self.k_true = rng.uniform(0.02, 0.05, n)
        self.k1 = np.full(n, 0.03)
        self.k2 = np.full(n, 0.03)
        L = np.arange(n - 1)
        self.case = SimpleNamespace(mesh=SimpleNamespace(edge_int_cells=np.stack([L, L + 1], axis=1)))
        self.rerecords = 0

    def set_param(self, name, v):
        v = np.broadcast_to(np.asarray(v, dtype=np.float64), (self.n,)).copy()
        if name in ("friction", "friction_1"):
            self.k1 = v.copy()
        if name in ("friction", "friction_2"):
            self.k2 = v.copy()

    def replay_cost(self):
        return float(np.sum(self.w * (self.k1 - self.k_true) ** 2) + np.sum(self.w * (self.k2 - self.k_true) ** 2))

    def rerecord(self):
        self.rerecords += 1
        return 10

    def adjoint(self, wrt=("friction_1", "friction_2")):
        g = {"friction_1": 2 * self.w * (self.k1 - self.k_true), "friction_2": 2 * self.w * (self.k2 - self.k_true)}
        return self.replay_cost(), {k: g[k] for k in wrt}


@pytest.mark.parametrize("mode", ["none", "clamp", "tanh"])
def test_transform_derivative_and_inverse(mode):
    T = A.ControlTransform(mode, lo=0.01, hi=0.1, lam=30.0)
    m = T.inverse(np.linspace(0.015, 0.095, 9))
    assert np.allclose(T.forward(m), np.linspace(0.015, 0.095, 9), rtol=1e-12)
    e = 1e-7
    fd = (T.forward(m + e) - T.forward(m - e)) / (2 * e)
    assert np.allclose(T.derivative(m), fd, rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("zonation", [False, True])
@pytest.mark.parametrize("mode", ["none", "tanh"])
def test_problem_gradient_matches_differences(zonation, mode):
    model = QuadraticModel()
    k_b = np.where(np.arange(model.n) < 20, 0.03, 0.04)
    free = np.arange(3, model.n - 2)
    prob = A.FrictionProblem(model, k_b, transform=A.ControlTransform(mode, lo=0.005, hi=0.2, lam=20.0), free=free,
                             zonation=zonation, alpha_reg=3.0, alpha_l1=0.01, alpha_spatial=5.0, alpha_ref=0.7,
                             k_ref=model.k_true)
    rng = np.random.default_rng(1)
    theta = prob.theta_start() + 0.1 * rng.standard_normal(prob.size()) * (0.01 if mode == "none" else 1.0)
    J, g = prob.grad(theta)
    assert J == pytest.approx(prob.func(theta), rel=1e-14)
    assert model.rerecords == 1
    for _ in range(5):
        v = rng.standard_normal(prob.size())
        e = 1e-7 if mode == "none" else 1e-6
        fd = (prob.func(theta + e * v) - prob.func(theta - e * v)) / (2 * e)
        assert abs(fd - float(np.dot(g, v))) <= 1e-5 * max(1e-12, abs(fd))


def test_fixed_cells_keep_background():
    model = QuadraticModel()
    k_b = np.full(model.n, 0.03)
    prob = A.FrictionProblem(model, k_b, free=np.arange(10))
    k = prob.control(prob.theta_start() + 0.01)
    assert np.all(k[10:] == 0.03) and np.allclose(k[:10], 0.04)


@pytest.mark.parametrize("algo", ["lbfgsb", "gd"])
def test_minimisers_reduce_the_cost_and_log(tmp_path, algo):
    model = QuadraticModel()
    d = str(tmp_path / "descent")
    prob = A.FrictionProblem(model, np.full(model.n, 0.03), transform=A.ControlTransform("clamp", lo=0.005, hi=0.2),
                             k_ref=model.k_true, descent_dir=d)
    res = A.run_minimization(prob, max_it=15, minimize_algo=algo, step=1.0)
    # L-BFGS-B solves the quadratic; the gradient descent contracts it (condition number 4)
    assert res["J_final"] < (1e-3 if algo == "lbfgsb" else 0.1) * res["J_init"]
    with open(os.path.join(d, "descent_log.csv")) as fh:
        rows = fh.read().splitlines()
    assert rows[0] == A.DESCENT_COLUMNS
    assert len(rows) - 1 == res["n_grad"]
    assert all(len(r.split(",")) == len(A.DESCENT_COLUMNS.split(",")) for r in rows[1:])
    maps = sorted(os.listdir(os.path.join(d, "friction_iter")))
    assert len(maps) == res["n_grad"] and maps[0] == "friction_iter_0001.txt"
    names, vals = pkg.case.read_map(os.path.join(d, "friction_iter", maps[-1]), 2, model.n)
    assert np.allclose(vals[0], res["k"])
