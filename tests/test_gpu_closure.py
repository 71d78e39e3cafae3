"""The learned closure inside the DIP step (sw2d_set_closure) and its data pipeline.

* A network whose outputs are exactly zero changes nothing: the run equals the run without
  closure (the plain closure inside the update is off while a network is attached).
* Out of the training hull every cell falls back to the plain momentum-dissipation closure
  applied to the step's increments: checked against that formula restated in numpy.
* The pipeline runs end to end on a small building layout: samples from the solver's own fine
  and coarse runs, tensor-core training (the loss falls), evaluation against the fine run.
"""
import copy

import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


@pytest.fixture(scope="module")
def urban(pkg):
    return pkg.closure.urban_cases(lx=120.0, ly=60.0, dx_fine=1.0, coarse_factor=6, seed=3)


def _zero_net(C):
    n = np.zeros(C.N_IN * 2 + C.N_OUT * 2, dtype=np.float32)
    n[C.N_IN:2 * C.N_IN] = 1.0
    n[2 * C.N_IN + C.N_OUT:] = 1.0
    return C.MLP(np.zeros_like(C.init_params()), n)


def _wide_hull():
    return np.full(10, -1e30, dtype=np.float32), np.full(10, 1e30, dtype=np.float32)


def test_zero_network_changes_nothing(pkg, urban):
    _, coarse, _ = urban
    a = pkg.SpModel(coarse)
    b = pkg.SpModel(coarse)
    net = _zero_net(pkg.closure)
    b.set_closure(net, *_wide_hull())
    assert a.step(60) == b.step(60)
    assert a.time == b.time
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)


def _dissipate(mu1, mu2, alpha_deg, h0, q0, r0, h, q, r):
    # the plain closure (dip/swDipHyp.cpp:295-324) on the step's increments
    a = alpha_deg * np.arctan(1.0) / 45.0
    ca, sa = np.cos(a), np.sin(a)
    dq, dr = q - q0, r - r0
    lq = ca * dq + sa * dr
    lr = -sa * dq + ca * dr
    rq, rr = mu1 * lq, mu2 * lr
    red_q = ca * rq - sa * rr
    red_r = sa * rq + ca * rr
    up = h > h0 + 1e-16
    return np.where(up, q - red_q, q), np.where(up, r - red_r, r)


def test_out_of_hull_falls_back_to_the_plain_closure(pkg, urban):
    _, coarse, _ = urban
    n = coarse.mesh.cell_nb
    case = copy.copy(coarse)
    case.opts = dict(coarse.opts, model_momentum_dissipation="active")
    rng = np.random.default_rng(0)
    case.mu = np.stack([rng.uniform(0, 0.5, n), rng.uniform(0, 0.5, n), rng.uniform(0, 90, n)])
    m = pkg.SpModel(case)
    m.step(30)
    s0 = m.state()
    t0, dt0 = m.time
    # the same step without any closure (plain closure off: a case without the mu map)
    plain = pkg.SpModel(coarse)
    plain.set_state(*s0)
    plain.set_time(t0, dt0)
    plain.step(1)
    h1, q1, r1 = plain.state()
    m.set_closure(_zero_net(pkg.closure), np.ones(10, np.float32), np.zeros(10, np.float32))  # empty hull
    m.step(1)
    h, q, r = m.state()
    assert np.array_equal(h, h1)
    eq, er = _dissipate(case.mu[0], case.mu[1], case.mu[2], s0[0], s0[1], s0[2], h1, q1, r1)
    assert np.allclose(q, eq, rtol=1e-13, atol=1e-15) and np.allclose(r, er, rtol=1e-13, atol=1e-15)


def test_pipeline_runs_and_trains(pkg, urban):
    C = pkg.closure
    fine, coarse, av = urban
    X, Y, T = C.generate_samples(fine, coarse, av, t_start=3.0, n_samples=40, spacing=0.2)
    assert X.shape[1] == 10 and Y.shape == (X.shape[0], 2) and np.all(np.isfinite(X)) and np.all(np.isfinite(Y))
    net, lo, hi, hist = C.train_closure(X, Y, epochs=15, batch=2048)
    assert hist[-1] < 0.2 * hist[0]
    res = C.evaluate(fine, coarse, av, 5.0, 12.0, net=net, hull=(lo, hi), mu=0.3)
    for key in ("none", "plain_mu", "learned"):
        assert np.all(np.isfinite(res[key]))


def test_fused_kernel_matches_the_gemm_path_and_the_reference(pkg, urban):
    """The in-step inference as one fused kernel (features, three tensor-core layers through
    shared memory and TMEM, apply) gives the same state bit for bit as the five-launch path
    (features, three GEMM launches, apply), and its correction matches the FP64 forward with the
    kernels' BF16 roundings."""
    C = pkg.closure
    _, coarse, _ = urban
    m0 = pkg.SpModel(coarse)
    m0.step(30)
    s0 = m0.state()
    t0 = m0.t
    plain = pkg.SpModel(coarse)
    plain.set_state(*s0)
    plain.set_time(t0, 0.0)
    plain.step(1)
    s1, dt = plain.state(), plain.dt
    f = C.features(s0, s1, coarse.phi, C.phig_min_of(coarse), dt)
    norm = np.concatenate([f.mean(0), np.maximum(f.std(0), 1e-6), np.zeros(2), np.full(2, 1e-3)]).astype(np.float32)
    p = C.init_params(seed=5)
    net = C.MLP(p, norm)
    runs = []
    for fused in (1, 0):
        m = pkg.SpModel(coarse)
        m.set_state(*s0)
        m.set_time(t0, 0.0)
        m.set_closure(net, *_wide_hull())
        m.set_option("closure_fused", fused)
        assert m.kernels_per_step == plain.kernels_per_step + (1 if fused else 5)
        m.step(1)
        one = m.state()
        m.step(20)
        runs.append((one, m.state(), m.t))
    for a, b in zip(runs[0][0] + runs[0][1], runs[1][0] + runs[1][1]):
        assert np.array_equal(a, b)
    assert runs[0][2] == runs[1][2]
    # the first step's correction against the FP64 forward (an FP32-accumulation difference can
    # move a BF16 rounding of a hidden activation: a tolerance of 1 % of the largest correction)
    y = C.reference_forward(p, norm, f)["y"]
    h, q, r = runs[0][0]
    assert np.array_equal(h, s1[0])
    for got, want in ((q - s1[1], y[:, 0]), (r - s1[2], y[:, 1])):
        assert np.abs(want).max() > 0
        assert np.max(np.abs(got - want)) <= 1e-2 * np.abs(want).max()
