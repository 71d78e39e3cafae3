"""The learned closure inside the DIP step (sw2d_set_closure) and its data pipeline.

* A network whose outputs are exactly zero changes nothing: the run equals the run without
  closure.
* Out of the training hull every cell gets the plain momentum-dissipation closure at its own
  site in the balance: the run equals the model without a network bit for bit.
* The network inside the update kernel: recorded features against the formula, outputs against
  the GEMM kernels (bit for bit) and the FP64 forward, the correction against the balanced
  state.
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


def _empty_hull():
    return np.ones(10, np.float32), np.zeros(10, np.float32)


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


def _with_mu(case, rng):
    n = case.mesh.cell_nb
    c = copy.copy(case)
    c.opts = dict(case.opts, model_momentum_dissipation="active")
    c.mu = np.stack([rng.uniform(0, 0.5, n), rng.uniform(0, 0.5, n), rng.uniform(0, 90, n)])
    return c


def test_out_of_hull_is_the_plain_closure(pkg, urban):
    """With an empty training hull every cell gets the plain closure (dip/swDipHyp.cpp:295-324)
    where the update applies it: the run equals the model without a network bit for bit."""
    _, coarse, _ = urban
    case = _with_mu(coarse, np.random.default_rng(0))
    a = pkg.SpModel(case)
    b = pkg.SpModel(case)
    b.set_closure(_zero_net(pkg.closure), *_empty_hull())
    assert a.step(80) == b.step(80)
    assert a.time == b.time
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    # and the plain closure does act on this case
    c = pkg.SpModel(coarse)
    c.step(80)
    assert not np.array_equal(c.state()[1], a.state()[1])


def test_in_update_network_matches_the_gemm_path_and_the_reference(pkg, urban):
    """The network inside the update kernel.  Its recorded features are the formula's on the
    state at the step's start and the balanced state; its outputs equal sw2d_mlp_infer's (the
    GEMM kernels) on the same features bit for bit, and the FP64 forward with the kernels' BF16
    roundings within 1 % of the largest output; the correction enters the balanced state as
    (double)(scale * output)."""
    C = pkg.closure
    _, coarse, _ = urban
    case = copy.copy(coarse)
    # no friction and no velocity cap: the balanced state is the step's result
    case.opts = dict(coarse.opts, model_friction="none", fr_max=1e30, v_max=1e30)
    m0 = pkg.SpModel(case)
    m0.step(30)
    s0 = m0.state()
    t0 = m0.t
    # the balanced state: one step with a network whose hull is empty (nothing applied)
    rec = pkg.SpModel(case)
    rec.set_state(*s0)
    rec.set_time(t0, 0.0)
    rec.set_closure(_zero_net(C), *_empty_hull())
    rec.set_option("closure_record", 1)
    rec.step(1)
    s1, dt = rec.state(), rec.dt
    f0 = rec.closure_record()[:, :10]
    # the formula on (s0, s1); s1 is the balanced state where the round-off flush (|x| < 1e-16
    # set to 0) left it alone
    f = C.features(s0, s1, case.phi, C.phig_min_of(case), dt)
    kept = np.all([np.abs(b) >= 1e-16 for b in s1], 0)
    assert kept.sum() >= 50
    bad = (f0 != f) & kept[:, None]
    assert not bad.any(), (bad.sum(0), f0[bad.any(1)][:3], f[bad.any(1)][:3])
    norm = np.concatenate([f.mean(0), np.maximum(f.std(0), 1e-6), np.zeros(2), np.full(2, 1e-3)]).astype(np.float32)
    p = C.init_params(seed=5)
    net = C.MLP(p, norm)
    scale = 0.75
    m = pkg.SpModel(case)
    m.set_state(*s0)
    m.set_time(t0, 0.0)
    m.set_closure(net, *_wide_hull(), scale)
    m.set_option("closure_record", 1)
    assert m.kernels_per_step == rec.kernels_per_step
    m.step(1)
    r = m.closure_record()
    assert np.array_equal(r[:, :10], f0)
    y = r[:, 10:]
    assert np.array_equal(y, net.infer(r[:, :10]))
    want = C.reference_forward(p, norm, r[:, :10])["y"]
    assert np.abs(want).max() > 0
    assert np.max(np.abs(y - want)) <= 1e-2 * np.abs(want).max()
    h, q, rr = m.state()
    assert np.array_equal(h, s1[0])
    corr = (np.float32(scale) * y).astype(np.float64)
    for got, base, c in ((q, s1[1], corr[:, 0]), (rr, s1[2], corr[:, 1])):
        exp = base + c
        exp = np.where(np.abs(exp) < 1e-16, 0.0, exp)
        assert np.array_equal(got[kept], exp[kept])
    # more steps run and stay finite; the record follows the last step
    m.step(20)
    assert all(np.all(np.isfinite(a)) for a in m.state())
    assert not np.array_equal(m.closure_record(), r)


def test_record_needs_a_closure(pkg, urban):
    _, coarse, _ = urban
    m = pkg.SpModel(coarse)
    with pytest.raises(RuntimeError):
        m.set_option("closure_record", 1)
    m.set_closure(_zero_net(pkg.closure), *_wide_hull())
    with pytest.raises(RuntimeError):
        m.closure_record()


def test_pipeline_runs_and_trains(pkg, urban):
    """Both generators on a small building layout: one-step pairs from the averaged fine state,
    on-trajectory pairs with nudging targets; training on the tensor cores lowers the loss; the
    evaluation runs every variant."""
    C = pkg.closure
    fine, coarse, av = urban
    X, Y, T = C.generate_samples(fine, coarse, av, t_start=3.0, n_samples=20, spacing=0.2)
    assert X.shape[1] == 10 and Y.shape == (X.shape[0], 2) and np.all(np.isfinite(X)) and np.all(np.isfinite(Y))
    X, Y = C.generate_trajectory_samples(fine, coarse, av, starts=(3.0, 8.0), window=4.0, tau=16.0, every=2)
    assert X.shape[1] == 10 and Y.shape == (X.shape[0], 2) and np.all(np.isfinite(X)) and np.all(np.isfinite(Y))
    net, lo, hi, hist = C.train_closure(X, Y, epochs=15, batch=2048)
    assert hist[-1] < 0.8 * hist[0]
    # a second round from the trajectories with the network attached (its hull, no plain closure)
    X2, Y2 = C.generate_trajectory_samples(fine, coarse, av, starts=(3.0,), window=4.0, tau=16.0, every=2,
                                           net=net, hull=(lo, hi))
    assert X2.shape[0] > 0 and np.all(np.isfinite(Y2))
    res = C.evaluate(fine, coarse, av, 5.0, 12.0, net=net, hull=(lo, hi))
    for key in ("none", "plain_mu0.1", "plain_mu0.3", "learned"):
        assert np.all(np.isfinite(res[key]))


def test_learned_closure_beats_the_plain_one_on_an_unseen_layout(pkg):
    """What the trained network gains: trained on three building layouts (on-trajectory samples,
    nudging targets), it is judged on a fourth against the fine run averaged onto the coarse
    cells.  Its errors in h and in (q, r) are below those of the run without closure and of the
    plain closure (mu = 0.1 and 0.3)."""
    C = pkg.closure
    mk = lambda seed: C.urban_cases(lx=240.0, ly=120.0, dx_fine=1.0, coarse_factor=8, seed=seed)
    net, lo, hi, hist, n = C.train_on_layouts([mk(1), mk(2), mk(3)], tau=16.0, epochs=20, batch=4096)
    assert n > 10000 and hist[-1] < hist[0]
    res = C.evaluate(*mk(7), 10.0, 30.0, net=net, hull=(lo, hi))
    print(res)
    for other in ("none", "plain_mu0.1", "plain_mu0.3"):
        assert res["learned"][0] < res[other][0], (other, res)
        assert res["learned"][1] < res[other][1], (other, res)
