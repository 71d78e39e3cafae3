"""Adjoint of the step on the GPU: the gradient of an observation misfit J along a recorded
trajectory with respect to the per-cell friction coefficients, the initial state and the bed.

The reference differentiates its replay (replay_trajectory_cost, assim/swSpE_checkpoint.cpp:
1380-1453) with Enzyme and checks the gradient with a Taylor test and finite differences
(assim/swSpE_checkpoint.cpp:1454-1663).  The Enzyme gradient cannot be produced here (no
clang/Enzyme), so these tests pin the GPU gradient by:

* central finite differences of sw2d_replay_cost in smooth random directions, per control;
* the Taylor ratio (J(m + e v) - J(m)) / (e g.v) -> 1;
* invariants of the implementation: the replay reproduces the recorded CFL run bit for bit,
  and the gradient does not depend on the checkpoint interval (bitwise).
"""
import zlib

import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu

N_STEPS = 60


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


def _smooth(case, seed):
    """A smooth random field over the cells, in [-1, 1]."""
    rng = np.random.default_rng(seed)
    x, y = case.mesh.cell_x, case.mesh.cell_y
    lx, ly = np.ptp(x) or 1.0, np.ptp(y) or 1.0
    f = np.zeros_like(x)
    for _ in range(4):
        kx, ky, ph = rng.uniform(0.5, 3.0), rng.uniform(0.5, 3.0), rng.uniform(0, 2 * np.pi)
        f += rng.uniform(-1, 1) * np.sin(2 * np.pi * (kx * x / lx + ky * y / ly) + ph)
    return f / np.max(np.abs(f))


CASES = {
    "dam_godunov": dict(kind="dam", scheme="godunov"),
    "dam_muscl": dict(kind="dam", scheme="muscl_evr"),
    "channel_muscl_blending": dict(kind="channel", scheme="muscl_evr", topo="blending"),
    "channel_godunov_discontinuous": dict(kind="channel", scheme="godunov", topo="discontinuous"),
}


def _case(pkg, spec, n_cells=3000):
    w = pkg.workloads
    if spec["kind"] == "dam":
        return w.dam_break(n_cells=n_cells, scheme=spec["scheme"], friction="manning")
    return w.channel_features(n_cells=n_cells, scheme=spec["scheme"], topo=spec["topo"], friction="manning",
                              head_loss=True, t_max=40.0)


def _twin(pkg, spec, every=16, n_gauges=24, obs_every=5, discharge=False, seed=3):
    """A model with a recorded trajectory and gauge observations from a twin replay whose
    friction is perturbed by a smooth +-20 % field."""
    case = _case(pkg, spec)
    model = pkg.SpModel(case)
    h0, q0, r0 = model.state()
    assert model.record(N_STEPS, every) == N_STEPS
    rng = np.random.default_rng(seed)
    wet = np.flatnonzero(h0 > 0.05)
    cells = np.sort(rng.choice(wet, size=n_gauges, replace=False))
    steps = np.arange(obs_every, N_STEPS + 1, obs_every)
    n1, n2 = model.get_param("friction_1"), model.get_param("friction_2")
    pert = 1.0 + 0.2 * _smooth(case, seed + 10)
    model.set_param("friction_1", n1 * pert)
    model.set_param("friction_2", n2 * pert)
    if discharge:
        ho, qo, ro = model.replay_sample(cells, steps, discharge=True)
    else:
        ho = model.replay_sample(cells, steps)
        qo = ro = None
    model.set_param("friction_1", n1)
    model.set_param("friction_2", n2)
    w_q = 0.5 if discharge else None
    model.set_observations(cells, steps, ho, w_h=rng.uniform(0.5, 2.0, cells.size), q_obs=qo, r_obs=ro, w_q=w_q)
    return model, case, (h0, q0, r0)


def test_replay_reproduces_the_recorded_run(pkg):
    spec = CASES["channel_muscl_blending"]
    plain = pkg.SpModel(_case(pkg, spec))
    assert plain.step(N_STEPS) == N_STEPS
    ref = plain.state()
    model = pkg.SpModel(_case(pkg, spec))
    model.record(N_STEPS, 7)
    after_record = model.state()
    for a, b in zip(ref, after_record):
        assert np.array_equal(a.view(np.int64), b.view(np.int64))
    model.set_observations([0], [N_STEPS], [[0.0]])
    model.replay_cost()
    for a, b in zip(ref, model.state()):
        assert np.array_equal(a.view(np.int64), b.view(np.int64))
    assert model.t == plain.t


@pytest.mark.parametrize("name", list(CASES))
def test_gradient_independent_of_checkpoint_interval(pkg, name):
    grads = []
    for every in (1, 7, N_STEPS):
        model, _, _ = _twin(pkg, CASES[name], every=every)
        J, g = model.adjoint()
        grads.append((J, g))
    J0, g0 = grads[0]
    for J, g in grads[1:]:
        assert J == J0
        for k in g0:
            assert np.array_equal(g0[k].view(np.int64), g[k].view(np.int64)), k


def test_adjoint_cost_equals_replay_cost_and_is_deterministic(pkg):
    model, _, _ = _twin(pkg, CASES["dam_muscl"], discharge=True)
    J1 = model.replay_cost()
    Ja, ga = model.adjoint()
    Jb, gb = model.adjoint()
    assert J1 == Ja == Jb and J1 > 0
    for k in ga:
        assert np.array_equal(ga[k].view(np.int64), gb[k].view(np.int64)), k


def _fd_check(model, case, start, control, seed, eps, tol):
    """Central difference of J along a smooth direction v of `control` against g . v."""
    h0, q0, r0 = start
    v = _smooth(case, seed)
    J, g = model.adjoint()
    if control in ("friction_1", "friction_2"):
        base = model.get_param(control)
        v = v * base                       # relative perturbation
        grad = g[control]

        def J_at(s):
            model.set_param(control, base + s * v)
            return model.replay_cost()

        restore = lambda: model.set_param(control, base)  # noqa: E731
    elif control == "z_b":
        base = model.get_param("z_b")
        grad = g["z_b"]

        def J_at(s):
            model.set_param("z_b", base + s * v)
            return model.replay_cost()

        restore = lambda: model.set_param("z_b", base)  # noqa: E731
    else:  # initial state: perturb wet cells only, so that no dry cell becomes wet
        k = {"h0": 0, "q0": 1, "r0": 2}[control]
        v = v * (h0 > 0.05)
        grad = g[control]

        def J_at(s):
            st = [h0, q0, r0]
            st[k] = st[k] + s * v
            model.set_trajectory_start(*st)
            return model.replay_cost()

        restore = lambda: model.set_trajectory_start(h0, q0, r0)  # noqa: E731
    ad = float(np.dot(grad, v))
    fd = (J_at(eps) - J_at(-eps)) / (2 * eps)
    restore()
    assert model.replay_cost() == J
    scale = float(np.sum(np.abs(grad * v)))
    assert abs(fd - ad) <= tol * max(abs(ad), scale, 1e-12), f"{control}: fd={fd:.10e} ad={ad:.10e}"
    return fd, ad


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("control", ["friction_1", "friction_2", "h0", "q0", "r0", "z_b"])
def test_gradient_matches_central_differences(pkg, name, control):
    model, case, start = _twin(pkg, CASES[name], discharge=(name == "dam_muscl"))
    eps = 1e-6
    _fd_check(model, case, start, control, seed=zlib.crc32(f"{name}/{control}".encode()) % 1000, eps=eps, tol=2e-5)


def test_taylor_ratio_tends_to_one(pkg):
    """The reference's Taylor protocol (assim/swSpE_checkpoint.cpp:1454-1663) on friction."""
    model, case, _ = _twin(pkg, CASES["channel_muscl_blending"])
    J, g = model.adjoint()
    base = model.get_param("friction_1")
    v = _smooth(case, 5) * base
    gv = float(np.dot(g["friction_1"], v))
    ratios = []
    for e in (1e-2, 1e-3, 1e-4, 1e-5):
        model.set_param("friction_1", base + e * v)
        ratios.append((model.replay_cost() - J) / (e * gv))
    model.set_param("friction_1", base)
    errs = [abs(r - 1.0) for r in ratios]
    assert errs[-1] < 1e-3
    assert errs[2] < errs[0]


def test_adjoint_errors(pkg):
    case = _case(pkg, CASES["dam_godunov"])
    model = pkg.SpModel(case)
    with pytest.raises(pkg.Sw2dError):
        model.adjoint()  # no trajectory
    model.record(10, 4)
    with pytest.raises(pkg.Sw2dError):
        model.adjoint()  # no observations
    with pytest.raises(pkg.Sw2dError):
        model.set_observations([3, 3], [5], [[0.0, 0.0]])  # repeated cell
    model.set_observations([3], [11], [[0.0]])
    with pytest.raises(pkg.Sw2dError):
        model.replay_cost()  # beyond the trajectory
    model.set_observations([3], [0, 10], [[0.0], [0.0]])
    J, g = model.adjoint()
    assert J > 0 and g["h0"][3] != 0.0
