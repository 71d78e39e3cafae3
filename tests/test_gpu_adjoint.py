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

J is only piecewise smooth.  Where the evaluation point itself sits on a switch, J has no
gradient and central differences average two one-sided slopes; the finite-difference tests
therefore start from states that do not: a free surface with small waves for MUSCL (a flat
surface puts every limiter test on its switch), directions that keep dry cells dry, and bed
directions that keep equal beds equal (the blending weight jumps there).  States at rest sit on
the round-off flush after the balance, which the adjoint differentiates as the identity (the
option adjoint_flush_branch selects the branch-taken derivative instead).
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


def _case(pkg, spec, n_cells=3000, wavy=False, opts=None):
    """The case of `spec`; with `wavy`, its initial free surface carries smooth waves of a few
    centimetres: a flat surface at rest sits exactly on the MUSCL limiter's switches (every
    reconstruction equals its neighbours' values), where J has no gradient, only one-sided
    directional derivatives."""
    w = pkg.workloads
    if spec["kind"] == "dam":
        case = w.dam_break(n_cells=n_cells, scheme=spec["scheme"], friction="manning")
    else:
        case = w.channel_features(n_cells=n_cells, scheme=spec["scheme"], topo=spec["topo"], friction="manning",
                                  head_loss=True, t_max=40.0)
    if wavy:
        wet = case.h0 > 0.0
        case.h0 = np.where(wet, np.maximum(0.0, case.h0 + 0.03 * _smooth(case, 101)), 0.0)
    if opts:
        case.opts.update(opts)
    return case


def _twin(pkg, spec, every=16, n_gauges=24, obs_every=5, discharge=False, seed=3, wavy=False, opts=None):
    """A model with a recorded trajectory and gauge observations from a twin replay whose
    friction is perturbed by a smooth +-20 % field."""
    case = _case(pkg, spec, wavy=wavy, opts=opts)
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


# central-difference steps tried, largest first: J is only piecewise smooth (limiter switches,
# wet/dry cut-offs, upwinding), so a large step may straddle a switch; a small one is limited by
# the rounding of J.  The check passes when one of them agrees with the adjoint.
EPS = (1e-5, 1e-6, 1e-7, 3e-8, 1e-8, 3e-9)


def _direction(model, case, start, control, seed):
    """A smooth perturbation of `control` that keeps dry cells dry and equal beds equal."""
    v = _smooth(case, seed)
    if control in ("friction_1", "friction_2"):
        return v * model.get_param(control)          # relative perturbation
    if control == "z_b" and case.opts.get("topo_discretization") == "blending":
        # a function of z_b itself: neighbours with equal beds (cells whose nodes lie on a
        # straight boundary of a planar bed) stay equal; the blending weight of the HLLC
        # solver is 0 there and jumps for any bed difference (swSpHyp.cpp:824-998)
        zb = model.get_param("z_b")
        return np.sin(7.0 * zb + seed) + 0.5 * np.cos(3.0 * zb)
    if control == "z_b":
        return v
    return v * (start[0] > 0.05)                     # initial state: wet cells only


def _J_along(model, start, control, base, v, s):
    if control in ("friction_1", "friction_2", "z_b"):
        model.set_param(control, base + s * v)
    else:
        st = list(start)
        k = {"h0": 0, "q0": 1, "r0": 2}[control]
        st[k] = st[k] + s * v
        model.set_trajectory_start(*st)
    return model.replay_cost()


def _restore(model, start, control, base):
    if control in ("friction_1", "friction_2", "z_b"):
        model.set_param(control, base)
    else:
        model.set_trajectory_start(*start)


def _fd_check(model, case, start, control, seed, tol):
    """Central differences of J along a smooth direction v of `control` against g . v;
    returns the best relative error over the steps of EPS."""
    v = _direction(model, case, start, control, seed)
    J, g = model.adjoint()
    base = model.get_param(control) if control in ("friction_1", "friction_2", "z_b") else None
    ad = float(np.dot(g[control], v))
    scale = max(abs(ad), 1e-300)
    errs = []
    for eps in EPS:
        fd = (_J_along(model, start, control, base, v, eps) - _J_along(model, start, control, base, v, -eps)) / (2 * eps)
        errs.append(abs(fd - ad) / scale)
        if errs[-1] <= tol:
            break
    _restore(model, start, control, base)
    assert model.replay_cost() == J
    assert min(errs) <= tol, f"{control}: ad={ad:.10e}, relative errors per step {dict(zip(EPS, errs))}"
    return min(errs)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("control", ["friction_1", "friction_2", "h0", "q0", "r0", "z_b"])
def test_gradient_matches_central_differences(pkg, name, control):
    """From a free surface with small waves (no state sits on a limiter switch)."""
    model, case, start = _twin(pkg, CASES[name], discharge=(name == "dam_muscl"), wavy=True)
    # MUSCL: states within 1e-16 of the round-off flush flip under any perturbation, which puts
    # a noise of order 1e-16 / eps on the differences; the channel's J is small (gauges far
    # from the inflow), so its differences are the noisiest
    tol = 1e-6 if CASES[name]["scheme"] == "godunov" else 5e-5
    _fd_check(model, case, start, control, seed=zlib.crc32(f"{name}/{control}".encode()) % 1000, tol=tol)


@pytest.mark.parametrize("control", ["friction_1", "h0", "q0", "r0", "z_b"])
def test_gradient_at_rest_matches_central_differences(pkg, control):
    """The dam break from rest (flat water on both sides, u = v = 0), first order: every cell
    at rest sits on the round-off flush, which the adjoint differentiates as the identity."""
    model, case, start = _twin(pkg, CASES["dam_godunov"])
    _fd_check(model, case, start, control, seed=zlib.crc32(f"rest/{control}".encode()) % 1000, tol=1e-6)


@pytest.mark.parametrize("control", ["friction_1", "h0", "q0"])
def test_gradient_with_the_velocity_cap_acting(pkg, control):
    """The dam break with v_max = 0.5 m/s: the velocity cap (swSp::correctVelocity) scales the
    discharge of the cells behind the front at every step, and the reverse takes the cap's
    branch from what the segment's recompute recorded."""
    spec = CASES["dam_godunov"]
    capped = {"v_max": 0.5}
    a = pkg.SpModel(_case(pkg, spec))
    b = pkg.SpModel(_case(pkg, spec, opts=capped))
    a.step(20)
    b.step(20)
    qa, qb = a.state()[1], b.state()[1]
    assert np.count_nonzero(qa != qb) > 100  # the cap acts
    model, case, start = _twin(pkg, spec, opts=capped)
    _fd_check(model, case, start, control, seed=zlib.crc32(f"cap/{control}".encode()) % 1000, tol=1e-5)


def test_flush_branch_option(pkg):
    """adjoint_flush_branch = 1 differentiates the flush as the branch taken (zero derivative
    for flushed values): from rest the discharge gradient then misses the first step's pressure
    imbalance.  J is the same; both gradients are deterministic."""
    model, _, _ = _twin(pkg, CASES["dam_godunov"])
    J0, g0 = model.adjoint()
    model.set_option("adjoint_flush_branch", 1)
    J1, g1 = model.adjoint()
    J2, g2 = model.adjoint()
    model.set_option("adjoint_flush_branch", 0)
    assert J0 == J1 == J2
    assert np.array_equal(g1["q0"], g2["q0"])
    assert not np.allclose(g0["q0"], g1["q0"])
    assert all(np.isfinite(g1[k]).all() for k in g1)


def test_taylor_ratio_tends_to_one(pkg):
    """The reference's Taylor protocol (assim/swSpE_checkpoint.cpp:1454-1663) on friction."""
    model, case, _ = _twin(pkg, CASES["channel_muscl_blending"], wavy=True)
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


def test_long_window_over_dry_islands_gives_a_finite_gradient(pkg):
    """500 steps over a bed with dry islands: near-dry cells carry the 1/max(h, 1e-16) factors
    of the wave speeds and velocities, and their adjoint can overflow (the reference sees the
    same and zeroes non-finite gradient entries, assim/swSpE_checkpoint.cpp:1196-1207).  The
    gradient handed back is finite, the count of zeroed entries is reported, and both are the
    same on a second sweep."""
    case = pkg.workloads.gaussian_bumps(n_cells=14000, seed_mesh=137)
    model = pkg.SpModel(case)
    model.record(500, 50)
    rng = np.random.default_rng(2)
    cells = np.sort(rng.choice(model.n, size=16, replace=False))
    steps = np.arange(10, 501, 10)
    model.set_observations(cells, steps, model.replay_sample(cells, steps) * 1.01)
    J, g = model.adjoint()
    counts = model.adjoint_nonfinite()
    assert np.isfinite(J) and all(np.isfinite(v).all() for v in g.values())
    assert set(counts) == set(g) and all(c >= 0 for c in counts.values())
    J2, g2 = model.adjoint()
    assert J2 == J and model.adjoint_nonfinite() == counts
    for k in g:
        assert np.array_equal(g[k].view(np.int64), g2[k].view(np.int64)), k


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


@pytest.mark.parametrize("scheme", ["muscl_evr", "godunov"])
def test_stored_states_give_the_same_gradient(pkg, scheme):
    """The segment recompute keeps each step's slopes and Riemann states for the reverse steps
    (option adjoint_store_states, the default) or the reverse steps rebuild them: the same bits."""
    case = pkg.workloads.dam_break(n_cells=4000, scheme=scheme)
    out = []
    for store in (1, 0):
        model = pkg.SpModel(case)
        model.set_option("adjoint_store_states", store)
        model.record(120, 25)
        rng = np.random.default_rng(3)
        cells = np.sort(rng.choice(model.n, size=16, replace=False))
        steps = np.arange(10, 121, 10)
        model.set_observations(cells, steps, model.replay_sample(cells, steps) * 1.02)
        out.append(model.adjoint())
    (J1, g1), (J0, g0) = out
    assert J1 == J0
    for k in g1:
        assert np.array_equal(g1[k].view(np.int64), g0[k].view(np.int64)), k


def test_lake_at_rest_reverse_growth(pkg):
    """Over a lake at rest (MUSCL-EVR) every wet cell's limiter tests sit on their kinks: the
    free surface is level to round-off, so each reconstruction equals its neighbours' values.
    The branch taken there (Enzyme's convention too) makes the reverse dynamics grow by orders of
    magnitude over 500 steps until they overflow; the non-finite entries are zeroed as the
    reference does, and counted.  The same lake under Godunov (no slopes): the adjoint stays
    bounded and nothing is zeroed."""
    out = {}
    for scheme in ("muscl_evr", "godunov"):
        case = pkg.workloads.gaussian_bumps(n_cells=20753, seed_mesh=105, scheme=scheme)
        model = pkg.SpModel(case)
        model.set_option("adjoint_trace", 1)
        model.record(500, 50)
        rng = np.random.default_rng(5)
        cells = np.sort(rng.choice(model.n, size=16, replace=False))
        steps = np.arange(10, 501, 10)
        model.set_observations(cells, steps, model.replay_sample(cells, steps) * 1.01)
        J, g = model.adjoint()
        out[scheme] = (g, sum(model.adjoint_nonfinite().values()), model.adjoint_trace())
        assert all(np.isfinite(v).all() for v in g.values())
    g, bad, tr = out["muscl_evr"]
    assert bad > 1000 and tr["nonfinite"].any()
    assert tr["max_h"][tr["nonfinite"] == 0].max() > 1e100
    g, bad, tr = out["godunov"]
    assert bad == 0 and not tr["nonfinite"].any() and tr["max_h"].max() < 1e3
