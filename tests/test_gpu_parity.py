"""Parity of the CUDA SP step (through the C ABI) with the reference and its CPU oracle.

Bar: bit for bit where the step uses only +, -, *, /, sqrt (no friction, no head loss, no
non-zero 'q' boundary); elsewhere within REL_TOL = 1e-10 relative (infinity norm per field),
the tolerance the specification states, since CUDA's exp/log may differ from the host libm
by an ulp.
"""
import numpy as np
import pytest

from tests.conftest import (REL_TOL, assert_state_close, golden_case, golden_names, load_pkg, rel_err,
                            sp_toce_case, uses_libm)

pytestmark = pytest.mark.gpu

oracle_binding = pytest.importorskip("oracle.binding")


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    oracle_binding.build(reference=False)
    return p


@pytest.mark.parametrize("name", golden_names())
def test_gpu_matches_reference_golden(pkg, name):
    case, fx = golden_case(name)
    model = pkg.SpModel(case)
    assert model.step(int(fx["steps"])) == int(fx["steps"])
    exact = not uses_libm(case)
    t, dt = model.time
    if exact:
        assert t == float(fx["t"]) and dt == float(fx["dt"])
    else:
        assert abs(t - float(fx["t"])) <= REL_TOL * abs(float(fx["t"]))
    assert_state_close(model.state(), (fx["h"], fx["q"], fx["r"]), exact, name)


def test_gpu_matches_reference_sp_toce(pkg):
    """The reference's own case: Godunov, blending topography, Strickler friction, singular
    head loss, 'q' inflow hydrograph and 'fr' outflow; 100 steps, then on to t_max (30 s)."""
    case, fx = sp_toce_case()
    model = pkg.SpModel(case)
    assert model.step(100) == int(fx["steps100"])
    assert_state_close(model.state(), (fx["h100"], fx["q100"], fx["r100"]), False, "sp_toce@100")
    n = model.execute()
    assert 100 + n == int(fx["steps_end"])
    assert model.t == float(fx["t_end"])
    assert_state_close(model.state(), (fx["h_end"], fx["q_end"], fx["r_end"]), False, "sp_toce@end")


@pytest.mark.parametrize("kind,kwargs", [
    ("dam_break", {"n_cells": 3000, "friction": "none"}),
    ("dam_break", {"n_cells": 3000, "friction": "none", "scheme": "godunov"}),
    ("gaussian_bumps", {"n_cells": 6000}),
    ("channel_features", {"n_cells": 2500, "scheme": "muscl_evr", "topo": "blending", "friction": "strickler",
                          "outflow": "fr"}),
])
def test_gpu_intermediates_match_oracle(pkg, kind, kwargs):
    """Step by step against the oracle: fluxes, wave speeds, slopes and state.  The first step
    is bit for bit in every configuration (its fluxes are computed before any exp/log)."""
    case = getattr(pkg.workloads, kind)(**kwargs)
    model = pkg.SpModel(case)
    o = oracle_binding.SpOracle(case)
    exact = not uses_libm(case)
    names = ["F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd", "lambda_max_int",
             "lambda_max_bnd"]
    if case.opts["num_scheme"] == "muscl_evr":
        names += ["slope_x", "slope_y"]
    for i, chunk in enumerate((1, 1, 5, 40, 150)):
        assert model.step(chunk) == o.step(chunk)
        first = i == 0
        for nm in names:
            a, b = model.array(nm), o.array(nm)
            if exact or first:
                assert np.array_equal(a.view(np.int64), b.view(np.int64)), f"{nm} after chunk {i}"
            else:
                assert rel_err(a, b) <= REL_TOL, nm
        assert_state_close(model.state(), o.state(), exact and True, f"{kind} chunk {i}")


def test_gpu_deterministic(pkg):
    case = pkg.workloads.gaussian_bumps(n_cells=20000)
    a = pkg.SpModel(case)
    b = pkg.SpModel(case)
    a.step(300)
    b.step(300)
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x.view(np.int64), y.view(np.int64))
    assert a.time == b.time


def test_gpu_mass_conservation(pkg):
    """Closed basin without wetting/drying clamps: sum(phi * A * h) is conserved to round-off."""
    case = pkg.workloads.dam_break(n_cells=8000, friction="none")
    model = pkg.SpModel(case)
    w = case.phi * case.mesh.cell_area
    m0 = float(np.sum(w * model.state()[0]))
    model.step(500)
    h = model.state()[0]
    assert h.min() > 1e-3
    m1 = float(np.sum(w * h))
    assert abs(m1 - m0) / m0 < 1e-12


def test_gpu_state_roundtrip_and_numbering(pkg):
    case = pkg.workloads.channel_features(n_cells=1500)
    model = pkg.SpModel(case)
    perm = model.cell_permutation()
    assert np.array_equal(np.sort(perm), np.arange(case.mesh.cell_nb))
    h, q, r = (np.random.default_rng(0).uniform(0, 1, case.mesh.cell_nb) for _ in range(3))
    model.set_state(h, q, r)
    for a, b in zip(model.state(), (h, q, r)):
        assert np.array_equal(a, b)
    model.set_time(1.5, 0.01)
    assert model.time == (1.5, 0.01)


def test_gpu_reports_impossible_hllc_configuration(pkg):
    """Where the reference stops (swSpHyp.cpp:728-739), the C ABI returns SW2D_E_HLLC_CONFIG."""
    case = pkg.workloads.channel_features(n_cells=3000, impervious=True, seed=7)
    model = pkg.SpModel(case)
    with pytest.raises(pkg.Sw2dError) as err:
        model.step(1)
    assert err.value.code == -4


def test_gpu_reports_bad_fr_boundary(pkg):
    case = pkg.workloads.channel_features(n_cells=1200, outflow="fr")
    case.bc.values[2][:] = 1.5        # 'fr' must lie in [0, 1] (swSpHyp.cpp:57-62)
    model = pkg.SpModel(case)
    with pytest.raises(pkg.Sw2dError) as err:
        model.step(3)
    assert err.value.code == -7


def test_gpu_execute_stops_at_t_max(pkg):
    case = pkg.workloads.channel_features(n_cells=1500, t_max=3.0)
    model = pkg.SpModel(case)
    o = oracle_binding.SpOracle(case)
    n = model.execute()
    assert n == o.step(10 ** 6)
    assert model.t == 3.0 and o.t == 3.0
    assert model.step(5) == 0


def test_gpu_full_size_properties(pkg):
    """The 4M-cell Gaussian-bump workload: a few steps against the oracle (within the
    tolerance: Manning friction), bit-identical reruns, finite and non-negative depths."""
    case = pkg.workloads.gaussian_bumps(n_cells=4_000_000)
    model = pkg.SpModel(case)
    o = oracle_binding.SpOracle(case)
    assert model.step(3) == 3 and o.step(3) == 3
    got, want = model.state(), o.state()
    assert_state_close(got, want, False, "4M cells")
    assert np.all(np.isfinite(got[0])) and got[0].min() >= 0.0
    again = pkg.SpModel(case)
    again.step(3)
    for x, y in zip(again.state(), got):
        assert np.array_equal(x.view(np.int64), y.view(np.int64))
