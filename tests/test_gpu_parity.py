"""Parity of the CUDA SP step (through the C ABI) with the reference and its CPU oracle.

Bars:
* bit for bit against the reference's own compiled objects linked with the portable exp/log
  the CUDA build uses (fixture fields ..._pm), and against the CPU oracle in that mode, in
  every configuration and over whole runs;
* within REL_TOL = 1e-10 relative (the specification's tolerance) against the reference linked
  with glibc wherever the reference itself is insensitive to its libm at that level (fixture
  flag libm_stable; the wetting/drying channel cases move by 1e-6..1e-1 when only the
  reference's libm changes, which no implementation can undercut).
"""
import os

import numpy as np
import pytest

from tests.conftest import GOLDEN, assert_state_close, golden_case, golden_names, load_pkg, sp_toce_case

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
    assert model.step(int(fx["steps"])) == int(fx["steps_pm"])
    assert model.time == (float(fx["t_pm"]), float(fx["dt_pm"]))
    state = model.state()
    assert_state_close(state, (fx["h_pm"], fx["q_pm"], fx["r_pm"]), True, name + " vs reference(portable libm)")
    if bool(fx["libm_stable"]):
        assert_state_close(state, (fx["h"], fx["q"], fx["r"]), False, name + " vs reference(glibc)")


def test_gpu_matches_reference_sp_toce(pkg):
    """The reference's own case: Godunov, blending topography, Strickler friction, singular
    head loss, 'q' inflow hydrograph and 'fr' outflow; 100 steps, then on to t_max (30 s)."""
    case, fx = sp_toce_case()
    model = pkg.SpModel(case)
    assert model.step(100) == int(fx["steps100"])
    st = model.state()
    assert_state_close(st, (fx["h100_pm"], fx["q100_pm"], fx["r100_pm"]), True, "sp_toce@100")
    assert_state_close(st, (fx["h100"], fx["q100"], fx["r100"]), False, "sp_toce@100 vs glibc")
    n = model.execute()
    assert 100 + n == int(fx["steps_end_pm"])
    assert model.t == float(fx["t_end_pm"])
    assert_state_close(model.state(), (fx["h_end_pm"], fx["q_end_pm"], fx["r_end_pm"]), True, "sp_toce@end")


@pytest.mark.parametrize("kind,kwargs", [
    ("dam_break", {"n_cells": 3000, "friction": "none"}),
    ("dam_break", {"n_cells": 3000, "friction": "none", "scheme": "godunov"}),
    ("gaussian_bumps", {"n_cells": 6000}),
    ("channel_features", {"n_cells": 2500, "scheme": "muscl_evr", "topo": "blending", "friction": "strickler",
                          "outflow": "fr"}),
])
def test_gpu_intermediates_match_oracle(pkg, kind, kwargs):
    """Step by step against the oracle (portable exp/log): fluxes, wave speeds, slopes and
    state, bit for bit."""
    case = getattr(pkg.workloads, kind)(**kwargs)
    model = pkg.SpModel(case)
    model.set_option("record_wave_speeds", 1)
    model.set_option("record_fluxes", 1)
    o = oracle_binding.SpOracle(case, portable_math=True)
    names = ["F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd", "lambda_max_int",
             "lambda_max_bnd"]
    if case.opts["num_scheme"] == "muscl_evr":
        names += ["slope_x", "slope_y"]
    for i, chunk in enumerate((1, 1, 5, 40, 150)):
        assert model.step(chunk) == o.step(chunk)
        assert model.time == (o.t, o.dt)
        for nm in names:
            a, b = model.array(nm), o.array(nm)
            assert np.array_equal(a.view(np.int64), b.view(np.int64)), f"{nm} after chunk {i}"
        assert_state_close(model.state(), o.state(), True, f"{kind} chunk {i}")


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
    o = oracle_binding.SpOracle(case, portable_math=True)
    n = model.execute()
    assert n == o.step(10 ** 6)
    assert model.t == 3.0 and o.t == 3.0
    assert_state_close(model.state(), o.state(), True, "execute")
    assert model.step(5) == 0


def test_gpu_full_size_properties(pkg):
    """The 4M-cell Gaussian-bump workload: a few steps bit for bit against the oracle,
    bit-identical reruns, finite and non-negative depths."""
    case = pkg.workloads.gaussian_bumps(n_cells=4_000_000)
    model = pkg.SpModel(case)
    o = oracle_binding.SpOracle(case, portable_math=True)
    assert model.step(3) == 3 and o.step(3) == 3
    got, want = model.state(), o.state()
    assert_state_close(got, want, True, "4M cells")
    assert np.all(np.isfinite(got[0])) and got[0].min() >= 0.0
    again = pkg.SpModel(case)
    again.step(3)
    for x, y in zip(again.state(), got):
        assert np.array_equal(x.view(np.int64), y.view(np.int64))


@pytest.mark.parametrize("friction", ["manning", "none"])
def test_gpu_c1_dam_break_delaunay_1000_steps(pkg, tmp_path, friction):
    """The plain SP dam break configuration at its stated size: ~20k cells of a seeded
    jittered-Delaunay mesh in a randomly permuted numbering, flat bed, h = 1.0 / 0.1 m, phi ~
    U[0.6, 1], Manning n = 0.03, MUSCL-EVR + the reference's limiter + HLLC, CFL 0.9, walls,
    1000 steps, against the reference's own solver run here on the same case folder.

    * Bit for bit with the reference linked with the portable exp/log of the CUDA build.
    * The reference linked with glibc: with Manning friction (exp and log every step in every wet
      cell) the reference itself moves by ~1e-6 over these 1000 steps when only its libm changes,
      so the GPU (equal to the portable-libm reference) is exactly that far from it, no closer
      and no further.  Without friction the step calls no exp or log (the walls' critical depth
      is exp(-inf) = 0 in both libms) and the glibc reference is matched within 1e-10."""
    case = pkg.workloads.dam_break(n_cells=20000, mesh="delaunay", friction=friction)
    assert 19000 <= case.mesh.cell_nb <= 21000
    if not oracle_binding.reference_available():
        pytest.skip("the reference solver library (oracle/_ref) is not built")
    folder = str(tmp_path / "c1")
    pkg.write_case(folder, case)
    model = pkg.SpModel(case)
    assert model.step(1000) == 1000
    got = model.state()
    ref_pm = oracle_binding.RefSolver(folder, portable_math=True)
    assert ref_pm.step(1000) == 1000
    assert model.t == ref_pm.t
    want_pm = ref_pm.state()
    assert_state_close(got, want_pm, True, "C1 vs reference(portable libm)")
    ref = oracle_binding.RefSolver(folder)
    assert ref.step(1000) == 1000
    want = ref.state()
    if friction == "none":
        assert_state_close(got, want, False, "C1 vs reference(glibc)")
    else:
        for a, b, c in zip(got, want, want_pm):
            assert np.array_equal(np.abs(a - b), np.abs(c - b))   # the reference's own libm sensitivity
    assert got[0].min() >= 0.0 and np.all(np.isfinite(got[0]))


@pytest.mark.parametrize("n_cells", [1_000_000, 4_000_000])
def test_gpu_c2_moving_bumps_vs_oracle(pkg, n_cells):
    """The large SP forward solve's bed under a dam break (free surface 5.0 m for x < 1 km, 3.5 m
    beyond, at rest): a moving, mostly wet flow with wet/dry fronts around the bumps, on the
    jittered-Delaunay mesh, 200 steps bit for bit against the CPU oracle.  The oracle takes
    minutes at these sizes, so tests/golden/make_c2_digest.py ran it once and kept the SHA-256 of
    its final (h, q, r) bits, its t and dt, and a digest of the inputs (which this test checks
    first).  The stored volume sum(phi A h) of the closed basin changes only by round-off and by
    the reference's negative-depth clamp at the wet/dry fronts (h < 0 -> 0, swSpHyp.cpp:197-209)."""
    import hashlib
    import json
    fx = json.load(open(os.path.join(GOLDEN, "c2_moving_digest.json")))[str(n_cells)]
    case = pkg.workloads.gaussian_bumps(n_cells=n_cells, mesh="delaunay", initial="dam")
    m = case.mesh
    d = hashlib.sha256()
    for a in (m.cell_x, m.cell_y, m.cell_z_b, m.cell_area, m.edge_int_cells, m.edge_int_nx, m.edge_int_ny,
              m.edge_int_length, m.edge_bnd_cell, case.h0, case.q0, case.r0, case.phi, case.friction):
        d.update(np.ascontiguousarray(a).tobytes())
    assert d.hexdigest() == fx["inputs_sha256"], "the case's inputs are not the ones the oracle ran"
    model = pkg.SpModel(case)
    w = case.phi * case.mesh.cell_area
    h0 = model.state()[0]
    wet0 = float(np.mean(h0 > 1e-5))
    assert wet0 > 0.75, f"the moving case should be mostly wet ({wet0:.2f})"
    v0 = float(np.sum(w * h0))
    steps = int(fx["steps"])
    assert model.step(steps) == steps
    got = model.state()
    assert model.time == (float(fx["t"]), float(fx["dt"]))
    d = hashlib.sha256()
    for a in got:
        d.update(np.ascontiguousarray(a, np.float64).tobytes())
    assert d.hexdigest() == fx["state_sha256"], f"moving bumps {n_cells} cells: state bits differ from the oracle's"
    moved = float(np.mean(np.abs(got[1]) + np.abs(got[2]) > 1e-6))
    # the dam line at x = 1 km: after 200 steps (about 10 s) the bores have run about 70 m each way
    # over the 2 km basin, so a band of about 1.5 % of the cells moves
    assert moved > 0.01, f"the flow should be moving ({moved:.3f} of the cells)"
    v1 = float(np.sum(w * got[0]))
    # measured 2.1e-9 (1M cells) and 1.2e-10 (4M cells) relative, the oracle's bits included
    assert abs(v1 - v0) / v0 < 1e-8, f"stored volume drifted by {abs(v1 - v0) / v0:.2e}"
