"""The host side of the porosity assimilation (porosity.py) against the reference's own readers
(assim/assimConfig.cpp, swSpE::load_all_observations, swSpE::load_phi_csv, through
oracle/ref_e_driver.cpp) on the reference's case sp_toce, and the penalties of PorosityProblem
against central differences.  The reference comparisons need the reference sources (present in
the build container) and skip elsewhere."""
import os

import numpy as np
import pytest

from tests.conftest import load_pkg, reference_case, reference_missing

CASE = reference_case("sp_toce")


def _ref():
    from oracle.binding import RefE, REF_E_SO
    if not os.path.isdir(CASE) or not os.path.exists(REF_E_SO):
        pytest.skip(reference_missing() or "the reference assimilation library (oracle/_ref) is not built")
    return RefE(CASE)


def test_config_matches_reference_parser():
    pkg = load_pkg()
    ref = _ref()
    rc = ref.config()
    case = pkg.read_case(CASE)
    c = pkg.porosity.AssimConfig.from_opts(case.opts)
    assert c.checkpoint_stride == rc["checkpoint_stride"] and c.windowed_assimilation == bool(rc["windowed"])
    assert c.assimilation_window_duration == rc["window_duration"] and c.assimilation_window_steps == rc["window_steps"]
    assert c.n_assimilation_windows == rc["n_windows"] and c.t_state_assimilation == rc["t_state_assimilation"]
    assert c.cost_normalize == bool(rc["cost_normalize"]) and c.phi_transform == "none" and rc["phi_transform"] == 0
    assert c.lambda_tanh == rc["lambda_tanh"] and c.dt_map_ad == rc["dt_map_ad"] and c.alpha_reg == rc["alpha_reg"]
    assert c.minimize_algo == "lbfgsb" and c.max_it == 50 and c.porosity_ebauche_map == "input/phi_init_ones.txt"


def test_observations_match_reference_reader():
    pkg = load_pkg()
    ref = _ref()
    t_ref, f_ref = ref.load_observations()
    n = ref.n
    t, f = pkg.porosity.load_observations(CASE, n, 10.0, 30.0)
    assert np.array_equal(t, t_ref)
    assert np.array_equal(f.view(np.int64), f_ref.view(np.int64))
    assert pkg.porosity.time_from_file_name("ResultHydro_p0001d02h03m04s056.txt") == 0.056 + 4 + 60 * (3 + 60 * (2 + 24))


def test_maps_match_reference_reader(tmp_path):
    pkg = load_pkg()
    ref = _ref()
    for name in ("phi_init_ones.txt", "SP_cell_porosity_map.txt", "phi_init_ebauche.txt"):
        path = os.path.join(CASE, "input", name)
        assert np.array_equal(pkg.porosity.load_map(path, ref.n), ref.load_phi_map(path))
    csv = tmp_path / "m.csv"
    vals = np.linspace(0.1, 0.9, ref.n)
    csv.write_text("cell_id,phi\n" + "\n".join(f"{i},{float(v)!r}" for i, v in enumerate(vals)) + "\n")
    assert np.array_equal(pkg.porosity.load_map(str(csv), ref.n), ref.load_phi_map(str(csv)))


class _FakeSpE:
    """J_data = sum(c * phi^2), with the transform of porosity.SpE."""

    def __init__(self, pkg, n, transform):
        cfg = pkg.porosity.AssimConfig(phi_transform=transform, alpha_l1=0.3, alpha_spatial=0.7, alpha_phi_ref=0.2,
                                       lambda_tanh=1.3)
        self.cfg = cfg
        self.n = n
        mesh = pkg.mesh.jittered_triangle_mesh(4, 3, 4.0, 3.0, seed=1)
        self.n = mesh.cell_nb

        class _M:
            pass

        self.model = _M()
        self.model.case = type("C", (), {"mesh": mesh})()
        self._c = np.linspace(0.5, 1.5, self.n)
        self.diag = {}
        self._spe = pkg.porosity.SpE.__new__(pkg.porosity.SpE)
        self._spe.cfg = cfg

    def phi_correct(self, m):
        return self._spe.phi_correct(m)

    def dphi_dm(self, m):
        return self._spe.dphi_dm(m)

    def m_from_phi(self, p):
        return self._spe.m_from_phi(p)

    def get_spatial_gradient_checkpointed(self, m, stride=None):
        phi = self.phi_correct(m)
        self.diag = {"J": float(np.sum(self._c * phi * phi)), "grad_l2": 0.0, "grad_max": 0.0, "grad_argmax": 0,
                     "dh_peak": 0.0}
        return 2.0 * self._c * phi * self.dphi_dm(m)

    def replay_trajectory_cost(self, m):
        phi = self.phi_correct(m)
        return float(np.sum(self._c * phi * phi))


@pytest.mark.parametrize("transform", ["none", "clamp", "tanh"])
def test_porosity_problem_gradient(transform):
    pkg = load_pkg()
    spe = _FakeSpE(pkg, 0, transform)
    rng = np.random.default_rng(3)
    phi_b = rng.uniform(0.4, 0.9, spe.n)
    prob = pkg.porosity.PorosityProblem(spe, phi_b, alpha_reg=0.5, phi_ref=rng.uniform(0.3, 1.0, spe.n), stride=1)
    spe.cfg.alpha_spatial = 0.0   # grad()'s J leaves the spatial term out (the reference's own J)
    theta = prob.theta_start() + rng.uniform(-0.05, 0.05, prob.size())
    J, g = prob.grad(theta)
    d = rng.standard_normal(prob.size())
    e = 1e-6
    fd = (prob.grad(theta + e * d)[0] - prob.grad(theta - e * d)[0]) / (2 * e)
    assert abs(fd - g @ d) <= 1e-6 * max(1.0, abs(fd))
    assert abs(prob.func(theta) - J) < 1e-12


def test_lbfgsb_probe_freezes_the_truncation_window():
    """run_minimization with L-BFGS-B and freeze_window (assim/swSpE_minimize.cpp:881-909): one probe evaluation at
    the start point, whose truncation segment + 1 becomes every gradient's first segment for the
    whole solve and is released after it; the probe and the solver's first evaluation are the same
    point (the reference's descent log opens with two equal rows); J_final is the solver's value."""
    pkg = load_pkg()
    spe = _FakeSpE(pkg, 0, "none")
    cfg = spe.cfg
    cfg.alpha_l1 = cfg.alpha_spatial = cfg.alpha_phi_ref = 0.0
    cfg.minimize_algo, cfg.max_it = "lbfgsb", 20
    frozen = []
    spe.set_forced_first_segment = frozen.append
    exact = spe.get_spatial_gradient_checkpointed

    def gradient(m, stride=None):
        g = exact(m, stride)
        spe.diag["truncation_segment"] = 6 if not frozen else 40   # the probe's truncation: segment 6
        return g

    spe.get_spatial_gradient_checkpointed = gradient
    res = pkg.porosity.run_minimization(spe, np.full(spe.n, 0.8), freeze_window=True)
    assert frozen == [7, -1]
    assert res["history"][0] == res["history"][1]
    assert res["J_final"] <= 1e-3 * res["J_init"]
    assert res["n_grad"] == len(res["history"])
    frozen.clear()
    res = pkg.porosity.run_minimization(spe, np.full(spe.n, 0.8))   # the default: each gradient's own window
    assert frozen == [] and res["J_final"] <= 1e-3 * res["J_init"]


def test_free_cells_zone_map(tmp_path):
    """porosity_free_zone_map (assim/swSpE_minimize.cpp:648-668): of the cells the dry mask leaves
    free (here all), only those whose zone value is below 0.5; an unreadable map leaves the set
    unchanged and is reported; an empty zone is reported."""
    from types import SimpleNamespace
    pkg = load_pkg()
    por = pkg.porosity
    n = 6
    (tmp_path / "zone.csv").write_text("cell_id,value\n" + "".join(f"{i},{v}\n" for i, v in
                                                                 enumerate([0, 1, 0.2, 0.7, 0.49, 1])))
    cfg = por.AssimConfig(porosity_free_zone_map="zone.csv")
    spe = SimpleNamespace(cfg=cfg, n=n, folder=str(tmp_path), diag={})
    assert por.free_cells(spe, np.ones(n)).tolist() == [0, 2, 4]
    assert spe.diag["porosity_free_zone_map"] == {"free_in_zone": 3, "free_before": 6}
    spe = SimpleNamespace(cfg=por.AssimConfig(porosity_free_zone_map="missing.csv"), n=n, folder=str(tmp_path), diag={})
    assert por.free_cells(spe, np.ones(n)).tolist() == list(range(n)) and "zone_map_error" in spe.diag
    (tmp_path / "none.csv").write_text("".join(f"{i},1\n" for i in range(n)))
    spe = SimpleNamespace(cfg=por.AssimConfig(porosity_free_zone_map="none.csv"), n=n, folder=str(tmp_path), diag={})
    assert por.free_cells(spe, np.ones(n)).size == 0 and "empty zone" in spe.diag["zone_map_error"]


def test_reference_map_file_name_and_format(tmp_path):
    """swIO::computeFileNameFromTime and createTxtFileMapDecimal, restated: the names and layout of
    the observation maps the reference's gen-ref-e mode writes (reference/ResultHydro_p*.txt)."""
    por = load_pkg().porosity
    assert por.result_file_name("ResultHydro_p", 10.0) == "ResultHydro_p0000d00h00m10s000.txt"
    assert por.result_file_name("ResultHydro_p", 29.5) == "ResultHydro_p0000d00h00m29s500.txt"
    assert por.result_file_name("ResultHydro_p", 90061.25) == "ResultHydro_p0001d01h01m01s250.txt"
    path = str(tmp_path / "m.txt")
    por.write_map_decimal(path, ["x", "unit_discharge_norm"], [np.array([7.006166665, -0.0]), np.array([1e-7, 2.5])], 10)
    lines = open(path).read().split("\n")
    assert lines[0] == "x" + " " * 16 + "\t" + "unit_discharge_norm\t"
    assert lines[1] == "7.0061666650e+00\t1.0000000000e-07\t"
    assert lines[2] == "-0.0000000000e+00\t2.5000000000e+00\t"
