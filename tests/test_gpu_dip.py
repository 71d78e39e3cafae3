"""Dual integral porosity (DIP) step on the GPU against the reference's own swDip.

The golden fixtures (tests/golden/dip_*.npz, made by the reference) are covered by
test_gpu_parity.test_gpu_matches_reference_golden.  These tests add, on the GPU box where the
reference library built from its sources travels (oracle/_ref):
* step-by-step parity, bit for bit, of the state and of every flux array, against the live
  reference linked with the portable exp/log, over the DIP options (schemes, topographies,
  inflow types q / phiWq, outflow types fr / h / z, momentum dissipation on and off);
* mass conservation (sum of phiW h A with walls only);
* the error the reference stops on (connectivity porosity below 1e-16 in a specific force).
"""
import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


CONFIGS = [
    dict(scheme="muscl_evr", topo="discontinuous", friction="manning", inflow="q", outflow="fr", dissipation=True),
    dict(scheme="godunov", topo="blending", friction="strickler", inflow="phiWq", outflow="h", dissipation=False),
    dict(scheme="muscl_evr", topo="blending", friction="chezy", inflow="q", outflow="z", dissipation=True,
         boussinesq=1.1),
    dict(scheme="godunov", topo="discontinuous", friction="none", inflow="phiWq", outflow="fr", dissipation=True),
]

FLUXES = ["F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd", "lambda_max_int",
          "lambda_max_bnd"]


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(str(v) for v in c.values()))
def test_dip_matches_live_reference(pkg, tmp_path, cfg):
    from oracle.binding import RefSolver, reference_available
    if not reference_available():
        pytest.skip("reference library (oracle/_ref) not built")
    case = pkg.workloads.dip_channel(n_cells=2500, **cfg)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    ref = RefSolver(folder, portable_math=True)
    model = pkg.SpModel(case)
    model.set_option("record_fluxes", 1)
    model.set_option("record_wave_speeds", 1)
    for chunk in (1, 1, 5, 40, 150):
        assert model.step(chunk) == ref.step(chunk)
        assert model.t == ref.t and model.dt == ref.dt
        for a, b in zip(model.state(), ref.state()):
            assert _bits_equal(a, b)
        for name in FLUXES:
            assert _bits_equal(model.array(name), ref.array(name)), name


def test_dip_mass_conservation(pkg):
    """Walls only and a wet bed (a wet/dry front adds mass through the negative-depth clamp,
    in the reference as here): the storage sum of phiW h A is conserved to round-off."""
    case = pkg.workloads.dip_channel(n_cells=3000, inflow="q", outflow="fr")
    bc = case.bc
    case.bc = type(bc)(codes=bc.codes, types=["q"] * len(bc.codes), times=bc.times, values=np.zeros_like(bc.values))
    case.h0 = 1.0 - case.mesh.cell_z_b + 0.05 * (case.mesh.cell_x < 20.0)
    model = pkg.SpModel(case)
    A = case.mesh.cell_area * case.phi

    def mass():
        return float(np.sum(model.state()[0] * A))

    m0 = mass()
    model.step(500)
    assert abs(mass() - m0) <= 1e-12 * m0


def test_dip_reports_zero_connectivity(pkg):
    """phiG = 0 on a wet boundary edge: the reference stops in specificForce
    (dip/swDip.cpp:1524-1528); the GPU step returns SW2D_E_PHIG."""
    case = pkg.workloads.dip_channel(n_cells=2000, inflow="q", outflow="fr")
    wet = case.h0[case.mesh.edge_bnd_cell] > 0.05
    k = int(np.flatnonzero(wet)[0])
    case.phi_g_bnd = case.phi_g_bnd.copy()
    case.phi_g_bnd[k] = 0.0
    model = pkg.SpModel(case)
    with pytest.raises(pkg.Sw2dError) as err:
        model.step(1)
    assert err.value.code == -10


def test_dip_rejects_connectivity_above_storage(pkg):
    case = pkg.workloads.dip_channel(n_cells=2000)
    case.phi_g_int = case.phi_g_int.copy()
    L = case.mesh.edge_int_cells[0, 0]
    case.phi_g_int[0] = min(1.0, case.phi[L] + 0.1)
    with pytest.raises(pkg.Sw2dError) as err:
        pkg.SpModel(case)
    assert err.value.code == -1


def test_dip_adjoint_not_available(pkg):
    model = pkg.SpModel(pkg.workloads.dip_channel(n_cells=1000))
    with pytest.raises(pkg.Sw2dError) as err:
        model.record(5, 5)
    assert err.value.code == -8
