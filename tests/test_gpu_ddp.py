"""Depth-dependent porosity (DDP) step on the GPU against the reference's own swDdp.

On the GPU box, where the reference library built from its sources travels (oracle/_ref):
* step-by-step parity, bit for bit, of the time, the time step, the state (thetaW, thetaW u,
  thetaW v), every flux array, the wave speeds and the map outputs, against the live reference
  linked with the portable exp/log, over the DDP options (every porosity-law type, friction
  laws, outflow types fr / h / z, singular head loss, momentum dissipation, Boussinesq > 1,
  h/z and q/u initial conditions, and both divergence corrections with their quirks), through
  single launches and through the CUDA-graph path;
* the tabulated porosity laws and thetaG(z_tab[0] + h_min_ddp) against the reference's tables;
* mass conservation with walls only; state round trip; the arguments the reference rejects.
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


def _ref(folder):
    from oracle.binding import RefSolver, reference_available
    if not reference_available():
        pytest.skip("reference library (oracle/_ref) not built")
    return RefSolver(folder, portable_math=True)


CONFIGS = {
    "mixed_fr_manning": dict(n_cells=2500, friction="manning", outflow="fr"),
    "mixed_h_strickler_headloss_diss_zuv": dict(n_cells=2500, friction="strickler", outflow="h", head_loss=True,
                                                 dissipation=True, moving=True, ic="zuv", seed=23),
    "mixed_z_chezy_b11_moving": dict(n_cells=2000, friction="chezy", outflow="z", boussinesq=1.1, moving=True,
                                     seed=25),
    "linear_fr_nofriction_ntab9": dict(n_cells=2000, friction="none", outflow="fr", laws="linear", n_por_tab_max=9,
                                       seed=33),
    "limit_timestep": dict(n_cells=2000, friction="manning", outflow="fr", div_corr="limit_timestep", seed=27),
    "limit_flux": dict(n_cells=2000, friction="manning", outflow="fr", div_corr="limit_flux", n_it_div_max=3,
                       seed=29),
}

FLUXES = ["F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd", "lambda_max_int",
          "lambda_max_bnd"]
OUTPUTS = ["water_depth", "unit_discharge_x", "unit_discharge_y", "surface_elevation"]


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_ddp_matches_live_reference(pkg, tmp_path, name):
    case = pkg.workloads.ddp_channel(t_max=40.0, **CONFIGS[name])
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    ref = _ref(folder)
    model = pkg.SpModel(case)
    model.set_option("record_fluxes", 1)
    model.set_option("record_wave_speeds", 1)
    for a, b in zip(model.state(), ref.state()):  # the initial-condition conversion
        assert _bits_equal(a, b)
    for chunk in (1, 1, 5, 40, 150):
        done = ref.step(chunk)
        if ref.failed:
            # the reference's execute() stops inside the step after `done` (a NaN mass flux,
            # swDdpHyp.cpp:460-483, before the balance): the model reports the same step
            assert model.step(done) == done
            assert model.t == ref.t
            for a, b in zip(model.state(), ref.state()):
                assert _bits_equal(a, b)
            with pytest.raises(pkg.solver.Sw2dError) as e:
                model.step(1)
            assert e.value.code == -3
            return
        assert model.step(chunk) == done
        assert model.t == ref.t and model.dt == ref.dt, (model.t, ref.t, model.dt, ref.dt)
        for k, (a, b) in enumerate(zip(model.state(), ref.state())):
            assert _bits_equal(a, b), (chunk, k, np.flatnonzero(a.view(np.int64) != b.view(np.int64))[:5])
        for nm in FLUXES:
            assert _bits_equal(model.array(nm), ref.array(nm)), nm
        for nm in OUTPUTS:
            assert _bits_equal(model.array(nm), ref.array(nm)), nm


def test_ddp_tables_match_reference(pkg, tmp_path):
    case = pkg.workloads.ddp_channel(n_cells=1500, t_max=1.0, seed=31)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    ref = _ref(folder)
    model = pkg.SpModel(case)
    m = case.mesh
    for which, count in (("cell", m.cell_nb), ("edge_int", m.edge_int_nb), ("edge_bnd", m.edge_bnd_nb)):
        for k in range(count):
            for a, b in zip(model.ddp_table(which, k), ref.ddp_table(which, k)):
                assert _bits_equal(a, b), (which, k)
    assert _bits_equal(model.array("thetaG_int_hmin"), ref.array("thetaG_int_hmin"))


def test_ddp_mass_conservation(pkg):
    """Walls only and a wet bed: sum(thetaW A) is conserved to round-off."""
    case = pkg.workloads.ddp_channel(n_cells=3000, outflow="fr", h_floor=0.3, laws="linear")
    bc = case.bc
    case.bc = type(bc)(codes=bc.codes, types=["q"] * len(bc.codes), times=bc.times, values=np.zeros_like(bc.values))
    model = pkg.SpModel(case)
    A = case.mesh.cell_area

    def mass():
        return float(np.sum(model.state()[0] * A))

    m0 = mass()
    model.step(400)
    assert abs(mass() - m0) <= 1e-12 * m0


def test_ddp_state_roundtrip_then_steps(pkg, tmp_path):
    case = pkg.workloads.ddp_channel(n_cells=1500, friction="manning", moving=True, seed=41)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    ref = _ref(folder)
    model = pkg.SpModel(case)
    ref.step(7)
    th, tu, tv = ref.state()
    model.set_state(th * 1.0, tu, tv)
    model.set_time(ref.t, ref.dt)
    for a, b in zip(model.state(), (th, tu, tv)):
        assert _bits_equal(a, b)
    assert model.step(20) == ref.step(20)
    for a, b in zip(model.state(), ref.state()):
        assert _bits_equal(a, b)


def test_ddp_rejections(pkg):
    err = pkg.solver.Sw2dError
    case = pkg.workloads.ddp_channel(n_cells=600, seed=43)
    case.opts["num_scheme"] = "muscl_evr"
    with pytest.raises(err) as e:
        pkg.SpModel(case)
    assert e.value.code == -8
    case = pkg.workloads.ddp_channel(n_cells=600, seed=43)
    recs = case.ddp_edge_int
    vals = recs.values.copy()
    r0 = recs.record(0)
    k = int(recs.offset[0])
    vals[k + 3] = 1.5 if r0[0] != -2 else 1.5  # a porosity above 1
    case.ddp_edge_int = type(recs)(recs.offset, vals)
    with pytest.raises(err) as e:
        pkg.SpModel(case)
    assert e.value.code == -1


def test_ddp_unknown_boundary_type_stops(pkg):
    case = pkg.workloads.ddp_channel(n_cells=600, seed=45)
    bc = case.bc
    types = list(bc.types)
    types[2] = "phiWq"  # DIP only
    case.bc = type(bc)(codes=bc.codes, types=types, times=bc.times, values=bc.values)
    model = pkg.SpModel(case)
    with pytest.raises(pkg.solver.Sw2dError) as e:
        model.step(1)
    assert e.value.code == -6
