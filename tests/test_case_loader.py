"""The library's own case-folder loader (csrc/sw2d_case.cpp: sw2d_case_read / sw2d_load_case)
against the Python readers of case.py, which restate the reference's readers: every table and
field the C ABI hands to the model, bit for bit, for SP, DIP and DDP folders and for the
reference's own functional case sp_toce (when the reference tree is present).  CPU only: the
reading needs no GPU.  tests/test_gpu_case_loader.py runs the loaded models."""
import os

import numpy as np
import pytest

from tests.conftest import load_pkg, reference_case, reference_missing

PKG = load_pkg()


@pytest.fixture(scope="module", autouse=True)
def built():
    PKG.build.build()


def _eq(a, b):
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def _check(folder):
    case = PKG.read_case(folder)
    cf = PKG.capi.CaseFolder(folder)
    m = case.mesh
    assert (cf.cell_nb, cf.edge_int_nb, cf.edge_bnd_nb) == (m.cell_nb, m.edge_int_nb, m.edge_bnd_nb)
    pairs = {"cell_area": m.cell_area, "cell_x": m.cell_x, "cell_y": m.cell_y, "cell_z_b": m.cell_z_b,
             "edge_int_cells": m.edge_int_cells, "edge_int_length": m.edge_int_length, "edge_int_nx": m.edge_int_nx,
             "edge_int_ny": m.edge_int_ny, "edge_int_mx": m.edge_int_mx, "edge_int_my": m.edge_int_my,
             "edge_int_mz": m.edge_int_mz, "edge_bnd_cell": m.edge_bnd_cell, "edge_bnd_length": m.edge_bnd_length,
             "edge_bnd_nx": m.edge_bnd_nx, "edge_bnd_ny": m.edge_bnd_ny, "edge_bnd_mz": m.edge_bnd_mz,
             "edge_bnd_code": m.edge_bnd_code, "boussinesq": case.boussinesq,
             "h0": case.h0, "q0": case.q0, "r0": case.r0, "bc_code": case.bc.codes,
             "bc_times": np.tile(case.bc.times, len(case.bc.codes)), "bc_values": np.asarray(case.bc.values)}
    if not case.is_ddp:
        pairs["phi"] = case.phi
    if case.friction is not None:
        pairs.update({"friction_1": case.friction[0], "friction_2": case.friction[1], "friction_alpha": case.friction[2]})
    if case.head_loss is not None:
        pairs.update({"hl_h_sing": case.head_loss[0], "hl_coeff_1": case.head_loss[1],
                      "hl_coeff_2": case.head_loss[2], "hl_alpha": case.head_loss[3]})
    if case.mu is not None:
        pairs.update({"mu_1": case.mu[0], "mu_2": case.mu[1], "mu_alpha": case.mu[2]})
    if case.is_dip:
        pairs.update({"phi_g_int": case.phi_g_int, "phi_g_bnd": case.phi_g_bnd})
    if case.is_ddp:
        for key, laws in (("cell", case.ddp_cell), ("edge_int", case.ddp_edge_int), ("edge_bnd", case.ddp_edge_bnd)):
            pairs[f"ddp_{key}_offset"] = laws.offset
            pairs[f"ddp_{key}_values"] = laws.values
        cols = (1 if case.ddp_ic[0] == "z" else 0) | (2 if case.ddp_ic[1] == "u" else 0) | \
               (4 if case.ddp_ic[2] == "v" else 0)
        assert cf.ic_columns == cols
    for name, want in pairs.items():
        assert _eq(cf.array(name), want), name
    types = [PKG.case.BC_TYPES.get(t, 99) for t in case.bc.types]
    assert _eq(cf.array("bc_type"), types)
    assert cf.model == {"sp": 0, "dip": 1, "ddp": 2}[str(case.opts["model_hyperb"]).lower()]
    for k, v in case.opts.items():
        got = cf.option(k)
        # keys absent from the file: the Python reader fills swSolverParam.h's defaults
        assert got == str(v) if got is not None else str(v) == PKG.case.SOLV_DEFAULTS.get(k), k
    cf.close()


CASES = {
    "dam_sp": lambda W: W.dam_break(n_cells=800),
    "chan_sp_headloss_strickler_fr": lambda W: W.channel_features(n_cells=700),
    "chan_sp_chezy_z": lambda W: W.channel_features(n_cells=700, friction="chezy", outflow="z", boussinesq=1.1),
    "dip_dissipation": lambda W: W.dip_channel(n_cells=700),
    "ddp_mixed_zuv_limit_flux": lambda W: W.ddp_channel(n_cells=600, ic="zuv", moving=True, div_corr="limit_flux",
                                                        dissipation=True, head_loss=True, friction="strickler"),
    "ddp_linear_hqr": lambda W: W.ddp_channel(n_cells=600, laws="linear"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_loader_reads_what_the_python_readers_read(tmp_path, name):
    case = CASES[name](PKG.workloads)
    folder = str(tmp_path / name)
    PKG.write_case(folder, case)
    _check(folder)


def test_loader_reads_sp_toce():
    src = reference_case("sp_toce")
    if not os.path.isdir(src):
        pytest.skip(reference_missing() or "the reference's functional case sp_toce is missing")
    _check(src)


def test_loader_reports_missing_files(tmp_path):
    case = PKG.workloads.dam_break(n_cells=400)
    folder = str(tmp_path / "c")
    PKG.write_case(folder, case)
    os.remove(os.path.join(folder, "input", "Boussinesq_map.txt"))
    with pytest.raises(ValueError, match="Boussinesq_map"):
        PKG.capi.CaseFolder(folder)
    with open(os.path.join(folder, "input", "Boussinesq_map.txt"), "w") as fh:
        fh.write("Unif\t1\n==== Default Param\nBeta\tgamma\n1.0\t2.0\n")
    with pytest.raises(ValueError, match="expecting 1 parameters"):
        PKG.capi.CaseFolder(folder)
