"""The binary map file's header (sw2d_result_header, host only) against the file the reference's
own solver writes (oracle/_ref/sw2dSolver_pm, output_format bin): the header is the file's prefix
byte for byte, for SP, DIP and DDP and each map_storage_mode; the rest of the reference's file
is whole frames of the stated layout (tests/result_file.py), at the times swSp::execute stores
maps.  tests/test_gpu_result.py compares whole files written by runs on the GPU."""
import copy
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import load_pkg
from tests.result_file import read_result

PKG = load_pkg()
oracle_binding = pytest.importorskip("oracle.binding")
needs_cli = pytest.mark.skipif(not os.path.exists(oracle_binding.REF_BIN_PM), reason="reference solver not built")

NAMES = {
    "default": ["bottom_elevation", "water_depth", "unit_discharge_x", "unit_discharge_y", "unit_discharge_norm"],
    "all": ["bottom_elevation", "water_depth", "unit_discharge_x", "unit_discharge_y", "unit_discharge_norm",
            "surface_elevation", "velocity_x", "velocity_y", "velocity_norm", "froude", "specific_head",
            "total_head", "phi_by_water_depth", "phi_by_unit_discharge_x", "phi_by_unit_discharge_y",
            "phi_by_unit_discharge_norm"],
    "none": ["bottom_elevation"],
}
MODEL = {"sp": 0, "dip": 1, "ddp": 2}


def result_case(kind, mode, dt_map="0.1", t_max="0.5"):
    """A small case of each model (Manning friction: the reference runs with the portable exp and
    log of the library, sw2dSolver_pm)."""
    w = PKG.workloads
    if kind == "sp":
        case = w.dam_break(n_cells=900, scheme="muscl_evr", seed_mesh=31, seed_phi=32)
    elif kind == "dip":
        case = w.dip_channel(n_cells=900)
    else:
        case = w.ddp_channel(n_cells=900, laws="linear")
    case = copy.copy(case)
    case.opts = dict(case.opts, output_format="bin", store_flag=mode, dt_map=dt_map,
                     t_max=t_max, t_0="0")
    return case


def run_reference(folder, case):
    """The reference solver (portable exp/log) on the written case; returns (its ResultHydro.bin,
    geometry.sw2d)."""
    PKG.write_case(folder, case)
    os.makedirs(os.path.join(folder, "output"), exist_ok=True)
    res = subprocess.run([oracle_binding.REF_BIN_PM, folder], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    with open(os.path.join(folder, "output", "ResultHydro.bin"), "rb") as fh:
        data = fh.read()
    with open(os.path.join(folder, "input", "geometry.sw2d"), "rb") as fh:
        geo = fh.read()
    return data, geo


@needs_cli
@pytest.mark.parametrize("kind,mode", [("sp", "default"), ("sp", "all"), ("sp", "none"), ("dip", "default"),
                                       ("dip", "all"), ("ddp", "default"), ("ddp", "all")])
def test_header_is_the_reference_files_prefix(tmp_path, kind, mode):
    case = result_case(kind, mode)
    data, geo = run_reference(str(tmp_path / "case"), case)
    ours = str(tmp_path / "ours.bin")
    lib = PKG.capi.load_library()
    geo_path = str(tmp_path / "case" / "input" / "geometry.sw2d")
    assert lib.sw2d_result_header(ours.encode(), geo_path.encode(), MODEL[kind], PKG.capi.RESULT_MODES[mode],
                                  0.0, 0.5, 0.1) == 0
    with open(ours, "rb") as fh:
        head = fh.read()
    assert data[:len(head)] == head
    names, times_cfg, times, frames = read_result(data, geo, case.mesh.cell_nb)
    expect = list(NAMES[mode])
    if kind == "ddp":  # swDdp::init's names (swDdp.cpp:794-805)
        expect[4] = "unit_disch_norm" if mode == "default" else "unit_disc_norm"
        if mode == "all":
            expect[12:] = ["phi_by_wat_depth", "phi_by_disc_x", "phi_by_disc_y", "phi_by_disc_norm"]
    assert names == expect
    assert times_cfg == (0.0, 0.5, 0.1)
    if mode == "none":
        assert len(times) == 0
        return
    # the run's first map, the storage times, and the last map (stored twice when t_max is one;
    # the DDP step snaps dt to the maps from the integer part of t, swDdpHyp.cpp:588-600, so
    # within 1 s it stores none between the first and the last)
    assert times[0] == 0.0 and times[-1] == 0.5
    if kind == "ddp":
        assert list(times) == [0.0, 0.5]
    else:
        assert times[-2] == 0.5 and len(times) >= 5
    assert np.all(np.diff(times) >= 0)
    # the first frame is the initial state, z_b first (DDP: the depth comes back from the volume)
    if kind != "ddp":
        np.testing.assert_array_equal(frames[0][:, 1], case.h0 if np.ndim(case.h0) else np.full(case.mesh.cell_nb, case.h0))


def test_header_rejects_bad_arguments(tmp_path):
    lib = PKG.capi.load_library()
    assert lib.sw2d_result_header(str(tmp_path / "x.bin").encode(), b"/nonexistent/geometry.sw2d", 0, 0, 0.0, 1.0,
                                  1.0) == -1
    assert lib.sw2d_result_header(str(tmp_path / "x.bin").encode(), b"g", 0, 3, 0.0, 1.0, 1.0) == -1
    assert lib.sw2d_result_header(str(tmp_path / "x.bin").encode(), b"g", 3, 0, 0.0, 1.0, 1.0) == -1
