"""The binary map file written by runs on the GPU (sw2d_result_open + sw2d_execute) against the
reference solver's own ResultHydro.bin on the same case folder: the whole file byte for byte,
for SP, DIP and DDP, map_storage_mode default / all / none, maps every 0.1 s or every step, the
case read by the library's loader (SpModel.load) or created from Python."""
import os
import shutil

import pytest

from tests.conftest import load_pkg
from tests.test_result_file import needs_cli, result_case, run_reference

pytestmark = pytest.mark.gpu
PKG = load_pkg()


@needs_cli
@pytest.mark.parametrize("kind,mode,dt_map", [("sp", "default", "0.1"), ("sp", "all", "-1"), ("sp", "none", "0.1"),
                                              ("dip", "default", "0.05"), ("dip", "all", "0.1"),
                                              ("ddp", "default", "0.1"), ("ddp", "all", "-1")])
def test_file_equals_the_reference_solvers(tmp_path, kind, mode, dt_map):
    PKG.build.build()
    case = result_case(kind, mode, dt_map=dt_map)
    ref_folder = str(tmp_path / "ref")
    data, _ = run_reference(ref_folder, case)
    ours = str(tmp_path / "ours")
    shutil.copytree(os.path.join(ref_folder, "input"), os.path.join(ours, "input"))
    m = PKG.SpModel.load(ours, results=True)
    m.execute()
    m.result_close()
    with open(os.path.join(ours, "output", "ResultHydro.bin"), "rb") as fh:
        got = fh.read()
    assert len(got) == len(data)
    assert got == data


@needs_cli
def test_python_created_model_and_reopen(tmp_path):
    """A model created from Python arrays writes the same file; closing twice is harmless; a
    second file opened on the same model restarts with the header."""
    PKG.build.build()
    case = result_case("sp", "default")
    data, geo = run_reference(str(tmp_path / "ref"), case)
    geo_path = str(tmp_path / "ref" / "input" / "geometry.sw2d")
    m = PKG.SpModel(case)
    out = str(tmp_path / "a.bin")
    m.result_open(out, geo_path, "default")
    m.execute()
    m.result_close()
    m.result_close()
    with open(out, "rb") as fh:
        assert fh.read() == data
    with pytest.raises(Exception):
        m.result_open(str(tmp_path / "b.bin"), str(tmp_path / "missing.sw2d"), "default")
