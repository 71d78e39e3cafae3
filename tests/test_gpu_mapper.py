"""The porosity mapper on the GPU (porosity_mapper.map_folder over sw2d_map_porosity) against
the reference's mapper program on the same case folder: every map file byte for byte (values
printed with 6 significant digits, as the reference prints them), for SP, DIP and DDP, on
hand-placed footprints, on a seeded building layout and on a raster of block buildings; and the
arrays against the reference's
values to 5e-6."""
import os
import shutil
import time

import numpy as np
import pytest

from tests.conftest import load_pkg
from tests.test_mapper import FILES, _values, mapper_case, needs_mapper, raster_case, run_reference_mapper

pytestmark = pytest.mark.gpu
PKG = load_pkg()


@needs_mapper
@pytest.mark.parametrize("urban", [False, True, "raster"], ids=["footprints", "layout", "raster"])
@pytest.mark.parametrize("model", ["sp", "dip", "ddp"])
def test_maps_equal_the_reference_mappers(tmp_path, model, urban):
    PKG.build.build()
    ref_folder = str(tmp_path / "ref")
    if urban == "raster":
        raster_case(ref_folder, model)
    else:
        mapper_case(ref_folder, model, n_cells=6000 if urban else 900, urban=urban)
    t0 = time.perf_counter()
    ref = run_reference_mapper(ref_folder)
    t_ref = time.perf_counter() - t0
    ours = str(tmp_path / "ours")
    shutil.copytree(ref_folder, ours, ignore=shutil.ignore_patterns("*porosity_map.txt"))
    t0 = time.perf_counter()
    res = PKG.porosity_mapper.map_folder(ours)
    t_ours = time.perf_counter() - t0
    print(model, urban, "reference", round(t_ref, 3), "s, ours", round(t_ours, 3), "s")
    for fn, key in zip(FILES[model], ["cell", "edge_bnd", "edge_int"]):
        with open(os.path.join(ours, "input", fn)) as fh:
            got = fh.read()
        want_vals, _ = _values(ref[fn], model == "ddp")
        assert np.max(np.abs(res[key] - want_vals)) <= 5e-6, fn
        assert got == ref[fn], fn
    assert res["cell"].min() < 0.99  # the buildings do cut the cells
