"""Models created by the library's own case-folder loader (sw2d_load_case) run exactly as the
models created from the Python readers' Case: same state, time and time step after the same
steps, for SP, DIP and DDP folders."""
import numpy as np
import pytest

from tests.conftest import load_pkg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


@pytest.mark.parametrize("builder,kwargs", [
    ("dam_break", {"n_cells": 3000}),
    ("channel_features", {"n_cells": 3000, "scheme": "muscl_evr"}),
    ("dip_channel", {"n_cells": 3000}),
    ("ddp_channel", {"n_cells": 3000, "ic": "zuv", "moving": True}),
])
def test_loaded_model_matches(pkg, tmp_path, builder, kwargs):
    case = getattr(pkg.workloads, builder)(**kwargs)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    a = pkg.SpModel(pkg.read_case(folder))
    b = pkg.SpModel.load(folder)
    assert a.step(137) == b.step(137)
    assert a.time == b.time
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x.view(np.int64), y.view(np.int64))
