"""The reference-side binding of INTEGRATION.md, compiled against the reference's own headers and
objects (oracle/b200_binding.cpp -> oracle/_ref/libsw2d_b200_binding.so): the reference reads a
case folder with its own swSp (swSp::init: input.solv, geometry.sw2d, maps, boundary series), the
model class swSpB200 hands the tables to the GPU through the C ABI and runs the whole time loop
there.  Its final state is compared with the reference's own solver (swSp's time loop on the
CPU) on the same folder: bit for bit with the reference linked with the portable exp/log the
CUDA build uses, within 1e-10 relative of the reference linked with glibc where the case is
insensitive to the last bit of exp/log."""
import os

import pytest

from tests.conftest import assert_state_close, load_pkg

pytestmark = pytest.mark.gpu

oracle_binding = pytest.importorskip("oracle.binding")

CASES = {
    "dam_muscl_manning_delaunay": ("dam_break", {"n_cells": 6000, "mesh": "delaunay", "t_max": 4.0}, True),
    "chan_godunov_blend_strickler_headloss_fr": ("channel_features", {"n_cells": 2500, "t_max": 6.0}, False),
    "chan_muscl_disc_chezy_z": ("channel_features", {"n_cells": 2500, "scheme": "muscl_evr", "topo": "discontinuous",
                                                     "friction": "chezy", "outflow": "z", "t_max": 6.0}, False),
}


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    return p


@pytest.mark.parametrize("name", sorted(CASES))
def test_binding_runs_the_reference_case_on_the_gpu(pkg, tmp_path, name):
    if not (oracle_binding.reference_available() and os.path.exists(oracle_binding.B200_BINDING_SO)):
        pytest.skip("the reference solver library or the compiled binding (oracle/_ref) is not built")
    kind, kwargs, libm_stable = CASES[name]
    case = getattr(pkg.workloads, kind)(**kwargs)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    b = oracle_binding.B200Binding(folder)
    n = b.execute()
    got = b.state()
    b.close()
    ref = oracle_binding.RefSolver(folder, portable_math=True)
    assert ref.step(10 ** 8) == n
    assert ref.t == float(kwargs["t_max"])
    assert_state_close(got, ref.state(), True, f"{name}: binding vs reference (portable libm)")
    if libm_stable:
        ref_g = oracle_binding.RefSolver(folder)
        ref_g.step(10 ** 8)
        assert_state_close(got, ref_g.state(), False, f"{name}: binding vs reference (glibc)")
