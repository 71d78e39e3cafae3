"""The CPU oracle (oracle/sp_oracle.c) pinned against the reference's own outputs.

* golden fixtures made by the reference compiled from its sources (tests/golden/);
* when the reference tree is present here, live step-by-step comparison with it.
Both bit for bit: the restatement keeps the reference's operand order and the host libm.
"""
import os
import shutil

import numpy as np
import pytest

from tests.conftest import golden_case, golden_names, load_pkg, sp_toce_case
from tests.golden.make_golden import DDP_BUILDERS, DIP_BUILDERS

oracle_binding = pytest.importorskip("oracle.binding")


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle_binding.build(reference=os.path.isdir(os.path.join(oracle_binding.REFERENCE_SRC, "src")))


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


@pytest.mark.parametrize("portable", [False, True], ids=["libm", "portable_math"])
@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_golden(name, portable):
    """The oracle with the host libm against the reference linked with glibc, and the oracle
    with the portable exp/log against the reference objects linked with them.  The C oracle
    restates the SP step; the DIP and DDP fixtures are pinned to the live reference instead (the
    reference re-run here must reproduce them bit for bit; the DDP host composition of
    tests/test_ddp_host.py is checked against them too)."""
    case, fx = golden_case(name)
    sfx = "_pm" if portable else ""
    if str(fx["builder"]) in DIP_BUILDERS | DDP_BUILDERS:
        if not oracle_binding.reference_available():
            pytest.skip("DIP and DDP fixtures are pinned to the live reference, whose library (oracle/_ref) is not built")
        import tempfile
        folder = tempfile.mkdtemp(prefix="sw2d_dip_")
        load_pkg().write_case(folder, case)
        ref = oracle_binding.RefSolver(folder, portable_math=portable)
        assert ref.step(int(fx["steps"])) == int(fx["steps"])
        h, q, r = ref.state()
        assert ref.t == float(fx["t" + sfx])
        assert _bits_equal(h, fx["h" + sfx]) and _bits_equal(q, fx["q" + sfx]) and _bits_equal(r, fx["r" + sfx])
        return
    o = oracle_binding.SpOracle(case, portable_math=portable)
    assert o.step(int(fx["steps"])) == int(fx["steps"])
    h, q, r = o.state()
    assert o.t == float(fx["t" + sfx]) and o.dt == float(fx["dt" + sfx])
    assert _bits_equal(h, fx["h" + sfx]) and _bits_equal(q, fx["q" + sfx]) and _bits_equal(r, fx["r" + sfx])


@pytest.mark.parametrize("portable", [False, True], ids=["libm", "portable_math"])
def test_oracle_matches_reference_sp_toce(portable):
    case, fx = sp_toce_case()
    sfx = "_pm" if portable else ""
    o = oracle_binding.SpOracle(case, portable_math=portable)
    assert o.step(100) == int(fx["steps100"])
    h, q, r = o.state()
    assert o.t == float(fx["t100" + sfx])
    assert _bits_equal(h, fx["h100" + sfx]) and _bits_equal(q, fx["q100" + sfx]) and _bits_equal(r, fx["r100" + sfx])
    n = o.step(10 ** 7)
    assert 100 + n == int(fx["steps_end" + sfx]) and o.t == float(fx["t_end" + sfx])
    h, q, r = o.state()
    assert _bits_equal(h, fx["h_end" + sfx]) and _bits_equal(q, fx["q_end" + sfx])
    assert _bits_equal(r, fx["r_end" + sfx])


needs_ref = pytest.mark.skipif(not oracle_binding.reference_available(),
                               reason="the reference solver library (oracle/_ref) is not built")


@needs_ref
@pytest.mark.parametrize("portable", [False, True], ids=["libm", "portable_math"])
@pytest.mark.parametrize("kind,kwargs", [
    ("dam_break", {"n_cells": 900, "seed_mesh": 11, "seed_phi": 12}),
    ("gaussian_bumps", {"n_cells": 1500, "seed_mesh": 13}),
    ("channel_features", {"n_cells": 1200, "scheme": "muscl_evr", "outflow": "fr", "seed": 21}),
    ("channel_features", {"n_cells": 1200, "topo": "discontinuous", "friction": "chezy", "outflow": "z", "seed": 22}),
])
def test_oracle_live_vs_reference(tmp_path, kind, kwargs, portable):
    """Step-by-step, every intermediate array the step produces, bit for bit."""
    pkg = load_pkg()
    case = getattr(pkg.workloads, kind)(**kwargs)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    ref = oracle_binding.RefSolver(folder, portable_math=portable)
    o = oracle_binding.SpOracle(case, portable_math=portable)
    names = ["F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd", "lambda_max_int",
             "lambda_max_bnd", "z_riemann_L", "z_riemann_R", "q_riemann_L", "r_riemann_R"]
    for chunk in (1, 1, 3, 25, 120):
        assert ref.step(chunk) == o.step(chunk)
        assert ref.t == o.t and ref.dt == o.dt
        for a, b in zip(ref.state(), o.state()):
            assert _bits_equal(a, b)
        for nm in names:
            assert _bits_equal(ref.array(nm), o.array(nm)), nm
    if case.opts["num_scheme"] == "muscl_evr":
        # limited slopes of the current state (computeMusclSlopes) against the oracle's, which
        # the next step recomputes from the same state
        sx, sy = ref.slopes()
        assert ref.step(1) == o.step(1)
        assert _bits_equal(sx, o.array("slope_x")) and _bits_equal(sy, o.array("slope_y"))


@needs_ref
def test_oracle_error_path_matches_reference(tmp_path):
    """Impervious cells next to dry ones: the reference stops on an impossible HLLC
    configuration (swSpHyp.cpp:728-739, exit status 1); the oracle returns SW2D_E_HLLC_CONFIG (-4)
    on the same first step.  The reference runs as a subprocess since it calls exit(1)."""
    import subprocess
    pkg = load_pkg()
    case = pkg.workloads.channel_features(n_cells=3000, impervious=True, seed=7)
    folder = str(tmp_path / "case")
    pkg.write_case(folder, case)
    res = subprocess.run([oracle_binding.REF_BIN, folder], capture_output=True, text=True, timeout=300)
    assert res.returncode == 1
    assert "Impossible flow configuration" in res.stderr
    o = oracle_binding.SpOracle(case)
    with pytest.raises(RuntimeError, match="status -4"):
        o.step(1)


def test_libm_sensitivity_recorded():
    """Where the reference's own results move by more than 1e-10 when only its libm changes
    (glibc vs the portable exp/log), the fixture says so; the stable cases agree to 1e-10."""
    from tests.golden.make_golden import state_rel_err
    for name in golden_names():
        _, fx = golden_case(name)
        e = state_rel_err((fx["h"], fx["q"], fx["r"]), (fx["h_pm"], fx["q_pm"], fx["r_pm"]))
        assert bool(fx["libm_stable"]) == (e <= 1e-10), name
