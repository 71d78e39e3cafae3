"""The reference's porosity-assimilation layer (assim/*.cpp, built with an Enzyme stub into
oracle/_ref/libsw2d_ref_e*.so) pinned against the case's own published numbers, and the
committed fixture tests/golden/sp_toce_assim.npz checked against it.

* Linked with the host libm, the reference's dry run + tiled replay at the first guess phi = 1 of
  configue_fonctionels/sp_toce gives J = 3.1042911536e+00, the first row of the case's
  descent_log_reference_-75.8pct.csv (the value its Enzyme build logged).  This pins the harness
  (observation reader, window and tiles restated from get_spatial_gradient_checkpointed).
* The fixture's observations decode to the doubles the reference's reader returns, and its
  recorded trajectory is the reference's (portable exp/log/cbrt build).
These need the reference sources (present in the build container only) and skip elsewhere.
"""
import json
import os

import numpy as np
import pytest

from tests.conftest import GOLDEN, reference_case, reference_missing

CASE = reference_case("sp_toce")
DESCENT_LOG_J_INIT = 3.1042911536e+00   # descent_log_reference_-75.8pct.csv, iteration 1, J_total


def _ref(pm):
    from oracle.binding import RefE, REF_E_SO, REF_E_PM_SO
    if not os.path.isdir(CASE) or not os.path.exists(REF_E_PM_SO if pm else REF_E_SO):
        pytest.skip(reference_missing() or "the reference assimilation library (oracle/_ref) is not built")
    return RefE(CASE, portable_math=pm)


def _run(ref):
    cfg = ref.config()
    ref.load_observations()
    m = ref.load_phi_map(os.path.join(CASE, "input", "phi_init_ones.txt"))
    K = ref.record(m, int(cfg["checkpoint_stride"]))
    first, tiles = ref.set_window()
    return cfg, m, K, first, tiles, ref.replay_cost(m)


def test_reference_assim_reproduces_descent_log_J():
    cfg, m, K, first, tiles, J = _run(_ref(False))
    assert cfg["checkpoint_stride"] == 30 and cfg["n_windows"] == 48 and cfg["window_duration"] == 20.0
    assert cfg["cost_normalize"] == 1.0 and cfg["phi_transform"] == 0.0
    assert np.all(m == 1.0)
    assert abs(J - DESCENT_LOG_J_INIT) < 5e-11, f"J = {J:.12e}"


def test_fixture_matches_reference():
    from tests.golden.make_assim_golden import decimals_to_float
    ref = _ref(True)
    ax = np.load(os.path.join(GOLDEN, "sp_toce_assim.npz"))
    times, frames = ref.load_observations()
    assert np.array_equal(times, ax["obs_times"])
    assert np.array_equal(decimals_to_float(ax["obs_mant"], ax["obs_exp"]).view(np.int64), frames.view(np.int64))
    cfg, m, K, first, tiles, J = _run(ref)
    assert json.loads(str(ax["config"])) == cfg
    segs = ref.segments()
    assert K == len(ax["seg_n"]) and first == int(ax["first_segment"]) and np.array_equal(tiles, ax["tiles"])
    assert np.array_equal(np.concatenate([s[1] for s in segs]).view(np.int64), ax["dt_seq"].view(np.int64))
    assert np.array_equal(np.concatenate([s[2] for s in segs]), ax["obs_trig"])
    assert J == float(ax["J_pm"])
    # the portable libm moves this chaotic run's cost by a few 1e-6 relative
    assert abs(J - DESCENT_LOG_J_INIT) / DESCENT_LOG_J_INIT < 2e-5


def test_reference_gen_ref_e_reproduces_the_shipped_maps():
    """The reference's gen-ref-e mode (generate_references_E) at the case's porosity_ref_map,
    linked with the host libm, writes the case's shipped reference/ResultHydro_p*.txt digit for
    digit: those maps are this mode's output.  Linked with the portable exp/log/cbrt instead, it
    gives the maps whose digests tests/golden/sp_toce_genref_pm.json keeps (the GPU's _E step
    uses the portable functions and is compared with those, tests/test_gpu_assim.py)."""
    import glob
    from tests.golden.make_assim_golden import frames_as_decimals
    from tests.golden.make_genref_digest import frame_digests
    fx = json.load(open(os.path.join(GOLDEN, "sp_toce_genref_pm.json")))
    for pm in (False, True):
        ref = _ref(pm)   # skips without the reference tree
        shipped = sorted(glob.glob(os.path.join(CASE, "reference", "ResultHydro_p*.txt")))
        ms, es = frames_as_decimals(shipped)
        try:
            phi = ref.load_phi_map(os.path.join(CASE, "input", "SP_cell_porosity_map.txt"))
            files = ref.generate_references(phi, int(ref.config()["checkpoint_stride"]))
            assert [os.path.basename(f) for f in files] == [os.path.basename(f) for f in shipped]
            if pm:
                assert frame_digests(files) == fx["sha256"]
                assert [os.path.basename(f) for f in files] == fx["names"]
            else:
                mant, expo = frames_as_decimals(files)
                same = (mant == ms) & ((expo == es) | (mant == 0))
                assert same.all(), f"{np.count_nonzero(~same)} printed values differ from the shipped maps"
        finally:
            ref.close()
