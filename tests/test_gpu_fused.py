"""The fused step (k_flux + k_update, sw2d_tile.cu) against the four-kernel step and the oracle.

The fused step computes the same arithmetic as the four-kernel step (k_slopes, k_edges, k_cfl,
k_update) with its operands staged per tile of cells in shared memory, so the two must agree bit
for bit: states, times, fluxes, wave speeds and slopes, on every scheme, topography, model and
tile size, on meshes with cells of every degree and a random input numbering.  Tile sizes as
small as 32 cells make most edges cross a tile boundary (edges computed by two tiles, ring-1
slopes recomputed), which is where a staging or indexing mistake would show.
"""
import numpy as np
import pytest

from tests.conftest import assert_state_close, load_pkg

pytestmark = pytest.mark.gpu

oracle_binding = pytest.importorskip("oracle.binding")

CASES = {
    "dam_muscl_nofriction": ("dam_break", {"n_cells": 3000, "friction": "none"}),
    "dam_godunov": ("dam_break", {"n_cells": 3000, "scheme": "godunov"}),
    "dam_delaunay": ("dam_break", {"n_cells": 5000, "mesh": "delaunay"}),
    "bumps_dam_delaunay": ("gaussian_bumps", {"n_cells": 8000, "mesh": "delaunay", "initial": "dam"}),
    "bumps_lake_delaunay": ("gaussian_bumps", {"n_cells": 8000, "mesh": "delaunay"}),
    "chan_muscl_blend_strickler_fr": ("channel_features", {"n_cells": 2500, "scheme": "muscl_evr", "topo": "blending",
                                                           "friction": "strickler", "outflow": "fr"}),
    "chan_godunov_blend_headloss": ("channel_features", {"n_cells": 2500}),
    "chan_muscl_disc_chezy_z": ("channel_features", {"n_cells": 2500, "scheme": "muscl_evr", "topo": "discontinuous",
                                                     "friction": "chezy", "outflow": "z", "head_loss": False}),
    "dip_muscl": ("dip_channel", {"n_cells": 3000}),
    "dip_godunov_blend": ("dip_channel", {"n_cells": 3000, "scheme": "godunov", "topo": "blending"}),
}

ARRAYS = ["F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int", "F1_bnd", "F2_bnd", "F3_bnd", "lambda_max_int",
          "lambda_max_bnd"]


@pytest.fixture(scope="module")
def pkg():
    p = load_pkg()
    p.build.build()
    oracle_binding.build(reference=False)
    return p


def _pair(pkg, case, tile, slopes_in=1):
    fused = pkg.SpModel(case)
    muscl = case.opts["num_scheme"] == "muscl_evr"
    assert fused.get_option("fused_step") == 0   # the four-kernel step is the default form
    fused.set_option("fused_step", 1)
    fused.set_option("fused_slopes", slopes_in)
    assert fused.kernels_per_step == (3 if muscl and not slopes_in else 2)
    if tile is not None:
        fused.set_option("tile_cells", tile)
    four = pkg.SpModel(case)
    four.set_option("fused_step", 0)
    assert four.kernels_per_step in (3, 4)
    for m in (fused, four):
        m.set_option("record_wave_speeds", 1)
        m.set_option("record_fluxes", 1)
    return fused, four


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


@pytest.mark.parametrize("tile,slopes_in", [(32, 1), (97, 1), (320, 1), (None, 1), (97, 0), (None, 0)])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_matches_four_kernel_step(pkg, name, tile, slopes_in):
    kind, kwargs = CASES[name]
    case = getattr(pkg.workloads, kind)(**kwargs)
    if not slopes_in and case.opts["num_scheme"] != "muscl_evr":
        pytest.skip("slopes exist only in the MUSCL-EVR scheme")
    fused, four = _pair(pkg, case, tile, slopes_in)
    names = list(ARRAYS)
    if case.opts["num_scheme"] == "muscl_evr":
        names += ["slope_x", "slope_y"]
    for i, chunk in enumerate((1, 1, 6, 40, 100)):
        assert fused.step(chunk) == four.step(chunk)
        assert fused.time == four.time, f"{name} tile {tile} chunk {i}: t, dt"
        for a, b, v in zip(fused.state(), four.state(), ("h", "q", "r")):
            assert _same(a, b), f"{name} tile {tile} chunk {i}: {v}"
        for nm in names:
            assert _same(fused.array(nm), four.array(nm)), f"{name} tile {tile} chunk {i}: {nm}"


def test_fused_matches_oracle_on_delaunay_mesh(pkg):
    """The dam break on the jittered-Delaunay mesh (cells of degree 1 to 3, random input
    numbering), stepped by the fused step, bit for bit against the CPU oracle at every chunk."""
    case = pkg.workloads.dam_break(n_cells=12000, mesh="delaunay")
    model = pkg.SpModel(case)
    o = oracle_binding.SpOracle(case, portable_math=True)
    for chunk in (1, 9, 90, 200):
        assert model.step(chunk) == o.step(chunk)
        assert model.time == (o.t, o.dt)
        assert_state_close(model.state(), o.state(), True, f"delaunay dam break after chunk {chunk}")


def test_fused_phase_labels_and_switch(pkg):
    case = pkg.workloads.dam_break(n_cells=2000)
    m = pkg.SpModel(case)
    assert list(m.phase_times(3)) == ["k_slopes", "k_edges", "k_cfl", "k_update"]   # MUSCL-EVR default
    m.set_option("fused_step", 1)
    assert list(m.phase_times(3)) == ["k_slopes", "k_flux", "k_update"]            # slopes first by default
    m.set_option("fused_slopes", 1)
    ph = m.phase_times(3)
    assert list(ph) == ["k_flux", "k_update"]
    m.set_option("fused_slopes", 0)
    assert list(m.phase_times(3)) == ["k_slopes", "k_flux", "k_update"] and m.kernels_per_step == 3
    m.set_option("fused_slopes", 1)
    m.set_option("fused_step", 0)
    ph = m.phase_times(3)
    assert list(ph) == ["k_slopes", "k_edges", "k_cfl", "k_update"]
    m.set_option("fused_step", 1)
    assert m.kernels_per_step == 2
    with pytest.raises(pkg.Sw2dError):
        m.set_option("tile_cells", 5)
    assert m.kernels_per_step == 2 and m.step(3) == 3   # the previous tiles are kept
    assert m.get_option("tile_cells") == 384
    with pytest.raises(pkg.Sw2dError, match="shared-memory"):
        m.set_option("tile_cells", 4096)                  # a stage beyond 200 KB is refused
    assert m.get_option("tile_cells") == 384 and m.step(2) == 2


def test_fused_autotune_keeps_results(pkg):
    """sw2d_autotune times every k_flux launch variant on the live state; the run is unchanged."""
    # a channel whose dt changes from step to step (the MUSCL-EVR step reads the previous dt)
    case = pkg.workloads.channel_features(n_cells=20000, scheme="muscl_evr")
    a = pkg.SpModel(case)
    b = pkg.SpModel(case)
    a.set_option("fused_step", 1)
    a.step(25)
    b.step(24)
    dt_before = b.dt
    b.step(1)
    assert b.dt != dt_before
    rep = pkg.tuning.autotune(a, iters=2, cache_path=None)
    assert "k_flux/" in rep["report"]
    assert a.step(50) == b.step(50)
    for x, y in zip(a.state(), b.state()):
        assert _same(x, y)
    assert a.time == b.time


@pytest.mark.parametrize("scheme", ["muscl_evr", "godunov"])
def test_autotune_step_keeps_results(pkg, scheme, tmp_path):
    """sw2d_autotune_step times the four-kernel step and the fused step at several tile sizes
    (and both places of the MUSCL-EVR slopes) on the live state, then sets the fastest form; the
    run continues with the same bits, and the cached choice is applied to a new model."""
    case = pkg.workloads.channel_features(n_cells=20000, scheme=scheme)   # dt changes every step
    a = pkg.SpModel(case)
    b = pkg.SpModel(case)
    a.step(25)
    b.step(24)
    dt_before = b.dt
    b.step(1)
    assert b.dt != dt_before
    cache = str(tmp_path / "tune.json")
    rep = pkg.tuning.autotune_step(a, iters=2, tile_sizes=(97, 256), cache_path=cache)
    assert "four-kernel=" in rep["report"] and "tile97" in rep["report"] and "chosen" in rep["report"]
    if scheme == "muscl_evr":
        assert "slopes-first/tile256" in rep["report"]
    assert rep["fused"] == a.get_option("fused_step")
    if rep["fused"]:
        assert a.get_option("tile_cells") == rep["tile"] and a.get_option("flux_variant") == rep["flux"]
    assert a.step(50) == b.step(50)
    for x, y in zip(a.state(), b.state()):
        assert _same(x, y)
    assert a.time == b.time
    c = pkg.SpModel(case)
    again = pkg.tuning.autotune_step(c, iters=2, tile_sizes=(97, 256), cache_path=cache)
    assert again["cached"] and c.get_option("fused_step") == rep["fused"]
    c.step(25)
    assert c.step(50) == 50
    for x, y in zip(c.state(), b.state()):
        assert _same(x, y)
