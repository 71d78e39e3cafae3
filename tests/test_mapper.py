"""The porosity mapper's host side against the reference's mapper program
(oracle/_ref/sw2dPorosityMapper, built from its sources): the buildings file and the level list
as its reader takes them, and the map files in its exact text layout (the reference's outputs,
read back and written again by porosity_mapper.write_maps, byte for byte).
tests/test_gpu_mapper.py compares the porosities computed on the GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.conftest import load_pkg

PKG = load_pkg()
M = PKG.porosity_mapper
oracle_binding = pytest.importorskip("oracle.binding")
needs_mapper = pytest.mark.skipif(not os.path.exists(oracle_binding.REF_MAPPER), reason="reference mapper not built")

FILES = {"sp": ["SP_cell_porosity_map.txt"],
         "dip": ["DIP_cell_porosity_map.txt", "DIP_edge_bnd_porosity_map.txt", "DIP_edge_int_porosity_map.txt"],
         "ddp": ["DDP_cell_porosity_map.txt", "DDP_edge_bnd_porosity_map.txt", "DDP_edge_int_porosity_map.txt"]}


def raster_case(folder, model, seed=5):
    """The dam-break channel (100 m x 20 m) under a 1 m raster of block buildings of heights 0, 3
    and 6 m (blocks of 2-6 pixels), with the raster input."""
    case = PKG.workloads.dam_break(n_cells=900, seed_mesh=seed, seed_phi=seed + 1)
    x = np.arange(100) + 0.5
    y = np.arange(20) + 0.5
    rng = np.random.default_rng(seed)
    hgt = np.zeros((20, 100))
    for _ in range(40):
        i, j = rng.integers(0, 96), rng.integers(0, 17)
        hgt[j:j + rng.integers(2, 5), i:i + rng.integers(2, 7)] = rng.choice([3.0, 6.0])
    PKG.write_case(folder, case)
    for fn in os.listdir(os.path.join(folder, "input")):
        if fn.endswith("porosity_map.txt"):
            os.remove(os.path.join(folder, "input", fn))
    os.makedirs(os.path.join(folder, "primary_files"), exist_ok=True)
    M.write_raster(os.path.join(folder, "primary_files", "buildings.txt"), x, y, hgt)
    with open(os.path.join(folder, "primary_files", "input.pmap"), "w") as fh:
        fh.write(f"model {model}\ninput raster\n")
    return case, x, y, hgt


def mapper_case(folder, model, n_cells=900, seed=31, urban=False):
    """A case folder with buildings: three hand-placed footprints (rectangles and a triangle,
    one across many cells) on the dam-break channel, or (urban=True) a seeded building layout."""
    if urban:
        case = PKG.workloads.gaussian_bumps(n_cells=n_cells, seed_mesh=seed)
        m = case.mesh
        lx, ly = float(np.ptp(m.node_x)), float(np.ptp(m.node_y))
        b = PKG.closure.building_layout(lx, ly, size=(0.04 * lx, 0.12 * lx), coverage=0.25, seed=seed, margin=0.02 * lx)
        x0, y0 = float(m.node_x.min()), float(m.node_y.min())
        xs = [np.array([p[0], p[2], p[2], p[0]]) + x0 for p in b]
        ys = [np.array([p[1], p[1], p[3], p[3]]) + y0 for p in b]
        hs = np.round(np.random.default_rng(seed).uniform(2.0, 12.0, len(xs)))
    else:
        case = PKG.workloads.dam_break(n_cells=n_cells, seed_mesh=seed, seed_phi=seed + 1)
        xs = [np.array([10.0, 18, 18, 10]), np.array([30.5, 41, 41, 30.5]), np.array([60.0, 66, 63]),
              np.array([75.0, 99, 99, 75])]
        ys = [np.array([2.0, 2, 9, 9]), np.array([11.0, 11, 17.5, 17.5]), np.array([5.0, 5, 12]),
              np.array([-1.0, -1, 6, 6])]
        hs = np.array([3.0, 6.0, 3.0, 4.5])
    PKG.write_case(folder, case)
    for fn in os.listdir(os.path.join(folder, "input")):  # the mapper writes these
        if fn.endswith("porosity_map.txt"):
            os.remove(os.path.join(folder, "input", fn))
    os.makedirs(os.path.join(folder, "primary_files"), exist_ok=True)
    M.write_buildings(os.path.join(folder, "primary_files", "buildings.txt"), xs, ys, hs)
    with open(os.path.join(folder, "primary_files", "input.pmap"), "w") as fh:
        fh.write(f"model {model}\ninput footprint\n")
    return case, xs, ys, hs


def run_reference_mapper(folder):
    res = subprocess.run([oracle_binding.REF_MAPPER, folder], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    out = {}
    for fn in sorted(os.listdir(os.path.join(folder, "input"))):
        if "porosity_map" in fn:
            with open(os.path.join(folder, "input", fn)) as fh:
                out[fn] = fh.read()
    return out


def _values(text, ddp):
    lines = text.split("\n")
    body = lines[lines.index("==== Distrib") + (2 if ddp else 1):]
    rows = [ln.split("\t") for ln in body if ln]
    if ddp:
        return np.array([[float(v) for v in r[2::2]] for r in rows]), [float(v) for v in rows[0][3::2]]
    return np.array([[float(r[0])] for r in rows]), None


def test_buildings_reader(tmp_path):
    _, xs, ys, hs = mapper_case(str(tmp_path / "c"), "ddp")
    rx, ry, rh, topo = M.read_buildings(str(tmp_path / "c" / "primary_files" / "buildings.txt"))
    assert len(rx) == 4 and all(np.array_equal(a, b) for a, b in zip(rx, xs)) and np.array_equal(rh, hs)
    assert topo == [0.0, 3.0, 4.5, 6.0]


def test_raster_reader(tmp_path):
    _, x, y, hgt = raster_case(str(tmp_path / "c"), "ddp")
    rx, ry, rh, topo = M.read_raster(str(tmp_path / "c" / "primary_files" / "buildings.txt"))
    assert np.array_equal(rx, x) and np.array_equal(ry, y) and np.array_equal(rh, hgt)
    assert topo == [0.0, 3.0, 6.0]


@needs_mapper
@pytest.mark.parametrize("raster", [False, True], ids=["footprint", "raster"])
@pytest.mark.parametrize("model", ["sp", "dip", "ddp"])
def test_writer_reproduces_the_reference_files(tmp_path, model, raster):
    folder = str(tmp_path / "c")
    (raster_case if raster else mapper_case)(folder, model)
    ref = run_reference_mapper(folder)
    assert sorted(ref) == sorted(FILES[model])
    ddp = model == "ddp"
    res, topo = {}, None
    for fn, key in zip(FILES[model], ["cell", "edge_bnd", "edge_int"]):
        res[key], t = _values(ref[fn], ddp)
        topo = t or topo
    if ddp:
        assert topo == ([0.0, 3.0, 6.0] if raster else [0.0, 3.0, 4.5, 6.0])
    out = str(tmp_path / "o")
    os.makedirs(os.path.join(out, "input"))
    M.write_maps(out, model, res, topo)
    for fn in FILES[model]:
        with open(os.path.join(out, "input", fn)) as fh:
            assert fh.read() == ref[fn], fn
