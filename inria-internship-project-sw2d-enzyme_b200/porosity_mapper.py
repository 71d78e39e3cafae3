"""The porosity mapper (the reference's sw2dPorosityMapper, footprint and raster inputs) with its
geometry on the GPU (C ABI sw2d_map_porosity, sw2d_map_porosity_raster).

``map_folder(folder)`` does what the reference's mapper program does on a case folder: it reads
``primary_files/input.pmap`` (model sp / dip / ddp, input footprint or raster),
``primary_files/buildings.txt`` (footprints, or a raster of building heights) and
``input/geometry.sw2d``, computes the storage porosity of
every cell and the connectivity porosity of every edge, and writes the model's porosity maps
into ``input/`` in the reference's text layout (swPorosityMapperPipeline::writeSp / writeDip /
writeDdp, src/sw2dPorosityMapper/swPorosityMapperPipeline.cpp:537-822; numbers as an
std::ostream prints them by default, %g).  ``map_porosity`` returns the arrays.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import capi
from .case import read_geometry


class _MapMesh(ctypes.Structure):
    _fields_ = [("cell_nb", ctypes.c_int64), ("node_nb", ctypes.c_int64), ("edge_int_nb", ctypes.c_int64),
                ("edge_bnd_nb", ctypes.c_int64), ("node_x", ctypes.c_void_p), ("node_y", ctypes.c_void_p),
                ("cell_node_offsets", ctypes.c_void_p), ("cell_nodes", ctypes.c_void_p),
                ("cell_area", ctypes.c_void_p), ("edge_int_nodes", ctypes.c_void_p),
                ("edge_int_length", ctypes.c_void_p), ("edge_bnd_nodes", ctypes.c_void_p),
                ("edge_bnd_length", ctypes.c_void_p)]


class _Raster(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p),
                ("height", ctypes.c_void_p)]


class _Buildings(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("offsets", ctypes.c_void_p), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p),
                ("height", ctypes.c_void_p)]


def read_buildings(path: str) -> Tuple[List[np.ndarray], List[np.ndarray], Optional[np.ndarray], List[float]]:
    """buildings.txt as swPorosityMapperPipeline::init reads it (:405-458): a header line, then
    one building per line, x1 y1 x2 y2 ... with an optional last value -height.  Returns
    (x per building, y per building, heights or None, the level list: 0 and every distinct
    height, ascending)."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    xs, ys, hs = [], [], []
    topo = [0.0]
    for ln in lines[1:]:
        tok = ln.replace("\r", "").split()
        if not tok:
            raise ValueError(f"{path}: empty building line (the reference reads past it)")
        vals = [float(t) for t in tok]
        if vals[-1] < 0:
            npts = (len(vals) - 1) // 2
            hs.append(-vals[-1])
            if -vals[-1] not in topo:
                topo.append(-vals[-1])
        else:
            npts = len(vals) // 2
        xs.append(np.array(vals[0:2 * npts:2]))
        ys.append(np.array(vals[1:2 * npts:2]))
    topo.sort()
    heights = np.array(hs) if hs else None
    if heights is not None and len(hs) != len(xs):
        raise ValueError(f"{path}: some buildings have a height and others not")
    return xs, ys, heights, topo


def write_buildings(path: str, xs, ys, heights=None) -> None:
    """buildings.txt for the reference mapper: no newline after the last building (its reader
    would read an empty building there)."""
    rows = []
    for k, (x, y) in enumerate(zip(xs, ys)):
        vals = [v for pair in zip(x, y) for v in pair]
        if heights is not None:
            vals.append(-float(heights[k]))
        rows.append(" ".join(repr(float(v)) for v in vals))
    with open(path, "w") as fh:
        fh.write("x y ... -height\n" + "\n".join(rows))


def read_raster(path: str) -> Tuple[np.ndarray, np.ndarray, np.ndarray, List[float]]:
    """A building raster as swRasterBuildings::build reads it (:35-128): a header line, then one
    pixel per line, x y height, row by row from the top (y descending, x ascending within a
    row).  Returns (x centres, y centres ascending, heights [ny x nx], the distinct heights
    ascending).  As with the reference's reader, a last line without a newline is not read."""
    with open(path) as fh:
        text = fh.read()
    # after the header; the last element of the split is empty after a final newline, or the
    # last line, which the reference's loop reads at end of file and does not use
    lines = text.split("\n")[1:-1]
    rows, xs, ys = [], [], []
    y0 = None
    for ln in lines:
        x, y, b = (float(t) for t in ln.split()[:3])
        if y0 is None:
            y0 = y
            rows.append([b])
            xs.append(x)
            ys.append(y)
        elif y != ys[-1]:
            rows.append([b])
            ys.append(y)
        else:
            rows[-1].append(b)
            if y == y0:
                xs.append(x)
    heights = np.array(rows[::-1], dtype=np.float64)
    topo = sorted(set(float(v) for v in heights.reshape(-1)))
    return np.array(xs), np.array(ys[::-1]), heights, topo


def write_raster(path: str, x: np.ndarray, y: np.ndarray, heights: np.ndarray) -> None:
    """A building raster for the reference mapper (top row first), ending with a newline."""
    out = ["x y height"]
    for j in range(len(y) - 1, -1, -1):
        out.extend(f"{float(x[i])!r} {float(y[j])!r} {float(heights[j, i])!r}" for i in range(len(x)))
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def _cell_nodes(mesh) -> Tuple[np.ndarray, np.ndarray]:
    flat = None if mesh.cell_nodes_flat is None else np.asarray(mesh.cell_nodes_flat, dtype=np.int64)
    if flat is not None and flat.ndim == 2:  # one node count for every cell
        off = np.arange(0, flat.size + 1, flat.shape[1], dtype=np.int64)
        return off, flat.reshape(-1)
    counts = np.array([len(c) for c in mesh.cell_nodes], dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return off, np.concatenate([np.asarray(c, dtype=np.int64) for c in mesh.cell_nodes])


def map_porosity(mesh, xs, ys, heights, levels, device: int = 0, edges: bool = True) -> Dict[str, np.ndarray]:
    """Porosities [element x level] of the cells and (edges=True) the internal and boundary
    edges; heights None: every building counts at every level."""
    lib = capi.load_library()
    off, cn = _cell_nodes(mesh)
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    nl = len(levels)
    nc, ni, nb = mesh.cell_nb, mesh.edge_int_nb, mesh.edge_bnd_nb
    mm = _MapMesh(nc, int(np.asarray(mesh.node_x).size), ni, nb, arr(mesh.node_x, np.float64),
                  arr(mesh.node_y, np.float64), arr(off, np.int64), arr(cn, np.int64), arr(mesh.cell_area, np.float64),
                  arr(mesh.edge_int_nodes, np.int64), arr(mesh.edge_int_length, np.float64),
                  arr(mesh.edge_bnd_nodes, np.int64), arr(mesh.edge_bnd_length, np.float64))
    counts = np.array([len(x) for x in xs], dtype=np.int64)
    boff = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    bx = np.concatenate(xs) if xs else np.zeros(0)
    by = np.concatenate(ys) if ys else np.zeros(0)
    bl = _Buildings(len(xs), arr(boff, np.int64), arr(bx, np.float64), arr(by, np.float64),
                    arr(heights, np.float64) if heights is not None else None)
    lev = np.ascontiguousarray(levels, dtype=np.float64)
    cell = np.empty((nc, nl))
    eint = np.empty((ni, nl)) if edges else None
    ebnd = np.empty((nb, nl)) if edges else None
    dp = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None
    st = lib.sw2d_map_porosity(int(device), ctypes.byref(mm), ctypes.byref(bl), lev.ctypes.data_as(ctypes.c_void_p),
                               nl, dp(cell), dp(eint), dp(ebnd))
    if st != 0:
        raise RuntimeError(f"sw2d_map_porosity failed ({st}): {lib.sw2d_map_last_error().decode()}")
    return {"cell": cell, "edge_int": eint, "edge_bnd": ebnd, "levels": lev}


def map_porosity_raster(mesh, x, y, heights, levels, device: int = 0, edges: bool = True) -> Dict[str, np.ndarray]:
    """Porosities [element x level] from a building raster (pixel centres x, y ascending,
    heights [ny x nx])."""
    lib = capi.load_library()
    off, cn = _cell_nodes(mesh)
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    nl = len(levels)
    nc, ni, nb = mesh.cell_nb, mesh.edge_int_nb, mesh.edge_bnd_nb
    mm = _MapMesh(nc, int(np.asarray(mesh.node_x).size), ni, nb, arr(mesh.node_x, np.float64),
                  arr(mesh.node_y, np.float64), arr(off, np.int64), arr(cn, np.int64), arr(mesh.cell_area, np.float64),
                  arr(mesh.edge_int_nodes, np.int64), arr(mesh.edge_int_length, np.float64),
                  arr(mesh.edge_bnd_nodes, np.int64), arr(mesh.edge_bnd_length, np.float64))
    ra = _Raster(len(x), len(y), arr(x, np.float64), arr(y, np.float64), arr(heights, np.float64))
    lev = np.ascontiguousarray(levels, dtype=np.float64)
    cell = np.empty((nc, nl))
    eint = np.empty((ni, nl)) if edges else None
    ebnd = np.empty((nb, nl)) if edges else None
    dp = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None
    st = lib.sw2d_map_porosity_raster(int(device), ctypes.byref(mm), ctypes.byref(ra),
                                      lev.ctypes.data_as(ctypes.c_void_p), nl, dp(cell), dp(eint), dp(ebnd))
    if st != 0:
        raise RuntimeError(f"sw2d_map_porosity_raster failed ({st}): {lib.sw2d_map_last_error().decode()}")
    return {"cell": cell, "edge_int": eint, "edge_bnd": ebnd, "levels": lev}


def _g(v: float) -> str:
    return "%g" % v


def _write_single(path: str, name: str, values) -> None:
    with open(path, "w") as fh:
        fh.write(f"Unif\t0\n==== Default Param\n{name}\n{_g(values[0])}\n==== Distrib\n")
        fh.write("".join(_g(v) + "\n" for v in values))


def _write_ddp(path: str, table: np.ndarray, topo, law: int = -2) -> None:
    n = len(topo)

    def row(r):
        return f"{law}\t{n}\t" + "\t".join(f"{_g(r[k])}\t{_g(topo[k])}" for k in range(n)) + "\n"

    with open(path, "w") as fh:
        fh.write(f"Unif\t0\nNtabMax\t{n}\n==== Default Param\nType\tParameters\n")
        fh.write(row(table[0]))
        fh.write("==== Distrib\nType\tParameters\n")
        fh.write("".join(row(r) for r in table))


def write_maps(folder: str, model: str, res: Dict[str, np.ndarray], topo=None) -> None:
    """The map files the reference mapper writes into <folder>/input."""
    inp = os.path.join(folder, "input")
    if model == "sp":
        _write_single(os.path.join(inp, "SP_cell_porosity_map.txt"), "PhiW", res["cell"][:, 0])
    elif model == "dip":
        _write_single(os.path.join(inp, "DIP_cell_porosity_map.txt"), "PhiW", res["cell"][:, 0])
        _write_single(os.path.join(inp, "DIP_edge_bnd_porosity_map.txt"), "PhiG", res["edge_bnd"][:, 0])
        _write_single(os.path.join(inp, "DIP_edge_int_porosity_map.txt"), "PhiG", res["edge_int"][:, 0])
    elif model == "ddp":
        _write_ddp(os.path.join(inp, "DDP_cell_porosity_map.txt"), res["cell"], topo)
        _write_ddp(os.path.join(inp, "DDP_edge_bnd_porosity_map.txt"), res["edge_bnd"], topo)
        _write_ddp(os.path.join(inp, "DDP_edge_int_porosity_map.txt"), res["edge_int"], topo)
    else:
        raise ValueError(f"model {model!r}")


def read_pmap(path: str) -> Dict[str, str]:
    """input.pmap (swPorosityMapperParam::readInputFile): 'model' and 'input' lines; '#' and '='
    start comments."""
    out = {}
    with open(path) as fh:
        for ln in fh:
            ln = ln.strip("\r\n")
            if not ln or ln[0] in "#=":
                continue
            tok = ln.split()
            if len(tok) != 2:
                raise ValueError(f"{path}: misformatted line {ln!r}")
            out[tok[0].lower()] = tok[1].lower()
    return out


def map_folder(folder: str, device: int = 0) -> Dict[str, np.ndarray]:
    """The mapper program on a case folder (footprint input)."""
    prm = read_pmap(os.path.join(folder, "primary_files", "input.pmap"))
    model, kind = prm.get("model"), prm.get("input")
    if model not in ("sp", "dip", "ddp"):
        raise ValueError(f"model {model!r}")
    if kind not in ("footprint", "raster"):
        raise ValueError(f"input {kind!r}")
    mesh = read_geometry(os.path.join(folder, "input", "geometry.sw2d"))
    if kind == "raster":
        x, y, hgt, topo = read_raster(os.path.join(folder, "primary_files", "buildings.txt"))
        levels = topo if model == "ddp" else [0.0]
        res = map_porosity_raster(mesh, x, y, hgt, levels, device, edges=(model != "sp"))
        write_maps(folder, model, res, topo)
        return res
    xs, ys, heights, topo = read_buildings(os.path.join(folder, "primary_files", "buildings.txt"))
    if model == "ddp":
        if heights is None:
            raise ValueError("the DDP mapping needs a height for every building")
        res = map_porosity(mesh, xs, ys, heights, topo, device)
    else:
        res = map_porosity(mesh, xs, ys, None, [0.0], device, edges=(model == "dip"))
    write_maps(folder, model, res, topo)
    return res
