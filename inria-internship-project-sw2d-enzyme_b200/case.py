"""SW2D case folders: the file formats the reference solver reads, restated in numpy.

A case folder holds ``input/input.solv`` (key/value options), ``input/geometry.sw2d`` (binary
mesh, version 2), per-cell parameter maps and ``input/hydro_boundary_time_series.txt``.  The
readers and writers here follow the reference's own parsers byte for byte:

* ``geometry.sw2d`` v2: ``swMesh::readGeometryFileV2`` (src/common/geometry/swMesh.cpp:213-471)
  and its writer ``swMesh::writeGeometryFile`` (swMesh.cpp:1221-1430);
* per-cell maps (``Unif 0|1`` / ``==== Default Param`` / ``==== Distrib``):
  ``swIO::readVectorParameterFile`` (src/common/swIO.cpp:1005-1191);
* boundary time series: ``swIO::readBoundaryTimeSeriesFile`` (swIO.cpp:687-817);
* ``input.solv``: ``swSolverParam::readInputFile`` (src/sw2dSolver/common/swSolverParam.cpp:663-890)
  with the defaults of swSolverParam.h:144-194.

Numbers are written with ``repr`` so that the reference's ``std::stod`` reads back the exact
binary64 value.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

# ---------------------------------------------------------------------------------------
# geometry.sw2d (version 2)
# ---------------------------------------------------------------------------------------
_CELL_DT = np.dtype([("idx", "<u8"), ("sms_id", "<u8"), ("nb_node", "<u8"), ("nb_edge_bnd", "<u8"),
                     ("nb_edge_int", "<u8"), ("nb_neigh", "<u8"), ("area", "<f8"), ("perimeter", "<f8"),
                     ("x", "<f8"), ("y", "<f8"), ("zb", "<f8")])
_NODE_DT = np.dtype([("idx", "<u8"), ("sms_id", "<u8"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                     ("nb_cell", "<u8"), ("nb_edge", "<u8")])
_BND_DT = np.dtype([("idx", "<u8"), ("n1", "<u8"), ("n2", "<u8"), ("mx", "<f8"), ("my", "<f8"), ("mz", "<f8"),
                    ("d_norm", "<f8"), ("length", "<f8"), ("nx", "<f8"), ("ny", "<f8"), ("bc_code", "<i4"),
                    ("cell", "<u8")])
_INT_DT = np.dtype([("idx", "<u8"), ("n1", "<u8"), ("n2", "<u8"), ("mx", "<f8"), ("my", "<f8"), ("mz", "<f8"),
                    ("d_norm", "<f8"), ("length", "<f8"), ("nx", "<f8"), ("ny", "<f8"), ("c0", "<u8"),
                    ("c1", "<u8")])
assert _CELL_DT.itemsize == 88 and _NODE_DT.itemsize == 56 and _BND_DT.itemsize == 92 and _INT_DT.itemsize == 96


@dataclass
class Mesh:
    """Mesh tables in the reference numbering (what ``swParent::setMeshTables`` builds)."""

    node_x: np.ndarray
    node_y: np.ndarray
    node_z: np.ndarray
    cell_nodes: List[np.ndarray]          # per cell, node indices (ccw)
    cell_area: np.ndarray
    cell_perimeter: np.ndarray
    cell_x: np.ndarray
    cell_y: np.ndarray
    cell_z_b: np.ndarray
    edge_int_cells: np.ndarray            # (n_int, 2) int64, L then R
    edge_int_nodes: np.ndarray            # (n_int, 2)
    edge_int_length: np.ndarray
    edge_int_nx: np.ndarray
    edge_int_ny: np.ndarray
    edge_int_mx: np.ndarray
    edge_int_my: np.ndarray
    edge_int_mz: np.ndarray
    edge_int_dnorm: np.ndarray
    edge_bnd_cell: np.ndarray             # (n_bnd,) int64
    edge_bnd_nodes: np.ndarray            # (n_bnd, 2)
    edge_bnd_length: np.ndarray
    edge_bnd_nx: np.ndarray
    edge_bnd_ny: np.ndarray
    edge_bnd_mx: np.ndarray
    edge_bnd_my: np.ndarray
    edge_bnd_mz: np.ndarray
    edge_bnd_dnorm: np.ndarray
    edge_bnd_code: np.ndarray             # (n_bnd,) int32, negative BC codes
    cell_nodes_flat: Optional[np.ndarray] = None   # (n_cell, 3) when all cells are triangles

    @property
    def cell_nb(self) -> int:
        return int(self.cell_area.shape[0])

    @property
    def edge_int_nb(self) -> int:
        return int(self.edge_int_cells.shape[0])

    @property
    def edge_bnd_nb(self) -> int:
        return int(self.edge_bnd_cell.shape[0])

    def bc_codes(self) -> List[int]:
        """Distinct boundary codes in order of first appearance (swMesh::assignBC, swMesh.cpp:126-143)."""
        seen: List[int] = []
        for c in self.edge_bnd_code.tolist():
            if c not in seen:
                seen.append(c)
        return seen


def _cell_lists(mesh: Mesh):
    """Per-cell boundary edges, internal edges and neighbours, by increasing edge index."""
    nc = mesh.cell_nb
    bcell = mesh.edge_bnd_cell
    border = np.argsort(bcell, kind="stable")
    bcount = np.bincount(bcell, minlength=nc)
    L = mesh.edge_int_cells[:, 0]
    R = mesh.edge_int_cells[:, 1]
    ne = mesh.edge_int_nb
    owner = np.concatenate([L, R])
    eidx = np.concatenate([np.arange(ne), np.arange(ne)])
    neigh = np.concatenate([R, L])
    order = np.lexsort((eidx, owner))
    icount = np.bincount(owner, minlength=nc)
    return border, bcount, eidx[order], neigh[order], icount


def write_geometry(path: str, mesh: Mesh) -> None:
    """Writes ``geometry.sw2d`` version 2 (layout of swMesh::writeGeometryFile, swMesh.cpp:1221-1430)."""
    nc, nb, ni = mesh.cell_nb, mesh.edge_bnd_nb, mesh.edge_int_nb
    nn = int(mesh.node_x.shape[0])
    codes = mesh.bc_codes()
    border, bcount, ci_edges, ci_neigh, icount = _cell_lists(mesh)
    if mesh.cell_nodes_flat is not None:
        nodes_per_cell = np.full(nc, mesh.cell_nodes_flat.shape[1], dtype=np.int64)
        cell_nodes_flat = mesh.cell_nodes_flat.reshape(-1).astype(np.int64)
    else:
        nodes_per_cell = np.array([len(c) for c in mesh.cell_nodes], dtype=np.int64)
        cell_nodes_flat = np.concatenate(mesh.cell_nodes).astype(np.int64)

    cells = np.zeros(nc, dtype=_CELL_DT)
    cells["idx"] = np.arange(nc)
    cells["sms_id"] = np.arange(1, nc + 1)
    cells["nb_node"] = nodes_per_cell
    cells["nb_edge_bnd"] = bcount
    cells["nb_edge_int"] = icount
    cells["nb_neigh"] = icount
    cells["area"] = mesh.cell_area
    cells["perimeter"] = mesh.cell_perimeter
    cells["x"] = mesh.cell_x
    cells["y"] = mesh.cell_y
    cells["zb"] = mesh.cell_z_b

    # node -> cells (sorted by cell), node -> edge counts
    owner_n = np.repeat(np.arange(nc), nodes_per_cell)
    norder = np.lexsort((owner_n, cell_nodes_flat))
    node_cells = owner_n[norder]
    ncount = np.bincount(cell_nodes_flat, minlength=nn)
    ecount = np.bincount(mesh.edge_int_nodes.reshape(-1), minlength=nn) + \
        np.bincount(mesh.edge_bnd_nodes.reshape(-1), minlength=nn)
    nodes = np.zeros(nn, dtype=_NODE_DT)
    nodes["idx"] = np.arange(nn)
    nodes["sms_id"] = np.arange(1, nn + 1)
    nodes["x"] = mesh.node_x
    nodes["y"] = mesh.node_y
    nodes["z"] = mesh.node_z
    nodes["nb_cell"] = ncount
    nodes["nb_edge"] = ecount

    bnd = np.zeros(nb, dtype=_BND_DT)
    bnd["idx"] = np.arange(nb)
    bnd["n1"] = mesh.edge_bnd_nodes[:, 0]
    bnd["n2"] = mesh.edge_bnd_nodes[:, 1]
    bnd["mx"] = mesh.edge_bnd_mx
    bnd["my"] = mesh.edge_bnd_my
    bnd["mz"] = mesh.edge_bnd_mz
    bnd["d_norm"] = mesh.edge_bnd_dnorm
    bnd["length"] = mesh.edge_bnd_length
    bnd["nx"] = mesh.edge_bnd_nx
    bnd["ny"] = mesh.edge_bnd_ny
    bnd["bc_code"] = mesh.edge_bnd_code
    bnd["cell"] = mesh.edge_bnd_cell

    ie = np.zeros(ni, dtype=_INT_DT)
    ie["idx"] = np.arange(ni)
    ie["n1"] = mesh.edge_int_nodes[:, 0]
    ie["n2"] = mesh.edge_int_nodes[:, 1]
    ie["mx"] = mesh.edge_int_mx
    ie["my"] = mesh.edge_int_my
    ie["mz"] = mesh.edge_int_mz
    ie["d_norm"] = mesh.edge_int_dnorm
    ie["length"] = mesh.edge_int_length
    ie["nx"] = mesh.edge_int_nx
    ie["ny"] = mesh.edge_int_ny
    ie["c0"] = mesh.edge_int_cells[:, 0]
    ie["c1"] = mesh.edge_int_cells[:, 1]

    # per-cell link record: nodes, boundary edges, internal edges, neighbours
    per_cell = nodes_per_cell + bcount + 2 * icount
    total = int(per_cell.sum())
    links = np.empty(total, dtype=np.uint64)
    start = np.concatenate([[0], np.cumsum(per_cell)[:-1]])
    # nodes
    pos_n = np.repeat(start, nodes_per_cell) + (np.arange(cell_nodes_flat.size) -
                                                np.repeat(np.cumsum(nodes_per_cell) - nodes_per_cell, nodes_per_cell))
    links[pos_n] = cell_nodes_flat
    # boundary edges
    b_start = start + nodes_per_cell
    bsorted_cells = mesh.edge_bnd_cell[border]
    rank_b = np.arange(nb) - np.repeat(np.cumsum(bcount) - bcount, bcount)
    links[b_start[bsorted_cells] + rank_b] = border
    # internal edges and neighbours
    i_start = b_start + bcount
    owners = np.repeat(np.arange(nc), icount)
    rank_i = np.arange(2 * ni) - np.repeat(np.cumsum(icount) - icount, icount)
    links[i_start[owners] + rank_i] = ci_edges
    links[i_start[owners] + icount[owners] + rank_i] = ci_neigh

    with open(path, "wb") as fh:
        fh.write(np.array([1], dtype="<u8").tobytes())
        fh.write(b"2")
        fh.write(np.array([nc, nb, ni, nn, len(codes)], dtype="<u8").tobytes())
        fh.write(cells.tobytes())
        fh.write(nodes.tobytes())
        fh.write(bnd.tobytes())
        fh.write(ie.tobytes())
        for code in codes:
            members = np.nonzero(mesh.edge_bnd_code == code)[0]
            fh.write(np.array([members.size], dtype="<u8").tobytes())
            fh.write(members.astype("<u8").tobytes())
        fh.write(np.array(codes, dtype="<i4").tobytes())
        fh.write(links.tobytes())
        fh.write(node_cells.astype("<u8").tobytes())


def read_geometry(path: str) -> Mesh:
    """Reads ``geometry.sw2d`` version 2 (swMesh::readGeometryFileV2, swMesh.cpp:213-471)."""
    raw = np.fromfile(path, dtype=np.uint8)
    off = 0

    def take(dtype, count):
        nonlocal off
        dt = np.dtype(dtype)
        arr = np.frombuffer(raw, dtype=dt, count=count, offset=off)
        off += dt.itemsize * count
        return arr

    vlen = int(take("<u8", 1)[0])
    version = raw[off:off + vlen].tobytes().decode()
    off += vlen
    if version != "2":
        raise ValueError(f"{path}: unsupported geometry version {version!r}")
    nc, nb, ni, nn, nbnd = (int(v) for v in take("<u8", 5))
    cells = take(_CELL_DT, nc)
    nodes = take(_NODE_DT, nn)
    bnd = take(_BND_DT, nb)
    ie = take(_INT_DT, ni)
    for _ in range(nbnd):
        size = int(take("<u8", 1)[0])
        take("<u8", size)
    codes = take("<i4", nbnd)
    del codes
    per_cell = (cells["nb_node"] + cells["nb_edge_bnd"] + cells["nb_edge_int"] + cells["nb_neigh"]).astype(np.int64)
    links = take("<u8", int(per_cell.sum())).astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(per_cell)[:-1]])
    npc = cells["nb_node"].astype(np.int64)
    if np.all(npc == npc[0]):
        idx = starts[:, None] + np.arange(npc[0])[None, :]
        flat = links[idx]
        cell_nodes = list(flat)
    else:
        flat = None
        cell_nodes = [links[s:s + k] for s, k in zip(starts, npc)]
    return Mesh(
        node_x=nodes["x"].copy(), node_y=nodes["y"].copy(), node_z=nodes["z"].copy(),
        cell_nodes=cell_nodes, cell_area=cells["area"].copy(), cell_perimeter=cells["perimeter"].copy(),
        cell_x=cells["x"].copy(), cell_y=cells["y"].copy(), cell_z_b=cells["zb"].copy(),
        edge_int_cells=np.stack([ie["c0"], ie["c1"]], axis=1).astype(np.int64),
        edge_int_nodes=np.stack([ie["n1"], ie["n2"]], axis=1).astype(np.int64),
        edge_int_length=ie["length"].copy(), edge_int_nx=ie["nx"].copy(), edge_int_ny=ie["ny"].copy(),
        edge_int_mx=ie["mx"].copy(), edge_int_my=ie["my"].copy(), edge_int_mz=ie["mz"].copy(),
        edge_int_dnorm=ie["d_norm"].copy(),
        edge_bnd_cell=bnd["cell"].astype(np.int64), edge_bnd_nodes=np.stack([bnd["n1"], bnd["n2"]], axis=1).astype(np.int64),
        edge_bnd_length=bnd["length"].copy(), edge_bnd_nx=bnd["nx"].copy(), edge_bnd_ny=bnd["ny"].copy(),
        edge_bnd_mx=bnd["mx"].copy(), edge_bnd_my=bnd["my"].copy(), edge_bnd_mz=bnd["mz"].copy(),
        edge_bnd_dnorm=bnd["d_norm"].copy(), edge_bnd_code=bnd["bc_code"].astype(np.int32),
        cell_nodes_flat=flat,
    )


# ---------------------------------------------------------------------------------------
# per-cell parameter maps
# ---------------------------------------------------------------------------------------
_TOKEN = re.compile(r"[a-zA-Z0-9\-_.+]+")


def _fmt(v: float) -> str:
    return repr(float(v))


def write_map(path: str, names: Sequence[str], columns: Sequence, n_records: int) -> None:
    """Writes a per-cell map.  A column given as a scalar is uniform; if every column is a
    scalar the file is written with ``Unif 1``."""
    uniform = all(np.ndim(c) == 0 for c in columns)
    with open(path, "w") as fh:
        fh.write(f"Unif\t{1 if uniform else 0}\n==== Default Param\n")
        fh.write("\t".join(names) + "\n")
        if uniform:
            fh.write("\t".join(_fmt(c) for c in columns) + "\n==== Distrib\n")
            return
        first = [c if np.ndim(c) == 0 else np.asarray(c)[0] for c in columns]
        fh.write("\t".join(_fmt(c) for c in first) + "\n==== Distrib\n")
        cols = [np.full(n_records, float(c)) if np.ndim(c) == 0 else np.asarray(c, dtype=np.float64)
                for c in columns]
        mat = np.stack(cols, axis=1)
        lines = ["\t".join(repr(v) for v in row) for row in mat.tolist()]
        fh.write("\n".join(lines) + "\n")


def read_map(path: str, n_params: int, n_records: int):
    """Reads a per-cell map (swIO::readVectorParameterFile, swIO.cpp:1005-1191).
    Returns (names, array of shape (n_params, n_records))."""
    with open(path) as fh:
        lines = [ln.rstrip("\r\n") for ln in fh]
    head = _TOKEN.findall(lines[0])
    if len(head) != 2 or head[1] not in ("0", "1"):
        raise ValueError(f"{path}: bad 'Unif' line")
    unif = head[1] == "1"
    names = _TOKEN.findall(lines[2])
    if len(names) != n_params:
        raise ValueError(f"{path}: expected {n_params} parameters, found {len(names)}")
    if unif:
        vals = [float(v) for v in _TOKEN.findall(lines[3])]
        if len(vals) != n_params:
            raise ValueError(f"{path}: bad uniform line")
        return names, np.repeat(np.array(vals)[:, None], n_records, axis=1)
    body = lines[5:5 + n_records]
    if len(body) < n_records:
        raise ValueError(f"{path}: not enough records ({len(body)} < {n_records})")
    arr = np.array([[float(v) for v in _TOKEN.findall(ln)] for ln in body], dtype=np.float64)
    if arr.shape != (n_records, n_params):
        raise ValueError(f"{path}: malformed records")
    return names, arr.T.copy()


# ---------------------------------------------------------------------------------------
# DDP porosity-law maps (DDP_cell_porosity_map.txt, DDP_edge_int/_bnd_porosity_map.txt)
# ---------------------------------------------------------------------------------------
# record length by law type, the count n included (swDdp::porosityLineSize, swDdp.cpp:1099-1211)
def _law_length(law: float, n: float) -> int:
    if law in (-2.0, -1.0):
        return 2 * int(n) + 2
    if law == 0.0:
        return int(n) + 2
    if law == 1.0:
        return 4
    if law == 2.0:
        return 6
    if law == 3.0:
        return 7
    raise ValueError(f"porosity law type {law!r} not in {{-2, -1, 0, 1, 2, 3}}")


@dataclass
class LawRecords:
    """Porosity-law records of one DDP map: record k is ``values[offset[k]:offset[k+1]]`` =
    {law type, n, parameters...} as swDdp::readPorosityFile reads a line (swDdp.cpp:1289-1481)."""

    offset: np.ndarray   # (n_records + 1,) int64
    values: np.ndarray   # float64

    @classmethod
    def uniform(cls, record: Sequence[float], n_records: int) -> "LawRecords":
        rec = np.asarray(record, dtype=np.float64)
        return cls(np.arange(n_records + 1, dtype=np.int64) * rec.size, np.tile(rec, n_records))

    @classmethod
    def from_list(cls, records: Sequence[Sequence[float]]) -> "LawRecords":
        lens = np.array([len(r) for r in records], dtype=np.int64)
        off = np.zeros(len(records) + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        vals = np.concatenate([np.asarray(r, dtype=np.float64) for r in records]) if records else np.zeros(0)
        return cls(off, vals)

    @property
    def count(self) -> int:
        return int(self.offset.shape[0] - 1)

    def record(self, k: int) -> np.ndarray:
        return self.values[self.offset[k]:self.offset[k + 1]]

    def is_uniform(self) -> bool:
        if self.count == 0:
            return True
        lens = np.diff(self.offset)
        if np.any(lens != lens[0]):
            return False
        return bool(np.all(self.values.reshape(self.count, -1) == self.record(0)[None, :]))


def _law_token(v: float, k: int) -> str:
    # law type and count are read with stringToInt: write them as integers
    return str(int(v)) if k < 2 else repr(float(v))


def write_porosity_laws(path: str, laws: LawRecords) -> None:
    """Writes a DDP porosity map (the layout swDdp::readPorosityFile reads, swDdp.cpp:1289-1481):
    ``Unif 1`` with one record when all records are equal, else ``Unif 0`` and one line per record."""
    uniform = laws.is_uniform()
    with open(path, "w") as fh:
        fh.write(f"Unif\t{1 if uniform else 0}\n==== Default Param\n")
        fh.write("law_type\tn\tparameters\n")
        first = laws.record(0) if laws.count else np.array([1.0, 2.0, 0.0, 1.0])
        line0 = "\t".join(_law_token(v, k) for k, v in enumerate(first.tolist()))
        if uniform:
            fh.write(line0 + "\n")
            return
        fh.write(line0 + "\n==== Distrib\n")
        out = []
        for k in range(laws.count):
            out.append("\t".join(_law_token(v, j) for j, v in enumerate(laws.record(k).tolist())))
        fh.write("\n".join(out) + "\n")


def read_porosity_laws(path: str, n_records: int) -> LawRecords:
    """Reads a DDP porosity map as swDdp::readPorosityFile does, with its per-line length check."""
    with open(path) as fh:
        lines = [ln.rstrip("\r\n") for ln in fh]
    head = _TOKEN.findall(lines[0])
    if len(head) != 2 or head[1] not in ("0", "1"):
        raise ValueError(f"{path}: bad 'Unif' line")

    def parse(ln: str) -> List[float]:
        tok = _TOKEN.findall(ln)
        vals = [float(t) for t in tok]
        if len(vals) < 2:
            raise ValueError(f"{path}: misformatted line {ln!r}")
        if len(vals) != _law_length(vals[0], vals[1]):
            raise ValueError(f"{path}: law type {vals[0]} is not compatible with {len(vals) - 1} parameters")
        return vals

    if head[1] == "1":
        return LawRecords.uniform(parse(lines[3]), n_records)
    body = lines[5:5 + n_records]
    if len(body) < n_records:
        raise ValueError(f"{path}: not enough records ({len(body)} < {n_records})")
    return LawRecords.from_list([parse(ln) for ln in body])


def ddp_law_table(record: Sequence[float], base: float, n_por_tab_max: int):
    """(z_tab, phi_tab, theta_tab) of one porosity-law record, restating swDdp::setPorosityCellMap
    (swDdp.cpp:1787-1935) and swDdp::tabulatePorosity (swDdp.cpp:2596-2645) operation for
    operation (Python floats are binary64, evaluated in the reference's order).  Raises where the
    reference would read outside its point list."""
    rec = [float(v) for v in record]
    law, ntab = rec[0], int(n_por_tab_max)

    def tabulate(z, phi):
        nv = len(z)
        dz = (z[nv - 1] - z[0]) / float(ntab - 1)
        zt = [z[0] + float(lv) * dz for lv in range(ntab)]
        interp = [0.0] * ntab
        index = 0
        for lv in range(1, ntab):
            while zt[lv] > z[index]:
                index += 1
                if index >= nv:
                    raise ValueError("tabulated level above the last point")
            if index == 0:
                raise ValueError("points not increasing")
            interp[lv] = phi[index - 1] + (phi[index] - phi[index - 1]) * (zt[lv] - z[index - 1]) / (z[index] - z[index - 1])
        pt = [(interp[lv + 1] + interp[lv]) * 0.5 for lv in range(ntab - 1)] + [phi[nv - 1]]
        return zt, pt

    if law in (-2.0, -1.0):
        nc = int(rec[1])
        z = [base + rec[2 + 2 * k] for k in range(nc)]
        phi = [rec[3 + 2 * k] for k in range(nc)]
        zt, pt = (z, phi) if law == -2.0 else tabulate(z, phi)
    elif law == 0.0:
        nl = int(rec[1])
        zt, pt = tabulate([base + rec[2 + k] for k in range(nl)], [float(k) * 1.0 / float(nl - 1) for k in range(nl)])
    elif law == 1.0:
        z = base + rec[2]
        zt, pt = tabulate([z, z + 1.0], [rec[3], rec[3]])
        pt[0] = rec[3]
    elif law in (2.0, 3.0):
        z0, z1 = base + rec[2], base + rec[4]
        phi0, phi1 = rec[3], rec[5]
        dz = (z1 - z0) / float(ntab - 1)
        dphi = (phi1 - phi0) / float(ntab - 1)
        zt = [z0 + float(lv) * dz for lv in range(ntab - 1)] + [z1]
        pt = [phi0 + (float(lv) + 0.5) * dphi for lv in range(ntab - 1)] + [phi1 if law == 2.0 else rec[6]]
    else:
        raise ValueError(f"porosity law type {law!r} not in {{-2, -1, 0, 1, 2, 3}}")
    theta, th = [0.0], 0.0
    for lv in range(1, len(zt)):
        th += (zt[lv] - zt[lv - 1]) * pt[lv - 1]
        theta.append(th)
    return np.array(zt), np.array(pt), np.array(theta)


# ---------------------------------------------------------------------------------------
# boundary time series
# ---------------------------------------------------------------------------------------
BC_TYPES = {"q": 0, "h": 1, "z": 2, "fr": 3, "phiWq": 4}   # phiWq: DIP only (dip/swDipHyp.cpp:88-101)


@dataclass
class BoundarySeries:
    codes: List[int]
    types: List[str]
    times: np.ndarray                     # (n_records,)
    values: np.ndarray                    # (n_series, n_records)


def write_bc_series(path: str, bc: BoundarySeries) -> None:
    """Writes hydro_boundary_time_series.txt in the layout swIO::readBoundaryTimeSeriesFile reads."""
    n = len(bc.codes)
    with open(path, "w") as fh:
        fh.write("BC\ttime\tseries\nnBCtypes\n")
        fh.write(f"{n}\n--\n")
        fh.write("\t".join(str(c) for c in bc.codes) + "\nTypes\n")
        fh.write("\t" + "\t".join(bc.types) + "\n--\n")
        fh.write("t\t" + "\t".join(f"bc{c}" for c in bc.codes) + "\n")
        for k, t in enumerate(np.asarray(bc.times).tolist()):
            fh.write("\t".join([repr(float(t))] + [repr(float(bc.values[j][k])) for j in range(n)]) + "\n")


def read_bc_series(path: str) -> BoundarySeries:
    with open(path) as fh:
        lines = [ln.rstrip("\r\n") for ln in fh]
    n = int(lines[2].strip())
    codes = [int(v) for v in lines[4].split()]
    types = lines[6].split()
    if len(codes) != n or len(types) != n:
        raise ValueError(f"{path}: inconsistent number of series")
    times, vals = [], [[] for _ in range(n)]
    for ln in lines[9:]:
        if not ln:
            continue
        parts = ln.split()
        times.append(float(parts[0]))
        for j in range(n):
            vals[j].append(float(parts[j + 1]))
    return BoundarySeries(codes=codes, types=types, times=np.array(times), values=np.array(vals))


# ---------------------------------------------------------------------------------------
# input.solv
# ---------------------------------------------------------------------------------------
SOLV_DEFAULTS: Dict[str, str] = {
    # src/sw2dSolver/common/swSolverParam.h:130-194 (the keys this path reads)
    "model_hyperb": "swes", "model_friction": "none", "model_singular_head_loss": "none",
    "num_scheme": "godunov", "topo_discretization": "discontinuous", "negative_depth_detection": "none",
    "cfl_max": "1", "dt_max": "10", "dt_map": "100", "dt_time_series": "100", "h_min": "1e-5",
    "phi_min": "1e-16", "v_max": "100", "fr_max": "100", "t_0": "0", "t_max": "100",
    "div_corr": "none", "store_flag": "default", "output_format": "all", "model_momentum_dissipation": "none",
}


def read_solv(path: str) -> Dict[str, str]:
    """Key/value pairs of input.solv; comment lines start with '#' or '=' (swSolverParam.cpp:690-700)."""
    opts = dict(SOLV_DEFAULTS)
    with open(path) as fh:
        for ln in fh:
            ln = ln.rstrip("\r\n")
            if not ln or ln[0] in "#=":
                continue
            parts = ln.split()
            if len(parts) < 2:
                raise ValueError(f"{path}: misformatted line {ln!r}")
            opts[parts[0].lower()] = parts[1]
    return opts


def write_solv(path: str, opts: Dict[str, object]) -> None:
    with open(path, "w") as fh:
        fh.write("= input.solv written by sw2d_b200\n")
        for k, v in opts.items():
            fh.write(f"{k}\t{v}\n")


# ---------------------------------------------------------------------------------------
# whole cases
# ---------------------------------------------------------------------------------------
@dataclass
class Case:
    """Everything the SP or DIP step needs, in the reference numbering."""

    mesh: Mesh
    opts: Dict[str, str]
    h0: np.ndarray
    q0: np.ndarray
    r0: np.ndarray
    phi: np.ndarray
    boussinesq: np.ndarray
    friction: Optional[np.ndarray] = None      # (3, n): coeff_1, coeff_2, alpha (degrees)
    head_loss: Optional[np.ndarray] = None     # (4, n): h_sing, k1, k2, alpha (degrees)
    bc: Optional[BoundarySeries] = None
    extra: Dict[str, object] = field(default_factory=dict)
    # DIP (model_hyperb dip): phi is the cell porosity phiW; these hold the connectivity porosity
    # of the internal and boundary edges and, with model_momentum_dissipation active, the
    # dissipation map (3, n): mu_1, mu_2, alpha (degrees)
    phi_g_int: Optional[np.ndarray] = None
    phi_g_bnd: Optional[np.ndarray] = None
    mu: Optional[np.ndarray] = None
    # DDP (model_hyperb ddp): porosity laws of the cells, internal and boundary edges; phi is
    # unused, h0/q0/r0 hold the initial-condition columns named by ddp_ic (h|z, q|u, r|v) and
    # mu the dissipation map as for DIP
    ddp_cell: Optional[LawRecords] = None
    ddp_edge_int: Optional[LawRecords] = None
    ddp_edge_bnd: Optional[LawRecords] = None
    ddp_ic: Sequence[str] = ("h", "q", "r")

    @property
    def is_dip(self) -> bool:
        return str(self.opts.get("model_hyperb", "sp")).lower() == "dip"

    @property
    def is_ddp(self) -> bool:
        return str(self.opts.get("model_hyperb", "sp")).lower() == "ddp"


FRICTION_FILES = {"chezy": "friction_chezy_map.txt", "manning": "friction_manning_map.txt",
                  "strickler": "friction_strickler_map.txt"}


def write_case(folder: str, case: Case) -> None:
    """Writes a case folder that the reference sw2dSolver runs unchanged."""
    inp = os.path.join(folder, "input")
    os.makedirs(inp, exist_ok=True)
    n = case.mesh.cell_nb
    write_geometry(os.path.join(inp, "geometry.sw2d"), case.mesh)
    write_solv(os.path.join(inp, "input.solv"), case.opts)
    ic_z = case.extra.get("ic_z") if case.extra else None
    if case.is_ddp:
        # swDdp::setInitialConditions (swDdp.cpp:1608-1726) reads h|z, q|u, r|v
        write_map(os.path.join(inp, "initial_conditions_map.txt"), list(case.ddp_ic),
                  [_collapse(case.h0), _collapse(case.q0), _collapse(case.r0)], n)
    elif ic_z is not None and not np.any(case.q0) and not np.any(case.r0):
        # uniform free surface at rest: "z u v" (swSp::setInitialConditions sets h = max(z - z_b, 0))
        write_map(os.path.join(inp, "initial_conditions_map.txt"), ["z", "u", "v"], [float(ic_z), 0.0, 0.0], n)
    else:
        write_map(os.path.join(inp, "initial_conditions_map.txt"), ["h", "q", "r"],
                  [_collapse(case.h0), _collapse(case.q0), _collapse(case.r0)], n)
    if case.is_dip:
        # swDip::setPorosityParameters / setMomentumDissipationParameters (dip/swDip.cpp:1302-1406)
        write_map(os.path.join(inp, "DIP_cell_porosity_map.txt"), ["DipPhiW"], [case.phi], n)
        write_map(os.path.join(inp, "DIP_edge_int_porosity_map.txt"), ["DipPhiG"], [case.phi_g_int],
                  case.mesh.edge_int_nb)
        write_map(os.path.join(inp, "DIP_edge_bnd_porosity_map.txt"), ["DipPhiG"], [case.phi_g_bnd],
                  case.mesh.edge_bnd_nb)
        if case.opts.get("model_momentum_dissipation", "none") != "none":
            mu = case.mu
            write_map(os.path.join(inp, "cell_momentum_dissipation_map.txt"), ["mu1", "mu2", "alpha"],
                      [mu[0], mu[1], mu[2]], n)
    elif case.is_ddp:
        # swDdp::setPorosityParameters (swDdp.cpp:2241-2316)
        write_porosity_laws(os.path.join(inp, "DDP_cell_porosity_map.txt"), case.ddp_cell)
        write_porosity_laws(os.path.join(inp, "DDP_edge_bnd_porosity_map.txt"), case.ddp_edge_bnd)
        write_porosity_laws(os.path.join(inp, "DDP_edge_int_porosity_map.txt"), case.ddp_edge_int)
        if case.opts.get("model_momentum_dissipation", "none") != "none":
            mu = case.mu
            write_map(os.path.join(inp, "cell_momentum_dissipation_map.txt"), ["mu1", "mu2", "alpha"],
                      [mu[0], mu[1], mu[2]], n)
    else:
        write_map(os.path.join(inp, "SP_cell_porosity_map.txt"), ["SpPhiW"], [case.phi], n)
    write_map(os.path.join(inp, "Boussinesq_map.txt"), ["Beta"], [_collapse(case.boussinesq)], n)
    fm = case.opts.get("model_friction", "none")
    if fm != "none":
        f = case.friction
        write_map(os.path.join(inp, FRICTION_FILES[fm]), ["K1", "K2", "alpha"], [f[0], f[1], f[2]], n)
    if case.opts.get("model_singular_head_loss", "none") != "none":
        hl = case.head_loss
        write_map(os.path.join(inp, "singular_head_loss_map.txt"), ["hsing", "ksing1", "ksing2", "alphasing"],
                  [hl[0], hl[1], hl[2], hl[3]], n)
    write_bc_series(os.path.join(inp, "hydro_boundary_time_series.txt"), case.bc)


def _collapse(arr: np.ndarray):
    """Scalar when uniform (keeps map files small), else the array."""
    a = np.asarray(arr, dtype=np.float64)
    return float(a[0]) if a.size and np.all(a == a[0]) else a


def read_case(folder: str) -> Case:
    """Reads a case folder the way swSp::init does (swSp.cpp:720-969)."""
    inp = os.path.join(folder, "input")
    opts = read_solv(os.path.join(inp, "input.solv"))
    mesh = read_geometry(os.path.join(inp, "geometry.sw2d"))
    n = mesh.cell_nb
    names, ic = read_map(os.path.join(inp, "initial_conditions_map.txt"), 3, n)
    if str(opts.get("model_hyperb", "sp")).lower() == "ddp":
        return _read_ddp_case(inp, opts, mesh, names, ic)
    # swSp::setInitialConditions (swSp.cpp:1119-1224): h or z, then q or u, then r or v
    h = np.zeros(n)
    if "h" in names:
        h = ic[names.index("h")].copy()
    if "z" in names:
        h = np.maximum(ic[names.index("z")] - mesh.cell_z_b, 0.0)
    if "h" not in names and "z" not in names:
        raise ValueError("initial conditions: neither h nor z")
    q = ic[names.index("q")].copy() if "q" in names else None
    if "u" in names:
        q = h * ic[names.index("u")]
    r = ic[names.index("r")].copy() if "r" in names else None
    if "v" in names:
        r = h * ic[names.index("v")]
    if q is None or r is None:
        raise ValueError("initial conditions: discharge columns missing")
    dip = str(opts.get("model_hyperb", "sp")).lower() == "dip"
    pgi = pgb = mu = None
    if dip:
        _, phi = read_map(os.path.join(inp, "DIP_cell_porosity_map.txt"), 1, n)
        _, pgi = read_map(os.path.join(inp, "DIP_edge_int_porosity_map.txt"), 1, mesh.edge_int_nb)
        _, pgb = read_map(os.path.join(inp, "DIP_edge_bnd_porosity_map.txt"), 1, mesh.edge_bnd_nb)
        pgi, pgb = pgi[0].copy(), pgb[0].copy()
        if opts.get("model_momentum_dissipation", "none") != "none":
            _, mu = read_map(os.path.join(inp, "cell_momentum_dissipation_map.txt"), 3, n)
    else:
        _, phi = read_map(os.path.join(inp, "SP_cell_porosity_map.txt"), 1, n)
    _, bous = read_map(os.path.join(inp, "Boussinesq_map.txt"), 1, n)
    fr = None
    fm = opts.get("model_friction", "none")
    if fm != "none":
        _, fr = read_map(os.path.join(inp, FRICTION_FILES[fm]), 3, n)
    hl = None
    if opts.get("model_singular_head_loss", "none") != "none":
        _, hl = read_map(os.path.join(inp, "singular_head_loss_map.txt"), 4, n)
    bc = read_bc_series(os.path.join(inp, "hydro_boundary_time_series.txt"))
    return Case(mesh=mesh, opts=opts, h0=h, q0=q, r0=r, phi=phi[0].copy(), boussinesq=bous[0].copy(),
                friction=fr, head_loss=hl, bc=bc, phi_g_int=pgi, phi_g_bnd=pgb, mu=mu)


def _read_ddp_case(inp: str, opts: Dict[str, str], mesh: Mesh, names: List[str], ic: np.ndarray) -> Case:
    """The DDP part of swDdp::init (swDdp.cpp:780-991): porosity laws, initial-condition columns
    (kept as read: the conversion to thetaW needs the tables), Boussinesq, friction, head loss,
    dissipation, boundary series."""
    n = mesh.cell_nb
    level = "z" if "z" in names else "h" if "h" in names else None
    xcol = "u" if "u" in names else "q" if "q" in names else None
    ycol = "v" if "v" in names else "r" if "r" in names else None
    if level is None or xcol is None or ycol is None:
        raise ValueError("initial conditions: DDP needs h|z, q|u and r|v columns")
    cell = read_porosity_laws(os.path.join(inp, "DDP_cell_porosity_map.txt"), n)
    ebnd = read_porosity_laws(os.path.join(inp, "DDP_edge_bnd_porosity_map.txt"), mesh.edge_bnd_nb)
    eint = read_porosity_laws(os.path.join(inp, "DDP_edge_int_porosity_map.txt"), mesh.edge_int_nb)
    mu = None
    if opts.get("model_momentum_dissipation", "none") != "none":
        _, mu = read_map(os.path.join(inp, "cell_momentum_dissipation_map.txt"), 3, n)
    _, bous = read_map(os.path.join(inp, "Boussinesq_map.txt"), 1, n)
    fr = None
    fm = opts.get("model_friction", "none")
    if fm != "none":
        _, fr = read_map(os.path.join(inp, FRICTION_FILES[fm]), 3, n)
    hl = None
    if opts.get("model_singular_head_loss", "none") != "none":
        _, hl = read_map(os.path.join(inp, "singular_head_loss_map.txt"), 4, n)
    bc = read_bc_series(os.path.join(inp, "hydro_boundary_time_series.txt"))
    return Case(mesh=mesh, opts=opts, h0=ic[names.index(level)].copy(), q0=ic[names.index(xcol)].copy(),
                r0=ic[names.index(ycol)].copy(), phi=np.ones(n), boussinesq=bous[0].copy(), friction=fr,
                head_loss=hl, bc=bc, mu=mu, ddp_cell=cell, ddp_edge_int=eint, ddp_edge_bnd=ebnd,
                ddp_ic=(level, xcol, ycol))
