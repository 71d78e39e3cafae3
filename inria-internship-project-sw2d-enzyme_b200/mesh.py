"""Synthetic unstructured triangle meshes and the derived SW2D geometry tables.

The generator jitters the interior nodes of a regular grid (seeded) and splits every quad
along the diagonal that satisfies the local Delaunay (empty circumcircle) criterion, which
is the Delaunay triangulation of the jittered points for moderate jitter.  Geometry follows
the reference's conventions so that a case written from it runs unchanged in the reference:

* cell area: shoelace formula (swCell::computeArea, src/common/geometry/swCell.cpp:85-101);
* cell centre and bottom level: vertex means (swCell::computeGravityCenter, swCell.cpp:104-125);
* edge midpoint, length and unit normal, normal oriented from cell L to cell R for internal
  edges and from the edge into the domain for boundary edges (swEdgeIntern.cpp:48-112,
  swEdgeBoundary.cpp:48-112).
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from .case import Mesh


def jittered_triangle_mesh(nx: int, ny: int, lx: float, ly: float, x0: float = 0.0, y0: float = 0.0,
                           jitter: float = 0.2, seed: int = 1,
                           z_fn: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None,
                           bc_code_fn: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None) -> Mesh:
    """Triangulates [x0, x0+lx] x [y0, y0+ly] with 2*nx*ny triangles.

    ``z_fn(x, y)`` gives the node elevations (default 0); ``bc_code_fn(mx, my)`` the negative
    boundary code of each boundary edge from its midpoint (default -1 everywhere).
    """
    x, y, z, tri = jittered_triangles(nx, ny, lx, ly, x0, y0, jitter, seed, z_fn)
    return mesh_from_triangles(x, y, z, tri, bc_code_fn)


def delaunay_triangle_mesh(n_cells: int, lx: float, ly: float, x0: float = 0.0, y0: float = 0.0,
                           jitter: float = 0.3, seed: int = 1, permute: bool = True,
                           z_fn: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None,
                           bc_code_fn: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None) -> Mesh:
    """Seeded jittered-Delaunay triangulation of [x0, x0+lx] x [y0, y0+ly] with about n_cells
    triangles.

    Nodes: a grid of cell-centred points (spacing d with lx*ly / d^2 ~ n_cells / 2), each moved
    by a seeded uniform jitter of +-jitter*d in x and y, plus points every d along the four sides
    (corners included).  Triangles: the Delaunay triangulation of those nodes
    (scipy.spatial.Delaunay, i.e. Qhull).  Cell degrees vary (1 to 3 internal neighbours), and
    with ``permute`` the triangles are listed in a seeded random order, so the cell and edge
    numbering a solver receives carries no locality of its own.
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    d = float(np.sqrt(lx * ly / max(n_cells / 2.0, 1.0)))
    nx = max(2, int(round(lx / d)))
    ny = max(2, int(round(ly / d)))
    dx, dy = lx / nx, ly / ny
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny))
    xi = x0 + (ii.reshape(-1) + 0.5) * dx + rng.uniform(-jitter, jitter, ii.size) * dx
    yi = y0 + (jj.reshape(-1) + 0.5) * dy + rng.uniform(-jitter, jitter, jj.size) * dy
    bx = x0 + np.arange(nx + 1) * dx
    by = y0 + np.arange(1, ny) * dy
    xb = np.concatenate([bx, bx, np.full(by.size, x0), np.full(by.size, x0 + lx)])
    yb = np.concatenate([np.full(bx.size, y0), np.full(bx.size, y0 + ly), by, by])
    x = np.concatenate([xb, xi])
    y = np.concatenate([yb, yi])
    tri = Delaunay(np.stack([x, y], 1)).simplices.astype(np.int64)
    # drop slivers of zero area (collinear boundary nodes)
    px, py = x[tri], y[tri]
    area2 = (px[:, 1] - px[:, 0]) * (py[:, 2] - py[:, 0]) - (px[:, 2] - px[:, 0]) * (py[:, 1] - py[:, 0])
    tri = tri[np.abs(area2) > 1e-12 * dx * dy]
    if permute:
        tri = tri[np.random.default_rng(seed + 1_000_003).permutation(tri.shape[0])]
    z = z_fn(x, y) if z_fn is not None else np.zeros_like(x)
    return mesh_from_triangles(x, y, np.asarray(z, dtype=np.float64), tri, bc_code_fn)


def jittered_triangles(nx: int, ny: int, lx: float, ly: float, x0: float = 0.0, y0: float = 0.0,
                       jitter: float = 0.2, seed: int = 1,
                       z_fn: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None):
    """Nodes (x, y, z) and triangles of jittered_triangle_mesh: the triangles of quad q of the
    grid (row-major, q = j nx + i) are rows 2q and 2q + 1."""
    rng = np.random.default_rng(seed)
    dx, dy = lx / nx, ly / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1))
    ii = ii.reshape(-1)
    jj = jj.reshape(-1)
    x = x0 + ii * dx
    y = y0 + jj * dy
    interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)
    jx = rng.uniform(-jitter, jitter, size=x.shape) * dx
    jy = rng.uniform(-jitter, jitter, size=y.shape) * dy
    x = np.where(interior, x + jx, x)
    y = np.where(interior, y + jy, y)
    z = z_fn(x, y) if z_fn is not None else np.zeros_like(x)
    z = np.asarray(z, dtype=np.float64)

    qi, qj = np.meshgrid(np.arange(nx), np.arange(ny))
    qi = qi.reshape(-1)
    qj = qj.reshape(-1)
    a = qj * (nx + 1) + qi
    b = a + 1
    c = a + (nx + 1) + 1
    d = a + (nx + 1)

    def angle(p, q0, q1):
        ux, uy = x[q0] - x[p], y[q0] - y[p]
        vx, vy = x[q1] - x[p], y[q1] - y[p]
        return np.arctan2(np.abs(ux * vy - uy * vx), ux * vx + uy * vy)

    # diagonal a-c is locally Delaunay iff the angles opposite to it sum to <= pi
    use_ac = angle(b, c, a) + angle(d, a, c) <= np.pi
    t0 = np.where(use_ac[:, None], np.stack([a, b, c], 1), np.stack([a, b, d], 1))
    t1 = np.where(use_ac[:, None], np.stack([a, c, d], 1), np.stack([b, c, d], 1))
    tri = np.empty((2 * qi.size, 3), dtype=np.int64)
    tri[0::2] = t0
    tri[1::2] = t1
    return x, y, z, tri


def mesh_from_triangles(x: np.ndarray, y: np.ndarray, z: np.ndarray, tri: np.ndarray,
                        bc_code_fn: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None) -> Mesh:
    """SW2D tables of a triangulation (counter-clockwise triangles not required)."""
    nc = tri.shape[0]
    px, py = x[tri], y[tri]
    cross = px * np.roll(py, -1, axis=1) - np.roll(px, -1, axis=1) * py
    area = np.abs(cross.sum(axis=1)) / 2
    side = np.sqrt((px - np.roll(px, -1, axis=1)) ** 2 + (py - np.roll(py, -1, axis=1)) ** 2)
    perim = side.sum(axis=1)
    cx = px.sum(axis=1) / 3
    cy = py.sum(axis=1) / 3
    czb = z[tri].sum(axis=1) / 3

    # edges: node pairs of each triangle, grouped
    e0 = tri.reshape(-1)
    e1 = np.roll(tri, -1, axis=1).reshape(-1)
    owner = np.repeat(np.arange(nc), 3)
    lo = np.minimum(e0, e1)
    hi = np.maximum(e0, e1)
    key = lo * (int(x.size) + 1) + hi
    order = np.lexsort((owner, key))
    key_s = key[order]
    first = np.ones(key_s.size, dtype=bool)
    first[1:] = key_s[1:] != key_s[:-1]
    grp = np.cumsum(first) - 1
    counts = np.bincount(grp)
    if counts.max() > 2:
        raise ValueError("non-manifold triangulation")
    starts = np.nonzero(first)[0]
    is_int = counts == 2
    s_int = starts[is_int]
    s_bnd = starts[~is_int]

    # internal edges: L = lower cell index, R = higher; ordered by (L, R)
    cL = owner[order[s_int]]
    cR = owner[order[s_int + 1]]
    n_a = lo[order[s_int]]
    n_b = hi[order[s_int]]
    eo = np.lexsort((cR, cL))
    cL, cR, n_a, n_b = cL[eo], cR[eo], n_a[eo], n_b[eo]
    length = np.sqrt((x[n_a] - x[n_b]) ** 2 + (y[n_a] - y[n_b]) ** 2)
    nxv = (y[n_b] - y[n_a]) / length
    nyv = -(x[n_b] - x[n_a]) / length
    flip = (nxv * (cx[cR] - cx[cL]) + nyv * (cy[cR] - cy[cL])) < 0
    nxv = np.where(flip, -nxv, nxv)
    nyv = np.where(flip, -nyv, nyv)
    n_first = np.where(flip, n_b, n_a)
    n_second = np.where(flip, n_a, n_b)
    mx = (x[n_a] + x[n_b]) / 2
    my = (y[n_a] + y[n_b]) / 2
    mz = (z[n_a] + z[n_b]) / 2
    dnorm = np.abs(nxv * (cx[cR] - cx[cL]) + nyv * (cy[cR] - cy[cL]))

    # boundary edges, ordered by cell
    bc_cell = owner[order[s_bnd]]
    b_a = lo[order[s_bnd]]
    b_b = hi[order[s_bnd]]
    bo = np.argsort(bc_cell, kind="stable")
    bc_cell, b_a, b_b = bc_cell[bo], b_a[bo], b_b[bo]
    blen = np.sqrt((x[b_a] - x[b_b]) ** 2 + (y[b_a] - y[b_b]) ** 2)
    bmx = (x[b_a] + x[b_b]) / 2
    bmy = (y[b_a] + y[b_b]) / 2
    bmz = (z[b_a] + z[b_b]) / 2
    bnx = (y[b_b] - y[b_a]) / blen
    bny = -(x[b_b] - x[b_a]) / blen
    bflip = (bnx * (cx[bc_cell] - bmx) + bny * (cy[bc_cell] - bmy)) < 0
    bnx = np.where(bflip, -bnx, bnx)
    bny = np.where(bflip, -bny, bny)
    bfirst = np.where(bflip, b_b, b_a)
    bsecond = np.where(bflip, b_a, b_b)
    bdn = np.abs(bnx * cx[bc_cell] + bny * cy[bc_cell])
    codes = (np.asarray(bc_code_fn(bmx, bmy), dtype=np.int32) if bc_code_fn is not None
             else np.full(bc_cell.size, -1, dtype=np.int32))

    tri_ccw = tri.copy()
    cw = cross.sum(axis=1) < 0
    tri_ccw[cw] = tri_ccw[cw][:, ::-1]
    return Mesh(
        node_x=x, node_y=y, node_z=z, cell_nodes=[], cell_area=area, cell_perimeter=perim,
        cell_x=cx, cell_y=cy, cell_z_b=czb,
        edge_int_cells=np.stack([cL, cR], 1).astype(np.int64), edge_int_nodes=np.stack([n_first, n_second], 1),
        edge_int_length=length, edge_int_nx=nxv, edge_int_ny=nyv, edge_int_mx=mx, edge_int_my=my,
        edge_int_mz=mz, edge_int_dnorm=dnorm,
        edge_bnd_cell=bc_cell.astype(np.int64), edge_bnd_nodes=np.stack([bfirst, bsecond], 1),
        edge_bnd_length=blen, edge_bnd_nx=bnx, edge_bnd_ny=bny, edge_bnd_mx=bmx, edge_bnd_my=bmy,
        edge_bnd_mz=bmz, edge_bnd_dnorm=bdn, edge_bnd_code=codes, cell_nodes_flat=tri_ccw,
    )
