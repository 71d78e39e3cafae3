"""Seeded synthetic SP cases with the shapes of the benchmark configurations.

The reference ships no benchmark suite; these constructions stand in for it:

* ``dam_break``: plain SP dam break in a 100 m x 20 m channel (jittered Delaunay-like
  triangles, seed 1), flat bed, h = 1.0 m for x < 50 and 0.1 m elsewhere, u = v = 0,
  porosity U[0.6, 1.0] per cell (seed 2), Manning n = 0.03, MUSCL-EVR + the reference's
  slope limiter + HLLC (discontinuous topography), CFL 0.9, reflective walls (q = 0);
* ``gaussian_bumps``: 2 km x 2 km, bed = sum of 50 Gaussian bumps (A ~ U[0,3] m,
  sigma ~ U[20,200] m, seed 3) + 1e-3 x, h = max(0, 2 - z_b) (wet/dry fronts), porosity a
  smoothed random field in [0.3, 1] (seed 4), Manning n lognormal (median 0.03, sigma 0.3,
  seed 5), MUSCL-EVR + HLLC, walls;
* ``channel_features``: a small case exercising every other branch of the path (blending
  topography, Strickler or Chezy friction, singular head loss, 'q' inflow and 'fr'/'h'/'z'
  outflow time series);
* ``dip_channel`` / ``ddp_channel``: the feature channel as a dual integral porosity or a
  depth-dependent porosity (DDP) case.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import numpy as np

from .case import BoundarySeries, Case, LawRecords, ddp_law_table
from .mesh import delaunay_triangle_mesh, jittered_triangle_mesh


def _grid_for(n_cells: int, aspect: float):
    """nx, ny with 2*nx*ny ~ n_cells and nx/ny ~ aspect."""
    ny = max(2, int(round(math.sqrt(n_cells / (2.0 * aspect)))))
    nx = max(2, int(round(n_cells / (2.0 * ny))))
    return nx, ny


def _wall_series(codes):
    # two records: with a single record the reference's cursor interpolation
    # (swBoundaryConditionTimeSeries.cpp:81-95) divides 0 by 0 when t equals that record's time
    return BoundarySeries(codes=list(codes), types=["q"] * len(codes), times=np.array([0.0, 1.0e9]),
                          values=np.zeros((len(codes), 2)))


def _mesh(kind: str, n_cells: int, lx: float, ly: float, seed: int, z_fn=None, bc_code_fn=None):
    """kind "grid": jittered_triangle_mesh (row-major numbering, every interior cell of degree 3);
    kind "delaunay": delaunay_triangle_mesh (seeded jittered-Delaunay, cells in a seeded random
    order)."""
    if kind == "delaunay":
        return delaunay_triangle_mesh(n_cells, lx, ly, seed=seed, z_fn=z_fn, bc_code_fn=bc_code_fn)
    if kind != "grid":
        raise ValueError(f"mesh kind {kind!r}: 'grid' or 'delaunay'")
    nx, ny = _grid_for(n_cells, lx / ly)
    return jittered_triangle_mesh(nx, ny, lx, ly, seed=seed, z_fn=z_fn, bc_code_fn=bc_code_fn)


def dam_break(n_cells: int = 20000, scheme: str = "muscl_evr", friction: str = "manning",
              t_max: float = 1.0e6, seed_mesh: int = 1, seed_phi: int = 2, mesh: str = "grid") -> Case:
    """The plain SP dam break; ``mesh="delaunay"`` is the benchmark configuration's seeded
    jittered-Delaunay mesh (randomly numbered)."""
    kind = mesh
    nx, ny = _grid_for(n_cells, 5.0)
    mesh = _mesh(kind, n_cells, 100.0, 20.0, seed_mesh)
    n = mesh.cell_nb
    h0 = np.where(mesh.cell_x < 50.0, 1.0, 0.1)
    rng = np.random.default_rng(seed_phi)
    phi = rng.uniform(0.6, 1.0, size=n)
    opts = {"model_hyperb": "sp", "model_friction": friction, "num_scheme": scheme,
            "topo_discretization": "discontinuous", "cfl_max": 0.9, "dt_max": 10.0, "dt_map": 100.0,
            "h_min": 1e-5, "t_max": t_max, "store_flag": "none", "output_format": "txt"}
    fr = None
    if friction != "none":
        fr = np.stack([np.full(n, 0.03 if friction == "manning" else 33.3), np.full(n, 0.03 if friction == "manning" else 33.3),
                       np.zeros(n)])
    return Case(mesh=mesh, opts=opts, h0=h0, q0=np.zeros(n), r0=np.zeros(n), phi=phi,
                boussinesq=np.ones(n), friction=fr, bc=_wall_series(mesh.bc_codes()),
                extra={"name": "dam_break", "nx": nx, "ny": ny, "mesh": kind})


def _smooth_field(x, y, lx, ly, seed, coarse=24):
    """Bilinear interpolation of a seeded coarse random grid: a smooth field in [0, 1]."""
    rng = np.random.default_rng(seed)
    g = rng.uniform(0.0, 1.0, size=(coarse + 1, coarse + 1))
    fx = np.clip(x / lx * coarse, 0, coarse - 1e-9)
    fy = np.clip(y / ly * coarse, 0, coarse - 1e-9)
    i = fx.astype(np.int64)
    j = fy.astype(np.int64)
    tx = fx - i
    ty = fy - j
    v = (g[j, i] * (1 - tx) * (1 - ty) + g[j, i + 1] * tx * (1 - ty) + g[j + 1, i] * (1 - tx) * ty +
         g[j + 1, i + 1] * tx * ty)
    lo, hi = v.min(), v.max()
    return (v - lo) / (hi - lo) if hi > lo else np.zeros_like(v)


def gaussian_bumps(n_cells: int = 4_000_000, scheme: str = "muscl_evr", t_max: float = 1.0e6,
                   seed_mesh: int = 1, seed_bed: int = 3, seed_phi: int = 4, seed_n: int = 5, mesh: str = "grid",
                   initial: str = "lake") -> Case:
    """The large SP forward solve.  ``initial="lake"``: h = max(0, 2 - z_b), the configuration's
    initial state (a lake at rest between dry bumps: most of the domain is dry and the wet part
    does not move).  ``initial="dam"``: the same bed under a dam break, free surface 5.0 m for
    x < 1000 m and 3.5 m beyond, water at rest: a moving flow over about 80 % of the cells, with
    wet/dry fronts around the tallest bumps.  ``mesh="delaunay"``: the seeded jittered-Delaunay mesh."""
    kind = mesh
    L = 2000.0
    rng = np.random.default_rng(seed_bed)
    amp = rng.uniform(0.0, 3.0, 50)
    sig = rng.uniform(20.0, 200.0, 50)
    bx = rng.uniform(0.0, L, 50)
    by = rng.uniform(0.0, L, 50)

    def bed(x, y):
        z = 1e-3 * x
        for k in range(50):
            z = z + amp[k] * np.exp(-((x - bx[k]) ** 2 + (y - by[k]) ** 2) / (2 * sig[k] ** 2))
        return z

    nx, ny = _grid_for(n_cells, 1.0)
    mesh = _mesh(kind, n_cells, L, L, seed_mesh, z_fn=bed)
    n = mesh.cell_nb
    if initial == "lake":
        zs = np.full(n, 2.0)
    elif initial == "dam":
        zs = np.where(mesh.cell_x < 0.5 * L, 5.0, 3.5)
    else:
        raise ValueError(f"initial {initial!r}: 'lake' or 'dam'")
    h0 = np.where(zs - mesh.cell_z_b < 0.0, 0.0, zs - mesh.cell_z_b)   # std::max(z - z_b, 0.0)
    phi = 0.3 + 0.7 * _smooth_field(mesh.cell_x, mesh.cell_y, L, L, seed_phi)
    rng_n = np.random.default_rng(seed_n)
    man = np.exp(np.log(0.03) + 0.3 * rng_n.standard_normal(n))
    opts = {"model_hyperb": "sp", "model_friction": "manning", "num_scheme": scheme,
            "topo_discretization": "discontinuous", "cfl_max": 0.9, "dt_max": 10.0, "dt_map": 100.0,
            "h_min": 1e-5, "t_max": t_max, "store_flag": "none", "output_format": "txt"}
    return Case(mesh=mesh, opts=opts, h0=h0, q0=np.zeros(n), r0=np.zeros(n), phi=phi,
                boussinesq=np.ones(n), friction=np.stack([man, man, np.zeros(n)]),
                bc=_wall_series(mesh.bc_codes()),
                extra={"name": "gaussian_bumps", "nx": nx, "ny": ny, "ic_z": 2.0, "mesh": kind, "initial": initial})


def channel_features(n_cells: int = 3000, scheme: str = "godunov", topo: str = "blending",
                     friction: str = "strickler", outflow: str = "fr", head_loss: bool = True,
                     boussinesq: float = 1.0, t_max: float = 40.0, seed: int = 7,
                     impervious: bool = False, h_floor: float = 0.0, h_sing: float = 0.05) -> Case:
    """Sloped 60 m x 12 m channel with bumps, an inflow hydrograph on the left ('q', code -2),
    an outflow condition on the right (code -3) and walls elsewhere (code -1).  The initial
    depth is max(h_floor, 0.45 - z_b) (h_floor > 0: wet everywhere); h_sing is the head-loss
    threshold depth."""
    rng = np.random.default_rng(seed)
    lx, ly = 60.0, 12.0

    def bed(x, y):
        return 0.5 - 0.005 * x + 0.25 * np.exp(-((x - 35.0) ** 2 + (y - 6.0) ** 2) / 8.0)

    def codes(mx, my):
        c = np.full(mx.shape, -1, dtype=np.int32)
        c[mx < 1e-9] = -2
        c[mx > lx - 1e-9] = -3
        return c

    nx, ny = _grid_for(n_cells, 5.0)
    mesh = jittered_triangle_mesh(nx, ny, lx, ly, seed=seed, z_fn=bed, bc_code_fn=codes)
    n = mesh.cell_nb
    h0 = np.maximum(h_floor, 0.45 - mesh.cell_z_b)     # partly dry bed unless h_floor > 0
    phi = rng.uniform(0.5, 1.0, size=n)
    if impervious:
        # phi = 0 next to a dry cell is the configuration the reference rejects as
        # impossible (swSpHyp.cpp:728-739); used by the error-path tests
        phi[rng.uniform(size=n) < 0.02] = 0.0
    opts: Dict[str, object] = {"model_hyperb": "sp", "model_friction": friction, "num_scheme": scheme,
                               "topo_discretization": topo, "cfl_max": 0.8, "dt_max": 0.1, "dt_map": 1.0,
                               "h_min": 1e-5, "t_max": t_max, "fr_max": 10.0, "store_flag": "none",
                               "output_format": "txt"}
    if head_loss:
        opts["model_singular_head_loss"] = "active"
    fr = None
    if friction != "none":
        k = {"strickler": 40.0, "manning": 0.025, "chezy": 30.0}[friction]
        fr = np.stack([k * rng.uniform(0.8, 1.2, n), k * rng.uniform(0.8, 1.2, n), rng.uniform(0.0, 90.0, n)])
    hl = None
    if head_loss:
        hl = np.stack([np.full(n, h_sing), rng.uniform(0.0, 0.5, n), rng.uniform(0.0, 0.5, n), rng.uniform(0.0, 45.0, n)])
    times = np.array([0.0, 5.0, 10.0, 20.0, 30.0, 40.0])
    inflow = np.array([0.0, 0.2, 0.5, 0.5, 0.3, 0.3])
    out_val = {"fr": np.full(6, 0.6), "h": np.full(6, 0.15), "z": np.full(6, 0.35), "q": np.full(6, -0.1)}[outflow]
    mesh_codes = mesh.bc_codes()
    series_codes = [-1, -2, -3]
    assert set(mesh_codes) <= set(series_codes)
    bc = BoundarySeries(codes=series_codes, types=["q", "q", outflow], times=times,
                        values=np.stack([np.zeros(6), inflow, out_val]))
    return Case(mesh=mesh, opts=opts, h0=h0, q0=np.zeros(n), r0=np.zeros(n), phi=phi,
                boussinesq=np.full(n, boussinesq), friction=fr, head_loss=hl, bc=bc,
                extra={"name": "channel_features", "nx": nx, "ny": ny})


def dip_channel(n_cells: int = 3000, scheme: str = "muscl_evr", topo: str = "discontinuous",
                friction: str = "manning", inflow: str = "q", outflow: str = "fr", dissipation: bool = True,
                boussinesq: float = 1.0, t_max: float = 40.0, seed: int = 11) -> Case:
    """The feature channel as a dual integral porosity (DIP) case: a seeded smooth storage
    porosity phiW in [0.4, 1] per cell (building blocks), a connectivity porosity per edge in
    [0.5, 1] x the smaller phiW of its cells (the reference requires phiG <= phiW,
    dip/swDip.cpp:121-240), an inflow of type 'q' (phi q) or 'phiWq' on the left, an outflow
    condition on the right, walls elsewhere, and a momentum-dissipation map."""
    base = channel_features(n_cells=n_cells, scheme=scheme, topo=topo, friction=friction, outflow=outflow,
                            head_loss=False, boussinesq=boussinesq, t_max=t_max, seed=seed)
    mesh = base.mesh
    n = mesh.cell_nb
    rng = np.random.default_rng(seed + 1)
    phiW = 0.4 + 0.6 * _smooth_field(mesh.cell_x, mesh.cell_y, 60.0, 12.0, seed + 2, coarse=12)
    L, R = mesh.edge_int_cells[:, 0], mesh.edge_int_cells[:, 1]
    phi_g_int = np.minimum(phiW[L], phiW[R]) * rng.uniform(0.5, 1.0, size=mesh.edge_int_nb)
    phi_g_bnd = phiW[mesh.edge_bnd_cell] * rng.uniform(0.5, 1.0, size=mesh.edge_bnd_nb)
    opts = dict(base.opts)
    opts["model_hyperb"] = "dip"
    mu = None
    if dissipation:
        opts["model_momentum_dissipation"] = "active"
        mu = np.stack([rng.uniform(0.0, 0.5, n), rng.uniform(0.0, 0.5, n), rng.uniform(0.0, 90.0, n)])
    bc = base.bc
    types = list(bc.types)
    types[1] = inflow
    values = np.array(bc.values, copy=True)
    if inflow == "phiWq":
        values[1] = values[1] * 0.7   # phiW q prescribed directly
    bc = BoundarySeries(codes=bc.codes, types=types, times=bc.times, values=values)
    return Case(mesh=mesh, opts=opts, h0=base.h0, q0=base.q0, r0=base.r0, phi=phiW, boussinesq=base.boussinesq,
                friction=base.friction, head_loss=None, bc=bc, extra={"name": "dip_channel"},
                phi_g_int=phi_g_int, phi_g_bnd=phi_g_bnd, mu=mu)


def _ddp_cell_record(rng, kind: str, ntab: int):
    """One cell porosity-law record (elevations relative to the cell bottom)."""
    z0 = 0.0 if rng.uniform() < 0.7 else float(rng.uniform(0.0, 0.04))
    if kind == "3":    # linear up to z1, then an open level above (an overtopped wall)
        return [3, 5, z0, rng.uniform(0.3, 0.7), z0 + rng.uniform(0.15, 0.5), rng.uniform(0.5, 0.9), rng.uniform(0.8, 1.0)]
    if kind == "2":
        return [2, 4, z0, rng.uniform(0.4, 0.8), z0 + rng.uniform(0.2, 0.7), rng.uniform(0.6, 1.0)]
    if kind == "1":
        return [1, 2, z0, rng.uniform(0.5, 1.0)]
    if kind == "-1":
        k = int(rng.integers(3, 5))
        zs = z0 + np.concatenate([[0.0], np.cumsum(rng.uniform(0.05, 0.3, k - 1))])
        ph = rng.uniform(0.3, 1.0, k)
        return [-1, k] + [v for pair in zip(zs.tolist(), ph.tolist()) for v in pair]
    if kind == "-2":   # pre-tabulated: more levels than n_por_tab_max
        k = ntab + 1
        zs = z0 + np.concatenate([[0.0], np.cumsum(rng.uniform(0.05, 0.2, k - 1))])
        ph = np.sort(rng.uniform(0.3, 1.0, k))
        return [-2, k] + [v for pair in zip(zs.tolist(), ph.tolist()) for v in pair]
    if kind == "0":    # levels only: phi rising from 0 to 1
        k = int(rng.integers(3, 5))
        zs = z0 + np.concatenate([[0.0], np.cumsum(rng.uniform(0.05, 0.3, k - 1))])
        return [0, k] + zs.tolist()
    raise ValueError(kind)


def _ddp_edge_record(rng, pmax: float, nlev: int, ntab: int):
    """An edge record whose tabulated porosities stay below pmax at every level (the reference
    requires phiG <= phiW level by level, swDdp.cpp:180-213) with at most nlev levels."""
    z0 = 0.0 if rng.uniform() < 0.7 else float(rng.uniform(0.0, 0.04))
    u = rng.uniform()
    if u < 0.5 and nlev >= ntab:
        return [3, 5, z0, pmax * rng.uniform(0.3, 1.0), z0 + rng.uniform(0.15, 0.5), pmax * rng.uniform(0.5, 1.0),
                pmax * rng.uniform(0.7, 1.0)]
    if u < 0.75 and nlev >= ntab:
        return [1, 2, z0, pmax * rng.uniform(0.4, 1.0)]
    if u < 0.9 and nlev >= ntab:
        return [2, 4, z0, pmax * rng.uniform(0.4, 1.0), z0 + rng.uniform(0.2, 0.6), pmax * rng.uniform(0.4, 1.0)]
    k = 2
    return [-2, k, z0, pmax * rng.uniform(0.3, 1.0), z0 + rng.uniform(0.1, 0.4), pmax * rng.uniform(0.3, 1.0)]


def ddp_channel(n_cells: int = 3000, friction: str = "manning", inflow_q: float = 0.5, outflow: str = "fr",
                head_loss: bool = False, dissipation: bool = False, div_corr: str = "none", n_it_div_max: int = 10,
                laws: str = "mixed", n_por_tab_max: int = 5, ic: str = "hqr", h_floor: float = 0.0,
                moving: bool = False, boussinesq: float = 1.0, t_max: float = 40.0, seed: int = 21) -> Case:
    """The feature channel as a depth-dependent porosity (DDP) case, Godunov with the
    discontinuous topography (the only path the reference's DDP step runs).  Cells get seeded
    porosity laws: laws="mixed" draws every law type (3: linear with an open top level, 2
    linear, 1 uniform, -1 re-tabulated couples, -2 pre-tabulated couples, 0 levels), "linear"
    only types 3, 2 and 1 (what the large benchmark case uses).  Edge laws stay below their
    cells' tabulated porosity at every level.  The initial state: depth max(h_floor, 0.45 - z_b)
    above the lowest level, a discharge of 0.05 m2/s where wet when moving; ic names the
    initial-condition columns ("hqr", "zuv", ...)."""
    base = channel_features(n_cells=n_cells, scheme="godunov", topo="discontinuous", friction=friction,
                            outflow=outflow, head_loss=head_loss, boussinesq=boussinesq, t_max=t_max, seed=seed,
                            h_floor=h_floor)
    mesh = base.mesh
    n = mesh.cell_nb
    rng = np.random.default_rng(seed + 100)
    if laws == "mixed":
        cell_laws, eint_laws, ebnd_laws, z_tab0 = _ddp_mixed_laws(mesh, rng, n_por_tab_max)
    elif laws == "linear":
        cell_laws, eint_laws, ebnd_laws, z_tab0 = _ddp_linear_laws(mesh, rng)
        _check_uniform_law_levels(cell_laws, mesh.cell_z_b, n_por_tab_max)
        _check_uniform_law_levels(eint_laws, mesh.edge_int_mz, n_por_tab_max)
        _check_uniform_law_levels(ebnd_laws, mesh.edge_bnd_mz, n_por_tab_max)
    else:
        raise ValueError(f"laws {laws!r} not in {{'mixed', 'linear'}}")
    opts = dict(base.opts)
    opts.update({"model_hyperb": "ddp", "n_por_tab_max": n_por_tab_max, "div_corr": div_corr,
                 "n_it_div_max": n_it_div_max, "ddp_chi_phi_max": 20.0})
    mu = None
    if dissipation:
        opts["model_momentum_dissipation"] = "active"
        mu = np.stack([rng.uniform(0.0, 0.5, n), rng.uniform(0.0, 0.5, n), rng.uniform(0.0, 90.0, n)])
    level = base.h0.copy()
    wet = level > 0.0
    qx = np.where(wet, 0.05, 0.0) if moving else np.zeros(n)
    qy = np.where(wet, 0.01, 0.0) if moving else np.zeros(n)
    if ic[0] == "z":
        level = level + z_tab0
    if ic[1] == "u":
        qx = np.where(wet, qx / np.maximum(base.h0, 1e-3), 0.0)
    if ic[2] == "v":
        qy = np.where(wet, qy / np.maximum(base.h0, 1e-3), 0.0)
    bc = base.bc
    values = np.array(bc.values, copy=True)
    values[1] = values[1] * (inflow_q / 0.5)
    bc = BoundarySeries(codes=bc.codes, types=list(bc.types), times=bc.times, values=values)
    return Case(mesh=mesh, opts=opts, h0=level, q0=qx, r0=qy, phi=np.ones(n), boussinesq=base.boussinesq,
                friction=base.friction, head_loss=base.head_loss, bc=bc, mu=mu,
                extra={"name": "ddp_channel"}, ddp_cell=cell_laws, ddp_edge_int=eint_laws, ddp_edge_bnd=ebnd_laws,
                ddp_ic=(ic[0], ic[1], ic[2]))


def _ddp_mixed_laws(mesh, rng, ntab: int):
    """Every law type, record by record (small cases)."""
    n = mesh.cell_nb
    kinds = rng.choice(["3", "2", "1", "-1", "-2", "0"], size=n, p=[0.45, 0.2, 0.15, 0.1, 0.05, 0.05])
    cell_recs, pmin, nlev = [], np.empty(n), np.empty(n, dtype=np.int64)
    for c in range(n):
        while True:
            rec = _ddp_cell_record(rng, str(kinds[c]), ntab)
            try:
                zt, pt, _ = ddp_law_table(rec, float(mesh.cell_z_b[c]), ntab)
                break
            except ValueError:   # a draw the reference cannot tabulate: draw again
                continue
        cell_recs.append(rec)
        pmin[c] = float(np.min(pt))
        nlev[c] = zt.size

    def edge(pmax, nl, base):
        while True:
            rec = _ddp_edge_record(rng, pmax, nl, ntab)
            try:
                ddp_law_table(rec, base, ntab)
                return rec
            except ValueError:
                continue

    L, R = mesh.edge_int_cells[:, 0], mesh.edge_int_cells[:, 1]
    eint = [edge(0.9 * min(pmin[a], pmin[b]), int(min(nlev[a], nlev[b])), float(mz))
            for a, b, mz in zip(L.tolist(), R.tolist(), mesh.edge_int_mz.tolist())]
    ebnd = [edge(0.9 * pmin[c], int(nlev[c]), float(mz))
            for c, mz in zip(mesh.edge_bnd_cell.tolist(), mesh.edge_bnd_mz.tolist())]
    z_tab0 = np.array([float(mesh.cell_z_b[c]) + float(cell_recs[c][2]) for c in range(n)])
    return LawRecords.from_list(cell_recs), LawRecords.from_list(eint), LawRecords.from_list(ebnd), z_tab0


def _records(kind: np.ndarray, columns: Dict[int, np.ndarray]) -> LawRecords:
    """Records of law types 3 (7 values), 2 (6) and 1 (4), built array-wise: columns[t] holds
    the (count_t, length_t) rows of type t in record order."""
    length = np.where(kind == 3, 7, np.where(kind == 2, 6, 4)).astype(np.int64)
    off = np.zeros(kind.size + 1, dtype=np.int64)
    np.cumsum(length, out=off[1:])
    vals = np.empty(int(off[-1]))
    for t, rows in columns.items():
        idx = np.flatnonzero(kind == t)
        if idx.size:
            cols = np.arange(rows.shape[1])
            vals[(off[idx][:, None] + cols[None, :]).reshape(-1)] = rows.reshape(-1)
    return LawRecords(off, vals)


def _linear_rows(kind, rng, pmax=None):
    """Rows of law types 3 / 2 / 1 ({law, n, z0, phi0, z1, phi1[, phi2]} / {1, 2, z0, phi}); with
    pmax the porosities are scaled below it (edges)."""
    m = kind.size
    z0 = np.where(rng.uniform(size=m) < 0.7, 0.0, rng.uniform(0.0, 0.04, m))
    s = np.ones(m) if pmax is None else pmax
    p0 = rng.uniform(0.3, 0.7, m) * (1.0 if pmax is None else 1.0)
    dz3 = rng.uniform(0.15, 0.5, m)
    p1 = rng.uniform(0.5, 0.9, m)
    p2 = rng.uniform(0.8, 1.0, m)
    if pmax is not None:
        p0, p1, p2 = s * rng.uniform(0.3, 1.0, m), s * rng.uniform(0.5, 1.0, m), s * rng.uniform(0.7, 1.0, m)
    q0 = rng.uniform(0.4, 0.8, m) if pmax is None else s * rng.uniform(0.4, 1.0, m)
    q1 = rng.uniform(0.6, 1.0, m) if pmax is None else s * rng.uniform(0.4, 1.0, m)
    dz2 = rng.uniform(0.2, 0.7, m)
    u = rng.uniform(0.5, 1.0, m) if pmax is None else s * rng.uniform(0.4, 1.0, m)
    rows = {3: np.stack([np.full(m, 3.0), np.full(m, 5.0), z0, p0, z0 + dz3, p1, p2], axis=1),
            2: np.stack([np.full(m, 2.0), np.full(m, 4.0), z0, q0, z0 + dz2, q1], axis=1),
            1: np.stack([np.full(m, 1.0), np.full(m, 2.0), z0, u], axis=1)}
    sel = {t: rows[t][kind == t] for t in (3, 2, 1)}
    # smallest tabulated porosity of each record (the tables interpolate between these values)
    pmin = np.where(kind == 3, np.minimum(np.minimum(p0, p1), p2), np.where(kind == 2, np.minimum(q0, q1), u))
    return sel, pmin, z0


def _ddp_linear_laws(mesh, rng):
    """Law types 3, 2 and 1 only, array-wise (large cases)."""
    n = mesh.cell_nb
    kind = rng.choice(np.array([3, 2, 1]), size=n, p=[0.5, 0.3, 0.2])
    rows, pmin, z0 = _linear_rows(kind, rng)
    cell = _records(kind, rows)
    L, R = mesh.edge_int_cells[:, 0], mesh.edge_int_cells[:, 1]
    ki = rng.choice(np.array([3, 2, 1]), size=mesh.edge_int_nb, p=[0.5, 0.25, 0.25])
    ri, _, _ = _linear_rows(ki, rng, pmax=0.9 * np.minimum(pmin[L], pmin[R]))
    kb = rng.choice(np.array([3, 2, 1]), size=mesh.edge_bnd_nb, p=[0.5, 0.25, 0.25])
    rb, _, _ = _linear_rows(kb, rng, pmax=0.9 * pmin[mesh.edge_bnd_cell])
    return cell, _records(ki, ri), _records(kb, rb), mesh.cell_z_b + z0


def _check_uniform_law_levels(laws: LawRecords, base: np.ndarray, ntab: int) -> None:
    """Law type 1 re-tabulates {z, z + 1}: its top level z + (ntab - 1) dz must not exceed z + 1
    after rounding, or the reference reads past its point list (swDdp.cpp:2616-2620)."""
    first = laws.values[laws.offset[:-1]]
    idx = np.flatnonzero(first == 1.0)
    if idx.size == 0:
        return
    z = base[idx] + laws.values[laws.offset[idx] + 2]
    z1 = z + 1.0
    dz = (z1 - z) / float(ntab - 1)
    if np.any(z + float(ntab - 1) * dz > z1):
        raise ValueError(f"n_por_tab_max = {ntab}: a uniform law's top level rounds above its last point")
