"""Porosity assimilation: the host-side mirror of the reference's assimilation front-end (class
swSpE, assim/swSpE*.cpp, and its driver assim/main_enzyme.cpp) over the GPU engine
(sw2d_assim_* of include/sw2d_b200.h).

* :class:`AssimConfig` — the assimilation keys of input.solv, parsed and defaulted as
  assim/assimConfig.cpp does.
* :class:`SpE` — a model with the reference's method names:
  ``build_checkpoint_records`` (the dry run), ``replay_trajectory_cost`` (``func``),
  ``get_spatial_gradient_checkpointed`` (``grad``; the reference differentiates with Enzyme,
  this one runs the GPU's hand-written reverse sweep).  ``SpE.from_folder`` reads a case folder
  the way main_enzyme.cpp does: the assimilation keys, the observations of
  reference/ResultHydro_p*.txt (or the gauge file), the cost weights.
* :class:`PorosityProblem` and :func:`run_minimization` — the reference's minimisation
  (assim/swSpE_minimize.cpp:264-1073): J_data + ridge + L1 + spatial (H1) + phi_ref penalty over
  the free cells, zonation, the descent log ``descent/descent_log.csv`` with the reference's
  columns and a porosity map per evaluation.  L-BFGS-B is scipy's (the reference links LBFGSpp,
  absent here); "gd" is the reference's projected gradient descent with Armijo backtracking.
"""
from __future__ import annotations

import glob
import math
import os
import re
import shutil
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .case import read_case, read_map, write_map
from .solver import SpModel

DESCENT_COLUMNS = ("iter,J_total,J_data,ridge,rel_init_pct,rel_prev_pct,gradJm_L2,gradJm_Linf,gradJm_argmax,"
                   "gradJphys_L2,gradJphys_max,gradJphys_argmax,dh_peak,phi_min,phi_max,phi_mean,n_phi_lt_0p5,"
                   "n_phi_lt_0p05,n_phi_upper_clamp,adam_step,sse_phi_ref")

_TRUE = ("1", "true", "yes", "on")


@dataclass
class AssimConfig:
    """The keys of assim/assimConfig.h:17-55 with their defaults."""
    minimize_algo: str = "bfgs"
    adam_step_size: float = 0.05
    adam_safe: bool = False
    alpha_l1: float = 0.0
    alpha_phi_ref: float = 0.0
    alpha_spatial: float = 0.0
    lambda_tanh: float = 1.0
    lbfgsb_epsilon: float = 1e-5
    lbfgsb_m: int = 6
    lbfgsb_max_linesearch: int = 20
    phi_transform: str = "none"
    phi_lower_bound: float = 0.0
    phi_upper_bound: float = 1.0
    t_state_assimilation: float = 0.0
    dt_map_ad: float = -1.0
    windowed_assimilation: bool = False
    assimilation_window_duration: float = -1.0
    assimilation_window_steps: int = -1
    n_assimilation_windows: int = 1
    zonation: bool = False
    mask_dry_cells: bool = False
    mask_wall_gradient: bool = False
    cost_normalize: bool = False
    obs_type: str = "cells"
    h_weight: str = "1.0"
    q_weight: str = "1.0"
    porosity_ref_map: str = ""
    porosity_free_zone_map: str = ""
    alpha_reg: float = 0.0
    checkpoint_stride: int = 30
    max_it: int = 3
    porosity_ebauche_map: str = ""

    @classmethod
    def from_opts(cls, opts: Dict[str, str]) -> "AssimConfig":
        """AssimConfig::load_and_filter (assim/assimConfig.cpp:94-147) on the key/value pairs of
        input.solv (keys lower-cased)."""
        c = cls()
        for name, f in cls.__dataclass_fields__.items():
            if name not in opts:
                continue
            v = str(opts[name])
            if f.type in ("bool", bool):
                setattr(c, name, v.lower() in _TRUE)
            elif f.type in ("int", int):
                setattr(c, name, int(v))
            elif f.type in ("float", float):
                setattr(c, name, float(v))
            else:
                setattr(c, name, v)
        c.phi_transform = c.phi_transform.lower()
        if c.phi_transform not in ("none", "clamp", "tanh", "normalize"):
            c.phi_transform = "none"
        return c


def time_from_file_name(name: str) -> float:
    """swIO::timeFromFileName (src/common/swIO.cpp:1194-1226): "ResultHydro_pDDDDdHHhMMmSSsMMM"."""
    base = os.path.basename(name)
    if base.startswith("ResultHydro_"):
        ts = base[13:30]
    elif base.startswith("ResultTime_"):
        ts = base[12:29]
    else:
        raise ValueError(f"file format not recognized: {base}")
    days, hours, minutes, seconds, ms = int(ts[0:4]), int(ts[5:7]), int(ts[8:10]), int(ts[11:13]), int(ts[14:17])
    return ms / 1000. + seconds + 60 * (minutes + 60 * (hours + 24 * days))


def load_observations(folder: str, n_cells: int, t_begin: float, t_end: float):
    """swSpE::load_all_observations + load_single_observation_file (assim/swSpE_ad.cpp:47-154):
    the maps reference/ResultHydro_p*.txt with t in [t_begin, t_end] (1e-6 tolerance), columns
    3..5 (h, qx, qy) of the first n_cells data lines.  Returns (times, frames[k][3][n])."""
    files = []
    for f in glob.glob(os.path.join(folder, "reference", "ResultHydro_p*.txt")):
        t = time_from_file_name(f)
        if t_begin - 1e-6 <= t <= t_end + 1e-6:
            files.append((t, f))
    files.sort()
    times, frames = [], []
    for t, f in files:
        frame = np.zeros((3, n_cells))
        with open(f) as fh:
            fh.readline()
            k = 0
            for line in fh:
                if k >= n_cells:
                    break
                if not line.strip():
                    continue
                tok = line.split()
                for col in range(3):
                    if 3 + col < len(tok):
                        frame[col, k] = float(tok[3 + col])
                k += 1
        times.append(t)
        frames.append(frame)
    return np.array(times), np.array(frames).reshape(len(times), 3, n_cells)


def load_gauge_observations(path: str, src_cols: Sequence[int], t_begin: float, t_end: float):
    """swSpE::load_gauge_observations (assim/swSpE_gauges.cpp:94-160): a probes time-series file
    (header lines, then "time ..." and rows time zb1 h1 q1 r1 zb2 ...); the depth of probe g is
    column 2 + 4 g.  Returns (times, values[k][gauge])."""
    times, rows = [], []
    header = False
    with open(path) as fh:
        for line in fh:
            if not line.strip():
                continue
            if not header:
                header = line.startswith("time")
                continue
            cols = [float(v) for v in line.split()]
            if not cols or cols[0] < t_begin - 1e-6 or cols[0] > t_end + 1e-6:
                continue
            idx = [2 + 4 * g for g in src_cols]
            if max(idx) >= len(cols):
                continue
            times.append(cols[0])
            rows.append([cols[i] for i in idx])
    return np.array(times), np.array(rows).reshape(len(times), len(src_cols))


def load_map(path: str, n_cells: int) -> np.ndarray:
    """The reader swSpE::load_phi_csv (assim/swSpE_minimize.cpp:130-197): the SW2D map format
    ("Unif ..." first line) or "cell_id,value" rows with an optional header."""
    with open(path) as fh:
        first = ""
        for first in fh:
            if first.strip():
                break
    if first.strip().lower().startswith("unif"):
        _, arr = read_map(path, 1, n_cells)
        return arr[0].copy()
    out = np.zeros(n_cells)
    count = 0
    with open(path) as fh:
        lines = fh.read().splitlines()
    if lines and not (lines[0][:1].isdigit() or lines[0][:1] in "+-"):
        lines = lines[1:]
    for line in lines:
        tok = line.replace(",", " ").split()
        if len(tok) < 2:
            continue
        i = int(tok[0])
        if i < 0 or i >= n_cells:
            raise ValueError(f"{path}: cell id {i} out of range")
        out[i] = float(tok[1])
        count += 1
    if count != n_cells:
        raise ValueError(f"{path}: {count} values for {n_cells} cells")
    return out


def result_file_name(prefix: str, t: float) -> str:
    """swIO::computeFileNameFromTime (src/common/swIO.cpp:51-87): prefix + DDDDdHHhMMmSSsmmm.txt,
    the digits taken the way the reference computes them (truncations of float quotients, the
    milliseconds rounded with +0.499999)."""
    nb_d = int(t / 86400.)
    nb_d_e3 = int(nb_d / 1000.)
    nb_d_e2 = int((nb_d - 1000. * nb_d_e3) / 100.)
    nb_d_e1 = int((nb_d - 1000. * nb_d_e3 - 100. * nb_d_e2) / 10.)
    nb_d_e0 = int(nb_d - 1000. * nb_d_e3 - 100. * nb_d_e2 - 10. * nb_d_e1)
    nb_h = int((t - float(np.float32(nb_d)) * 86400.) / 3600.)
    nb_h_e1 = int(nb_h / 10.)
    nb_h_e0 = int(nb_h - 10. * nb_h_e1)
    nb_m = int((t - nb_d * 86400. - nb_h * 3600.) / 60.)
    nb_m_e1 = int(nb_m / 10.)
    nb_m_e0 = int(nb_m - 10. * nb_m_e1)
    nb_s = int(t - 86400. * nb_d - 3600. * nb_h - 60. * nb_m)
    nb_s_e1 = int(nb_s / 10.)
    nb_s_e0 = int(nb_s - 10. * nb_s_e1)
    nb_mill = int((t - int(t)) * 1000. + 0.499999)
    nb_mill_e2 = int(nb_mill / 100.)
    nb_mill_e1 = int((nb_mill - 100 * nb_mill_e2) / 10.)
    nb_mill_e0 = int(nb_mill - 100 * nb_mill_e2 - 10 * nb_mill_e1)
    return (f"{prefix}{nb_d_e3}{nb_d_e2}{nb_d_e1}{nb_d_e0}d{nb_h_e1}{nb_h_e0}h{nb_m_e1}{nb_m_e0}m"
            f"{nb_s_e1}{nb_s_e0}s{nb_mill_e2}{nb_mill_e1}{nb_mill_e0}.txt")


def write_map_decimal(path: str, names: Sequence[str], cols: Sequence[np.ndarray], precision: int) -> None:
    """swIO::createTxtFileMapDecimal (src/common/swIO.cpp:182-222): a header of the names, each
    padded with spaces to precision + 7 characters and followed by a tab, then one line per cell
    of the values in scientific notation with `precision` digits, each followed by a tab."""
    width = precision + 7
    lines = ["".join(nm + " " * max(0, width - len(nm)) + "\t" for nm in names)]
    fmt = f"{{:.{precision}e}}\t"
    arrs = [np.asarray(c, dtype=np.float64) for c in cols]
    for i in range(arrs[0].size):
        lines.append("".join(fmt.format(float(a[i])) for a in arrs))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def resolve_weight(spec: str, folder: str, n_cells: int) -> np.ndarray:
    """swSpE::resolve_cost_weight (assim/swSpE_core.cpp:268-298): a number (uniform weight) or a
    map path relative to the case folder; an unreadable map gives weight 1."""
    try:
        return np.full(n_cells, float(spec))
    except ValueError:
        pass
    try:
        return load_map(os.path.join(folder, spec), n_cells)
    except (OSError, ValueError):
        return np.ones(n_cells)


def locate_gauges(mesh, xs: Sequence[float], ys: Sequence[float]) -> Tuple[List[int], List[int]]:
    """swSpE::locate_gauges (assim/swSpE_gauges.cpp:41-92): the cell containing each probe
    (probes outside the mesh are left out).  Returns (cells, probe indices kept)."""
    cells, kept = [], []
    nx, ny = np.asarray(mesh.node_x), np.asarray(mesh.node_y)
    for i, (x, y) in enumerate(zip(xs, ys)):
        found = -1
        order = np.argsort((mesh.cell_x - x) ** 2 + (mesh.cell_y - y) ** 2)
        for c in order[:32]:
            nodes = np.asarray(mesh.cell_nodes[c])
            px, py = nx[nodes], ny[nodes]
            inside = True
            k = len(nodes)
            for a in range(k):
                b = (a + 1) % k
                if (px[b] - px[a]) * (y - py[a]) - (py[b] - py[a]) * (x - px[a]) < -1e-12:
                    inside = False
                    break
            if inside:
                found = int(c)
                break
        if found >= 0:
            cells.append(found)
            kept.append(i)
    return cells, kept


class SpE:
    """The reference's swSpE over the GPU: an SP model with the assimilation engine configured."""

    def __init__(self, model: SpModel, config: AssimConfig, folder: Optional[str] = None):
        self.model = model
        self.cfg = config
        self.folder = folder
        self.n = model.n
        c = config
        self._conf = dict(phi_transform=c.phi_transform, lambda_tanh=c.lambda_tanh,
                          windowed=c.windowed_assimilation, window_duration=c.assimilation_window_duration,
                          window_steps=c.assimilation_window_steps, n_windows=max(1, c.n_assimilation_windows),
                          t_state_assimilation=c.t_state_assimilation, cost_normalize=c.cost_normalize,
                          mask_wall_gradient=c.mask_wall_gradient)
        model.assim_configure(**self._conf)
        self.diag: Dict[str, object] = {}

    def set_forced_first_segment(self, seg: int) -> None:
        """forced_first_seg_ of the reference's L-BFGS-B driver (assim/swSpE_minimize.cpp:881-903):
        while it is >= 0 every gradient's window starts at that segment; -1 lets each gradient cut
        its window at its own truncation point again."""
        self.model.assim_configure(**self._conf, forced_first_segment=int(seg))

    @classmethod
    def from_folder(cls, folder: str, device: int = 0, load_obs: bool = True) -> "SpE":
        """assim/main_enzyme.cpp:76-131 and 196-219: read the case and its assimilation keys, then
        the observations (obs_type cells: reference/ResultHydro_p*.txt in [t_state_assimilation,
        t_max]; gauges: reference/gauges.txt at the probes of input/probes_location.txt)."""
        case = read_case(folder)
        cfg = AssimConfig.from_opts(case.opts)
        model = SpModel(case, device)
        spe = cls(model, cfg, folder)
        if load_obs:
            spe.load_observations()
        return spe

    def load_observations(self) -> int:
        c, folder = self.cfg, self.folder
        t_end = float(self.model.case.opts.get("t_max", 0.0))
        if c.obs_type == "gauges":
            xs, ys = _read_probes(os.path.join(folder, "input", "probes_location.txt"))
            cells, kept = locate_gauges(self.model.case.mesh, xs, ys)
            times, vals = load_gauge_observations(os.path.join(folder, "reference", "gauges.txt"), kept,
                                                  c.t_state_assimilation, t_end)
            self.set_gauges(times, cells, np.ones(len(cells)), vals)
        else:
            times, frames = load_observations(folder, self.n, c.t_state_assimilation, t_end)
            wh = resolve_weight(c.h_weight, folder, self.n)
            wq = resolve_weight(c.q_weight, folder, self.n)
            self.set_frames(times, frames, wh, wq)
        return len(times)

    def set_frames(self, times, frames, h_weight=None, q_weight=None) -> None:
        self.model.assim_set_frames(times, frames, h_weight, q_weight)

    def set_gauges(self, times, cells, weights, values) -> None:
        self.model.assim_set_gauges(times, cells, weights, values)

    # ---- the reference's methods
    def build_checkpoint_records(self, phi_map, stride: Optional[int] = None) -> Tuple[int, int]:
        return self.model.assim_record(phi_map, stride or self.cfg.checkpoint_stride)

    def replay_trajectory_cost(self, phi_map) -> float:
        return self.model.assim_replay_cost(phi_map)

    def get_spatial_gradient_checkpointed(self, phi_map, stride: Optional[int] = None) -> np.ndarray:
        """dJ/dm at phi_map (the optimisation variable m: phi = phi_correct(m)); the diagnostics
        (grad_l2, grad_max, grad_argmax, dh_peak, window, tiles, J) go to self.diag."""
        g, info = self.model.assim_gradient(phi_map, stride or self.cfg.checkpoint_stride)
        self.diag = info
        return g

    def observation_grid(self) -> np.ndarray:
        """The observation times generate_references_E synthesises (swSpE_checkpoint.cpp:482-496):
        the multiples of dt_map_ad in [t_state_assimilation, t_max] (1e-16 slack at both ends)."""
        c = self.cfg
        dt_ref = float(c.dt_map_ad)
        if not dt_ref > 1e-16:
            raise ValueError(f"generate_references_E: invalid dt_map_ad ({dt_ref})")
        t_max = float(self.model.case.opts["t_max"])
        k0 = max(0, int(math.ceil((c.t_state_assimilation - 1e-16) / dt_ref)))
        times = []
        k = k0
        while True:
            tt = float(k) * dt_ref
            if tt > t_max + 1e-16:
                break
            if tt >= c.t_state_assimilation - 1e-16:
                times.append(tt)
            k += 1
        if not times:
            raise ValueError(f"generate_references_E: no observation time in [{c.t_state_assimilation}, {t_max}] "
                             f"(dt_map_ad = {dt_ref})")
        return np.array(times)

    def generate_references_E(self, phi_map, out_dir: str, stride: Optional[int] = None) -> List[str]:
        """The reference's gen-ref-e mode (swSpE::generate_references_E,
        assim/swSpE_checkpoint.cpp:470-515): the _E forward (the dry run at control phi_map) on the
        synthesised observation grid, and at every observation it lands on, the state written as
        storeReferenceMap does (swSpE_core.cpp:300-340): out_dir/ResultHydro_p<time>.txt with the
        columns x, y, zb, water_depth, unit_discharge_x, unit_discharge_y, unit_discharge_norm, in
        n_decimal-digit scientific notation.  Returns the files written.  Replaying the same _E
        trajectory at phi_map against these maps then gives J = 0 up to their printed digits."""
        times = self.observation_grid()
        n = self.n
        self.set_frames(times, np.zeros((times.size, 3, n)))
        m = np.ascontiguousarray(phi_map, dtype=np.float64)
        self.model.assim_record(m, stride or self.cfg.checkpoint_stride)
        h, q, r, landed = self.model.assim_trigger_states(m, times.size)
        dt, trig = self.model.assim_steps()
        # the time after each step, accumulated as the engine does (t_{j+1} = t_j + dt_j)
        t = float(self.model.assim_segments()[0][0]) if dt.size else 0.0
        t_after = np.empty(dt.size)
        for j in range(dt.size):
            t = t + float(dt[j])
            t_after[j] = t
        mesh = self.model.case.mesh
        digits = int(self.model.case.opts.get("n_decimal", 10))
        os.makedirs(out_dir, exist_ok=True)
        written = []
        for j in np.nonzero(trig >= 0)[0]:
            k = int(trig[j])
            if k >= times.size:
                continue
            path = os.path.join(out_dir, result_file_name("ResultHydro_p", float(t_after[j])))
            cols = [mesh.cell_x, mesh.cell_y, mesh.cell_z_b, h[k], q[k], r[k], np.sqrt(q[k] * q[k] + r[k] * r[k])]
            write_map_decimal(path, ["x", "y", "zb", "water_depth", "unit_discharge_x", "unit_discharge_y",
                                     "unit_discharge_norm"], cols, digits)
            written.append(path)
        self.diag["gen_ref_e"] = {"observations": int(times.size), "written": len(written), "landed": landed}
        return written

    # ---- swSpE::phi_correct / dphi_dm / m_from_phi (assim/swSpE.h:59-107)
    def phi_correct(self, m) -> np.ndarray:
        m = np.asarray(m, dtype=np.float64)
        t = self.cfg.phi_transform
        if t == "clamp":
            return np.clip(m, 0.0, 1.05)
        if t == "tanh":
            return 1.0 / (1.0 + np.exp(-self.cfg.lambda_tanh * m))
        if t == "normalize":
            lo, hi = float(m.min()), float(m.max())
            return (m - lo) / (hi - lo) if hi - lo >= 1e-12 else m.copy()
        return m.copy()

    def dphi_dm(self, m) -> np.ndarray:
        m = np.asarray(m, dtype=np.float64)
        t = self.cfg.phi_transform
        if t == "clamp":
            return np.where((m < 0.0) | (m > 1.05), 0.0, 1.0)
        if t == "tanh":
            s = 1.0 / (1.0 + np.exp(-self.cfg.lambda_tanh * m))
            return self.cfg.lambda_tanh * s * (1.0 - s)
        if t == "normalize":
            lo, hi = float(m.min()), float(m.max())
            return np.full_like(m, 1.0 / (hi - lo)) if hi - lo >= 1e-12 else np.ones_like(m)
        return np.ones_like(m)

    def m_from_phi(self, phi) -> np.ndarray:
        phi = np.asarray(phi, dtype=np.float64)
        t = self.cfg.phi_transform
        if t == "tanh":
            p = np.clip(phi, 1e-2, 1.0 - 1e-2)
            return np.log(p / (1.0 - p)) / self.cfg.lambda_tanh
        if t == "clamp":
            return np.clip(phi, 0.0, 1.05)
        return phi.copy()


def _read_probes(path: str):
    xs, ys = [], []
    with open(path) as fh:
        for line in fh:
            tok = line.split()
            nums = []
            for t in tok:
                try:
                    nums.append(float(t))
                except ValueError:
                    pass
            if len(nums) >= 2:
                xs.append(nums[-2])
                ys.append(nums[-1])
    return xs, ys


class PorosityProblem:
    """PorosityProblem (assim/swSpE_minimize.cpp:264-580): f(theta) over the free cells, theta =
    m per free cell, or per zone of free cells sharing a first-guess value (zonation)."""

    def __init__(self, spe: SpE, phi_b, free: Optional[Sequence[int]] = None, zonation: bool = False,
                 alpha_reg: float = 0.0, phi_ref=None, descent_dir: Optional[str] = None,
                 stride: Optional[int] = None):
        self.spe = spe
        self.n = spe.n
        self.phi_b = np.asarray(phi_b, dtype=np.float64).copy()
        self.free = np.arange(self.n) if free is None else np.asarray(free, dtype=np.int64)
        self.zonation = zonation
        if zonation:
            self.zone_value, self.zone_of_free = np.unique(self.phi_b[self.free], return_inverse=True)
        self.alpha = alpha_reg
        self.phi_ref = None if phi_ref is None else np.asarray(phi_ref, dtype=np.float64)
        self.stride = stride or spe.cfg.checkpoint_stride
        mesh = spe.model.case.mesh
        self._L = mesh.edge_int_cells[:, 0].astype(np.int64)
        self._R = mesh.edge_int_cells[:, 1].astype(np.int64)
        self.m_buf = spe.m_from_phi(self.phi_b)
        self.grad_calls = 0
        self.J_init = None
        self.J_prev = None
        self.descent_dir = descent_dir
        self._csv = None
        if descent_dir:
            shutil.rmtree(descent_dir, ignore_errors=True)
            os.makedirs(os.path.join(descent_dir, "phi_iter"), exist_ok=True)

    def size(self) -> int:
        return len(self.zone_value) if self.zonation else len(self.free)

    def theta_start(self) -> np.ndarray:
        v = self.zone_value if self.zonation else self.phi_b[self.free]
        return self.spe.m_from_phi(v)

    def _map_theta(self, theta) -> np.ndarray:
        theta = np.asarray(theta, dtype=np.float64)
        self.m_buf[self.free] = theta[self.zone_of_free] if self.zonation else theta
        return self.m_buf

    # penalties of func()/grad() (swSpE_minimize.cpp:339-396)
    def _penalties(self):
        cfg = self.spe.cfg
        phi = self.spe.phi_correct(self.m_buf)
        d = phi[self.free] - self.phi_b[self.free]
        ridge = 0.5 * self.alpha * float(np.dot(d, d))
        l1 = cfg.alpha_l1 * float(np.sum(np.abs(d)))
        sp = 0.0
        if cfg.alpha_spatial > 0:
            e = phi[self._L] - phi[self._R]
            sp = 0.5 * cfg.alpha_spatial * float(np.dot(e, e))
        ref = 0.0
        if cfg.alpha_phi_ref > 0 and self.phi_ref is not None:
            r = phi[self.free] - self.phi_ref[self.free]
            ref = 0.5 * cfg.alpha_phi_ref * float(np.dot(r, r))
        return ridge, l1, sp, ref

    def func(self, theta) -> float:
        self._map_theta(theta)
        return self.spe.replay_trajectory_cost(self.m_buf) + sum(self._penalties())

    def grad(self, theta):
        """(f, df/dtheta) (swSpE_minimize.cpp:405-511): records at theta, the GPU gradient of
        J_data, the penalties' analytic gradients chained by dphi/dm."""
        cfg = self.spe.cfg
        m = self._map_theta(theta)
        g_data = self.spe.get_spatial_gradient_checkpointed(m, self.stride)
        J_data = float(self.spe.diag["J"])
        phi = self.spe.phi_correct(m)
        dphidm = self.spe.dphi_dm(m)
        free = self.free
        d = phi[free] - self.phi_b[free]
        gval = g_data[free] + self.alpha * d * dphidm[free]
        if cfg.alpha_l1 > 0:
            gval = gval + cfg.alpha_l1 * np.where(d > 1e-12, 1.0, np.where(d < -1e-12, -1.0, 0.0)) * dphidm[free]
        if cfg.alpha_spatial > 0:
            gs = np.zeros(self.n)
            e = cfg.alpha_spatial * (phi[self._L] - phi[self._R])
            np.add.at(gs, self._L, e)
            np.add.at(gs, self._R, -e)
            gval = gval + gs[free] * dphidm[free]
        if cfg.alpha_phi_ref > 0 and self.phi_ref is not None:
            gval = gval + cfg.alpha_phi_ref * (phi[free] - self.phi_ref[free]) * dphidm[free]
        g_theta = np.bincount(self.zone_of_free, weights=gval, minlength=self.size()) if self.zonation else gval
        ridge, l1, sp, ref = self._penalties()
        J = J_data + ridge + l1 + ref   # the reference's grad() leaves the spatial term out of J
        self.grad_calls += 1
        if self.J_init is None:
            self.J_init = J
        self._log(J, J_data, ridge, gval, g_data, phi)
        self.J_prev = J
        return J, g_theta

    def _log(self, J, J_data, ridge, gval, g_data, phi):
        if not self.descent_dir:
            return
        if self._csv is None:
            self._csv = open(os.path.join(self.descent_dir, "descent_log.csv"), "w")
            self._csv.write(DESCENT_COLUMNS + "\n")
        diag = self.spe.diag
        rel = (J - self.J_init) / self.J_init * 100.0 if self.J_init else 0.0
        rel_prev = (J - self.J_prev) / self.J_prev * 100.0 if self.J_prev else 0.0
        pf = phi[self.free]
        ag = np.abs(gval)
        sse = float(np.sum((phi - self.phi_ref) ** 2)) if self.phi_ref is not None else -1.0
        row = [self.grad_calls, f"{J:.10e}", f"{J_data:.10e}", f"{ridge:.10e}", f"{rel:.6e}", f"{rel_prev:.6e}",
               f"{float(np.sqrt(np.dot(gval, gval))):.6e}", f"{float(ag.max()) if ag.size else 0.0:.6e}",
               int(self.free[int(np.argmax(ag))]) if ag.size else -1,
               f"{float(diag.get('grad_l2', 0.0)):.6e}", f"{float(diag.get('grad_max', 0.0)):.6e}",
               int(diag.get("grad_argmax", -1)), f"{float(diag.get('dh_peak', 0.0)):.6e}",
               f"{float(pf.min()):.6e}", f"{float(pf.max()):.6e}", f"{float(pf.mean()):.6e}",
               int(np.sum(pf < 0.5)), int(np.sum(pf < 0.05)), int(np.sum(pf > 1.049)),
               f"{self.spe.cfg.adam_step_size:.6e}", f"{sse:.10e}"]
        self._csv.write(",".join(str(x) for x in row) + "\n")
        self._csv.flush()
        write_map(os.path.join(self.descent_dir, "phi_iter", f"phi_iter_{self.grad_calls:04d}.txt"), ["SpPhiW"],
                  [phi], self.n)

    def close(self):
        if self._csv is not None:
            self._csv.close()
            self._csv = None


def free_cells(spe: SpE, phi_start) -> np.ndarray:
    """The cells the minimisation moves (swSpE::run_minimization, assim/swSpE_minimize.cpp:604-668).

    * mask_dry_cells: a native forward run (swSp::execute) of the case to t_max with the
      first-guess porosity; cells still dry at its end (h <= 1e-4) never see water, their
      porosity has no observable effect and stays at the first guess.  Otherwise every cell.
    * porosity_free_zone_map ("cell_id,value" or SW2D map, path relative to the case folder):
      of those, only the cells whose value is below 0.5.  An unreadable map leaves the set as
      it is (the reference logs an error and carries on); an empty zone is reported."""
    cfg = spe.cfg
    n = spe.n
    if cfg.mask_dry_cells:
        import dataclasses

        case = dataclasses.replace(spe.model.case, phi=np.ascontiguousarray(phi_start, dtype=np.float64))
        fwd = SpModel(case, device=getattr(spe.model, "device", 0))
        try:
            fwd.execute()
            h_end = fwd.state()[0]
        finally:
            fwd.close()
        free = np.nonzero(h_end > 1e-4)[0]
        spe.diag["mask_dry_cells"] = {"fixed": int(n - free.size), "free": int(free.size)}
    else:
        free = np.arange(n)
    if cfg.porosity_free_zone_map:
        path = cfg.porosity_free_zone_map
        if spe.folder and not os.path.isabs(path):
            path = os.path.join(spe.folder, path)
        try:
            zone = load_map(path, n)
        except (OSError, ValueError) as exc:
            spe.diag["zone_map_error"] = f"{path}: {exc}; zonation ignored"
        else:
            before = free.size
            free = free[zone[free] < 0.5]
            spe.diag["porosity_free_zone_map"] = {"free_in_zone": int(free.size), "free_before": int(before)}
            if free.size == 0:
                spe.diag["zone_map_error"] = f"{path}: empty zone (no cell with value < 0.5)"
    return free


def run_minimization(spe: SpE, phi_start, max_it: Optional[int] = None, alpha_reg: Optional[float] = None,
                     descent_dir: Optional[str] = None, free=None, phi_ref=None,
                     freeze_window: bool = False) -> Dict[str, object]:
    """swSpE::run_minimization (assim/swSpE_minimize.cpp:582-1073) with minimize_algo "lbfgsb"
    (scipy's L-BFGS-B on the box [phi_lower_bound, phi_upper_bound]) or "gd" (projected gradient
    descent with Armijo backtracking: c1 = 1e-4, shrink 0.5, grow 4, 40 backtracks).  Returns
    {"phi", "J_final", "J_init", "n_grad", "history"}.

    freeze_window (L-BFGS-B): the reference's probe evaluation at the start point, whose
    truncation segment then stays the first segment of every gradient's window for the whole
    solve (swSpE_minimize.cpp:881-903), J_final being the solver's value on that window.  Off by
    default: on sp_toce with this gradient the frozen window stops the descent at J = 2.836
    (-8.7 %), against 1.924 (-38 %) with each gradient's own window."""
    cfg = spe.cfg
    max_it = cfg.max_it if max_it is None else max_it
    alpha = cfg.alpha_reg if alpha_reg is None else alpha_reg
    if free is None:
        free = free_cells(spe, phi_start)
    prob = PorosityProblem(spe, phi_start, free=free, zonation=cfg.zonation, alpha_reg=alpha, phi_ref=phi_ref,
                           descent_dir=descent_dir)
    theta = prob.theta_start()
    history: List[float] = []
    algo = cfg.minimize_algo.lower()
    if algo in ("lbfgsb", "bfgs"):
        from scipy.optimize import minimize

        def fg(th):
            J, g = prob.grad(th)
            history.append(J)
            return J, g

        bounds = [(cfg.phi_lower_bound, cfg.phi_upper_bound)] * prob.size() if algo == "lbfgsb" else None
        # the reference's LBFGSpp settings: m corrections (lbfgsb_m), at most lbfgsb_max_linesearch
        # line-search trials, convergence at a projected gradient below lbfgsb_epsilon
        opts = {"maxiter": max_it}
        if algo == "lbfgsb":
            opts.update(maxcor=int(cfg.lbfgsb_m), maxls=int(cfg.lbfgsb_max_linesearch), gtol=float(cfg.lbfgsb_epsilon))
        frozen = False
        if algo == "lbfgsb" and freeze_window:
            # the reference's probe (swSpE_minimize.cpp:881-892): one evaluation at the start point
            # fixes the segment where the adjoint's window is cut, and the window stays there for
            # the whole solve, so that every line-search trial computes J over the same window
            # (a window that moves with theta makes J jump between trials and the line search fail)
            fg(theta)
            spe.set_forced_first_segment(max(0, int(spe.diag.get("truncation_segment", -1)) + 1))
            frozen = True
        try:
            res = minimize(fg, theta, jac=True, method="L-BFGS-B" if algo == "lbfgsb" else "BFGS", bounds=bounds,
                           options=opts)
        finally:
            if frozen:
                spe.set_forced_first_segment(-1)
        theta = res.x
        if frozen:
            # J_final is the solver's value, on the frozen window (swSpE_minimize.cpp:906-909)
            prob.close()
            phi = spe.phi_correct(prob._map_theta(theta))
            return {"phi": phi, "J_final": float(res.fun), "J_init": prob.J_init, "n_grad": prob.grad_calls,
                    "history": history}
    elif algo == "gd":
        project = cfg.phi_transform in ("none", "clamp")
        c1, shrink, grow, max_bt = 1e-4, 0.5, 4.0, 40
        t = cfg.adam_step_size if cfg.adam_step_size > 0 else 1e-6
        best_theta, best_J = theta.copy(), math.inf
        for _ in range(max_it):
            J, g = prob.grad(theta)
            history.append(J)
            if J < best_J:
                best_J, best_theta = J, theta.copy()
            if not np.dot(g, g) > 0.0:
                break
            t_try, accepted = t * grow, False
            for _ in range(max_bt):
                trial = theta - t_try * g
                if project:
                    trial = np.clip(trial, 0.0, 1.0)
                pg = float(np.dot(g, theta - trial))
                Jn = prob.func(trial)
                if np.isfinite(Jn) and Jn <= J - c1 * pg and pg > 0.0:
                    accepted = True
                    break
                t_try *= shrink
            if not accepted:
                break
            theta, t = trial, t_try
        theta = best_theta
    else:
        raise ValueError(f"unknown minimize_algo {cfg.minimize_algo!r}")
    J_final, _ = prob.grad(theta)
    history.append(J_final)
    prob.close()
    phi = spe.phi_correct(prob._map_theta(theta))
    return {"phi": phi, "J_final": J_final, "J_init": prob.J_init, "n_grad": prob.grad_calls, "history": history}
