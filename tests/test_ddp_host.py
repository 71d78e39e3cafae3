"""DDP model on the CPU: the porosity-law tabulation and the arithmetic of the DDP kernels
against the reference's own swDdp.

* ``case.ddp_law_table`` (the Python restatement of swDdp::setPorosity*Map + tabulatePorosity)
  gives the reference's tables bit for bit, for every law type;
* tests/ddp_step_check.cpp composes the device functions of csrc/ddp_math.cuh in the
  reference's serial order (g++ -ffp-contract=off); N steps of it reproduce the reference's
  state, time step and fluxes bit for bit, with every divergence-correction mode.

The reference is the one built by oracle/Makefile (the portable exp/log build, as the CUDA
library uses those).
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.conftest import load_pkg

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "inria-internship-project-sw2d-enzyme_b200", "csrc")
SRC = os.path.join(HERE, "ddp_step_check.cpp")

PKG = load_pkg()
case_mod = PKG.case
workloads = PKG.workloads

D = ctypes.POINTER(ctypes.c_double)
I64 = ctypes.POINTER(ctypes.c_int64)
I32 = ctypes.POINTER(ctypes.c_int32)


class HostCase(ctypes.Structure):
    _fields_ = [("nc", ctypes.c_int64), ("ni", ctypes.c_int64), ("nb", ctypes.c_int64),
                ("area", D), ("zb", D), ("bous", D), ("L", I64), ("R", I64), ("nx", D), ("ny", D), ("len", D),
                ("bcell", I64), ("bnx", D), ("bny", D), ("blen", D), ("bbc", I32),
                ("ctoff", I64), ("cz", D), ("cphi", D), ("ctheta", D),
                ("etoff", I64), ("ez", D), ("ephi", D), ("etheta", D),
                ("bctype", I32), ("bcoff", I64), ("bct", D), ("bcv", D),
                ("h_min", ctypes.c_double), ("cfl_max", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("dt_map", ctypes.c_double), ("t_max", ctypes.c_double), ("v_max", ctypes.c_double),
                ("fr_max", ctypes.c_double), ("chi_phi_max", ctypes.c_double), ("h_min_ddp", ctypes.c_double),
                ("friction", ctypes.c_int32), ("head_loss", ctypes.c_int32), ("dissipation", ctypes.c_int32),
                ("div_corr", ctypes.c_int32), ("n_it_div_max", ctypes.c_int32), ("neg_detect", ctypes.c_int32),
                ("f1", D), ("f2", D), ("fa", D), ("hs", D), ("hk1", D), ("hk2", D), ("ha", D),
                ("mu1", D), ("mu2", D), ("mua", D)]


class HostState(ctypes.Structure):
    _fields_ = [("theta", D), ("tu", D), ("tv", D), ("t", D), ("dt", D),
                ("F1i", D), ("F2i", D), ("F3i", D), ("s2Li", D), ("s2Ri", D),
                ("F1b", D), ("F2b", D), ("F3b", D), ("s2Rb", D), ("lmi", D), ("lmb", D), ("status", I32)]


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    so = str(tmp_path_factory.mktemp("ddp") / "libddp_host.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC", "-I", CSRC, SRC, "-o", so],
                   check=True, capture_output=True, text=True)
    lib = ctypes.CDLL(so)
    lib.ddp_host_steps.argtypes = [ctypes.POINTER(HostCase), ctypes.POINTER(HostState), ctypes.c_int]
    lib.ddp_host_steps.restype = ctypes.c_int
    return lib


def _ref_or_skip():
    from oracle import binding
    if not os.path.exists(binding.REF_PM_SO):
        pytest.skip("reference not built (make -C oracle ref)")
    return binding


def _ptr(a, t):
    return a.ctypes.data_as(t)


class HostModel:
    """The host composition of the DDP step on a Case, in the reference numbering."""

    def __init__(self, lib, case):
        self.lib = lib
        m = case.mesh
        o = case.opts
        ntab = int(o.get("n_por_tab_max", 5))
        keep = []

        def arr(a, dtype=np.float64):
            x = np.ascontiguousarray(a, dtype=dtype)
            keep.append(x)
            return x

        def tables(recs, base):
            off, z, p, t = [0], [], [], []
            for k in range(recs.count):
                zt, pt, tt = case_mod.ddp_law_table(recs.record(k), float(base[k]), ntab)
                z += zt.tolist()
                p += pt.tolist()
                t += tt.tolist()
                off.append(len(z))
            return arr(off, np.int64), arr(z), arr(p), arr(t)

        co, cz, cp, ct = tables(case.ddp_cell, m.cell_z_b)
        eo, ez, ep, et = tables(case.ddp_edge_int, m.edge_int_mz)
        codes = list(case.bc.codes)
        bbc = arr([codes.index(int(c)) for c in m.edge_bnd_code], np.int32)
        ns = len(codes)
        nrec = case.bc.times.shape[0]
        bctype = arr([case_mod.BC_TYPES[t] for t in case.bc.types], np.int32)
        bcoff = arr(np.arange(ns + 1) * nrec, np.int64)
        bct = arr(np.tile(case.bc.times, ns))
        bcv = arr(np.asarray(case.bc.values).reshape(-1))
        fr, hl, mu = case.friction, case.head_loss, case.mu
        friction = {"none": 0, "chezy": 1, "manning": 2, "strickler": 3}[o.get("model_friction", "none")]
        null = D()
        self.L = arr(m.edge_int_cells[:, 0], np.int64)
        self.R = arr(m.edge_int_cells[:, 1], np.int64)

        def f(k, d):
            return float(o.get(k, d))

        self.c = HostCase(
            m.cell_nb, m.edge_int_nb, m.edge_bnd_nb, _ptr(arr(m.cell_area), D), _ptr(arr(m.cell_z_b), D),
            _ptr(arr(case.boussinesq), D), _ptr(self.L, I64), _ptr(self.R, I64), _ptr(arr(m.edge_int_nx), D),
            _ptr(arr(m.edge_int_ny), D), _ptr(arr(m.edge_int_length), D), _ptr(arr(m.edge_bnd_cell, np.int64), I64),
            _ptr(arr(m.edge_bnd_nx), D), _ptr(arr(m.edge_bnd_ny), D), _ptr(arr(m.edge_bnd_length), D), _ptr(bbc, I32),
            _ptr(co, I64), _ptr(cz, D), _ptr(cp, D), _ptr(ct, D), _ptr(eo, I64), _ptr(ez, D), _ptr(ep, D), _ptr(et, D),
            _ptr(bctype, I32), _ptr(bcoff, I64), _ptr(bct, D), _ptr(bcv, D),
            f("h_min", 1e-5), f("cfl_max", 1.0), f("dt_max", 10.0), f("dt_map", 100.0), f("t_max", 100.0),
            f("v_max", 100.0), f("fr_max", 100.0), f("ddp_chi_phi_max", 20.0), f("h_min_ddp", 1e-3),
            friction, int(o.get("model_singular_head_loss", "none") != "none"),
            int(o.get("model_momentum_dissipation", "none") != "none"),
            {"none": 0, "limit_flux": 1, "limit_timestep": 2}[o.get("div_corr", "none")], int(o.get("n_it_div_max", 10)),
            int(o.get("negative_depth_detection", "none") == "active"),
            _ptr(arr(fr[0]), D) if fr is not None else null, _ptr(arr(fr[1]), D) if fr is not None else null,
            _ptr(arr(fr[2]), D) if fr is not None else null,
            *([_ptr(arr(hl[k]), D) for k in range(4)] if hl is not None else [null] * 4),
            *([_ptr(arr(mu[k]), D) for k in range(3)] if mu is not None else [null] * 3))
        self.keep = keep
        n, ni, nb = m.cell_nb, m.edge_int_nb, m.edge_bnd_nb
        self.theta, self.tu, self.tv = np.zeros(n), np.zeros(n), np.zeros(n)
        self.t = np.array([f("t_0", 0.0)])
        self.dt = np.zeros(1)
        self.fi = {k: np.zeros(ni) for k in ("F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int")}
        self.fb = {k: np.zeros(nb) for k in ("F1_bnd", "F2_bnd", "F3_bnd", "s2R_bnd")}
        self.lmi, self.lmb = np.zeros(ni), np.zeros(nb)
        self.status = np.zeros(1, dtype=np.int32)
        self.s = HostState(_ptr(self.theta, D), _ptr(self.tu, D), _ptr(self.tv, D), _ptr(self.t, D), _ptr(self.dt, D),
                           *[_ptr(self.fi[k], D) for k in ("F1_int", "F2_int", "F3_int", "s2L_int", "s2R_int")],
                           *[_ptr(self.fb[k], D) for k in ("F1_bnd", "F2_bnd", "F3_bnd", "s2R_bnd")],
                           _ptr(self.lmi, D), _ptr(self.lmb, D), _ptr(self.status, I32))

    def set_state(self, th, tu, tv):
        self.theta[:] = th
        self.tu[:] = tu
        self.tv[:] = tv

    def step(self, k=1):
        return self.lib.ddp_host_steps(ctypes.byref(self.c), ctypes.byref(self.s), int(k))


CASES = {
    # name: ddp_channel keyword arguments
    "mixed_fr_manning": dict(n_cells=500, friction="manning", outflow="fr", t_max=30.0, h_floor=0.0),
    "mixed_h_strickler_headloss_diss": dict(n_cells=500, friction="strickler", outflow="h", head_loss=True,
                                            dissipation=True, moving=True, ic="zuv", t_max=30.0, seed=23),
    "mixed_z_chezy_b11": dict(n_cells=400, friction="chezy", outflow="z", boussinesq=1.1, moving=True, t_max=30.0,
                              seed=25),
    "limit_timestep": dict(n_cells=400, friction="manning", outflow="fr", div_corr="limit_timestep", t_max=30.0,
                           seed=27),
    "limit_flux": dict(n_cells=400, friction="manning", outflow="fr", div_corr="limit_flux", n_it_div_max=3,
                       t_max=30.0, seed=29),
}


def test_tables_match_reference(tmp_path):
    """Every law type tabulated by the Python restatement equals the reference's tables."""
    binding = _ref_or_skip()
    case = workloads.ddp_channel(n_cells=400, t_max=1.0, seed=31)
    case_mod.write_case(str(tmp_path), case)
    ref = binding.RefSolver(str(tmp_path), portable_math=True)
    m = case.mesh
    seen = set()
    for which, recs, base, count in (("cell", case.ddp_cell, m.cell_z_b, m.cell_nb),
                                     ("edge_int", case.ddp_edge_int, m.edge_int_mz, m.edge_int_nb),
                                     ("edge_bnd", case.ddp_edge_bnd, m.edge_bnd_mz, m.edge_bnd_nb)):
        for k in range(count):
            rec = recs.record(k)
            seen.add(int(rec[0]))
            want = ref.ddp_table(which, k)
            got = case_mod.ddp_law_table(rec, float(base[k]), 5)
            for a, b in zip(got, want):
                assert a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64)), (which, k, rec)
    assert seen == {-2, -1, 0, 1, 2, 3}
    # the reference's theta_G at z_tab[0] + h_min_ddp
    hmin = ref.array("thetaG_int_hmin")
    for k in range(m.edge_int_nb):
        z, p, t = case_mod.ddp_law_table(case.ddp_edge_int.record(k), float(m.edge_int_mz[k]), 5)
        zz = z[0] + 1e-3
        lv = int(np.searchsorted(z, zz, side="left"))  # first level with z >= zz  -> scan stops there
        want = t[lv - 1] + (zz - z[lv - 1]) * p[lv - 1]
        assert hmin[k] == want


@pytest.mark.parametrize("name", sorted(CASES))
def test_host_steps_match_reference(hostlib, tmp_path, name):
    binding = _ref_or_skip()
    case = workloads.ddp_channel(**CASES[name])
    case_mod.write_case(str(tmp_path), case)
    ref = binding.RefSolver(str(tmp_path), portable_math=True)
    host = HostModel(hostlib, case)
    host.set_state(*ref.state())
    n_steps = 60
    for k in range(n_steps):
        a = ref.step(1)
        b = host.step(1)
        assert a == b
        if a == 0:
            break
        assert host.status[0] == 0
        assert ref.dt == host.dt[0] and ref.t == host.t[0], (k, ref.dt, host.dt[0])
        for nm, got in zip(("h", "q", "r"), (host.theta, host.tu, host.tv)):
            want = ref.array(nm)
            bad = np.flatnonzero(want.view(np.uint64) != got.view(np.uint64))
            assert bad.size == 0, (name, k, nm, bad[:5], want[bad[:3]], got[bad[:3]])
        for nm, got in list(host.fi.items()) + list(host.fb.items()):
            want = ref.array(nm)
            assert np.array_equal(want.view(np.uint64), got.view(np.uint64)), (name, k, nm)
        for nm, got in (("lambda_max_int", host.lmi), ("lambda_max_bnd", host.lmb)):
            assert np.array_equal(ref.array(nm).view(np.uint64), got.view(np.uint64)), (name, k, nm)
    th, _, _ = ref.state()
    assert np.any(th > 0)


def _ddp_golden_names():
    from tests.conftest import golden_names
    return [n for n in golden_names() if n.startswith("ddp_")]


@pytest.mark.parametrize("name", _ddp_golden_names())
def test_host_steps_match_golden(hostlib, name):
    """The host composition against the fixtures the reference (portable exp/log) made: needs
    no reference at run time."""
    from tests.conftest import golden_case
    case, fx = golden_case(name)
    host = HostModel(hostlib, case)
    # the reference's initial state: thetaW from the initial-condition columns
    # (swDdp::setInitialConditions, restated here with the tabulated laws)
    m = case.mesh
    ntab = int(case.opts.get("n_por_tab_max", 5))
    th, tu, tv = np.zeros(m.cell_nb), np.zeros(m.cell_nb), np.zeros(m.cell_nb)
    for c in range(m.cell_nb):
        z, p, t = case_mod.ddp_law_table(case.ddp_cell.record(c), float(m.cell_z_b[c]), ntab)
        level = case.h0[c] if case.ddp_ic[0] == "z" else case.h0[c] + z[0]
        th[c] = _theta_of_z(z, p, t, level)
        zz = _z_of_theta(z, p, t, th[c])
        hq = max(1e-16, zz - z[0])
        tu[c] = th[c] * case.q0[c] if case.ddp_ic[1] == "u" else th[c] * case.q0[c] / hq
        tv[c] = th[c] * case.r0[c] if case.ddp_ic[2] == "v" else th[c] * case.r0[c] / hq
    host.set_state(th, tu, tv)
    assert host.step(int(fx["steps_pm"])) == int(fx["steps_pm"])
    assert host.t[0] == float(fx["t_pm"]) and host.dt[0] == float(fx["dt_pm"])
    for got, key in ((host.theta, "h_pm"), (host.tu, "q_pm"), (host.tv, "r_pm")):
        assert np.array_equal(got.view(np.uint64), np.asarray(fx[key]).view(np.uint64)), key


def _theta_of_z(z, p, t, zz):
    # thetaWOfZ (swDdp.cpp:2708-2736)
    if zz <= z[0]:
        return 0.0
    lv = 0
    while lv < z.size and zz > z[lv]:
        lv += 1
    th = float(t[lv - 1])
    if zz > z[lv - 1]:
        th += (zz - float(z[lv - 1])) * float(p[lv - 1])
    return th


def _z_of_theta(z, p, t, th):
    # zOfThetaW (swDdp.cpp:3368-3388)
    if th <= 0:
        return float(z[0])
    lv = 0
    while lv < t.size and th > t[lv]:
        lv += 1
    return float(z[lv - 1]) + (th - float(t[lv - 1])) / float(p[lv - 1])
