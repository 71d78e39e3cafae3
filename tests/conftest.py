"""Shared fixtures.  `gpu` marks tests that need a CUDA device (run with -m gpu)."""
from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
PKG_NAME = "inria-internship-project-sw2d-enzyme_b200"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def reference_missing():
    """Why the reference's source tree is unavailable to a test ("" when it is available): its
    root comes from the environment variable SW2D_REFERENCE."""
    root = os.environ.get("SW2D_REFERENCE", "")
    if not root:
        return "SW2D_REFERENCE is not set (root of the reference's source tree)"
    if not os.path.isdir(root):
        return f"SW2D_REFERENCE={root} is not a directory"
    return ""


def reference_case(name):
    """Folder of the reference's functional case `name` under SW2D_REFERENCE ("" when unset)."""
    root = os.environ.get("SW2D_REFERENCE", "")
    return os.path.join(root, "configue_fonctionels", name) if root else ""


def load_pkg():
    return importlib.import_module(PKG_NAME)


@pytest.fixture(scope="session")
def pkg():
    return load_pkg()


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and not f.startswith("sp_toce"))


def golden_case(name):
    """(case, fixture) for a synthetic golden case; the inputs are rebuilt from their seeds and
    checked against the digest recorded when the reference produced the fixture."""
    pkg = load_pkg()
    from tests.golden.make_golden import build_case, case_digest
    fx = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    case = build_case(str(fx["builder"]), json.loads(str(fx["kwargs"])))
    assert case_digest(case) == str(fx["digest"]), f"{name}: regenerated inputs differ from the fixture's"
    return case, fx


def sp_toce_case():
    """The reference's functional case sp_toce, rebuilt from tests/golden/sp_toce.npz."""
    pkg = load_pkg()
    fx = np.load(os.path.join(GOLDEN, "sp_toce.npz"), allow_pickle=False)
    M = pkg.case.Mesh
    mesh = M(node_x=np.zeros(0), node_y=np.zeros(0), node_z=np.zeros(0), cell_nodes=[],
             cell_area=fx["cell_area"], cell_perimeter=np.zeros_like(fx["cell_area"]), cell_x=fx["cell_x"],
             cell_y=fx["cell_y"], cell_z_b=fx["cell_z_b"], edge_int_cells=fx["edge_int_cells"].astype(np.int64),
             edge_int_nodes=np.zeros((0, 2), np.int64), edge_int_length=fx["edge_int_length"],
             edge_int_nx=fx["edge_int_nx"], edge_int_ny=fx["edge_int_ny"], edge_int_mx=fx["edge_int_mx"],
             edge_int_my=fx["edge_int_my"], edge_int_mz=np.zeros(0), edge_int_dnorm=np.zeros(0),
             edge_bnd_cell=fx["edge_bnd_cell"].astype(np.int64), edge_bnd_nodes=np.zeros((0, 2), np.int64),
             edge_bnd_length=fx["edge_bnd_length"], edge_bnd_nx=fx["edge_bnd_nx"], edge_bnd_ny=fx["edge_bnd_ny"],
             edge_bnd_mx=np.zeros(0), edge_bnd_my=np.zeros(0), edge_bnd_mz=np.zeros(0), edge_bnd_dnorm=np.zeros(0),
             edge_bnd_code=fx["edge_bnd_code"].astype(np.int32))
    bc = pkg.case.BoundarySeries(codes=[int(c) for c in fx["bc_codes"]], types=json.loads(str(fx["bc_types"])),
                                 times=fx["bc_times"], values=fx["bc_values"])
    case = pkg.case.Case(mesh=mesh, opts=json.loads(str(fx["opts"])), h0=fx["h0"], q0=fx["q0"], r0=fx["r0"],
                         phi=fx["phi"], boussinesq=fx["boussinesq"], friction=fx["friction"],
                         head_loss=fx["head_loss"], bc=bc)
    return case, fx


# parity bar of the floating-point comparisons: within 1e-10 relative of the reference in h, hu, hv
REL_TOL = 1e-10


def rel_err(a, b, scale=None):
    """Infinity-norm relative error of a against b (0 when both are exactly zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if b.size else 0.0
    if scale is not None:
        s = max(s, scale)
    diff = np.max(np.abs(a - b)) if a.size else 0.0
    return 0.0 if diff == 0.0 else diff / max(s, 1e-300)


def assert_state_close(got, want, exact, what=""):
    """Bit for bit, or within REL_TOL.  Discharges are judged relative to
    max(|q|max, h_max sqrt(g h_max)) so that water at rest (round-off-sized q) is measured on
    the flow's own scale."""
    hmax = float(np.max(np.abs(want[0]))) if np.asarray(want[0]).size else 0.0
    qscale = hmax * np.sqrt(9.81 * hmax)
    for k, (name, a, b) in enumerate(zip(("h", "hu", "hv"), got, want)):
        if exact:
            nbad = int(np.count_nonzero(np.asarray(a).view(np.int64) != np.asarray(b).view(np.int64)))
            assert nbad == 0, f"{what} {name}: {nbad} values differ bitwise (max abs {np.max(np.abs(a - b))})"
        else:
            e = rel_err(a, b, qscale if k > 0 else None)
            assert e <= REL_TOL, f"{what} {name}: relative error {e:.3e} > {REL_TOL}"
