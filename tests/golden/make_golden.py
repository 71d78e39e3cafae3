"""Generates the golden fixtures of tests/golden/ by running the REFERENCE solver, compiled from
its own sources (oracle/Makefile -> oracle/_ref/libsw2d_ref.so), on:

* the synthetic cases of ``CASES`` (inputs are regenerated from their seeds by the tests; the
  fixture stores a digest of those inputs and the reference's state after ``STEPS`` steps);
* the reference's own functional case ``configue_fonctionels/sp_toce`` (native input.solv keys
  only; the fixture stores the mesh tables and parameters the SP step reads, and the
  reference's state after 100 steps and at t_max).

Each state is recorded twice: from the reference linked with the host libm (glibc, fields
h/q/r...) and from the same reference objects linked with the portable exp/log of the CUDA
build (oracle/_ref/libsw2d_ref_pm.so, fields ..._pm).  ``libm_stable`` records whether the two
agree within 1e-10 (relative, infinity norm; discharges scaled by max(|q|max, h_max sqrt(g h_max))).

The dip_* cases are dual integral porosity cases (the reference's swDip), the ddp_* cases
depth-dependent porosity cases (swDdp; their state is thetaW, thetaW u, thetaW v).

Run here (the reference tree must be present):  python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import hashlib
import importlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
pkg = importlib.import_module("inria-internship-project-sw2d-enzyme_b200")
W = pkg.workloads

STEPS = 200
CASES = {
    "dam_muscl_manning": ("dam_break", {"n_cells": 2000}),
    "dam_godunov_manning": ("dam_break", {"n_cells": 2000, "scheme": "godunov"}),
    "dam_muscl_nofriction": ("dam_break", {"n_cells": 2000, "friction": "none"}),
    "bumps_muscl_manning": ("gaussian_bumps", {"n_cells": 3000}),
    "chan_godunov_blending_strickler_fr": ("channel_features", {}),
    "chan_muscl_disc_manning_h": ("channel_features", {"scheme": "muscl_evr", "topo": "discontinuous",
                                                       "friction": "manning", "outflow": "h"}),
    "chan_muscl_blend_chezy_z_b11": ("channel_features", {"scheme": "muscl_evr", "topo": "blending",
                                                          "friction": "chezy", "outflow": "z", "boussinesq": 1.1}),
    "chan_godunov_disc_none_q": ("channel_features", {"friction": "none", "outflow": "q", "head_loss": False}),
    # dual integral porosity (model_hyperb dip)
    "dip_muscl_disc_manning_q_fr": ("dip_channel", {"n_cells": 2000}),
    "dip_godunov_blend_strickler_phiwq_h": ("dip_channel", {"n_cells": 2000, "scheme": "godunov", "topo": "blending",
                                                             "friction": "strickler", "inflow": "phiWq",
                                                             "outflow": "h", "dissipation": False}),
    "dip_muscl_blend_chezy_q_z_b11": ("dip_channel", {"n_cells": 2000, "topo": "blending", "friction": "chezy",
                                                       "outflow": "z", "boussinesq": 1.1}),
    # depth-dependent porosity (model_hyperb ddp)
    "ddp_mixed_manning_fr": ("ddp_channel", {"n_cells": 2000}),
    "ddp_linear_strickler_h_hl_diss": ("ddp_channel", {"n_cells": 2000, "friction": "strickler", "outflow": "h",
                                                        "head_loss": True, "dissipation": True, "moving": True,
                                                        "laws": "linear", "seed": 51}),
    "ddp_mixed_chezy_z_limit_flux": ("ddp_channel", {"n_cells": 2000, "friction": "chezy", "outflow": "z",
                                                      "div_corr": "limit_flux", "n_it_div_max": 4, "seed": 53}),
}
DIP_BUILDERS = {"dip_channel"}
DDP_BUILDERS = {"ddp_channel"}
NATIVE_KEYS = ["model_hyperb", "model_friction", "model_singular_head_loss", "num_scheme", "topo_discretization",
               "t_max", "dt_max", "dt_map", "dt_time_series", "h_min", "fr_max", "store_flag"]


def build_case(builder: str, kwargs: dict):
    return getattr(W, builder)(**kwargs)


def case_digest(case) -> str:
    """Digest of every input the step reads (detects drift of the seeded generators)."""
    m = case.mesh
    h = hashlib.sha256()
    for a in (m.cell_area, m.cell_x, m.cell_y, m.cell_z_b, m.edge_int_cells, m.edge_int_length, m.edge_int_nx,
              m.edge_int_ny, m.edge_int_mx, m.edge_int_my, m.edge_bnd_cell, m.edge_bnd_length, m.edge_bnd_nx,
              m.edge_bnd_ny, m.edge_bnd_code, case.h0, case.q0, case.r0, case.phi, case.boussinesq):
        h.update(np.ascontiguousarray(a).tobytes())
    for a in (case.friction, case.head_loss, case.phi_g_int, case.phi_g_bnd, case.mu):
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    for laws in (case.ddp_cell, case.ddp_edge_int, case.ddp_edge_bnd):
        if laws is not None:
            h.update(np.ascontiguousarray(laws.offset).tobytes())
            h.update(np.ascontiguousarray(laws.values).tobytes())
    if case.ddp_cell is not None:
        h.update(np.ascontiguousarray(m.edge_int_mz).tobytes())
        h.update(np.ascontiguousarray(m.edge_bnd_mz).tobytes())
        h.update("".join(case.ddp_ic).encode())
    h.update(json.dumps(case.opts, sort_keys=True, default=str).encode())
    return h.hexdigest()


def state_rel_err(got, want) -> float:
    """max over (h, q, r) of the infinity-norm relative error; discharges are scaled by
    max(|q|max, Q) with Q = h_max sqrt(g h_max), the discharge of the deepest water at the wave
    speed, so that fields at rest (round-off-sized q) are judged on the flow's own scale."""
    h = np.asarray(want[0])
    hmax = float(np.max(np.abs(h))) if h.size else 0.0
    qs = hmax * np.sqrt(9.81 * hmax)
    errs = []
    for k, (a, b) in enumerate(zip(got, want)):
        a = np.asarray(a, dtype=np.float64)
        b = np.asarray(b, dtype=np.float64)
        d = float(np.max(np.abs(a - b))) if a.size else 0.0
        scale = float(np.max(np.abs(b))) if b.size else 0.0
        if k > 0:
            scale = max(scale, qs)
        errs.append(0.0 if d == 0.0 else d / max(scale, 1e-300))
    return max(errs)


def main(only=None):
    """Regenerates every fixture, or only the named ones (command-line arguments)."""
    from oracle.binding import RefSolver, build, reference_available
    build(reference=True)
    assert reference_available(), "reference sources not found: cannot make golden fixtures"
    tmp = tempfile.mkdtemp(prefix="sw2d_golden_")
    try:
        for name, (builder, kwargs) in CASES.items():
            if only and name not in only:
                continue
            case = build_case(builder, kwargs)
            folder = os.path.join(tmp, name)
            pkg.write_case(folder, case)
            ref = RefSolver(folder)
            done = ref.step(STEPS)
            h, q, r = ref.state()
            pm = RefSolver(folder, portable_math=True)
            done_pm = pm.step(STEPS)
            hp, qp, rp = pm.state()
            stable = state_rel_err((h, q, r), (hp, qp, rp)) <= 1e-10
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), builder=builder, kwargs=json.dumps(kwargs),
                                digest=case_digest(case), steps=done, t=ref.t, dt=ref.dt, h=h, q=q, r=r,
                                steps_pm=done_pm, t_pm=pm.t, dt_pm=pm.dt, h_pm=hp, q_pm=qp, r_pm=rp,
                                libm_stable=stable)
            print(name, case.mesh.cell_nb, done, ref.t, "libm-stable" if stable else "libm-sensitive",
                  "%.2e" % state_rel_err((h, q, r), (hp, qp, rp)))

        if only and "sp_toce" not in only:
            return
        root = os.environ.get("SW2D_REFERENCE", "")
        if not root:
            raise SystemExit("make_golden.py: set SW2D_REFERENCE to the reference's source tree")
        src = os.path.join(root, "configue_fonctionels", "sp_toce")
        folder = os.path.join(tmp, "sp_toce")
        shutil.copytree(src, folder)
        solv = os.path.join(folder, "input", "input.solv")
        lines = [ln for ln in open(solv).read().splitlines() if ln.strip() and ln.split()[0].lower() in NATIVE_KEYS]
        open(solv, "w").write("\n".join(lines) + "\n")
        case = pkg.read_case(folder)
        ref = RefSolver(folder)
        s100 = ref.step(100)
        h100, q100, r100 = ref.state()
        t100 = ref.t
        s_end = s100 + ref.step(10 ** 7)
        h, q, r = ref.state()
        pm = RefSolver(folder, portable_math=True)
        pm.step(100)
        h100p, q100p, r100p = pm.state()
        t100p = pm.t
        s_end_p = 100 + pm.step(10 ** 7)
        hp, qp, rp = pm.state()
        m = case.mesh
        np.savez_compressed(
            os.path.join(HERE, "sp_toce.npz"), opts=json.dumps(case.opts),
            cell_area=m.cell_area, cell_x=m.cell_x, cell_y=m.cell_y, cell_z_b=m.cell_z_b,
            edge_int_cells=m.edge_int_cells.astype(np.int32), edge_int_length=m.edge_int_length,
            edge_int_nx=m.edge_int_nx, edge_int_ny=m.edge_int_ny, edge_int_mx=m.edge_int_mx,
            edge_int_my=m.edge_int_my, edge_bnd_cell=m.edge_bnd_cell.astype(np.int32),
            edge_bnd_length=m.edge_bnd_length, edge_bnd_nx=m.edge_bnd_nx, edge_bnd_ny=m.edge_bnd_ny,
            edge_bnd_code=m.edge_bnd_code, h0=case.h0, q0=case.q0, r0=case.r0, phi=case.phi,
            boussinesq=case.boussinesq, friction=case.friction, head_loss=case.head_loss,
            bc_codes=np.array(case.bc.codes), bc_types=json.dumps(case.bc.types), bc_times=case.bc.times,
            bc_values=case.bc.values, steps100=s100, t100=t100, h100=h100, q100=q100, r100=r100,
            steps_end=s_end, t_end=ref.t, h_end=h, q_end=q, r_end=r,
            t100_pm=t100p, h100_pm=h100p, q100_pm=q100p, r100_pm=r100p,
            steps_end_pm=s_end_p, t_end_pm=pm.t, h_end_pm=hp, q_end_pm=qp, r_end_pm=rp,
            libm_stable=state_rel_err((h, q, r), (hp, qp, rp)) <= 1e-10)
        print("sp_toce", m.cell_nb, s100, s_end, ref.t, "%.2e" % state_rel_err((h, q, r), (hp, qp, rp)))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1:])
