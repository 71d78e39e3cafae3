"""Digest fixture of the moving C2 parity case: the oracle (oracle/sp_oracle.c, the C restatement
of the reference's SP step, pinned bit for bit to the reference by tests/test_oracle.py) run on
the Gaussian-bump bed under a dam break (workloads.gaussian_bumps(initial="dam"), seeded
jittered-Delaunay mesh) for STEPS steps at 1M and 4M cells.  The CPU oracle needs minutes at
these sizes, so the fixture keeps the SHA-256 of its final state bits (h, q, r in the caller's
numbering), its t and dt, and a digest of the inputs; tests/test_gpu_parity.py compares the GPU
run's bits against it.

Run here:  python tests/golden/make_c2_digest.py
"""
from __future__ import annotations

import hashlib
import importlib
import json
import os
import sys
from concurrent.futures import ProcessPoolExecutor
import multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

STEPS = 200
SIZES = (1_000_000, 4_000_000)
OUT = os.path.join(HERE, "c2_moving_digest.json")


def state_digest(h, q, r) -> str:
    import numpy as np
    d = hashlib.sha256()
    for a in (h, q, r):
        d.update(np.ascontiguousarray(a, np.float64).tobytes())
    return d.hexdigest()


def input_digest(case) -> str:
    import numpy as np
    m = case.mesh
    d = hashlib.sha256()
    for a in (m.cell_x, m.cell_y, m.cell_z_b, m.cell_area, m.edge_int_cells, m.edge_int_nx, m.edge_int_ny,
              m.edge_int_length, m.edge_bnd_cell, case.h0, case.q0, case.r0, case.phi, case.friction):
        d.update(np.ascontiguousarray(a).tobytes())
    return d.hexdigest()


def run(n_cells: int) -> dict:
    pkg = importlib.import_module("inria-internship-project-sw2d-enzyme_b200")
    from oracle import binding
    case = pkg.workloads.gaussian_bumps(n_cells=n_cells, mesh="delaunay", initial="dam")
    o = binding.SpOracle(case, portable_math=True)
    assert o.step(STEPS) == STEPS
    h, q, r = o.state()
    return {"cells": int(case.mesh.cell_nb), "steps": STEPS, "inputs_sha256": input_digest(case),
            "state_sha256": state_digest(h, q, r), "t": repr(float(o.t)), "dt": repr(float(o.dt))}


def main():
    from oracle import binding
    binding.build(reference=False)
    with ProcessPoolExecutor(max_workers=len(SIZES), mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(run, SIZES))
    out = {str(n): r for n, r in zip(SIZES, res)}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
