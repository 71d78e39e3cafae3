"""Builds tests/golden/sp_toce_assim.npz: the reference's porosity-assimilation case sp_toce as the
GPU tests need it, and what the reference's own assimilation layer (assim/*.cpp, run through
oracle/ref_e_driver.cpp) computes on it.

Contents:
* the observations: the 41 maps reference/ResultHydro_p*.txt (t = 10 .. 30 s) as the reference
  reads them (swSpE::load_all_observations); each value "d.dddddddddde+XX" of the text is stored
  as its decimal digits (an integer mantissa and a power of ten), from which float() gives the
  double the reference's stream extraction gives, checked here against the reference's reading;
* the assimilation keys of input.solv as the reference's AssimConfig parses them;
* from the reference linked with the portable exp/log/cbrt of the CUDA build, at phi = 1 (the
  case's first guess input/phi_init_ones.txt): the recorded time steps, observation triggers and
  segment starts, a SHA-256 of every checkpoint state, the window's first segment and tiles, the
  replay cost, and the replay cost at m +- eps d (eps = 1e-6, 1e-7, 1e-8) for two smooth bumps d
  centred on cells 3931 and 509.  (This case's cost is not differentiable in generic directions:
  the _E step switches on h > h_min and h > h_sing at its wetting and drying fronts, so central
  differences in a random direction over all cells do not converge; along these bumps they do.);
* from the reference linked with the host libm, the replay cost at phi = 1 (which equals the first
  row of the case's descent_log_reference_-75.8pct.csv, 3.1042911536e+00).

Run from the repository root, in a container where the reference sources are present:
    make -C oracle ref && python tests/golden/make_assim_golden.py
"""
from __future__ import annotations

import decimal
import glob
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.binding import RefE, REFERENCE_SRC  # noqa: E402

# the reference's functional case (under SW2D_REFERENCE; "" when unset: main() then stops)
CASE = os.path.join(REFERENCE_SRC, "configue_fonctionels", "sp_toce") if REFERENCE_SRC else ""
OUT = os.path.join(ROOT, "tests", "golden", "sp_toce_assim.npz")
EPS = (1e-6, 1e-7, 1e-8)


def ck_hash(h, q, r) -> str:
    d = hashlib.sha256()
    for a in (h, q, r):
        d.update(np.ascontiguousarray(a, np.float64).tobytes())
    return d.hexdigest()


def directions(x: np.ndarray, y: np.ndarray, centres=(3931, 509)):
    """Gaussian bumps of 0.5 m width centred on the given cells."""
    return [np.exp(-((x - x[c]) ** 2 + (y - y[c]) ** 2) / (2.0 * 0.5 ** 2)) for c in centres]


def frames_as_decimals(files):
    """(mantissa, exponent) with value = mantissa * 10^exponent exactly, for columns 3..5."""
    mant, expo = [], []
    for f in files:
        with open(f) as fh:
            fh.readline()
            rm, re_ = [], []
            for line in fh:
                tok = line.split()
                if not tok:
                    continue
                ms, es = [], []
                for t in tok[3:6]:
                    sign, digits, e = decimal.Decimal(t).as_tuple()
                    v = int("".join(map(str, digits)))
                    ms.append(-v if sign else v)
                    es.append(e)
                rm.append(ms)
                re_.append(es)
        mant.append(np.array(rm, dtype=np.int64).T)
        expo.append(np.array(re_, dtype=np.int8).T)
    return np.stack(mant), np.stack(expo)


def decimals_to_float(mant, expo):
    flat = [float(f"{m}e{e}") for m, e in zip(mant.ravel().tolist(), expo.ravel().tolist())]
    return np.array(flat, dtype=np.float64).reshape(mant.shape)


def main():
    if not CASE:
        raise SystemExit("make_assim_golden.py: set SW2D_REFERENCE to the reference's source tree")
    ref = RefE(CASE, portable_math=True)
    cfg = ref.config()
    times, frames = ref.load_observations()
    names = sorted(glob.glob(os.path.join(CASE, "reference", "ResultHydro_p*.txt")))
    mant, expo = frames_as_decimals(names)
    assert np.array_equal(decimals_to_float(mant, expo).view(np.int64), frames.view(np.int64)), "decimal encoding"
    m = ref.load_phi_map(os.path.join(CASE, "input", "phi_init_ones.txt"))
    K = ref.record(m, int(cfg["checkpoint_stride"]))
    segs = ref.segments()
    first, tiles = ref.set_window()
    J_pm = ref.replay_cost(m)
    h_end, q_end, r_end = ref.state()
    # bumps around the cell the descent log names as the gradient's argmax (3931), and another
    import importlib
    pkg = importlib.import_module("inria-internship-project-sw2d-enzyme_b200")
    case = pkg.read_case(CASE)
    dirs = directions(case.mesh.cell_x, case.mesh.cell_y)
    fd = [[(ref.replay_cost(m + e * d), ref.replay_cost(m - e * d)) for e in EPS] for d in dirs]
    ref_glibc = RefE(CASE, portable_math=False)
    ref_glibc.load_observations()
    ref_glibc.record(m, int(cfg["checkpoint_stride"]))
    ref_glibc.set_window()
    J_glibc = ref_glibc.replay_cost(m)
    np.savez_compressed(
        OUT,
        config=json.dumps(cfg), obs_times=times, obs_mant=mant, obs_exp=expo, m=m,
        seg_t_start=np.array([s[0] for s in segs]), seg_n=np.array([len(s[1]) for s in segs], dtype=np.int64),
        dt_seq=np.concatenate([s[1] for s in segs]), obs_trig=np.concatenate([s[2] for s in segs]),
        ck_sha256=np.array([ck_hash(*s[3]) for s in segs]), end_sha256=ck_hash(h_end, q_end, r_end),
        first_segment=first, tiles=tiles, J_pm=J_pm, J_glibc=J_glibc, eps=np.array(EPS),
        fd_dirs=np.stack(dirs), fd_J=np.array(fd))
    print(f"K={K} first={first} tiles={len(tiles)} J_pm={J_pm:.12e} J_glibc={J_glibc:.12e} -> {OUT} "
          f"({os.path.getsize(OUT) / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
