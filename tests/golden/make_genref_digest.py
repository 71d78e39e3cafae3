"""Digest fixture of the reference's gen-ref-e mode on sp_toce (swSpE::generate_references_E,
assim/swSpE_checkpoint.cpp:470-515), run from the reference's own objects built with the
portable exp/log/cbrt of the CUDA build (oracle/_ref/libsw2d_ref_e_pm.so) at the case's
porosity_ref_map.  The case's shipped reference/ResultHydro_p*.txt maps were written by the same
mode with the host libm (tests/test_oracle_assim.py checks that they are reproduced digit for
digit from the host-libm build); the two libms' trajectories part at the wet/dry fronts, so the
GPU, whose _E step uses the portable functions, is pinned to this fixture instead: per map, the
SHA-256 of its printed water_depth, unit_discharge_x and unit_discharge_y.

Run here (the reference tree must be present, SW2D_REFERENCE set):
    python tests/golden/make_genref_digest.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "sp_toce_genref_pm.json")


def frame_digests(files):
    """Per map: SHA-256 of the printed decimals (mantissa, exponent) of columns 3..5 (the
    exponent of a printed zero is not part of it)."""
    import numpy as np
    from tests.golden.make_assim_golden import frames_as_decimals
    mant, expo = frames_as_decimals(files)
    out = []
    for k in range(mant.shape[0]):
        e = np.where(mant[k] == 0, 0, expo[k]).astype(np.int8)
        d = hashlib.sha256()
        d.update(np.ascontiguousarray(mant[k], np.int64).tobytes())
        d.update(np.ascontiguousarray(e).tobytes())
        out.append(d.hexdigest())
    return out


def main():
    from oracle import binding
    case = os.path.join(binding.REFERENCE_SRC, "configue_fonctionels", "sp_toce")
    ref = binding.RefE(case, portable_math=True)
    try:
        phi = ref.load_phi_map(os.path.join(case, "input", "SP_cell_porosity_map.txt"))
        files = ref.generate_references(phi, int(ref.config()["checkpoint_stride"]))
        res = {"names": [os.path.basename(f) for f in files], "sha256": frame_digests(files)}
    finally:
        ref.close()
    with open(OUT, "w") as fh:
        json.dump(res, fh, indent=1)
    print(len(res["names"]), "maps;", OUT)


if __name__ == "__main__":
    main()
