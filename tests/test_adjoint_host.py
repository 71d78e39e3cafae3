"""Hand-written reverse functions of the step, checked against central finite differences.

The forward device functions (csrc/sp_math.cuh) and their reverses (csrc/sp_adjoint.cuh) are
plain host/device C++; tests/adjoint_fd_check.cpp builds them with g++ and compares, for
thousands of random inputs per function, the reverse's vector-Jacobian product with a central
difference of the forward.  The HLLC reverse is checked with both sides wet and with one side
dry (for both topography discretisations), the boundary reverse for every boundary type wet and
dry, the cell update for every friction law with and without head loss and velocity cap, and
the slope limiter for 2 to 6 neighbours.  A sample whose evaluation point lies within the step
of a branch switch (a limiter trigger, the velocity cap) can differ; at most 0.2 % of the
samples of a function may.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "inria-internship-project-sw2d-enzyme_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "adjoint_fd_check.cpp")

EXPECTED = (["godunov_side", "evr_side_left", "evr_side_right"] +
            [f"hllc_{t}_{r}" for t in ("discontinuous", "blending") for r in ("wet", "left_dry", "right_dry")] +
            [f"boundary_flux_{b}_{w}" for b in ("q", "h", "z", "fr") for w in ("wet", "dry")] +
            [f"update_friction{f}_headloss{h}_cap{c}" for f in range(4) for h in range(2) for c in range(2)] +
            [f"slopes_n{n}" for n in range(2, 7)])


def _compiler():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    pytest.skip("no C++ compiler")


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("fd") / "adjoint_fd_check")
    subprocess.run([_compiler(), "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, SRC, "-o", exe], check=True,
                   capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.splitlines():
        name, n, fail, worst = line.split()
        res[name] = (int(n), int(fail), float(worst))
    return res


def test_every_reverse_function_was_checked(results):
    assert sorted(results) == sorted(EXPECTED)


@pytest.mark.parametrize("name", EXPECTED)
def test_reverse_matches_central_differences(results, name):
    n, fail, worst = results[name]
    assert n >= 500, f"{name}: only {n} samples"
    assert fail <= max(1, int(0.002 * n)), f"{name}: {fail} of {n} samples differ (worst relative error {worst:.2e})"
