"""Reverse functions of the differentiated step (csrc/spe_math.cuh), checked against central
finite differences on the host.

tests/spe_fd_check.cpp builds the device functions with g++ and compares, for thousands of random
inputs per function, the reverse's vector-Jacobian product with a central difference of the
forward: desingularised velocity, Godunov and MUSCL-EVR sides, the smooth-porosity HLLC in each
regime, the boundary flux of every type wet and dry, the cell update (flush, clamp,
semi-implicit Strickler friction, head loss) and the porosity transforms.  A sample whose
evaluation point lies within the step of a branch switch can differ; at most 0.2 % may.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "inria-internship-project-sw2d-enzyme_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "spe_fd_check.cpp")

EXPECTED = (["desing", "god_side", "evr_bnd_side", "evr_side_left", "evr_side_right",
             "hllc_wet", "hllc_left_dry", "hllc_right_dry"] +
            [f"boundary_flux_{b}_{w}" for b in ("q", "h", "z", "fr") for w in ("wet", "dry")] +
            [f"cell_update_friction{f}_headloss{h}" for f in range(2) for h in range(2)] +
            [f"transform_{k}" for k in ("none", "clamp", "tanh", "normalize")])


def _compiler():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    pytest.skip("no C++ compiler")


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("spe_fd") / "spe_fd_check")
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


STEP_SRC = os.path.join(ROOT, "tests", "spe_step_check.cpp")


def test_whole_steps_match_central_differences(tmp_path):
    """tests/spe_step_check.cpp: 12 steps of the _E step on a small triangulated channel, composed
    as the CUDA kernels compose them, and their reverse composed as the reverse kernels: the
    gradient of a misfit with respect to porosity and the initial depth against central
    differences (Godunov and MUSCL-EVR, 6 seeded trials x 3 directions each)."""
    exe = str(tmp_path / "spe_step_check")
    subprocess.run([_compiler(), "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, STEP_SRC, "-o", exe], check=True,
                   capture_output=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    res = {ln.split()[0]: ln.split()[1:] for ln in out.splitlines()}
    assert sorted(res) == ["step_godunov", "step_muscl_evr"]
    for name, (n, fail, worst) in res.items():
        assert int(n) >= 18 and int(fail) == 0, f"{name}: {fail} of {n} differ (worst {worst})"
