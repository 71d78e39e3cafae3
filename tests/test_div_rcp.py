"""sw2d::div_rcp (csrc/sp_math.cuh), the division by a shared reciprocal the slope kernels use,
against the IEEE division on the host: tests/div_rcp_check.cpp runs it on about 60 million
inputs (random significands over wide exponent ranges, the slope arithmetic's own magnitudes,
divisors with significands near 1 and near 2, quotients at rounding midpoints, zeros,
subnormals, huge values, infinities and NaN) and counts the quotients whose bits differ.  The
device side is checked on 33 million inputs of the same families by
test_device_div_rcp_is_the_ieee_quotient (sw2d_eval_div)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "inria-internship-project-sw2d-enzyme_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "div_rcp_check.cpp")
CASES = ["random_wide", "mesh_like", "divisor_edges", "midpoints", "specials"]


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    cxx = next((c for c in ("/usr/bin/g++", shutil.which("g++")) if c and os.path.exists(c)), None)
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("div") / "div_rcp_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, SRC, "-o", exe], check=True,
                   capture_output=True)
    run = subprocess.run([exe], check=True, capture_output=True, text=True)
    res = {}
    for line in run.stdout.splitlines():
        name, n, bad = line.split()
        res[name] = (int(n), int(bad))
    return res, run.stderr


def test_every_family_ran(results):
    assert sorted(results[0]) == sorted(CASES)


@pytest.mark.parametrize("name", CASES)
def test_div_rcp_is_the_ieee_quotient(results, name):
    n, bad = results[0][name]
    assert n > 10000
    assert bad == 0, f"{name}: {bad} of {n} quotients differ\n{results[1]}"


def _families(rng, n):
    """Random significands over wide exponents, mesh-like magnitudes, divisors with significands
    near 1 and 2, quotients at rounding midpoints, and special values (as the host check)."""
    def bits(sign, exp, mant):
        return ((sign.astype(np.uint64) << np.uint64(63)) | ((exp + 1023).astype(np.uint64) << np.uint64(52))
                | mant.astype(np.uint64)).view(np.float64)
    m52 = np.uint64(0xFFFFFFFFFFFFF)
    mant = lambda: rng.integers(0, 2**63, n, dtype=np.uint64) & m52
    a1 = bits(rng.integers(0, 2, n), rng.integers(-800, 801, n), mant())
    b1 = bits(np.zeros(n, np.int64), rng.integers(-59, 60, n), mant())
    dz = rng.uniform(-5, 5, n) * 10.0 ** rng.integers(-12, 1, n)
    dx = rng.uniform(-200, 200, n)
    a2, b2 = dz * dx, np.sqrt(dx * dx + rng.uniform(0, 200, n) ** 2) + 1e-3
    k = rng.integers(0, 2**16, n, dtype=np.uint64)
    e = rng.integers(-40, 41, n)
    b3 = np.concatenate([bits(np.zeros(n, np.int64), e, m52 - k), bits(np.zeros(n, np.int64), e, k)])
    a3 = bits(rng.integers(0, 2, 2 * n), rng.integers(-500, 501, 2 * n), rng.integers(0, 2**63, 2 * n, dtype=np.uint64) & m52)
    q = bits(rng.integers(0, 2, n), rng.integers(-300, 301, n), mant())
    mid = q + (np.nextafter(q, 2 * q) - q) * 0.5
    b4 = bits(np.zeros(n, np.int64), rng.integers(-50, 51, n), mant())
    a4 = mid * b4
    a4 = np.concatenate([a4, np.nextafter(a4, 0.0), np.nextafter(a4, 2 * a4), q * b4])
    b4 = np.tile(b4, 4)
    sp = np.array([0.0, -0.0, 5e-324, -5e-324, 2.0**-1022, 2.0**-960, 2.0**-901, 2.0**-899, 2.0**899, 2.0**901,
                   1.7976931348623157e308, -1.7976931348623157e308, np.inf, -np.inf, np.nan, 1.0, -1.0, 3.0])
    a5 = np.repeat(sp, 200)
    b5 = bits(np.zeros(a5.size, np.int64), rng.integers(-59, 60, a5.size), rng.integers(0, 2**63, a5.size, dtype=np.uint64) & m52)
    return np.concatenate([a1, a2, a3, a4, a5]), np.concatenate([b1, b2, b3, b4, b5])


@pytest.mark.gpu
def test_device_div_rcp_is_the_ieee_quotient():
    """On the device, both the IEEE division and div_rcp give numpy's (IEEE) quotient bits."""
    from tests.conftest import load_pkg
    pkg = load_pkg()
    pkg.build.build()
    rng = np.random.default_rng(20240607)
    for _ in range(4):
        a, b = _families(rng, 1 << 21)
        with np.errstate(all="ignore"):
            want = a / b
        for shared in (False, True):
            got = pkg.solver.eval_div(a, b, shared)
            same = (got.view(np.uint64) == want.view(np.uint64)) | (np.isnan(got) & np.isnan(want))
            assert same.all(), (f"shared={shared}: {np.count_nonzero(~same)} of {a.size} differ, "
                                f"first a={a[~same][0]!r} b={b[~same][0]!r}")
