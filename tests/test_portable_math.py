"""The portable exp/log/cbrt of the CUDA build (csrc/portable_math.h): accuracy against the host
libm (cbrt: against the 80-bit long-double cube root), special values, and (GPU) identical bits
on the device and the host, within a few ulp of CUDA's own functions."""
import ctypes
import math
import os

import numpy as np
import pytest

from tests.conftest import ROOT, load_pkg

HDR = os.path.join(ROOT, "inria-internship-project-sw2d-enzyme_b200", "csrc", "portable_math.h")


@pytest.fixture(scope="module")
def host_pm(tmp_path_factory):
    """The header compiled for the host with the flags of the oracle (-ffp-contract=off)."""
    import subprocess
    d = tmp_path_factory.mktemp("pm")
    src = d / "pm.c"
    src.write_text(f'#include "{HDR}"\ndouble pexp(double x) {{ return sw2d_exp(x); }}\n'
                   'double plog(double x) { return sw2d_log(x); }\n'
                   'double pcbrt(double x) { return sw2d_cbrt(x); }\n')
    so = d / "libpm.so"
    subprocess.run(["gcc", "-std=c11", "-O2", "-fPIC", "-ffp-contract=off", "-shared", "-o", str(so), str(src)],
                   check=True)
    lib = ctypes.CDLL(str(so))
    for f in (lib.pexp, lib.plog, lib.pcbrt):
        f.argtypes = [ctypes.c_double]
        f.restype = ctypes.c_double
    return lib


def _ulps(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    sp = np.abs(np.spacing(b))
    return np.where(a == b, 0.0, np.abs(a - b) / sp)


def _samples():
    rng = np.random.default_rng(5)
    xe = np.concatenate([rng.uniform(-745, 709.7, 20000), rng.uniform(-40, 40, 20000), rng.uniform(-1e-3, 1e-3, 5000),
                         -np.logspace(-3, 4, 5000)])
    xl = np.concatenate([np.exp(rng.uniform(-700, 700, 20000)), rng.uniform(0.5, 2.0, 20000),
                         np.logspace(-16, 2, 5000), rng.uniform(1e-5, 10, 5000)])
    return xe, xl


def test_portable_math_accuracy(host_pm):
    xe, xl = _samples()
    pe = np.array([host_pm.pexp(float(v)) for v in xe])
    pl = np.array([host_pm.plog(float(v)) for v in xl])
    assert _ulps(pe, np.exp(xe)).max() <= 2.0
    assert _ulps(pl, np.log(xl)).max() <= 2.0


def _cbrt_samples():
    rng = np.random.default_rng(6)
    x = np.concatenate([np.ldexp(rng.uniform(0.5, 1.0, 20000), rng.integers(-1070, 1020, 20000)),
                        rng.uniform(1e-16, 10.0, 20000), np.logspace(-16, 2, 5000), -rng.uniform(0.0, 5.0, 2000)])
    return x


def test_portable_cbrt_accuracy(host_pm):
    """Within 1 ulp of the cube root taken in 80-bit long double (the host libm's double cbrt
    itself is off by up to ~3.5 ulp on these samples)."""
    x = _cbrt_samples()
    p = np.array([host_pm.pcbrt(float(v)) for v in x])
    truth = np.cbrt(x.astype(np.longdouble))
    err = np.abs(p.astype(np.longdouble) - truth) / np.abs(np.spacing(truth.astype(np.float64))).astype(np.longdouble)
    assert float(err.max()) <= 1.0
    for v in (0.0, -0.0, 1.0, 8.0, 27.0, 0.125, -8.0, 1e-300, 5e-324):
        assert host_pm.pcbrt(v) == v if v == 0.0 else abs(host_pm.pcbrt(v) - math.cbrt(v)) <= 2 * math.ulp(math.cbrt(v))
    assert host_pm.pcbrt(float("inf")) == float("inf") and math.isnan(host_pm.pcbrt(float("nan")))
    assert math.copysign(1.0, host_pm.pcbrt(-0.0)) < 0


def test_portable_math_special_values(host_pm):
    inf = float("inf")
    assert host_pm.pexp(0.0) == 1.0 and host_pm.pexp(-inf) == 0.0 and host_pm.pexp(inf) == inf
    assert math.isnan(host_pm.pexp(float("nan"))) and host_pm.pexp(800.0) == inf and host_pm.pexp(-800.0) == 0.0
    assert host_pm.plog(1.0) == 0.0 and host_pm.plog(0.0) == -inf and host_pm.plog(inf) == inf
    assert math.isnan(host_pm.plog(-1.0)) and math.isnan(host_pm.plog(float("nan")))
    assert abs(host_pm.plog(5e-324) - math.log(5e-324)) <= 2 * abs(math.ulp(math.log(5e-324)))


@pytest.mark.gpu
def test_portable_math_device_matches_host(host_pm):
    pkg = load_pkg()
    pkg.build.build()
    xe, xl = _samples()
    de = pkg.solver.eval_math("exp", xe)
    dl = pkg.solver.eval_math("log", xl)
    he = np.array([host_pm.pexp(float(v)) for v in xe])
    hl = np.array([host_pm.plog(float(v)) for v in xl])
    assert np.array_equal(de.view(np.int64), he.view(np.int64))
    assert np.array_equal(dl.view(np.int64), hl.view(np.int64))
    ce = pkg.solver.eval_math("cuda_exp", xe)
    cl = pkg.solver.eval_math("cuda_log", xl)
    assert _ulps(de, ce).max() <= 2.0
    assert _ulps(dl, cl).max() <= 2.0
    dc = pkg.solver.eval_math("cbrt", _cbrt_samples())
    hc = np.array([host_pm.pcbrt(float(v)) for v in _cbrt_samples()])
    assert np.array_equal(dc.view(np.int64), hc.view(np.int64))
    assert _ulps(dc, pkg.solver.eval_math("cuda_cbrt", _cbrt_samples())).max() <= 2.0
