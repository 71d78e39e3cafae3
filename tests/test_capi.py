"""The C-ABI library builds for sm_100a, loads without a GPU and exports every entry point
that include/sw2d_b200.h declares (no compute call is made here)."""
import ctypes
import os
import re

from tests.conftest import ROOT, load_pkg


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^[A-Za-z_][\w \*]*?\b(sw2d_\w+)\s*\(", txt, flags=re.M))
    return names


def test_library_exports_declared_symbols():
    pkg = load_pkg()
    path = pkg.build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    declared = _declared()
    assert {"sw2d_create", "sw2d_step_n", "sw2d_get_state", "sw2d_destroy"} <= declared
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(pkg.capi.EXPORTED) == declared
    assert lib.sw2d_abi_version() == 3


def test_params_from_input_solv_keys():
    pkg = load_pkg()
    p = pkg.capi.params_from_opts({"num_scheme": "muscl_evr", "topo_discretization": "blending",
                                   "model_friction": "strickler", "model_singular_head_loss": "active",
                                   "cfl_max": "0.8", "t_max": "30."})
    assert (p.scheme, p.topo, p.friction, p.singular_head_loss) == (1, 1, 3, 1)
    assert p.cfl_max == 0.8 and p.t_max == 30.0 and p.h_min == 1e-5 and p.phi_min == 1e-16
    assert p.dt_max == 10.0 and p.dt_map == 100.0 and p.v_max == 100.0 and p.fr_max == 100.0
