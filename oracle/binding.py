"""ctypes bindings of the two CPU checkers (TEST INFRASTRUCTURE, never the product path).

* :class:`SpOracle` — the plain-C restatement ``sp_oracle.c`` (built into ``_build/``);
* :class:`RefSolver` — the reference's own native solver compiled from its sources with
  ``ref_driver.cpp`` (``_ref/libsw2d_ref.so``), run on a case folder;
* :class:`RefE` — the reference's assimilation layer (class swSpE, assim/*.cpp, with an Enzyme
  stub) through ``ref_e_driver.cpp`` (``_ref/libsw2d_ref_e.so``): its dry run, its segment
  function and its frozen-trajectory cost.
"""
from __future__ import annotations

import ctypes
import importlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libsp_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsw2d_ref.so")
REF_PM_SO = os.path.join(HERE, "_ref", "libsw2d_ref_pm.so")
REF_BIN = os.path.join(HERE, "_ref", "sw2dSolver")
REF_BIN_PM = os.path.join(HERE, "_ref", "sw2dSolver_pm")
REF_MAPPER = os.path.join(HERE, "_ref", "sw2dPorosityMapper")
REF_E_SO = os.path.join(HERE, "_ref", "libsw2d_ref_e.so")
REF_E_PM_SO = os.path.join(HERE, "_ref", "libsw2d_ref_e_pm.so")
B200_BINDING_SO = os.path.join(HERE, "_ref", "libsw2d_b200_binding.so")
# root of the reference's source tree (the environment variable SW2D_REFERENCE; empty when unset)
REFERENCE_SRC = os.environ.get("SW2D_REFERENCE", "")

_pkg = importlib.import_module("inria-internship-project-sw2d-enzyme_b200")
capi = _pkg.capi


def build(reference: bool = True) -> None:
    """Compiles the C restatement and, when the reference sources are present, the reference."""
    targets = ["oracle"]
    if reference and os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-j8", f"REF={REFERENCE_SRC}"] + targets, cwd=HERE, check=True)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


_P = ctypes.c_void_p
_D = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def _oracle_lib():
    if not os.path.exists(ORACLE_SO):
        build(reference=False)
    lib = ctypes.CDLL(ORACLE_SO)
    lib.spo_create.argtypes = [ctypes.POINTER(capi.Sw2dMesh), ctypes.POINTER(capi.Sw2dParams),
                               ctypes.POINTER(capi.Sw2dCellFields), ctypes.POINTER(capi.Sw2dBcTable),
                               capi.c_double_p, capi.c_double_p, capi.c_double_p]
    lib.spo_create.restype = _P
    lib.spo_step.argtypes = [_P, ctypes.c_int]
    lib.spo_step.restype = ctypes.c_int
    lib.spo_get_state.argtypes = [_P, _D, _D, _D]
    lib.spo_set_state.argtypes = [_P, _D, _D, _D]
    lib.spo_time.argtypes = [_P]
    lib.spo_time.restype = ctypes.c_double
    lib.spo_dt.argtypes = [_P]
    lib.spo_dt.restype = ctypes.c_double
    lib.spo_set_time.argtypes = [_P, ctypes.c_double, ctypes.c_double]
    lib.spo_get_array.argtypes = [_P, ctypes.c_char_p, _D]
    lib.spo_get_array.restype = ctypes.c_long
    lib.spo_destroy.argtypes = [_P]
    lib.spo_set_portable_math.argtypes = [_P, ctypes.c_int]
    return lib


class SpOracle:
    """The C restatement of the native SP step on a :class:`Case`.  ``portable_math`` selects the
    portable exp/log of the CUDA build instead of the host libm."""

    def __init__(self, case, portable_math: bool = False):
        self.lib = _oracle_lib()
        self.case = case
        self.n = case.mesh.cell_nb
        self._in = capi.native_inputs(case)
        i = self._in
        self.h = self.lib.spo_create(ctypes.byref(i.mesh), ctypes.byref(i.params), ctypes.byref(i.fields),
                                     ctypes.byref(i.bc), capi._dp(i.h0), capi._dp(i.q0), capi._dp(i.r0))
        self.lib.spo_set_portable_math(self.h, 1 if portable_math else 0)

    def step(self, n: int) -> int:
        k = self.lib.spo_step(self.h, int(n))
        if k < 0:
            raise RuntimeError(f"oracle step failed with status {k}")
        return k

    def state(self):
        h, q, r = (np.empty(self.n) for _ in range(3))
        self.lib.spo_get_state(self.h, h, q, r)
        return h, q, r

    def set_state(self, h, q, r):
        self.lib.spo_set_state(self.h, *(np.ascontiguousarray(a, dtype=np.float64) for a in (h, q, r)))

    @property
    def t(self) -> float:
        return self.lib.spo_time(self.h)

    @property
    def dt(self) -> float:
        return self.lib.spo_dt(self.h)

    def array(self, name: str) -> np.ndarray:
        m = self.case.mesh
        out = np.empty(max(m.cell_nb, m.edge_int_nb, m.edge_bnd_nb, 1))
        k = self.lib.spo_get_array(self.h, name.encode(), out)
        if k < 0:
            raise KeyError(name)
        return out[:k].copy()

    def __del__(self):
        try:
            self.lib.spo_destroy(self.h)
        except Exception:
            pass


class RefSolver:
    """The reference's native SP, DIP or DDP solver (built from its own sources) on a case
    folder.  ``portable_math`` loads the build linked with the portable exp/log of the CUDA
    build.  For a DDP case ``state()`` is (thetaW, thetaW u, thetaW v)."""

    def __init__(self, folder: str, quiet: bool = True, portable_math: bool = False):
        so = REF_PM_SO if portable_math else REF_SO
        if not os.path.exists(so):
            raise RuntimeError(f"reference library not built ({so})")
        lib = ctypes.CDLL(so)
        lib.sw2dref_open.argtypes = [ctypes.c_char_p, ctypes.c_int]
        lib.sw2dref_open.restype = _P
        lib.sw2dref_step.argtypes = [_P, ctypes.c_int]
        lib.sw2dref_step.restype = ctypes.c_int
        lib.sw2dref_run.argtypes = [_P]
        for f in ("sw2dref_time", "sw2dref_dt", "sw2dref_t_max"):
            getattr(lib, f).argtypes = [_P]
            getattr(lib, f).restype = ctypes.c_double
        for f in ("sw2dref_cell_nb", "sw2dref_edge_int_nb", "sw2dref_edge_bnd_nb"):
            getattr(lib, f).argtypes = [_P]
            getattr(lib, f).restype = ctypes.c_long
        lib.sw2dref_get_state.argtypes = [_P, _D, _D, _D]
        lib.sw2dref_set_state.argtypes = [_P, _D, _D, _D]
        lib.sw2dref_get_array.argtypes = [_P, ctypes.c_char_p, _D]
        lib.sw2dref_get_array.restype = ctypes.c_int
        lib.sw2dref_slopes.argtypes = [_P, _D, _D]
        lib.sw2dref_ddp_table.argtypes = [_P, ctypes.c_int, ctypes.c_long, _D, _D, _D, ctypes.c_long]
        lib.sw2dref_ddp_table.restype = ctypes.c_long
        lib.sw2dref_failed.argtypes = [_P]
        lib.sw2dref_failed.restype = ctypes.c_int
        self.lib = lib
        self.h = lib.sw2dref_open(folder.encode(), 1 if quiet else 0)
        if not self.h:
            raise RuntimeError(f"reference failed to open {folder}")
        self.n = lib.sw2dref_cell_nb(self.h)
        self.ni = lib.sw2dref_edge_int_nb(self.h)
        self.nb = lib.sw2dref_edge_bnd_nb(self.h)

    def step(self, n: int) -> int:
        return self.lib.sw2dref_step(self.h, int(n))

    def run(self) -> int:
        return self.lib.sw2dref_run(self.h)

    @property
    def failed(self) -> bool:
        """True once a step failed where the reference's execute() stops with EXIT_FAILURE."""
        return bool(self.lib.sw2dref_failed(self.h))

    def state(self):
        h, q, r = (np.empty(self.n) for _ in range(3))
        self.lib.sw2dref_get_state(self.h, h, q, r)
        return h, q, r

    def set_state(self, h, q, r):
        self.lib.sw2dref_set_state(self.h, *(np.ascontiguousarray(a, dtype=np.float64) for a in (h, q, r)))

    @property
    def t(self) -> float:
        return self.lib.sw2dref_time(self.h)

    @property
    def dt(self) -> float:
        return self.lib.sw2dref_dt(self.h)

    def array(self, name: str) -> np.ndarray:
        out = np.empty(max(self.n, self.ni, self.nb, 1))
        k = self.lib.sw2dref_get_array(self.h, name.encode(), out)
        if k < 0:
            raise KeyError(name)
        return out[:k].copy()

    def slopes(self):
        sx, sy = np.empty(self.n), np.empty(self.n)
        self.lib.sw2dref_slopes(self.h, sx, sy)
        return sx, sy

    def ddp_table(self, which: str, record: int):
        """(z, phi, theta) levels of a DDP cell / internal edge / boundary edge table."""
        k = {"cell": 0, "edge_int": 1, "edge_bnd": 2}[which]
        buf = [np.empty(4096) for _ in range(3)]
        n = self.lib.sw2dref_ddp_table(self.h, k, int(record), buf[0], buf[1], buf[2], 4096)
        if n < 0:
            raise KeyError(f"{which}[{record}]")
        return tuple(b[:n].copy() for b in buf)


class RefE:
    """The reference's porosity-assimilation engine (swSpE) on a case folder whose input.solv may
    hold the assimilation keys.  ``portable_math`` loads the build whose exp, log and cbrt are the
    portable versions of the CUDA build."""

    def __init__(self, folder: str, quiet: bool = True, portable_math: bool = False):
        so = REF_E_PM_SO if portable_math else REF_E_SO
        if not os.path.exists(so):
            raise RuntimeError(f"reference assimilation library not built ({so})")
        lib = ctypes.CDLL(so)
        L = ctypes.c_long
        lib.sw2dref_e_open.argtypes = [ctypes.c_char_p, ctypes.c_int]
        lib.sw2dref_e_open.restype = _P
        lib.sw2dref_e_cell_nb.argtypes = [_P]
        lib.sw2dref_e_cell_nb.restype = L
        lib.sw2dref_e_config.argtypes = [_P, _D]
        lib.sw2dref_e_get_phi.argtypes = [_P, _D]
        lib.sw2dref_e_load_phi_map.argtypes = [_P, ctypes.c_char_p, _D]
        lib.sw2dref_e_load_phi_map.restype = ctypes.c_int
        lib.sw2dref_e_set_options.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        lib.sw2dref_e_set_weights.argtypes = [_P, _D, _D]
        lib.sw2dref_e_set_window_keys.argtypes = [_P, ctypes.c_int, ctypes.c_double, L, L, ctypes.c_double]
        lib.sw2dref_e_load_observations.argtypes = [_P, ctypes.c_int]
        lib.sw2dref_e_load_observations.restype = ctypes.c_int
        lib.sw2dref_e_get_observation.argtypes = [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _D]
        lib.sw2dref_e_set_frames.argtypes = [_P, ctypes.c_int, _D, _D]
        _I = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        lib.sw2dref_e_set_gauges.argtypes = [_P, ctypes.c_int, _D, ctypes.c_int, _I, _D, _D]
        lib.sw2dref_e_record.argtypes = [_P, _D, L, ctypes.c_int]
        lib.sw2dref_e_record.restype = L
        lib.sw2dref_e_segment.argtypes = [_P, L, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]
        lib.sw2dref_e_segment.restype = L
        lib.sw2dref_e_set_window.argtypes = [_P, ctypes.POINTER(L), _I]
        lib.sw2dref_e_set_window.restype = ctypes.c_int
        lib.sw2dref_e_set_truncation.argtypes = [_P, L]
        lib.sw2dref_e_replay_cost.argtypes = [_P, _D, ctypes.c_int]
        lib.sw2dref_e_replay_cost.restype = ctypes.c_double
        lib.sw2dref_e_get_state.argtypes = [_P, _D, _D, _D]
        lib.sw2dref_e_time.argtypes = [_P]
        lib.sw2dref_e_time.restype = ctypes.c_double
        lib.sw2dref_e_close.argtypes = [_P]
        lib.sw2dref_e_folder.argtypes = [_P]
        lib.sw2dref_e_folder.restype = ctypes.c_char_p
        lib.sw2dref_e_generate_references.argtypes = [_P, _D, L, ctypes.c_int]
        lib.sw2dref_e_generate_references.restype = L
        self.lib = lib
        self.h = lib.sw2dref_e_open(folder.encode(), 1 if quiet else 0)
        if not self.h:
            raise RuntimeError(f"reference assimilation layer failed to open {folder}")
        self.n = lib.sw2dref_e_cell_nb(self.h)
        self.K = 0

    CONFIG = ("checkpoint_stride", "windowed", "window_duration", "window_steps", "n_windows",
              "t_state_assimilation", "cost_normalize", "phi_transform", "lambda_tanh", "dt_map_ad",
              "mask_wall_gradient", "alpha_reg", "t_0", "t_max")

    def generate_references(self, phi, stride: int, quiet: bool = True):
        """The reference's gen-ref-e mode (generate_references_E) at porosity phi: the maps it
        writes (into this handle's temporary folder), sorted by name."""
        n = self.lib.sw2dref_e_generate_references(self.h, np.ascontiguousarray(phi, dtype=np.float64), int(stride),
                                                   1 if quiet else 0)
        if n < 0:
            raise RuntimeError("the reference's generate_references_E failed")
        folder = os.path.join(self.lib.sw2dref_e_folder(self.h).decode(), "reference")
        return sorted(os.path.join(folder, f) for f in os.listdir(folder) if f.startswith("ResultHydro_p"))

    def config(self) -> dict:
        out = np.zeros(len(self.CONFIG))
        self.lib.sw2dref_e_config(self.h, out)
        return dict(zip(self.CONFIG, out.tolist()))

    def phi(self) -> np.ndarray:
        out = np.empty(self.n)
        self.lib.sw2dref_e_get_phi(self.h, out)
        return out

    def load_phi_map(self, path: str) -> np.ndarray:
        out = np.zeros(self.n)
        if self.lib.sw2dref_e_load_phi_map(self.h, path.encode(), out) != 0:
            raise RuntimeError(f"cannot read {path}")
        return out

    def set_options(self, cost_normalize: bool, phi_transform: int = 0, lambda_tanh: float = 1.0) -> None:
        self.lib.sw2dref_e_set_options(self.h, int(cost_normalize), int(phi_transform), float(lambda_tanh))

    def set_window_keys(self, windowed: bool, duration: float = -1.0, steps: int = -1, n_windows: int = 1,
                        t_state: float = 0.0) -> None:
        self.lib.sw2dref_e_set_window_keys(self.h, int(windowed), float(duration), int(steps), int(n_windows),
                                           float(t_state))

    def set_weights(self, wh, wq) -> None:
        self.lib.sw2dref_e_set_weights(self.h, np.ascontiguousarray(wh, np.float64), np.ascontiguousarray(wq, np.float64))

    def load_observations(self):
        """The reference's reader of reference/ResultHydro_p*.txt: (times, frames[k][3][n])."""
        n_obs = self.lib.sw2dref_e_load_observations(self.h, 1)
        if n_obs < 0:
            raise RuntimeError("observations could not be loaded")
        times = np.zeros(n_obs)
        frames = np.zeros((n_obs, 3, self.n))
        t = ctypes.c_double()
        for k in range(n_obs):
            buf = np.zeros(3 * self.n)
            self.lib.sw2dref_e_get_observation(self.h, k, ctypes.byref(t), buf)
            times[k] = t.value
            frames[k] = buf.reshape(3, self.n)
        return times, frames

    def set_frames(self, times, frames) -> None:
        t = np.ascontiguousarray(times, np.float64)
        self.lib.sw2dref_e_set_frames(self.h, len(t), t, np.ascontiguousarray(frames, np.float64).ravel())

    def set_gauges(self, times, cells, weights, values) -> None:
        t = np.ascontiguousarray(times, np.float64)
        c = np.ascontiguousarray(cells, np.int64)
        self.lib.sw2dref_e_set_gauges(self.h, len(t), t, len(c), c, np.ascontiguousarray(weights, np.float64),
                                      np.ascontiguousarray(values, np.float64).ravel())

    def record(self, m, stride: int) -> int:
        self.K = int(self.lib.sw2dref_e_record(self.h, np.ascontiguousarray(m, np.float64), int(stride), 1))
        return self.K

    def segments(self):
        """[(t_start, dt_seq, obs_trig, (h, q, r) checkpoint)] of the record."""
        out = []
        for k in range(self.K):
            ts = ctypes.c_double()
            n = self.lib.sw2dref_e_segment(self.h, k, ctypes.addressof(ts), None, None, None, None, None)
            dt = np.zeros(n)
            tr = np.zeros(n, dtype=np.int32)
            h, q, r = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
            self.lib.sw2dref_e_segment(self.h, k, None, dt.ctypes.data, tr.ctypes.data, h.ctypes.data, q.ctypes.data,
                                       r.ctypes.data)
            out.append((ts.value, dt, tr, (h, q, r)))
        return out

    def set_window(self):
        """The window and tiles get_spatial_gradient_checkpointed would set: (first, tiles)."""
        first = ctypes.c_long()
        tiles = np.zeros(max(1, self.K), dtype=np.int64)
        nt = self.lib.sw2dref_e_set_window(self.h, ctypes.byref(first), tiles)
        return first.value, tiles[:nt].copy()

    def set_truncation(self, seg: int) -> None:
        self.lib.sw2dref_e_set_truncation(self.h, int(seg))

    def replay_cost(self, m) -> float:
        return float(self.lib.sw2dref_e_replay_cost(self.h, np.ascontiguousarray(m, np.float64), 1))

    def state(self):
        h, q, r = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        self.lib.sw2dref_e_get_state(self.h, h, q, r)
        return h, q, r

    def close(self) -> None:
        if self.h:
            self.lib.sw2dref_e_close(self.h)
            self.h = None


class B200Binding:
    """The reference-side binding of INTEGRATION.md (oracle/b200_binding.cpp, compiled against the
    reference's headers and objects): the reference reads the case folder with its own swSp and
    the model class swSpB200 runs the time loop on the GPU through the C ABI."""

    def __init__(self, folder: str, device: int = 0):
        if not os.path.exists(B200_BINDING_SO):
            raise RuntimeError(f"binding library not built ({B200_BINDING_SO})")
        lib = ctypes.CDLL(B200_BINDING_SO)
        lib.b200_open.argtypes = [ctypes.c_char_p, ctypes.c_int]
        lib.b200_open.restype = _P
        lib.b200_execute.argtypes = [_P, ctypes.POINTER(ctypes.c_int64)]
        lib.b200_execute.restype = ctypes.c_int
        lib.b200_cell_nb.argtypes = [_P]
        lib.b200_cell_nb.restype = ctypes.c_long
        lib.b200_state.argtypes = [_P, _D, _D, _D]
        lib.b200_error.argtypes = [_P]
        lib.b200_error.restype = ctypes.c_char_p
        lib.b200_close.argtypes = [_P]
        self.lib = lib
        self.h = lib.b200_open(folder.encode(), int(device))
        if not self.h:
            raise RuntimeError(f"binding failed to open {folder}")
        err = lib.b200_error(self.h).decode()
        if err:
            raise RuntimeError(f"binding init: {err}")
        self.n = lib.b200_cell_nb(self.h)

    def execute(self) -> int:
        steps = ctypes.c_int64(0)
        if self.lib.b200_execute(self.h, ctypes.byref(steps)) != 0:
            raise RuntimeError(f"binding execute: {self.lib.b200_error(self.h).decode()}")
        return int(steps.value)

    def state(self):
        h, q, r = (np.empty(self.n) for _ in range(3))
        self.lib.b200_state(self.h, h, q, r)
        return h, q, r

    def close(self):
        if self.h:
            self.lib.b200_close(self.h)
            self.h = None
