"""SpModel: the host-side mirror of the reference's SP model interface over the C ABI.

The reference drives a model through ``swParent::create`` / ``importAttributesFromSolverParam``
/ ``init(mesh)`` / ``execute()`` (src/sw2dSolver/models/swParent.h:19-27, called from
src/sw2dSolver/main.cpp:138-173).  ``SpModel`` keeps those names and meanings:

* ``SpModel.from_folder(folder)`` / ``SpModel(case)`` — read the case and ``init`` (upload,
  renumber, edge factors, t = t_0);
* ``execute()`` — run until t >= t_max (no result storage), returns the number of steps;
* ``step(n)`` — at most n passes of the time-loop body;
* ``state()``, ``set_state()``, ``t``, ``dt``, ``array(name)``.

Where the reference calls ``exit(1)`` (src/common/swMessage.cpp:74-84), SpModel raises
:class:`Sw2dError` carrying the C status code and message.  There is no CPU fallback: without
the CUDA library or a GPU the constructor raises.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import capi
from .case import Case, read_case


class Sw2dError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"sw2d error {code}: {message}")
        self.code = code
        self.message = message


class SpModel:
    """SW2D porosity model (single porosity, or dual integral porosity when the case says
    model_hyperb dip) running on one GPU."""

    def __init__(self, case: Case, device: int = 0):
        self.lib = capi.load_library()
        self.case = case
        self.n = case.mesh.cell_nb
        self.ni = case.mesh.edge_int_nb
        self.nb = case.mesh.edge_bnd_nb
        self._in = capi.native_inputs(case)
        i = self._in
        handle = ctypes.c_void_p()
        if i.dip is not None:  # model_hyperb dip: swDip
            st = self.lib.sw2d_create_dip(ctypes.byref(i.mesh), ctypes.byref(i.params), ctypes.byref(i.fields),
                                          ctypes.byref(i.dip), ctypes.byref(i.bc), capi._dp(i.h0), capi._dp(i.q0),
                                          capi._dp(i.r0), int(device), ctypes.byref(handle))
        else:
            st = self.lib.sw2d_create(ctypes.byref(i.mesh), ctypes.byref(i.params), ctypes.byref(i.fields),
                                      ctypes.byref(i.bc), capi._dp(i.h0), capi._dp(i.q0), capi._dp(i.r0),
                                      int(device), ctypes.byref(handle))
        if st != 0:
            raise Sw2dError(st, self.lib.sw2d_last_error(None).decode())
        self.handle = handle

    @classmethod
    def from_folder(cls, folder: str, device: int = 0) -> "SpModel":
        case = read_case(folder)
        if str(case.opts.get("model_hyperb", "sp")).lower() not in ("sp", "dip"):
            raise Sw2dError(-8, f"model_hyperb {case.opts.get('model_hyperb')!r}: only 'sp' and 'dip' are implemented")
        return cls(case, device)

    def _check(self, st: int) -> None:
        if st != 0:
            raise Sw2dError(st, self.lib.sw2d_last_error(self.handle).decode())

    def step(self, n: int) -> int:
        done = ctypes.c_int64(0)
        self._check(self.lib.sw2d_step_n(self.handle, int(n), ctypes.byref(done)))
        return int(done.value)

    def execute(self) -> int:
        done = ctypes.c_int64(0)
        self._check(self.lib.sw2d_execute(self.handle, ctypes.byref(done)))
        return int(done.value)

    def state(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        h, q, r = (np.empty(self.n) for _ in range(3))
        self._check(self.lib.sw2d_get_state(self.handle, h.ctypes.data, q.ctypes.data, r.ctypes.data))
        return h, q, r

    def set_state(self, h, q, r) -> None:
        h, q, r = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, q, r))
        self._check(self.lib.sw2d_set_state(self.handle, h.ctypes.data, q.ctypes.data, r.ctypes.data))

    def get_state_device(self, h_ptr: int, q_ptr: int, r_ptr: int) -> None:
        self._check(self.lib.sw2d_get_state_device(self.handle, h_ptr, q_ptr, r_ptr))

    def set_state_device(self, h_ptr: int, q_ptr: int, r_ptr: int) -> None:
        self._check(self.lib.sw2d_set_state_device(self.handle, h_ptr, q_ptr, r_ptr))

    @property
    def time(self) -> Tuple[float, float]:
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.sw2d_get_time(self.handle, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    @property
    def t(self) -> float:
        return self.time[0]

    @property
    def dt(self) -> float:
        return self.time[1]

    def set_time(self, t: float, dt: float) -> None:
        self._check(self.lib.sw2d_set_time(self.handle, float(t), float(dt)))

    def array(self, name: str) -> np.ndarray:
        out = np.empty(max(self.n, self.ni, self.nb, 1))
        k = self.lib.sw2d_get_array(self.handle, name.encode(), out.ctypes.data_as(capi.c_double_p), out.size)
        if k < 0:
            self._check(int(k))
        return out[:k].copy()

    def cell_permutation(self) -> np.ndarray:
        perm = np.empty(self.n, dtype=np.int64)
        self._check(self.lib.sw2d_get_cell_permutation(self.handle, perm.ctypes.data_as(capi.c_int64_p)))
        return perm

    def phase_times(self, n_steps: int):
        """{kernel name: average device ms per step} over n_steps steps (which advance the run)."""
        ms = np.zeros(8)
        k = self.lib.sw2d_phase_times(self.handle, int(n_steps), ms.ctypes.data_as(capi.c_double_p), ms.size)
        if k < 0:
            self._check(int(k))
        return {self.lib.sw2d_phase_name(i).decode(): float(ms[i]) for i in range(k)}

    def set_option(self, name: str, value: int) -> None:
        self._check(self.lib.sw2d_set_option(self.handle, name.encode(), int(value)))

    @property
    def stream(self) -> int:
        return int(self.lib.sw2d_get_stream(self.handle) or 0)

    @property
    def kernels_per_step(self) -> int:
        return int(self.lib.sw2d_kernels_per_step(self.handle))

    # ---- adjoint: J and its gradient along a recorded trajectory (frozen dt) -------------------
    # The reference's assimilation front-end (swSpE, assim/swSpE.h) records a dry run, then
    # replays it with the control for J (replay_trajectory_cost) and differentiates the replay
    # (get_spatial_gradient_checkpointed).  These methods are the same steps over the C ABI.

    GRADIENTS = ("h0", "q0", "r0", "z_b", "friction_1", "friction_2")

    def record(self, n_steps: int, checkpoint_every: int = 100) -> int:
        """Runs n_steps CFL-driven steps from the current state and records them as the
        trajectory (dt sequence, checkpoints every `checkpoint_every` steps).  Returns the number
        of steps recorded (fewer when t_max is reached)."""
        done = ctypes.c_int64(0)
        self._check(self.lib.sw2d_record(self.handle, int(n_steps), int(checkpoint_every), ctypes.byref(done)))
        return int(done.value)

    def rerecord(self) -> int:
        """Records the trajectory again from its initial state with the current parameters."""
        done = ctypes.c_int64(0)
        self._check(self.lib.sw2d_rerecord(self.handle, ctypes.byref(done)))
        return int(done.value)

    def trajectory_info(self) -> dict:
        n, k = ctypes.c_int64(), ctypes.c_int64()
        t0, t1 = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.sw2d_trajectory_info(self.handle, ctypes.byref(n), ctypes.byref(k), ctypes.byref(t0),
                                                  ctypes.byref(t1)))
        return {"n_steps": n.value, "checkpoint_every": k.value, "t_start": t0.value, "t_end": t1.value}

    def trajectory_dt(self) -> np.ndarray:
        n = self.trajectory_info()["n_steps"]
        dt = np.empty(n)
        self._check(self.lib.sw2d_get_trajectory_dt(self.handle, dt.ctypes.data_as(capi.c_double_p), n))
        return dt

    def set_trajectory_start(self, h, q, r) -> None:
        h, q, r = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, q, r))
        self._check(self.lib.sw2d_set_trajectory_start(self.handle, h.ctypes.data, q.ctypes.data, r.ctypes.data))

    def set_param(self, name: str, values) -> None:
        """Per-cell parameter: "friction_1", "friction_2", "friction" (both) or "z_b"."""
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(values, dtype=np.float64), (self.n,)))
        self._check(self.lib.sw2d_set_param(self.handle, name.encode(), v.ctypes.data))

    def get_param(self, name: str) -> np.ndarray:
        v = np.empty(self.n)
        self._check(self.lib.sw2d_get_param(self.handle, name.encode(), v.ctypes.data))
        return v

    def set_observations(self, cells, steps, h_obs, w_h=None, q_obs=None, r_obs=None, w_q=None,
                         normalize: bool = False) -> None:
        """Observation set of J: `cells` (distinct cell indices), `steps` (increasing step
        indices after the trajectory's start), h_obs[k, p] (and q_obs, r_obs with weights w_q)."""
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        steps = np.ascontiguousarray(steps, dtype=np.int64)
        npts, nt = cells.size, steps.size
        h_obs = np.ascontiguousarray(np.asarray(h_obs, dtype=np.float64).reshape(nt, npts))
        w_h = np.ascontiguousarray(np.broadcast_to(np.asarray(1.0 if w_h is None else w_h, dtype=np.float64), (npts,)))
        o = capi.Sw2dObs()
        o.n_points, o.cells, o.w_h = npts, cells.ctypes.data_as(capi.c_int64_p), w_h.ctypes.data_as(capi.c_double_p)
        o.n_times, o.steps = nt, steps.ctypes.data_as(capi.c_int64_p)
        o.h_obs = h_obs.ctypes.data_as(capi.c_double_p)
        keep = [cells, steps, h_obs, w_h]
        if w_q is not None:
            w_q = np.ascontiguousarray(np.broadcast_to(np.asarray(w_q, dtype=np.float64), (npts,)))
            q_obs = np.ascontiguousarray(np.asarray(q_obs, dtype=np.float64).reshape(nt, npts))
            r_obs = np.ascontiguousarray(np.asarray(r_obs, dtype=np.float64).reshape(nt, npts))
            o.w_q, o.q_obs, o.r_obs = (a.ctypes.data_as(capi.c_double_p) for a in (w_q, q_obs, r_obs))
            keep += [w_q, q_obs, r_obs]
        o.normalize = 1 if normalize else 0
        self._check(self.lib.sw2d_set_observations(self.handle, ctypes.byref(o)))
        del keep

    def replay_cost(self) -> float:
        J = ctypes.c_double()
        self._check(self.lib.sw2d_replay_cost(self.handle, ctypes.byref(J)))
        return J.value

    def replay_sample(self, cells, steps, discharge: bool = False):
        """h[k, p] (and q, r) at the given cells after each given step of the replayed trajectory."""
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        steps = np.ascontiguousarray(steps, dtype=np.int64)
        h = np.empty((steps.size, cells.size))
        q = np.empty_like(h) if discharge else None
        r = np.empty_like(h) if discharge else None
        self._check(self.lib.sw2d_replay_sample(self.handle, cells.size, cells.ctypes.data_as(capi.c_int64_p),
                                                steps.size, steps.ctypes.data_as(capi.c_int64_p), h.ctypes.data,
                                                q.ctypes.data if discharge else None,
                                                r.ctypes.data if discharge else None))
        return (h, q, r) if discharge else h

    def adjoint(self, wrt=GRADIENTS):
        """(J, {name: dJ/dname}) for the names in `wrt` (a subset of GRADIENTS)."""
        g = capi.Sw2dGradient()
        out = {}
        for name in wrt:
            if name not in self.GRADIENTS:
                raise ValueError(f"unknown gradient {name!r}")
            out[name] = np.empty(self.n)
            setattr(g, name, out[name].ctypes.data_as(capi.c_double_p))
        J = ctypes.c_double()
        self._check(self.lib.sw2d_adjoint(self.handle, ctypes.byref(J), ctypes.byref(g)))
        return J.value, out

    def adjoint_nonfinite(self) -> dict:
        """Entries of the last gradient that were NaN or infinite and were set to 0, per control."""
        c = np.zeros(6, dtype=np.int64)
        self._check(self.lib.sw2d_adjoint_nonfinite(self.handle, c.ctypes.data_as(capi.c_int64_p)))
        return dict(zip(self.GRADIENTS, (int(v) for v in c)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.sw2d_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def eval_math(fn: str, x, device: int = 0) -> np.ndarray:
    """Device evaluation of the step's elementary functions: fn in ("exp", "log", "cbrt") for
    the portable versions the step uses, ("cuda_exp", "cuda_log", "cuda_cbrt") for CUDA's."""
    lib = capi.load_library()
    code = {"exp": 0, "log": 1, "cuda_exp": 2, "cuda_log": 3, "cbrt": 4, "cuda_cbrt": 5}[fn]
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    st = lib.sw2d_eval_math(int(device), code, x.ctypes.data_as(capi.c_double_p), y.ctypes.data_as(capi.c_double_p),
                            x.size)
    if st != 0:
        raise Sw2dError(st, lib.sw2d_last_error(None).decode())
    return y


def run_case(folder: str, device: int = 0, n_steps: Optional[int] = None):
    """`sw2dSolver <folder>` without result storage: returns (model, steps taken)."""
    model = SpModel.from_folder(folder, device)
    steps = model.execute() if n_steps is None else model.step(n_steps)
    return model, steps
