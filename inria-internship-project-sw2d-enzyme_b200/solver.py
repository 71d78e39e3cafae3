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
import os
from typing import Optional, Tuple

import numpy as np

from . import capi
from .case import Case, read_case, read_solv


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(capi.c_double_p)


class Sw2dError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"sw2d error {code}: {message}")
        self.code = code
        self.message = message


class SpModel:
    """SW2D porosity model running on one GPU: single porosity, dual integral porosity when the
    case says model_hyperb dip, depth-dependent porosity when it says ddp (then ``state()`` is
    the model's own (thetaW, thetaW u, thetaW v), and ``array("water_depth")`` etc. give the map
    outputs)."""

    def __init__(self, case: Case, device: int = 0):
        self.lib = capi.load_library()
        self.case = case
        self.device = int(device)
        self.n = case.mesh.cell_nb
        self.ni = case.mesh.edge_int_nb
        self.nb = case.mesh.edge_bnd_nb
        self._in = capi.native_inputs(case)
        i = self._in
        handle = ctypes.c_void_p()
        if i.ddp is not None:  # model_hyperb ddp: swDdp (h0/q0/r0 are the initial-condition columns)
            st = self.lib.sw2d_create_ddp(ctypes.byref(i.mesh), ctypes.byref(i.params), ctypes.byref(i.fields),
                                          ctypes.byref(i.ddp), ctypes.byref(i.bc), capi._dp(i.h0), capi._dp(i.q0),
                                          capi._dp(i.r0), int(device), ctypes.byref(handle))
        elif i.dip is not None:  # model_hyperb dip: swDip
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
        if str(case.opts.get("model_hyperb", "sp")).lower() not in ("sp", "dip", "ddp"):
            raise Sw2dError(-8, f"model_hyperb {case.opts.get('model_hyperb')!r}: only 'sp', 'dip' and 'ddp' are "
                                "implemented")
        return cls(case, device)

    @classmethod
    def load(cls, folder: str, device: int = 0, results: bool = False) -> "SpModel":
        """The model a case folder names, read and created by the library itself
        (sw2d_load_case: the C++ readers of input.solv, geometry.sw2d and the maps).  With
        results=True and output_format bin or all, output/ResultHydro.bin is opened with the
        folder's store_flag (the reference's map_storage_mode), as its init does."""
        self = cls.__new__(cls)
        self.lib = capi.load_library()
        self.case = None
        cf = capi.CaseFolder(folder)
        self.n, self.ni, self.nb = cf.cell_nb, cf.edge_int_nb, cf.edge_bnd_nb
        handle = ctypes.c_void_p()
        st = self.lib.sw2d_case_create(cf.ptr, int(device), ctypes.byref(handle))
        cf.close()
        if st != 0:
            msg = self.lib.sw2d_last_error(None).decode() or self.lib.sw2d_case_last_error().decode()
            raise Sw2dError(st, msg)
        self.handle = handle
        if results:
            opts = read_solv(os.path.join(folder, "input", "input.solv"))
            if str(opts.get("output_format", "all")).lower() in ("bin", "all"):
                out = os.path.join(folder, "output")
                os.makedirs(out, exist_ok=True)
                self.result_open(os.path.join(out, "ResultHydro.bin"), os.path.join(folder, "input", "geometry.sw2d"),
                                 str(opts.get("store_flag", "default")).lower())
        return self

    def result_open(self, path: str, geometry_path: str, mode: str = "default") -> None:
        """Creates the binary map file (ResultHydro.bin layout) and attaches it: execute() then
        appends the run's maps (first, every storage time, last)."""
        if mode not in capi.RESULT_MODES:
            raise ValueError(f"map_storage_mode {mode!r}")
        self._check(self.lib.sw2d_result_open(self.handle, path.encode(), geometry_path.encode(),
                                              capi.RESULT_MODES[mode]))

    def result_close(self) -> None:
        self._check(self.lib.sw2d_result_close(self.handle))

    def _check(self, st: int) -> None:
        if st != 0:
            raise Sw2dError(st, self.lib.sw2d_last_error(self.handle).decode())

    def step(self, n: int) -> int:
        done = ctypes.c_int64(0)
        self._check(self.lib.sw2d_step_n(self.handle, int(n), ctypes.byref(done)))
        return int(done.value)

    def save_point(self) -> None:
        """Saves the run's point on the device (state, balance slots, time); restore_point
        returns to it with the same bits as from the saved point."""
        self._check(self.lib.sw2d_save_point(self.handle))

    def restore_point(self) -> None:
        self._check(self.lib.sw2d_restore_point(self.handle))

    def prepare(self) -> None:
        """Captures the step graph that ``step`` launches (no step taken), so that a timed run
        does not include the capture."""
        self._check(self.lib.sw2d_prepare_steps(self.handle))

    def execute(self) -> int:
        done = ctypes.c_int64(0)
        self._check(self.lib.sw2d_execute(self.handle, ctypes.byref(done)))
        return int(done.value)

    def ddp_table(self, which: str, record: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Tabulated porosity law (z, phi, theta) of a DDP cell ("cell"), internal edge ("edge_int")
        or boundary edge ("edge_bnd"), as swDdp keeps it (cell_z_tab / phiW_tab / thetaW_tab ...)."""
        k = {"cell": 0, "edge_int": 1, "edge_bnd": 2}[which]
        n = self.lib.sw2d_ddp_get_table(self.handle, k, int(record), None, None, None, 0)
        if n < 0:
            self._check(int(n))
        z, phi, theta = np.empty(n), np.empty(n), np.empty(n)
        self.lib.sw2d_ddp_get_table(self.handle, k, int(record), _p(z), _p(phi), _p(theta), n)
        return z, phi, theta

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

    def set_t_max(self, t_max: float) -> None:
        """Moves the run's end time (the time step is clipped to it)."""
        self._check(self.lib.sw2d_set_t_max(self.handle, float(t_max)))

    def set_closure(self, net, hull_lo=None, hull_hi=None, scale: float = 1.0) -> None:
        """Attaches a closure.MLP (None detaches) with its training hull [lo, hi] per feature; the
        network's correction is applied times `scale`."""
        fp = ctypes.POINTER(ctypes.c_float)
        if net is None:
            self._check(self.lib.sw2d_set_closure(self.handle, None, None, None, 1.0))
            self._closure = None
            return
        lo = np.ascontiguousarray(hull_lo, dtype=np.float32)
        hi = np.ascontiguousarray(hull_hi, dtype=np.float32)
        self._check(self.lib.sw2d_set_closure(self.handle, net.h, lo.ctypes.data_as(fp), hi.ctypes.data_as(fp),
                                              float(scale)))
        self._closure = net  # keep the network alive while attached

    def closure_record(self) -> np.ndarray:
        """[n x 12] float32: the ten closure features and the network's two outputs of every cell
        in the last step taken with option "closure_record" on (caller's cell order)."""
        out = np.empty((self.n, 12), dtype=np.float32)
        k = self.lib.sw2d_closure_record(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), out.size)
        if k < 0:
            self._check(int(k))
        return out

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
        return {self.lib.sw2d_phase_label(self.handle, i).decode(): float(ms[i]) for i in range(k)}

    def get_option(self, name: str) -> int:
        v = ctypes.c_int64(0)
        self._check(self.lib.sw2d_get_option(self.handle, name.encode(), ctypes.byref(v)))
        return int(v.value)

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

    def adjoint_trace(self) -> dict:
        """With the option "adjoint_trace": the last gradient's state adjoint after each reverse
        step (trajectory order): non-finite entries, largest finite |adjoint| of h and of q/r, and
        the first cell holding a non-finite entry (-1: none)."""
        n = int(self.lib.sw2d_adjoint_trace(self.handle, None, None, None, None, 0))
        if n < 0:
            self._check(n)
        nf, fc = np.zeros(n, np.int64), np.zeros(n, np.int64)
        mh, mq = np.zeros(n), np.zeros(n)
        self._check(min(0, self.lib.sw2d_adjoint_trace(self.handle, nf.ctypes.data_as(capi.c_int64_p), _p(mh), _p(mq),
                                                       fc.ctypes.data_as(capi.c_int64_p), n)))
        return {"nonfinite": nf, "max_h": mh, "max_qr": mq, "first_cell": fc}

    # ---- porosity assimilation with the reference's differentiated step (sw2d_assim_*) ----
    PHI_TRANSFORMS = {"none": 0, "clamp": 1, "tanh": 2, "normalize": 3}

    def assim_configure(self, phi_transform: str = "none", lambda_tanh: float = 1.0, windowed: bool = False,
                        window_duration: float = -1.0, window_steps: int = -1, n_windows: int = 1,
                        t_state_assimilation: float = 0.0, cost_normalize: bool = False,
                        mask_wall_gradient: bool = False, forced_first_segment: int = -1) -> None:
        """The assimilation keys of input.solv (assim/assimConfig.h); the trajectory starts from the
        model's state and time at the first call."""
        p = capi.Sw2dAssimParams(self.PHI_TRANSFORMS[phi_transform.lower()], float(lambda_tanh), int(bool(windowed)),
                                 float(window_duration), int(window_steps), int(n_windows),
                                 float(t_state_assimilation), int(bool(cost_normalize)), int(bool(mask_wall_gradient)),
                                 int(forced_first_segment))
        self._check(self.lib.sw2d_assim_configure(self.handle, ctypes.byref(p)))

    def assim_set_frames(self, times, frames, h_weight=None, q_weight=None) -> None:
        """Full-field observations: frames[k] = (h, qx, qy) of every cell at times[k]."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        f = np.ascontiguousarray(frames, dtype=np.float64).reshape(len(t), 3, self.n)
        wh = None if h_weight is None else np.ascontiguousarray(h_weight, dtype=np.float64)
        wq = None if q_weight is None else np.ascontiguousarray(q_weight, dtype=np.float64)
        o = capi.Sw2dAssimObs(0, len(t), _p(t), _p(f), _p(wh), _p(wq), 0, None, None, None)
        self._check(self.lib.sw2d_assim_set_observations(self.handle, ctypes.byref(o)))

    def assim_set_gauges(self, times, cells, weights, values) -> None:
        """Gauge observations: values[k][g] is the depth at cells[g] at times[k]."""
        t = np.ascontiguousarray(times, dtype=np.float64)
        c = np.ascontiguousarray(cells, dtype=np.int64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(len(t), len(c))
        o = capi.Sw2dAssimObs(1, len(t), _p(t), None, None, None, len(c), c.ctypes.data_as(capi.c_int64_p), _p(w), _p(v))
        self._check(self.lib.sw2d_assim_set_observations(self.handle, ctypes.byref(o)))

    def assim_record(self, m, stride: int = 30) -> Tuple[int, int]:
        """build_checkpoint_records at control m: (steps, segments)."""
        mm = np.ascontiguousarray(m, dtype=np.float64)
        ns, nk = ctypes.c_int64(0), ctypes.c_int64(0)
        self._check(self.lib.sw2d_assim_record(self.handle, _p(mm), int(stride), ctypes.byref(ns), ctypes.byref(nk)))
        return ns.value, nk.value

    def assim_replay_cost(self, m) -> float:
        """replay_trajectory_cost at control m on the recorded trajectory."""
        mm = np.ascontiguousarray(m, dtype=np.float64)
        J = ctypes.c_double(0.0)
        self._check(self.lib.sw2d_assim_replay_cost(self.handle, _p(mm), ctypes.byref(J)))
        return J.value

    def assim_gradient(self, m, stride: int = 30, extras: bool = False):
        """get_spatial_gradient_checkpointed at control m: (dJ/dm, info); with extras also
        {"k1", "k2", "h0", "q0", "r0"} (Strickler coefficients, state at the window start)."""
        mm = np.ascontiguousarray(m, dtype=np.float64)
        g = np.zeros(self.n)
        k1 = np.zeros(self.n) if extras else None
        k2 = np.zeros(self.n) if extras else None
        s0 = np.zeros(3 * self.n) if extras else None
        inf = capi.Sw2dAssimInfo()
        self._check(self.lib.sw2d_assim_gradient(self.handle, _p(mm), int(stride), _p(g), _p(k1), _p(k2), _p(s0),
                                                 ctypes.byref(inf)))
        info = {name: getattr(inf, name) for name, _ in capi.Sw2dAssimInfo._fields_}
        if not extras:
            return g, info
        n = self.n
        return g, info, {"k1": k1, "k2": k2, "h0": s0[:n], "q0": s0[n:2 * n], "r0": s0[2 * n:]}

    def assim_segments(self) -> Tuple[np.ndarray, np.ndarray]:
        """(t_start, n_steps) of each recorded segment."""
        cap = 1
        while True:
            t = np.zeros(cap)
            n = np.zeros(cap, dtype=np.int64)
            st = self.lib.sw2d_assim_segments(self.handle, _p(t), n.ctypes.data_as(capi.c_int64_p), cap)
            if st == 0:
                k = int(np.count_nonzero(n))
                return t[:k], n[:k]
            if cap > 1 << 26:
                self._check(st)
            cap *= 4

    def assim_steps(self) -> Tuple[np.ndarray, np.ndarray]:
        """(dt, observation trigger) of each recorded step."""
        _, n = self.assim_segments()
        total = int(n.sum())
        dt = np.zeros(max(1, total))
        tr = np.zeros(max(1, total), dtype=np.int32)
        self._check(self.lib.sw2d_assim_steps(self.handle, _p(dt), tr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                              max(1, total)))
        return dt[:total], tr[:total]

    def assim_set_start(self, h, q, r) -> None:
        h, q, r = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, q, r))
        self._check(self.lib.sw2d_assim_set_start(self.handle, _p(h), _p(q), _p(r)))

    def assim_trigger_states(self, m, n_obs: int):
        """The recorded trajectory replayed at control m: the state after each step that lands on
        an observation, as arrays [n_obs, n_cells] (h, qx, qy), and the number of observations
        landed on."""
        mm = np.ascontiguousarray(m, dtype=np.float64)
        h, q, r = (np.full((n_obs, self.n), np.nan) for _ in range(3))
        k = ctypes.c_int64(0)
        self._check(self.lib.sw2d_assim_trigger_states(self.handle, _p(mm), _p(h), _p(q), _p(r), int(n_obs),
                                                       ctypes.byref(k)))
        return h, q, r, int(k.value)

    def assim_checkpoint(self, k: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        h, q, r = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self._check(self.lib.sw2d_assim_checkpoint(self.handle, int(k), _p(h), _p(q), _p(r)))
        return h, q, r

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
