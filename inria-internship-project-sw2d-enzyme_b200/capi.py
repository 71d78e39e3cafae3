"""ctypes view of the C ABI in include/sw2d_b200.h and the loader of the CUDA library.

``native_inputs(case)`` turns a :class:`Case` into the C structures (keeping the numpy arrays
alive); ``load_library()`` loads ``libsw2d_b200.so`` built in-tree and fails loudly when it is
missing: there is no CPU fallback for the product path.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .case import BC_TYPES, Case

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsw2d_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_int32_p = ctypes.POINTER(ctypes.c_int32)

SCHEMES = {"godunov": 0, "muscl_evr": 1}
TOPOS = {"discontinuous": 0, "blending": 1}
# map_storage_mode -> enum sw2d_result_mode
RESULT_MODES = {"default": 0, "all": 1, "none": 2}
FRICTIONS = {"none": 0, "chezy": 1, "manning": 2, "strickler": 3}


class Sw2dMesh(ctypes.Structure):
    _fields_ = [("cell_nb", ctypes.c_int64), ("edge_int_nb", ctypes.c_int64), ("edge_bnd_nb", ctypes.c_int64),
                ("cell_area", c_double_p), ("cell_x", c_double_p), ("cell_y", c_double_p),
                ("cell_z_b", c_double_p), ("edge_int_cells", c_int64_p), ("edge_int_length", c_double_p),
                ("edge_int_nx", c_double_p), ("edge_int_ny", c_double_p), ("edge_int_mx", c_double_p),
                ("edge_int_my", c_double_p), ("edge_bnd_cell", c_int64_p), ("edge_bnd_length", c_double_p),
                ("edge_bnd_nx", c_double_p), ("edge_bnd_ny", c_double_p), ("edge_bnd_bc", c_int32_p)]


class Sw2dParams(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int32), ("topo", ctypes.c_int32), ("friction", ctypes.c_int32),
                ("singular_head_loss", ctypes.c_int32), ("negative_depth_detection", ctypes.c_int32),
                ("variant", ctypes.c_int32), ("cfl_max", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("dt_map", ctypes.c_double), ("h_min", ctypes.c_double), ("phi_min", ctypes.c_double),
                ("v_max", ctypes.c_double), ("fr_max", ctypes.c_double), ("t_0", ctypes.c_double),
                ("t_max", ctypes.c_double)]


class Sw2dCellFields(ctypes.Structure):
    _fields_ = [("phi", c_double_p), ("boussinesq", c_double_p), ("friction_1", c_double_p),
                ("friction_2", c_double_p), ("friction_alpha", c_double_p), ("hl_h_sing", c_double_p),
                ("hl_coeff_1", c_double_p), ("hl_coeff_2", c_double_p), ("hl_alpha", c_double_p)]


class Sw2dBcTable(ctypes.Structure):
    _fields_ = [("bc_nb", ctypes.c_int32), ("type", c_int32_p), ("offset", c_int64_p), ("times", c_double_p),
                ("values", c_double_p)]


class Sw2dDipFields(ctypes.Structure):
    _fields_ = [("phi_g_int", c_double_p), ("phi_g_bnd", c_double_p), ("momentum_dissipation", ctypes.c_int32),
                ("mu_1", c_double_p), ("mu_2", c_double_p), ("mu_alpha", c_double_p)]


class Sw2dDdpRecords(ctypes.Structure):
    _fields_ = [("offset", c_int64_p), ("values", c_double_p)]


class Sw2dDdpFields(ctypes.Structure):
    _fields_ = [("cell", Sw2dDdpRecords), ("edge_int", Sw2dDdpRecords), ("edge_bnd", Sw2dDdpRecords),
                ("edge_int_mz", c_double_p), ("edge_bnd_mz", c_double_p), ("n_por_tab_max", ctypes.c_int64),
                ("h_min_ddp", ctypes.c_double), ("chi_phi_max", ctypes.c_double), ("chi_theta_max", ctypes.c_double),
                ("div_corr", ctypes.c_int32), ("ic_columns", ctypes.c_int32), ("n_it_div_max", ctypes.c_int64),
                ("momentum_dissipation", ctypes.c_int32), ("pad", ctypes.c_int32), ("mu_1", c_double_p),
                ("mu_2", c_double_p), ("mu_alpha", c_double_p)]


DIV_CORR = {"none": 0, "limit_flux": 1, "limit_timestep": 2}
DDP_IC_LEVEL_Z, DDP_IC_X_VELOCITY, DDP_IC_Y_VELOCITY = 1, 2, 4


class Sw2dObs(ctypes.Structure):
    _fields_ = [("n_points", ctypes.c_int64), ("cells", c_int64_p), ("w_h", c_double_p), ("w_q", c_double_p),
                ("n_times", ctypes.c_int64), ("steps", c_int64_p), ("h_obs", c_double_p), ("q_obs", c_double_p),
                ("r_obs", c_double_p), ("normalize", ctypes.c_int)]


class Sw2dGradient(ctypes.Structure):
    _fields_ = [("h0", c_double_p), ("q0", c_double_p), ("r0", c_double_p), ("z_b", c_double_p),
                ("friction_1", c_double_p), ("friction_2", c_double_p)]


class Sw2dAssimParams(ctypes.Structure):
    _fields_ = [("phi_transform", ctypes.c_int32), ("lambda_tanh", ctypes.c_double), ("windowed", ctypes.c_int32),
                ("window_duration", ctypes.c_double), ("window_steps", ctypes.c_int64), ("n_windows", ctypes.c_int64),
                ("t_state_assimilation", ctypes.c_double), ("cost_normalize", ctypes.c_int32),
                ("mask_wall_gradient", ctypes.c_int32), ("forced_first_segment", ctypes.c_int64)]


class Sw2dAssimObs(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n_obs", ctypes.c_int32), ("times", c_double_p), ("frames", c_double_p),
                ("h_weight", c_double_p), ("q_weight", c_double_p), ("n_gauges", ctypes.c_int32),
                ("gauge_cells", c_int64_p), ("gauge_weight", c_double_p), ("gauge_h", c_double_p)]


class Sw2dAssimInfo(ctypes.Structure):
    _fields_ = [("J", ctypes.c_double), ("grad_l2", ctypes.c_double), ("grad_max", ctypes.c_double),
                ("grad_argmax", ctypes.c_int64), ("dh_peak", ctypes.c_double), ("n_steps", ctypes.c_int64),
                ("n_segments", ctypes.c_int64), ("first_segment", ctypes.c_int64),
                ("truncation_segment", ctypes.c_int64), ("n_tiles", ctypes.c_int64),
                ("exploded_segment", ctypes.c_int64), ("n_nonfinite", ctypes.c_int64), ("n_masked", ctypes.c_int64)]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(c_double_p)


@dataclass
class NativeInputs:
    mesh: Sw2dMesh
    params: Sw2dParams
    fields: Sw2dCellFields
    bc: Sw2dBcTable
    h0: np.ndarray
    q0: np.ndarray
    r0: np.ndarray
    keep: List[np.ndarray]
    dip: Optional[Sw2dDipFields] = None
    ddp: Optional[Sw2dDdpFields] = None


def params_from_opts(opts) -> Sw2dParams:
    """input.solv keys -> sw2d_params (defaults of swSolverParam.h:144-194)."""
    def f(k, d):
        return float(opts.get(k, d))
    scheme = str(opts.get("num_scheme", "godunov")).lower()
    topo = str(opts.get("topo_discretization", "discontinuous")).lower()
    fric = str(opts.get("model_friction", "none")).lower()
    if scheme not in SCHEMES:
        raise ValueError(f"num_scheme {scheme!r} not implemented")
    if topo not in TOPOS:
        raise ValueError(f"topo_discretization {topo!r} not recognised")
    if fric not in FRICTIONS:
        raise ValueError(f"model_friction {fric!r} not handled")
    model = str(opts.get("model_hyperb", "sp")).lower()
    if model != "ddp" and str(opts.get("div_corr", "none")).lower() != "none":
        raise ValueError("div_corr other than 'none' is outside the SP/DIP path (the reference's SP and DIP "
                         "steps ignore it)")
    return Sw2dParams(
        scheme=SCHEMES[scheme], topo=TOPOS[topo], friction=FRICTIONS[fric],
        singular_head_loss=int(str(opts.get("model_singular_head_loss", "none")).lower() != "none"),
        negative_depth_detection=int(str(opts.get("negative_depth_detection", "none")).lower() == "active"),
        variant=0, cfl_max=f("cfl_max", 1.0), dt_max=f("dt_max", 10.0), dt_map=f("dt_map", 100.0),
        h_min=f("h_min", 1e-5), phi_min=f("phi_min", 1e-16), v_max=f("v_max", 100.0), fr_max=f("fr_max", 100.0),
        t_0=f("t_0", 0.0), t_max=f("t_max", 100.0))


def native_inputs(case: Case) -> NativeInputs:
    m = case.mesh
    keep: List[np.ndarray] = []

    def d(a):
        arr = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(arr)
        return _dp(arr)

    cells = np.ascontiguousarray(m.edge_int_cells, dtype=np.int64).reshape(-1)
    bcell = np.ascontiguousarray(m.edge_bnd_cell, dtype=np.int64)
    series_codes = list(case.bc.codes)
    try:
        bc_index = np.array([series_codes.index(int(c)) for c in m.edge_bnd_code], dtype=np.int32)
    except ValueError as exc:
        raise ValueError("a boundary code of the mesh has no time series") from exc
    keep += [cells, bcell, bc_index]
    mesh = Sw2dMesh(m.cell_nb, m.edge_int_nb, m.edge_bnd_nb, d(m.cell_area), d(m.cell_x), d(m.cell_y),
                    d(m.cell_z_b), cells.ctypes.data_as(c_int64_p), d(m.edge_int_length), d(m.edge_int_nx),
                    d(m.edge_int_ny), d(m.edge_int_mx), d(m.edge_int_my), bcell.ctypes.data_as(c_int64_p),
                    d(m.edge_bnd_length), d(m.edge_bnd_nx), d(m.edge_bnd_ny), bc_index.ctypes.data_as(c_int32_p))
    params = params_from_opts(case.opts)
    null = c_double_p()
    fr = case.friction
    hl = case.head_loss
    fields = Sw2dCellFields(d(case.phi), d(case.boussinesq),
                            d(fr[0]) if fr is not None else null, d(fr[1]) if fr is not None else null,
                            d(fr[2]) if fr is not None else null,
                            d(hl[0]) if hl is not None else null, d(hl[1]) if hl is not None else null,
                            d(hl[2]) if hl is not None else null, d(hl[3]) if hl is not None else null)
    ns = len(series_codes)
    types = np.array([BC_TYPES.get(t, 99) for t in case.bc.types], dtype=np.int32)  # exact, as the reference
    nrec = case.bc.times.shape[0]
    offset = np.arange(ns + 1, dtype=np.int64) * nrec
    times = np.tile(np.asarray(case.bc.times, dtype=np.float64), ns)
    values = np.ascontiguousarray(np.asarray(case.bc.values, dtype=np.float64).reshape(-1))
    keep += [types, offset, times, values]
    bc = Sw2dBcTable(ns, types.ctypes.data_as(c_int32_p), offset.ctypes.data_as(c_int64_p), _dp(times), _dp(values))
    h0 = np.ascontiguousarray(case.h0, dtype=np.float64)
    q0 = np.ascontiguousarray(case.q0, dtype=np.float64)
    r0 = np.ascontiguousarray(case.r0, dtype=np.float64)
    dip = None
    if case.is_dip:
        mu = case.mu
        diss = str(case.opts.get("model_momentum_dissipation", "none")).lower() == "active"
        dip = Sw2dDipFields(d(case.phi_g_int), d(case.phi_g_bnd), 1 if diss else 0,
                            d(mu[0]) if diss else null, d(mu[1]) if diss else null, d(mu[2]) if diss else null)
    ddp = None
    if case.is_ddp:
        ddp = ddp_fields(case, keep)
    return NativeInputs(mesh, params, fields, bc, h0, q0, r0, keep, dip, ddp)


def ddp_fields(case: Case, keep: List[np.ndarray]) -> Sw2dDdpFields:
    """input.solv DDP keys and maps -> sw2d_ddp_fields (defaults of swSolverParam.h:161-181;
    h_min_ddp has no input.solv key in the reference and stays 1e-3)."""
    o = case.opts
    m = case.mesh

    def recs(lr):
        off = np.ascontiguousarray(lr.offset, dtype=np.int64)
        val = np.ascontiguousarray(lr.values, dtype=np.float64)
        keep.extend([off, val])
        return Sw2dDdpRecords(off.ctypes.data_as(c_int64_p), _dp(val))

    def d(a):
        arr = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(arr)
        return _dp(arr)

    div = str(o.get("div_corr", "none")).lower()
    if div not in DIV_CORR:
        raise ValueError(f"div_corr {div!r} not in {sorted(DIV_CORR)}")
    level, xcol, ycol = case.ddp_ic
    cols = (DDP_IC_LEVEL_Z if level == "z" else 0) | (DDP_IC_X_VELOCITY if xcol == "u" else 0) | \
           (DDP_IC_Y_VELOCITY if ycol == "v" else 0)
    diss = str(o.get("model_momentum_dissipation", "none")).lower() == "active"
    null = c_double_p()
    mu = case.mu
    return Sw2dDdpFields(recs(case.ddp_cell), recs(case.ddp_edge_int), recs(case.ddp_edge_bnd), d(m.edge_int_mz),
                         d(m.edge_bnd_mz), int(o.get("n_por_tab_max", 5)), float(o.get("h_min_ddp", 1e-3)),
                         float(o.get("ddp_chi_phi_max", 20.0)), float(o.get("ddp_chi_theta_max", 20.0)),
                         DIV_CORR[div], cols, int(o.get("n_it_div_max", 10)), 1 if diss else 0, 0,
                         d(mu[0]) if diss else null, d(mu[1]) if diss else null, d(mu[2]) if diss else null)


_LIB = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library (fails loudly when it was not built: no CPU fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with __graft_entry__.build() (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    lib.sw2d_create.argtypes = [ctypes.POINTER(Sw2dMesh), ctypes.POINTER(Sw2dParams), ctypes.POINTER(Sw2dCellFields),
                                ctypes.POINTER(Sw2dBcTable), c_double_p, c_double_p, c_double_p, ctypes.c_int,
                                ctypes.POINTER(P)]
    lib.sw2d_create.restype = ctypes.c_int
    lib.sw2d_create_dip.argtypes = [ctypes.POINTER(Sw2dMesh), ctypes.POINTER(Sw2dParams),
                                    ctypes.POINTER(Sw2dCellFields), ctypes.POINTER(Sw2dDipFields),
                                    ctypes.POINTER(Sw2dBcTable), c_double_p, c_double_p, c_double_p, ctypes.c_int,
                                    ctypes.POINTER(P)]
    lib.sw2d_create_dip.restype = ctypes.c_int
    lib.sw2d_create_ddp.argtypes = [ctypes.POINTER(Sw2dMesh), ctypes.POINTER(Sw2dParams),
                                    ctypes.POINTER(Sw2dCellFields), ctypes.POINTER(Sw2dDdpFields),
                                    ctypes.POINTER(Sw2dBcTable), c_double_p, c_double_p, c_double_p, ctypes.c_int,
                                    ctypes.POINTER(P)]
    lib.sw2d_create_ddp.restype = ctypes.c_int
    lib.sw2d_ddp_get_table.argtypes = [P, ctypes.c_int, ctypes.c_int64, c_double_p, c_double_p, c_double_p,
                                       ctypes.c_int64]
    lib.sw2d_ddp_get_table.restype = ctypes.c_int64
    lib.sw2d_load_case.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(P)]
    lib.sw2d_load_case.restype = ctypes.c_int
    lib.sw2d_case_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(P)]
    lib.sw2d_case_read.restype = ctypes.c_int
    lib.sw2d_case_array.argtypes = [P, ctypes.c_char_p, c_double_p, ctypes.c_int64]
    lib.sw2d_case_array.restype = ctypes.c_int64
    lib.sw2d_case_info.argtypes = [P, c_int64_p]
    lib.sw2d_case_info.restype = ctypes.c_int
    lib.sw2d_case_option.argtypes = [P, ctypes.c_char_p]
    lib.sw2d_case_option.restype = ctypes.c_char_p
    lib.sw2d_case_create.argtypes = [P, ctypes.c_int, ctypes.POINTER(P)]
    lib.sw2d_case_create.restype = ctypes.c_int
    lib.sw2d_case_free.argtypes = [P]
    lib.sw2d_case_free.restype = None
    lib.sw2d_case_last_error.argtypes = []
    lib.sw2d_case_last_error.restype = ctypes.c_char_p
    c_float_p = ctypes.POINTER(ctypes.c_float)
    lib.sw2d_mlp_param_count.argtypes = []
    lib.sw2d_mlp_param_count.restype = ctypes.c_int
    lib.sw2d_mlp_create.argtypes = [ctypes.c_int, c_float_p, c_float_p, ctypes.POINTER(P)]
    lib.sw2d_mlp_create.restype = ctypes.c_int
    lib.sw2d_mlp_destroy.argtypes = [P]
    lib.sw2d_mlp_destroy.restype = ctypes.c_int
    lib.sw2d_mlp_last_error.argtypes = [P]
    lib.sw2d_mlp_last_error.restype = ctypes.c_char_p
    lib.sw2d_mlp_get_params.argtypes = [P, c_float_p]
    lib.sw2d_mlp_get_params.restype = ctypes.c_int
    lib.sw2d_mlp_infer.argtypes = [P, c_float_p, ctypes.c_int64, c_float_p, c_float_p]
    lib.sw2d_mlp_infer.restype = ctypes.c_int
    lib.sw2d_mlp_loss_grad.argtypes = [P, c_float_p, c_float_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                                       c_float_p]
    lib.sw2d_mlp_loss_grad.restype = ctypes.c_int
    lib.sw2d_mlp_adam_step.argtypes = [P, ctypes.c_float]
    lib.sw2d_mlp_adam_step.restype = ctypes.c_int
    lib.sw2d_mlp_set_wait_polls.argtypes = [P, ctypes.c_int64]
    lib.sw2d_mlp_set_wait_polls.restype = ctypes.c_int
    lib.sw2d_set_closure.argtypes = [P, P, c_float_p, c_float_p, ctypes.c_float]
    lib.sw2d_set_closure.restype = ctypes.c_int
    lib.sw2d_map_porosity.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int, P, P, P]
    lib.sw2d_map_porosity.restype = ctypes.c_int
    lib.sw2d_map_porosity_raster.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int, P, P, P]
    lib.sw2d_map_porosity_raster.restype = ctypes.c_int
    lib.sw2d_map_last_error.argtypes = []
    lib.sw2d_map_last_error.restype = ctypes.c_char_p
    lib.sw2d_result_header.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double]
    lib.sw2d_result_header.restype = ctypes.c_int
    lib.sw2d_result_open.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
    lib.sw2d_result_open.restype = ctypes.c_int
    lib.sw2d_result_close.argtypes = [P]
    lib.sw2d_result_close.restype = ctypes.c_int
    lib.sw2d_closure_record.argtypes = [P, c_float_p, ctypes.c_int64]
    lib.sw2d_closure_record.restype = ctypes.c_int64
    lib.sw2d_set_t_max.argtypes = [P, ctypes.c_double]
    lib.sw2d_set_t_max.restype = ctypes.c_int
    lib.sw2d_step_n.argtypes = [P, ctypes.c_int64, c_int64_p]
    lib.sw2d_step_n.restype = ctypes.c_int
    lib.sw2d_save_point.argtypes = [P]
    lib.sw2d_save_point.restype = ctypes.c_int
    lib.sw2d_restore_point.argtypes = [P]
    lib.sw2d_restore_point.restype = ctypes.c_int
    lib.sw2d_prepare_steps.argtypes = [P]
    lib.sw2d_prepare_steps.restype = ctypes.c_int
    lib.sw2d_execute.argtypes = [P, c_int64_p]
    lib.sw2d_execute.restype = ctypes.c_int
    for name in ("sw2d_get_state", "sw2d_set_state", "sw2d_get_state_device", "sw2d_set_state_device"):
        fn = getattr(lib, name)
        fn.argtypes = [P, P, P, P]
        fn.restype = ctypes.c_int
    lib.sw2d_get_time.argtypes = [P, c_double_p, c_double_p]
    lib.sw2d_get_time.restype = ctypes.c_int
    lib.sw2d_set_time.argtypes = [P, ctypes.c_double, ctypes.c_double]
    lib.sw2d_set_time.restype = ctypes.c_int
    lib.sw2d_get_array.argtypes = [P, ctypes.c_char_p, c_double_p, ctypes.c_int64]
    lib.sw2d_get_array.restype = ctypes.c_int64
    lib.sw2d_get_array_noalloc.argtypes = [P, ctypes.c_char_p, c_double_p, ctypes.c_int64]
    lib.sw2d_get_array_noalloc.restype = ctypes.c_int64
    lib.sw2d_get_cell_permutation.argtypes = [P, c_int64_p]
    lib.sw2d_get_cell_permutation.restype = ctypes.c_int
    lib.sw2d_get_stream.argtypes = [P]
    lib.sw2d_get_stream.restype = P
    lib.sw2d_kernels_per_step.argtypes = [P]
    lib.sw2d_kernels_per_step.restype = ctypes.c_int
    lib.sw2d_destroy.argtypes = [P]
    lib.sw2d_destroy.restype = ctypes.c_int
    lib.sw2d_last_error.argtypes = [P]
    lib.sw2d_last_error.restype = ctypes.c_char_p
    lib.sw2d_phase_times.argtypes = [P, ctypes.c_int64, c_double_p, ctypes.c_int]
    lib.sw2d_phase_times.restype = ctypes.c_int
    lib.sw2d_phase_name.argtypes = [ctypes.c_int]
    lib.sw2d_phase_name.restype = ctypes.c_char_p
    lib.sw2d_phase_label.argtypes = [P, ctypes.c_int]
    lib.sw2d_phase_label.restype = ctypes.c_char_p
    lib.sw2d_get_option.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
    lib.sw2d_get_option.restype = ctypes.c_int
    lib.sw2d_set_option.argtypes = [P, ctypes.c_char_p, ctypes.c_int64]
    lib.sw2d_set_option.restype = ctypes.c_int
    lib.sw2d_eval_math.argtypes = [ctypes.c_int, ctypes.c_int, c_double_p, c_double_p, ctypes.c_int64]
    lib.sw2d_eval_math.restype = ctypes.c_int
    lib.sw2d_autotune.argtypes = [P, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    lib.sw2d_autotune.restype = ctypes.c_int
    lib.sw2d_autotune_step.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_char_p,
                                       ctypes.c_int]
    lib.sw2d_autotune_step.restype = ctypes.c_int
    lib.sw2d_get_launch_config.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.sw2d_get_launch_config.restype = ctypes.c_int
    lib.sw2d_set_launch_config.argtypes = [P, ctypes.c_int, ctypes.c_int]
    lib.sw2d_set_launch_config.restype = ctypes.c_int
    lib.sw2d_abi_version.argtypes = []
    lib.sw2d_abi_version.restype = ctypes.c_int
    # adjoint
    lib.sw2d_record.argtypes = [P, ctypes.c_int64, ctypes.c_int64, c_int64_p]
    lib.sw2d_record.restype = ctypes.c_int
    lib.sw2d_rerecord.argtypes = [P, c_int64_p]
    lib.sw2d_rerecord.restype = ctypes.c_int
    lib.sw2d_trajectory_info.argtypes = [P, c_int64_p, c_int64_p, c_double_p, c_double_p]
    lib.sw2d_trajectory_info.restype = ctypes.c_int
    lib.sw2d_get_trajectory_dt.argtypes = [P, c_double_p, ctypes.c_int64]
    lib.sw2d_get_trajectory_dt.restype = ctypes.c_int
    lib.sw2d_set_trajectory_start.argtypes = [P, P, P, P]
    lib.sw2d_set_trajectory_start.restype = ctypes.c_int
    lib.sw2d_set_param.argtypes = [P, ctypes.c_char_p, P]
    lib.sw2d_set_param.restype = ctypes.c_int
    lib.sw2d_get_param.argtypes = [P, ctypes.c_char_p, P]
    lib.sw2d_get_param.restype = ctypes.c_int
    lib.sw2d_set_observations.argtypes = [P, ctypes.POINTER(Sw2dObs)]
    lib.sw2d_set_observations.restype = ctypes.c_int
    lib.sw2d_replay_cost.argtypes = [P, c_double_p]
    lib.sw2d_replay_cost.restype = ctypes.c_int
    lib.sw2d_replay_sample.argtypes = [P, ctypes.c_int64, c_int64_p, ctypes.c_int64, c_int64_p, P, P, P]
    lib.sw2d_replay_sample.restype = ctypes.c_int
    lib.sw2d_adjoint.argtypes = [P, c_double_p, ctypes.POINTER(Sw2dGradient)]
    lib.sw2d_adjoint.restype = ctypes.c_int
    lib.sw2d_adjoint_nonfinite.argtypes = [P, c_int64_p]
    lib.sw2d_adjoint_nonfinite.restype = ctypes.c_int
    lib.sw2d_adjoint_trace.argtypes = [P, c_int64_p, c_double_p, c_double_p, c_int64_p, ctypes.c_int64]
    lib.sw2d_adjoint_trace.restype = ctypes.c_int
    # ensembles
    lib.sw2d_batch_create.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.POINTER(P)]
    lib.sw2d_batch_create.restype = ctypes.c_int
    lib.sw2d_batch_step_n.argtypes = [P, ctypes.c_int64, c_int64_p]
    lib.sw2d_batch_step_n.restype = ctypes.c_int
    lib.sw2d_batch_adjoint.argtypes = [P, c_double_p, ctypes.POINTER(Sw2dGradient), ctypes.c_int]
    lib.sw2d_batch_adjoint.restype = ctypes.c_int
    lib.sw2d_batch_configure.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.sw2d_batch_configure.restype = ctypes.c_int
    c_int_p = ctypes.POINTER(ctypes.c_int)
    lib.sw2d_batch_get_config.argtypes = [P, c_int_p, c_int_p, c_int_p, c_int_p]
    lib.sw2d_batch_get_config.restype = ctypes.c_int
    lib.sw2d_batch_autotune.argtypes = [P, ctypes.c_int, c_int_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    lib.sw2d_batch_autotune.restype = ctypes.c_int
    lib.sw2d_batch_set_wait_polls.argtypes = [P, ctypes.c_int64]
    lib.sw2d_batch_set_wait_polls.restype = ctypes.c_int
    lib.sw2d_batch_stream.argtypes = [P]
    lib.sw2d_batch_stream.restype = ctypes.c_void_p
    lib.sw2d_batch_size.argtypes = [P]
    lib.sw2d_batch_size.restype = ctypes.c_int
    lib.sw2d_batch_destroy.argtypes = [P]
    lib.sw2d_batch_destroy.restype = ctypes.c_int
    lib.sw2d_batch_last_error.argtypes = [P]
    lib.sw2d_batch_last_error.restype = ctypes.c_char_p
    # porosity assimilation (the differentiated step)
    lib.sw2d_assim_configure.argtypes = [P, ctypes.POINTER(Sw2dAssimParams)]
    lib.sw2d_assim_configure.restype = ctypes.c_int
    lib.sw2d_assim_set_observations.argtypes = [P, ctypes.POINTER(Sw2dAssimObs)]
    lib.sw2d_assim_set_observations.restype = ctypes.c_int
    lib.sw2d_assim_record.argtypes = [P, c_double_p, ctypes.c_int64, c_int64_p, c_int64_p]
    lib.sw2d_assim_record.restype = ctypes.c_int
    lib.sw2d_assim_replay_cost.argtypes = [P, c_double_p, c_double_p]
    lib.sw2d_assim_replay_cost.restype = ctypes.c_int
    lib.sw2d_assim_gradient.argtypes = [P, c_double_p, ctypes.c_int64, c_double_p, c_double_p, c_double_p, c_double_p,
                                        ctypes.POINTER(Sw2dAssimInfo)]
    lib.sw2d_assim_gradient.restype = ctypes.c_int
    lib.sw2d_assim_segments.argtypes = [P, c_double_p, c_int64_p, ctypes.c_int64]
    lib.sw2d_assim_segments.restype = ctypes.c_int
    lib.sw2d_assim_steps.argtypes = [P, c_double_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_int64]
    lib.sw2d_assim_steps.restype = ctypes.c_int
    lib.sw2d_assim_set_start.argtypes = [P, c_double_p, c_double_p, c_double_p]
    lib.sw2d_assim_set_start.restype = ctypes.c_int
    lib.sw2d_assim_checkpoint.argtypes = [P, ctypes.c_int64, c_double_p, c_double_p, c_double_p]
    lib.sw2d_assim_checkpoint.restype = ctypes.c_int
    lib.sw2d_assim_trigger_states.argtypes = [P, c_double_p, c_double_p, c_double_p, c_double_p, ctypes.c_int64,
                                              ctypes.POINTER(ctypes.c_int64)]
    lib.sw2d_assim_trigger_states.restype = ctypes.c_int
    _LIB = lib
    return lib


# every symbol include/sw2d_b200.h declares (checked by the CPU test suite)
EXPORTED = ["sw2d_create", "sw2d_create_dip", "sw2d_create_ddp", "sw2d_ddp_get_table", "sw2d_load_case",
            "sw2d_case_read", "sw2d_case_array", "sw2d_case_info", "sw2d_case_option", "sw2d_case_create",
            "sw2d_case_free", "sw2d_case_last_error", "sw2d_mlp_param_count", "sw2d_mlp_create",
            "sw2d_mlp_destroy", "sw2d_mlp_last_error", "sw2d_mlp_get_params", "sw2d_mlp_infer",
            "sw2d_mlp_loss_grad", "sw2d_mlp_adam_step", "sw2d_mlp_set_wait_polls", "sw2d_set_closure", "sw2d_closure_record", "sw2d_set_t_max",
            "sw2d_result_header", "sw2d_result_open", "sw2d_result_close", "sw2d_map_porosity", "sw2d_map_porosity_raster",
            "sw2d_map_last_error", "sw2d_step_n", "sw2d_prepare_steps", "sw2d_save_point", "sw2d_restore_point", "sw2d_execute", "sw2d_get_state", "sw2d_set_state",
            "sw2d_get_state_device", "sw2d_set_state_device", "sw2d_get_time", "sw2d_set_time",
            "sw2d_get_array", "sw2d_get_cell_permutation", "sw2d_get_stream", "sw2d_kernels_per_step",
            "sw2d_destroy", "sw2d_last_error", "sw2d_abi_version", "sw2d_phase_times", "sw2d_phase_name", "sw2d_phase_label", "sw2d_get_option",
            "sw2d_set_option", "sw2d_eval_math", "sw2d_autotune", "sw2d_autotune_step", "sw2d_get_launch_config",
            "sw2d_set_launch_config", "sw2d_get_array_noalloc", "sw2d_record", "sw2d_rerecord", "sw2d_trajectory_info",
            "sw2d_get_trajectory_dt", "sw2d_set_trajectory_start", "sw2d_set_param", "sw2d_get_param",
            "sw2d_set_observations", "sw2d_replay_cost", "sw2d_replay_sample", "sw2d_adjoint", "sw2d_adjoint_nonfinite", "sw2d_adjoint_trace",
            "sw2d_batch_create", "sw2d_batch_step_n", "sw2d_batch_adjoint", "sw2d_batch_size",
            "sw2d_batch_configure", "sw2d_batch_get_config", "sw2d_batch_autotune", "sw2d_batch_set_wait_polls",
            "sw2d_batch_stream",
            "sw2d_batch_destroy", "sw2d_batch_last_error", "sw2d_assim_configure", "sw2d_assim_set_observations",
            "sw2d_assim_record", "sw2d_assim_replay_cost", "sw2d_assim_gradient", "sw2d_assim_segments",
            "sw2d_assim_steps", "sw2d_assim_checkpoint", "sw2d_assim_set_start", "sw2d_assim_trigger_states"]


class CaseFolder:
    """A case folder read by the library's own loader (sw2d_case_read): the tables and fields as
    the C ABI will hand them to the model, for inspection; ``create(device)`` builds the model."""

    def __init__(self, folder: str):
        self.lib = load_library()
        self.ptr = ctypes.c_void_p()
        st = self.lib.sw2d_case_read(folder.encode(), ctypes.byref(self.ptr))
        if st != 0:
            raise ValueError(f"sw2d_case_read: {self.lib.sw2d_case_last_error().decode()}")
        info = np.zeros(5, dtype=np.int64)
        self.lib.sw2d_case_info(self.ptr, info.ctypes.data_as(c_int64_p))
        self.cell_nb, self.edge_int_nb, self.edge_bnd_nb, self.model, self.ic_columns = (int(v) for v in info)

    def array(self, name: str) -> np.ndarray:
        cap = 8 * max(self.cell_nb, self.edge_int_nb, self.edge_bnd_nb, 1) + 1024
        while True:
            out = np.empty(cap)
            k = self.lib.sw2d_case_array(self.ptr, name.encode(), _dp(out), cap)
            if k >= 0:
                return out[:k].copy()
            if cap > 1 << 31:
                raise KeyError(name)
            cap *= 4

    def option(self, key: str) -> Optional[str]:
        v = self.lib.sw2d_case_option(self.ptr, key.encode())
        return None if v is None else v.decode()

    def close(self) -> None:
        if self.ptr:
            self.lib.sw2d_case_free(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
