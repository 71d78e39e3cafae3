"""Friction assimilation driven by the GPU adjoint: the minimisation front-end of the
reference (``swSpE::run_minimization`` and ``PorosityProblem``, assim/swSpE_minimize.cpp) with
the per-cell friction coefficient as the control.

The reference fits per-cell porosity; here the control is the coefficient of both friction
directions (isotropic: Manning n for the Manning law, Strickler K, Chezy C).  The problem has
the reference's structure (PorosityProblem::func / grad, assim/swSpE_minimize.cpp:398-511):

    f(theta) = J_data + 0.5 a_reg sum_free (k - k_b)^2 + a_l1 sum_free |k - k_b|
                      + 0.5 a_sp sum_internal edges (k_L - k_R)^2 + 0.5 a_ref sum (k - k_ref)^2

with k = T(m) on the free cells (control transform, assim/swSpE.h:59-107: none, clamp, tanh)
and the optimisation variable theta = m per free cell, or per zone of free cells sharing the
same background value (zonation).  J_data is the replayed misfit on the recorded trajectory
(sw2d_replay_cost); its gradient comes from sw2d_adjoint, and the penalties' gradients are
analytic.  As in the reference, every gradient evaluation records the trajectory again at the
current control (the dry run) and the line searches in between replay that recording.

Algorithms (minimize_algo): "lbfgsb" (L-BFGS-B with the box of the transform; the reference
uses LBFGSpp's, here scipy's) and "gd" (projected gradient descent with Armijo backtracking,
the reference's "gd" branch, assim/swSpE_minimize.cpp:749-840).  Each gradient evaluation
appends a row to ``descent_log.csv`` with the reference's columns (the porosity columns carry
the friction control; see DESCENT_COLUMNS) and writes the control map
``friction_iter/friction_iter_XXXX.txt`` in the map-file format.
"""
from __future__ import annotations

import math
import os
import shutil
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from .case import write_map

DESCENT_COLUMNS = ("iter,J_total,J_data,ridge,rel_init_pct,rel_prev_pct,gradJm_L2,gradJm_Linf,gradJm_argmax,"
                   "gradJphys_L2,gradJphys_max,gradJphys_argmax,dh_peak,phi_min,phi_max,phi_mean,n_phi_lt_0p5,"
                   "n_phi_lt_0p05,n_phi_upper_clamp,adam_step,sse_phi_ref")


@dataclass
class ControlTransform:
    """k = T(m) (phi_correct / dphi_dm / m_from_phi of assim/swSpE.h:59-107, with the box
    [lo, hi] of the friction coefficient in place of porosity's [0, 1.05] and (0, 1))."""
    mode: str = "none"
    lo: float = 0.0
    hi: float = math.inf
    lam: float = 1.0

    def __post_init__(self):
        if self.mode not in ("none", "clamp", "tanh"):
            raise ValueError(f"unknown transform {self.mode!r}")
        if self.mode == "tanh" and not math.isfinite(self.hi):
            raise ValueError("the tanh transform needs a finite upper bound")

    def forward(self, m):
        m = np.asarray(m, dtype=np.float64)
        if self.mode == "clamp":
            return np.clip(m, self.lo, self.hi)
        if self.mode == "tanh":
            return self.lo + (self.hi - self.lo) / (1.0 + np.exp(-self.lam * m))
        return m.copy()

    def derivative(self, m):
        m = np.asarray(m, dtype=np.float64)
        if self.mode == "clamp":
            return np.where((m < self.lo) | (m > self.hi), 0.0, 1.0)
        if self.mode == "tanh":
            s = 1.0 / (1.0 + np.exp(-self.lam * m))
            return (self.hi - self.lo) * self.lam * s * (1.0 - s)
        return np.ones_like(m)

    def inverse(self, k):
        k = np.asarray(k, dtype=np.float64)
        if self.mode == "tanh":
            eps = 1e-2
            p = np.clip((k - self.lo) / (self.hi - self.lo), eps, 1.0 - eps)
            return np.log(p / (1.0 - p)) / self.lam
        if self.mode == "clamp":
            return np.clip(k, self.lo, self.hi)
        return k.copy()

    def bounds(self):
        """Box of the optimisation variable (L-BFGS-B), or None."""
        if self.mode in ("none", "clamp"):
            lo = self.lo if math.isfinite(self.lo) else None
            hi = self.hi if math.isfinite(self.hi) else None
            return (lo, hi)
        return None


@dataclass
class FrictionProblem:
    """f(theta) and its gradient over the recorded trajectory of `model` (an SpModel with a
    trajectory and observations)."""
    model: object
    k_b: np.ndarray                         # background (first guess) per cell
    transform: ControlTransform = field(default_factory=ControlTransform)
    free: Optional[np.ndarray] = None       # free cells (default: all)
    zonation: bool = False                  # one parameter per set of free cells with equal k_b
    alpha_reg: float = 0.0
    alpha_l1: float = 0.0
    alpha_spatial: float = 0.0
    alpha_ref: float = 0.0
    k_ref: Optional[np.ndarray] = None      # truth map, for the sse column and the a_ref term
    rerecord: bool = True                   # record the trajectory again at each gradient
    descent_dir: Optional[str] = None

    def __post_init__(self):
        n = self.model.n
        self.k_b = np.asarray(self.k_b, dtype=np.float64).copy()
        self.free = np.arange(n) if self.free is None else np.asarray(self.free, dtype=np.int64)
        if self.zonation:
            vals, self.zone_of_free = np.unique(self.k_b[self.free], return_inverse=True)
            self.zone_value = vals
        mesh = self.model.case.mesh
        self._L = mesh.edge_int_cells[:, 0].astype(np.int64)
        self._R = mesh.edge_int_cells[:, 1].astype(np.int64)
        self.grad_calls = 0
        self.J_init = None
        self.J_prev = None
        self._csv = None
        if self.descent_dir:
            shutil.rmtree(self.descent_dir, ignore_errors=True)
            os.makedirs(os.path.join(self.descent_dir, "friction_iter"), exist_ok=True)

    # ---- parameterisation
    def size(self) -> int:
        return len(self.zone_value) if self.zonation else len(self.free)

    def theta_start(self) -> np.ndarray:
        v = self.zone_value if self.zonation else self.k_b[self.free]
        return self.transform.inverse(v)

    def _m_free(self, theta):
        theta = np.asarray(theta, dtype=np.float64)
        return theta[self.zone_of_free] if self.zonation else theta

    def control(self, theta) -> np.ndarray:
        """Physical friction map for theta (fixed cells keep k_b)."""
        k = self.k_b.copy()
        k[self.free] = self.transform.forward(self._m_free(theta))
        return k

    def _apply(self, theta) -> np.ndarray:
        k = self.control(theta)
        self.model.set_param("friction", k)
        return k

    # ---- penalties
    def _penalties(self, k):
        d = k[self.free] - self.k_b[self.free]
        ridge = 0.5 * self.alpha_reg * float(np.dot(d, d))
        l1 = self.alpha_l1 * float(np.sum(np.abs(d)))
        sp = 0.0
        if self.alpha_spatial > 0:
            e = k[self._L] - k[self._R]
            sp = 0.5 * self.alpha_spatial * float(np.dot(e, e))
        ref = 0.0
        if self.alpha_ref > 0 and self.k_ref is not None:
            r = k - self.k_ref
            ref = 0.5 * self.alpha_ref * float(np.dot(r, r))
        return ridge, l1, sp, ref

    def func(self, theta) -> float:
        """f(theta) on the current recording (a replay, no gradient)."""
        k = self._apply(theta)
        return self.model.replay_cost() + sum(self._penalties(k))

    def grad(self, theta):
        """(f(theta), df/dtheta); records the trajectory again first when `rerecord`."""
        k = self._apply(theta)
        if self.rerecord:
            self.model.rerecord()
        J_data, g = self.model.adjoint(wrt=("friction_1", "friction_2"))
        g_k = g["friction_1"] + g["friction_2"]           # both directions carry the control
        ridge, l1, sp, ref = self._penalties(k)
        free = self.free
        d = k[free] - self.k_b[free]
        g_phys = g_k[free] + self.alpha_reg * d
        if self.alpha_l1 > 0:
            g_phys = g_phys + self.alpha_l1 * np.where(d > 1e-12, 1.0, np.where(d < -1e-12, -1.0, 0.0))
        if self.alpha_spatial > 0:
            gs = np.zeros(self.model.n)
            e = self.alpha_spatial * (k[self._L] - k[self._R])
            np.add.at(gs, self._L, e)
            np.add.at(gs, self._R, -e)
            g_phys = g_phys + gs[free]
        if self.alpha_ref > 0 and self.k_ref is not None:
            g_phys = g_phys + self.alpha_ref * (k[free] - self.k_ref[free])
        m = self._m_free(theta)
        g_m = g_phys * self.transform.derivative(m)
        g_theta = np.bincount(self.zone_of_free, weights=g_m, minlength=self.size()) if self.zonation else g_m
        J = J_data + ridge + l1 + sp + ref
        self.grad_calls += 1
        if self.J_init is None:
            self.J_init = J
        self._log(J, J_data, ridge, g_theta, g_k, k)
        self.J_prev = J
        return J, g_theta

    # ---- descent log (assim/swSpE_minimize.cpp:527-580)
    def _log(self, J, J_data, ridge, g_theta, g_phys_all, k):
        if not self.descent_dir:
            return
        if self._csv is None:
            self._csv = open(os.path.join(self.descent_dir, "descent_log.csv"), "w")
            self._csv.write(DESCENT_COLUMNS + "\n")
        rel = (J - self.J_init) / self.J_init * 100.0 if self.J_init else 0.0
        rel_prev = (J - self.J_prev) / self.J_prev * 100.0 if self.J_prev else 0.0
        kf = k[self.free]
        kb = self.k_b[self.free]
        upper = self.transform.hi if math.isfinite(self.transform.hi) else math.inf
        sse = float(np.sum((k - self.k_ref) ** 2)) if self.k_ref is not None else -1.0
        gl = np.abs(g_theta)
        gp = np.abs(g_phys_all)
        row = [self.grad_calls, f"{J:.10e}", f"{J_data:.10e}", f"{ridge:.10e}", f"{rel:.6e}", f"{rel_prev:.6e}",
               f"{float(np.sqrt(np.dot(g_theta, g_theta))):.6e}", f"{float(gl.max()) if gl.size else 0.0:.6e}",
               int(self.free[int(np.argmax(gl))]) if gl.size and not self.zonation else int(np.argmax(gl)) if gl.size else -1,
               f"{float(np.sqrt(np.dot(g_phys_all, g_phys_all))):.6e}", f"{float(gp.max()):.6e}", int(np.argmax(gp)),
               "-1", f"{float(kf.min()):.6e}", f"{float(kf.max()):.6e}", f"{float(kf.mean()):.6e}",
               int(np.sum(kf < 0.5 * kb)), int(np.sum(kf < 0.05 * kb)), int(np.sum(kf >= 0.999 * upper)), "-1",
               f"{sse:.10e}"]
        self._csv.write(",".join(str(x) for x in row) + "\n")
        self._csv.flush()
        write_map(os.path.join(self.descent_dir, "friction_iter", f"friction_iter_{self.grad_calls:04d}.txt"),
                  ["friction_coeff_1", "friction_coeff_2"], [k, k], self.model.n)

    def close(self):
        if self._csv is not None:
            self._csv.close()
            self._csv = None


def run_minimization(problem: FrictionProblem, max_it: int = 20, minimize_algo: str = "lbfgsb",
                     step: float = 0.0) -> Dict[str, object]:
    """Minimises problem.f from the background; returns {"theta", "k", "J_final", "J_init",
    "n_grad", "history"} and leaves the best control in the model (swSpE::run_minimization,
    assim/swSpE_minimize.cpp:582-)."""
    theta0 = problem.theta_start()
    history = []
    if minimize_algo == "lbfgsb":
        from scipy.optimize import minimize

        def fg(theta):
            J, g = problem.grad(theta)
            history.append(J)
            return J, g

        b = problem.transform.bounds()
        bounds = [b] * problem.size() if b is not None else None
        res = minimize(fg, theta0, jac=True, method="L-BFGS-B", bounds=bounds,
                       options={"maxiter": max_it, "maxfun": 2 * max_it + 5})
        theta = res.x
    elif minimize_algo == "gd":
        theta = _projected_gd(problem, theta0, max_it, step, history)
    else:
        raise ValueError(f"unknown minimize_algo {minimize_algo!r}")
    J_final, _ = problem.grad(theta)
    history.append(J_final)
    problem.close()
    return {"theta": theta, "k": problem.control(theta), "J_final": J_final, "J_init": problem.J_init,
            "n_grad": problem.grad_calls, "history": history}


def _projected_gd(problem, theta, max_it, step, history):
    """Projected gradient descent with Armijo backtracking (c1 = 1e-4, shrink 0.5, grow 4,
    40 backtracks at most), keeping the best iterate."""
    c1, shrink, grow, max_bt = 1e-4, 0.5, 4.0, 40
    b = problem.transform.bounds()

    def project(x):
        if b is None:
            return x
        lo = -np.inf if b[0] is None else b[0]
        hi = np.inf if b[1] is None else b[1]
        return np.clip(x, lo, hi)

    t = step if step > 0 else 1e-6
    best_theta, best_J = theta.copy(), math.inf
    for _ in range(max_it):
        J, g = problem.grad(theta)
        history.append(J)
        if J < best_J:
            best_J, best_theta = J, theta.copy()
        if not np.all(np.isfinite(g)) or not np.any(g):
            break
        t_try = t * grow
        accepted = False
        for _ in range(max_bt):
            trial = project(theta - t_try * g)
            Jt = problem.func(trial)
            if np.isfinite(Jt) and Jt <= J - c1 * float(np.dot(g, theta - trial)):
                theta, t, accepted = trial, t_try, True
                break
            t_try *= shrink
        if not accepted:
            break
    return best_theta if best_J <= problem.func(theta) else theta
