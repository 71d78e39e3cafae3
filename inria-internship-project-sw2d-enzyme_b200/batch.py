"""Ensembles of independent simulations advanced together on one GPU (sw2d_batch_* of the C
ABI): one CUDA graph launch steps every member, each on its own stream branch; member results
are those of the member run alone, bit for bit.  The reference runs one simulation per process
and evaluates line-search trial points and perturbed members one after another."""
from __future__ import annotations

import ctypes
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import capi
from .solver import SpModel, Sw2dError


class Batch:
    def __init__(self, models: Sequence[SpModel]):
        self.lib = capi.load_library()
        self.models = list(models)
        arr = (ctypes.c_void_p * len(self.models))(*[m.handle.value for m in self.models])
        out = ctypes.c_void_p()
        st = self.lib.sw2d_batch_create(arr, len(self.models), ctypes.byref(out))
        if st != 0:
            raise Sw2dError(st, self.lib.sw2d_batch_last_error(None).decode())
        self.handle = out

    def _check(self, st: int) -> None:
        if st != 0:
            raise Sw2dError(st, self.lib.sw2d_batch_last_error(self.handle).decode())

    def step(self, n: int) -> np.ndarray:
        """At most n steps of every member; returns the steps each took."""
        done = np.zeros(len(self.models), dtype=np.int64)
        self._check(self.lib.sw2d_batch_step_n(self.handle, int(n), done.ctypes.data_as(capi.c_int64_p)))
        return done

    def adjoint(self, wrt=SpModel.GRADIENTS, n_threads: int = 16) -> List[Tuple[float, Dict[str, np.ndarray]]]:
        """(J, {name: gradient}) of every member (each with its recorded trajectory and observations)."""
        M = len(self.models)
        grads = (capi.Sw2dGradient * M)()
        outs = []
        for i, m in enumerate(self.models):
            d = {}
            for name in wrt:
                d[name] = np.empty(m.n)
                setattr(grads[i], name, d[name].ctypes.data_as(capi.c_double_p))
            outs.append(d)
        J = np.zeros(M)
        self._check(self.lib.sw2d_batch_adjoint(self.handle, J.ctypes.data_as(capi.c_double_p), grads, int(n_threads)))
        return [(float(J[i]), outs[i]) for i in range(M)]

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.sw2d_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
