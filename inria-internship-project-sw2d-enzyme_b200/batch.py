"""Ensembles of independent simulations advanced together on one GPU (sw2d_batch_* of the C
ABI).  Members that are SP models of one scheme run as one persistent kernel over a work queue
of (step, phase, member, tile) items (``mode == QUEUE``); any other mix runs as one CUDA graph
with a stream branch per member (``mode == BRANCHES``).  Member results are those of the member
run alone, bit for bit, in both forms.  The reference runs one simulation per process and
evaluates line-search trial points and perturbed members one after another."""
from __future__ import annotations

import ctypes
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import capi
from .solver import SpModel, Sw2dError


class Batch:
    BRANCHES, QUEUE = 0, 1

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

    @property
    def config(self) -> Dict[str, int]:
        """{"mode", "variant", "cells_per_tile", "edges_per_tile"} of the batch's step."""
        v = [ctypes.c_int() for _ in range(4)]
        self._check(self.lib.sw2d_batch_get_config(self.handle, *(ctypes.byref(x) for x in v)))
        return dict(zip(("mode", "variant", "cells_per_tile", "edges_per_tile"), (x.value for x in v)))

    def configure(self, mode: int, variant: int = -1, cells_per_tile: int = 0, edges_per_tile: int = 0) -> None:
        self._check(self.lib.sw2d_batch_configure(self.handle, int(mode), int(variant), int(cells_per_tile),
                                                  int(edges_per_tile)))

    def autotune(self, steps: int = 8, tile_sizes: Sequence[int] = ()) -> str:
        """Times the work queue over its launch variants and tile sizes on the members' current
        states (restored after each trial) and keeps the fastest; returns the report."""
        tiles = (ctypes.c_int * max(1, len(tile_sizes)))(*[int(t) for t in tile_sizes])
        buf = ctypes.create_string_buffer(8192)
        self._check(self.lib.sw2d_batch_autotune(self.handle, int(steps), tiles, len(tile_sizes), buf, len(buf)))
        return buf.value.decode()

    def set_wait_polls(self, polls: int) -> None:
        """Poll limit of the work queue's waits (< 0: the default)."""
        self._check(self.lib.sw2d_batch_set_wait_polls(self.handle, int(polls)))

    @property
    def stream(self) -> int:
        return int(self.lib.sw2d_batch_stream(self.handle) or 0)

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
