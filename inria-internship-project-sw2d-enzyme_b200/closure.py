"""The learned momentum-exchange closure: a small MLP on the tensor cores (C ABI sw2d_mlp_*).

``MLP`` owns a network of 10 features -> 64 -> 64 -> 2 outputs (GELU) on one GPU: inference,
loss and gradient, Adam steps, all in the library's tcgen05 kernels (BF16 operands, FP32
accumulation).  ``reference_forward`` / ``reference_loss_grad`` restate the same network in
numpy FP64 with the kernels' BF16 roundings, for the tests' gradient checks.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import capi

N_IN, N_HID, N_OUT = 10, 64, 2
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,))]


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation of the parameter vector (layout of sw2d_mlp_create)."""
    rng = np.random.default_rng(seed)
    out = []
    for name, shape in SHAPES:
        if name.startswith("W"):
            out.append(rng.normal(0.0, np.sqrt(2.0 / shape[1]), size=shape).reshape(-1))
        else:
            out.append(np.zeros(shape))
    return np.concatenate(out).astype(np.float32)


def unpack(p: np.ndarray):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(x):
    k0, k1 = 0.7978845608028654, 0.044715
    return 0.5 * x * (1.0 + np.tanh(k0 * (x + k1 * x ** 3)))


def gelu_grad(x):
    k0, k1 = 0.7978845608028654, 0.044715
    t = np.tanh(k0 * (x + k1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * k0 * (1.0 + 3.0 * k1 * x * x)


def reference_forward(p: np.ndarray, norm: np.ndarray, x: np.ndarray, rounding: bool = True):
    """FP64 forward with the kernels' BF16 roundings (inputs, weights, hidden activations), or
    without any rounding (rounding=False, for finite-difference checks of the formulas)."""
    rd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    w = unpack(p)
    xm, xs, ym, ys = norm[:N_IN], norm[N_IN:2 * N_IN], norm[2 * N_IN:2 * N_IN + N_OUT], norm[2 * N_IN + N_OUT:]
    xn = rd(((np.asarray(x, np.float32) - xm.astype(np.float32)) / xs.astype(np.float32)))
    z1 = xn @ rd(w["W1"]).T + w["b1"]
    h1 = rd(gelu(z1))
    z2 = h1 @ rd(w["W2"]).T + w["b2"]
    h2 = rd(gelu(z2))
    yn = h2 @ rd(w["W3"]).T + w["b3"]
    return dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2, yn=yn, y=yn * ys + ym)


def reference_loss_grad(p: np.ndarray, norm: np.ndarray, x: np.ndarray, t: np.ndarray,
                        rounding: bool = True) -> Tuple[float, np.ndarray]:
    """Loss (mean squared error of the normalised outputs) and its FP64 gradient, with the
    kernels' BF16 roundings of dY, dZ2 and dZ1 (or none: rounding=False)."""
    rd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    w = unpack(p)
    f = reference_forward(p, norm, x, rounding)
    ym, ys = norm[2 * N_IN:2 * N_IN + N_OUT], norm[2 * N_IN + N_OUT:]
    tn = ((np.asarray(t, np.float32) - ym.astype(np.float32)) / ys.astype(np.float32)).astype(np.float64)
    n = x.shape[0]
    d = f["yn"] - tn
    loss = float(np.sum(d * d) / (n * N_OUT))
    dy = rd(2.0 * d / (n * N_OUT))
    dz2 = rd((dy @ rd(w["W3"])) * gelu_grad(f["z2"]))
    dz1 = rd((dz2 @ rd(w["W2"])) * gelu_grad(f["z1"]))
    g = dict(W3=dy.T @ f["h2"], b3=dy.sum(0), W2=dz2.T @ f["h1"], b2=dz2.sum(0), W1=dz1.T @ f["xn"],
             b1=dz1.sum(0))
    return loss, np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])


class MLP:
    """The closure network on one GPU (the library's tcgen05 kernels)."""

    def __init__(self, params: Optional[np.ndarray] = None, norm: Optional[np.ndarray] = None, device: int = 0):
        self.lib = capi.load_library()
        n = self.lib.sw2d_mlp_param_count()
        p = init_params() if params is None else np.asarray(params, dtype=np.float32)
        if p.size != n:
            raise ValueError(f"expected {n} parameters")
        if norm is None:
            norm = np.concatenate([np.zeros(N_IN), np.ones(N_IN), np.zeros(N_OUT), np.ones(N_OUT)])
        self.norm = np.ascontiguousarray(norm, dtype=np.float32)
        self.h = ctypes.c_void_p()
        fp = ctypes.POINTER(ctypes.c_float)
        st = self.lib.sw2d_mlp_create(int(device), np.ascontiguousarray(p).ctypes.data_as(fp),
                                      self.norm.ctypes.data_as(fp), ctypes.byref(self.h))
        if st != 0:
            raise RuntimeError(f"sw2d_mlp_create failed ({st})")

    def _fp(self, a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def _check(self, st):
        if st != 0:
            raise RuntimeError(f"sw2d_mlp error {st}: {self.lib.sw2d_mlp_last_error(self.h).decode()}")

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.lib.sw2d_mlp_param_count(), dtype=np.float32)
        self._check(self.lib.sw2d_mlp_get_params(self.h, self._fp(out)))
        return out

    def infer(self, x, layers: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        y = np.empty((n, N_OUT), dtype=np.float32)
        lay = np.empty((4, n, N_HID), dtype=np.float32) if layers else None
        self._check(self.lib.sw2d_mlp_infer(self.h, self._fp(x), n, self._fp(y),
                                            self._fp(lay) if layers else None))
        return (y, lay) if layers else y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_double()
        g = np.empty(self.lib.sw2d_mlp_param_count(), dtype=np.float32)
        self._check(self.lib.sw2d_mlp_loss_grad(self.h, self._fp(x), self._fp(t), x.shape[0], ctypes.byref(loss),
                                                self._fp(g)))
        return loss.value, g

    def adam_step(self, lr: float) -> None:
        self._check(self.lib.sw2d_mlp_adam_step(self.h, float(lr)))

    def train(self, x, t, epochs: int = 10, batch: int = 4096, lr: float = 2e-3, seed: int = 0):
        """Mini-batch Adam over seeded shuffles; returns the per-epoch mean losses."""
        rng = np.random.default_rng(seed)
        n = x.shape[0]
        hist = []
        for _ in range(epochs):
            order = rng.permutation(n)
            tot, cnt = 0.0, 0
            for s in range(0, n, batch):
                idx = order[s:s + batch]
                loss, _ = self.loss_grad(x[idx], t[idx])
                self.adam_step(lr)
                tot += loss * idx.size
                cnt += idx.size
            hist.append(tot / max(cnt, 1))
        return hist

    def close(self):
        if self.h:
            self.lib.sw2d_mlp_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
