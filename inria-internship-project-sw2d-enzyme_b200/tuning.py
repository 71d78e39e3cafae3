"""Launch-configuration autotuner with a persistent JSON cache.

``autotune(model)`` asks the library (sw2d_autotune) to time every {threads per block,
register cap} variant of the step's heaviest kernels on the model's current state (k_flux for
the fused step; k_slopes and k_edges for the four-kernel step) and keeps the fastest; the
choice is stored in a JSON file keyed by GPU, scheme, options, step kind, tile size and mesh
size (power-of-two bucket), and reused by later runs without timing again.

``autotune_step(model)`` (sw2d_autotune_step) also chooses the step form: the four-kernel step
or the fused step, its tile size and, for MUSCL-EVR, where the slopes are computed; its cache
key leaves out the step kind and tile size, which are what it chooses.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from typing import Dict, Optional

CACHE = os.path.join(os.environ.get("XDG_CACHE_HOME", os.path.expanduser("~/.cache")), "sw2d_b200", "autotune.json")


def _device_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:  # noqa: BLE001 - the key only needs to be stable
        return f"cuda{device}"


def _base_key(model, device: int) -> list:
    o = model.case.opts
    bucket = int(math.log2(max(1, model.n)))
    return [_device_name(device), str(o.get("model_hyperb", "sp")), str(o.get("num_scheme", "godunov")),
            str(o.get("topo_discretization", "discontinuous")), str(o.get("model_friction", "none")),
            str(o.get("model_singular_head_loss", "none")), f"2^{bucket}"]


def _key(model, device: int) -> str:
    return "|".join(_base_key(model, device) + [f"fused{model.get_option('fused_step')}",
                                                 f"tile{model.get_option('tile_cells')}"])


def _store(cache_path: Optional[str], db: Dict[str, dict], key: str, entry: dict) -> None:
    if not cache_path:
        return
    db[key] = entry
    try:
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(db, fh, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    except OSError:
        pass


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def autotune(model, iters: int = 10, device: int = 0, cache_path: Optional[str] = CACHE, force: bool = False) -> dict:
    """Chooses the launch variants for `model`; returns {"slopes", "edges", "report", "cached"}."""
    key = _key(model, device)
    db = _load(cache_path) if cache_path else {}
    if not force and key in db:
        e = db[key]
        model._check(model.lib.sw2d_set_launch_config(model.handle, int(e["slopes"]), int(e["edges"])))
        if "flux" in e and model.get_option("fused_step"):
            model.set_option("flux_variant", int(e["flux"]))
        return {**e, "cached": True}
    buf = ctypes.create_string_buffer(4096)
    model._check(model.lib.sw2d_autotune(model.handle, int(iters), buf, len(buf)))
    sv, ev = ctypes.c_int(), ctypes.c_int()
    model._check(model.lib.sw2d_get_launch_config(model.handle, ctypes.byref(sv), ctypes.byref(ev)))
    entry = {"slopes": sv.value, "edges": ev.value, "flux": model.get_option("flux_variant"),
             "report": buf.value.decode()}
    _store(cache_path, db, key, entry)
    return {**entry, "cached": False}


def autotune_step(model, iters: int = 10, device: int = 0, tile_sizes=(), cache_path: Optional[str] = CACHE,
                  force: bool = False) -> dict:
    """Chooses the step form, tile size and launch variants for `model` (sw2d_autotune_step);
    returns {"fused", "fused_slopes", "tile", "slopes", "edges", "flux", "report", "cached"}."""
    key = "|".join(_base_key(model, device) + ["step"])
    db = _load(cache_path) if cache_path else {}
    if not force and key in db:
        e = db[key]
        if e["fused"]:
            if model.get_option("fused_slopes") != e["fused_slopes"]:
                model.set_option("fused_slopes", int(e["fused_slopes"]))
            if model.get_option("tile_cells") != e["tile"]:
                model.set_option("tile_cells", int(e["tile"]))
            model.set_option("flux_variant", int(e["flux"]))
        model.set_option("fused_step", int(e["fused"]))
        model._check(model.lib.sw2d_set_launch_config(model.handle, int(e["slopes"]), int(e["edges"])))
        return {**e, "cached": True}
    tiles = (ctypes.c_int * max(1, len(tile_sizes)))(*[int(t) for t in tile_sizes])
    buf = ctypes.create_string_buffer(8192)
    model._check(model.lib.sw2d_autotune_step(model.handle, int(iters), tiles, len(tile_sizes), buf, len(buf)))
    sv, ev = ctypes.c_int(), ctypes.c_int()
    model._check(model.lib.sw2d_get_launch_config(model.handle, ctypes.byref(sv), ctypes.byref(ev)))
    entry = {"fused": model.get_option("fused_step"), "fused_slopes": model.get_option("fused_slopes"),
             "tile": model.get_option("tile_cells"), "slopes": sv.value, "edges": ev.value,
             "flux": model.get_option("flux_variant"), "report": buf.value.decode()}
    _store(cache_path, db, key, entry)
    return {**entry, "cached": False}
