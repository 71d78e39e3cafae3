"""Builds the CUDA library ``lib/libsw2d_b200.so`` in-tree with nvcc for sm_100a.

``-fmad=false`` keeps every multiply and add separately rounded, as the reference's host
build does (g++ on x86-64 without FMA), which is what makes the FP64 results bit-identical.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
SOURCES = ["sw2d_sp.cu", "sw2d_tile.cu", "sw2d_queue.cu", "sw2d_adjoint.cu", "sw2d_batch.cu", "sw2d_assim.cu", "sw2d_ddp.cu", "sw2d_case.cpp", "sw2d_mlp.cu",
           "sw2d_result.cu", "sw2d_mapper.cu"]
HEADERS = ["sw2d_internal.cuh", "sp_math.cuh", "dip_math.cuh", "sp_adjoint.cuh", "portable_math.h", "adjoint_common.cuh",
           "spe_math.cuh", "ddp_math.cuh", "umma.cuh"]
OUT = os.path.join(LIBDIR, "libsw2d_b200.so")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
              "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "-shared", "-Xptxas", "-v"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler():
    # the system g++ links libstdc++ dynamically, which a library loaded by Python needs
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else None


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "sw2d_b200.h"))
    deps.append(__file__)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _compile(src: str, obj: str, hc) -> subprocess.CompletedProcess:
    cmd = [_nvcc()] + [f for f in NVCC_FLAGS if f != "-shared"] + ["-c"]
    if hc:
        cmd += ["-ccbin", hc]
    cmd += ["-o", obj + ".tmp", src]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode == 0:
        os.replace(obj + ".tmp", obj)
    return res


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object in lib/obj (in parallel, one nvcc per source) and links
    the shared library; the -Xptxas -v report of all sources goes to lib/ptxas.log."""
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    hc = _host_compiler()
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    objs = [os.path.join(objdir, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda so: _compile(so[0], so[1], hc), zip(srcs, objs)))
    log = "".join(r.stderr for r in results)
    if any(r.returncode != 0 for r in results):
        sys.stderr.write("".join(r.stdout + r.stderr for r in results if r.returncode != 0))
        raise RuntimeError("nvcc failed")
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared"]
    if hc:
        cmd += ["-ccbin", hc]
    cmd += ["-o", OUT + ".tmp"] + objs
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed")
    if verbose:
        sys.stderr.write(log)
    os.replace(OUT + ".tmp", OUT)
    with open(os.path.join(LIBDIR, "ptxas.log"), "w") as fh:
        fh.write(log)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
