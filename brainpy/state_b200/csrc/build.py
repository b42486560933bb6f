"""Build libbspk.so (sm_100a) in-tree with nvcc.

    python -m brainpy.state_b200.csrc.build      # or build() from Python

Objects go to ``csrc/_build/``; the library to ``brainpy/state_b200/libbspk.so``.
``lif_exact.cu`` is compiled with ``-fmad=false`` (the deterministic FP64
kernel rounds every multiply and add separately).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(os.path.dirname(PKG))
OUT = os.path.join(PKG, "libbspk.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
          "-I" + HERE, "-I" + os.path.join(ROOT, "include")]
SOURCES = {
    "plan.cpp": [],
    "lif_fast.cu": [],
    "lif_tiled.cu": [],
    "lif_exact.cu": ["-fmad=false"],
    "per_step.cu": [],
    "batch.cu": [],
    "batch_host.cpp": [],
    "conn_gen.cu": [],
    "adjoint.cu": ["-fmad=false"],
    "checkpoint.cpp": [],
    "xla_ffi.cpp": [],
    "jax_rng.cpp": [],
    "umma_gemm.cu": [],
}
HEADERS = ["common.cuh", "device_types.h", "lif_args.h", "aeif_args.h", "stdp_args.h",
           "host_rng.h", "batch_args.h", "plan_internal.h", "conn_gen.h", "conn_gen.cuh",
           "coef_cast.h", "jax_rng.h", "umma.h"]


def _mtime(p):
    try:
        return os.path.getmtime(p)
    except OSError:
        return 0.0


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr_t = max([_mtime(os.path.join(HERE, h)) for h in HEADERS] +
                [_mtime(os.path.join(ROOT, "include", "bspk.h")), _mtime(__file__)])
    objs = []
    for src, extra in SOURCES.items():
        path = os.path.join(HERE, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _mtime(obj) < max(_mtime(path), hdr_t):
            lang = ["-x", "cu"] if src.endswith(".cpp") else []
            cmd = [NVCC] + ARCH + COMMON + extra + lang + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _mtime(OUT) < max(_mtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
