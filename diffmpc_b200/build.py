"""Builds ``diffmpc_b200/libdmpc.so`` for sm_100a with nvcc (in-tree).

Usage: ``python -m diffmpc_b200.build [--force]``.  Rebuilds only when a
source under ``csrc/`` or ``include/`` is newer than the library.

The SQP kernels (``csrc/k_sqp.cu``) are compiled once per launch
configuration (``-DDMPC_CFG=0``: up to 512 threads and one CTA per SM;
``1``: up to 256 threads, one CTA per SM, up to 255 registers a thread; ``2``:
256 threads and two CTAs per SM; ``3``: up to 384 threads, one CTA per SM, up to
168 registers a thread), in parallel with the host side and the
dense-layout kernels (``csrc/solver.cu``) and the XLA custom-call handler
core (``csrc/xla_ffi.cc``; its XLA FFI symbols too when ``DMPC_XLA_INCLUDE`` names jaxlib's
include directory); the objects are linked into one shared library.
"""

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdmpc.so")
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
UNITS = [
    ("solver.o", os.path.join(CSRC, "solver.cu"), []),
    ("k_sqp_cfg0.o", os.path.join(CSRC, "k_sqp.cu"), ["-DDMPC_CFG=0"]),
    ("k_sqp_cfg1.o", os.path.join(CSRC, "k_sqp.cu"), ["-DDMPC_CFG=1"]),
    ("k_sqp_cfg2.o", os.path.join(CSRC, "k_sqp.cu"), ["-DDMPC_CFG=2"]),
    ("k_sqp_cfg3.o", os.path.join(CSRC, "k_sqp.cu"), ["-DDMPC_CFG=3"]),
]
# XLA custom-call handlers: the core always; the XLA FFI symbols when DMPC_XLA_INCLUDE names
# jaxlib's include directory (the one holding xla/ffi/api/ffi.h)
_XLA_INC = os.environ.get("DMPC_XLA_INCLUDE")
UNITS.append(("xla_ffi.o", os.path.join(CSRC, "xla_ffi.cc"),
              ["-DDMPC_WITH_XLA_FFI", "-I", _XLA_INC] if _XLA_INC else []))
DEPS = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.exists(cand) or cand == "nvcc"):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def _compile(unit, verbose):
    obj, src, defs = unit
    cmd = [nvcc()] + NVCC_FLAGS + defs + ["-c", src, "-o", os.path.join(BUILD, obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        for f in [ex.submit(_compile, u, verbose) for u in UNITS]:
            f.result()
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + [os.path.join(BUILD, u[0]) for u in UNITS]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
