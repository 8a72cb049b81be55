"""Build ``libwakis_b200.so`` in-tree with nvcc for sm_100a.

    python -m wakis_b200.build [--force]

The library has no dependency on PyTorch: it links only the CUDA runtime.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libwakis_b200.so")
SOURCES = ["abi.cu", "fit_step.cu", "fit_march.cu", "fit_fused.cu", "fit_comp.cu", "fit_tma.cu", "fit_tma_comp.cu",
           "wake.cu", "adjoint.cu", "monitor.cu"]
HEADERS = ["abi_internal.h", "fit_common.cuh", "fit_kernels.cuh", "fit_comp.cuh", "tma_util.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "wakis_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force=False, verbose=True, extra=()):
    if not force and not _stale():
        return OUT
    srcs = [os.path.join(CSRC, f) for f in SOURCES]
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-o", tmp, *srcs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
