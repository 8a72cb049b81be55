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
SOURCES = ["abi.cu", "fit_step.cu", "fit_fused.cu", "fit_comp.cu", "fit_tma.cu", "fit_tma2.cu", "fit_tma_comp.cu",
           "fit_batch.cu", "wake.cu", "adjoint.cu", "monitor.cu", "sources.cu"]
HEADERS = ["abi_internal.h", "fit_common.cuh", "fit_kernels.cuh", "fit_comp.cuh", "fit_tma_comp.cuh",
           "tma_util.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC",
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
    """Compile every translation unit to an object file (in parallel, one
    nvcc per source) and link them into the shared library."""
    if not force and not _stale():
        return OUT
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    inc = ["-I", os.path.join(ROOT, "include")]
    with tempfile.TemporaryDirectory(prefix="wk_build_") as tmpdir:
        def compile_one(src):
            obj = os.path.join(tmpdir, os.path.splitext(src)[0] + ".o")
            cmd = [nvcc(), *NVCC_FLAGS, *extra, *inc, "-c", "-o", obj, os.path.join(CSRC, src)]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}{r.stderr}")
            if r.stderr and verbose:
                print(r.stderr, end="", flush=True)
            return obj
        with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
            objs = list(ex.map(compile_one, SOURCES))
        tmp = OUT + ".tmp"
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
               "-Xcompiler", "-fPIC", "-o", tmp, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
