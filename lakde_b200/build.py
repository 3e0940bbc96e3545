"""Builds the CUDA library of the package in-tree for sm_100a.

    python -m lakde_b200.build [--verbose] [--ptxas-info]

Each ``csrc/*.cu`` is compiled by nvcc to an object under ``_build/`` and the
objects are linked into ``lakde_b200/_lib/liblakde_b200.so``.  Objects are
rebuilt only when a source or header is newer.
"""

import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "liblakde_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "-DLAKDE_BUILD",
] + ARCH


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    if os.path.exists(cand):
        return cand
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found; set CUDA_HOME")
    return found


def lib_path():
    return os.path.join(LIBDIR, LIBNAME)


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src, ptxas_info=False, verbose=False):
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    newest_dep = max(os.path.getmtime(p) for p in [src] + _headers())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep and not ptxas_info:
        return obj, ""
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def build(verbose=False, ptxas_info=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or min(len(sources), os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_info, verbose), sources))
    if ptxas_info:
        for _, log in results:
            sys.stdout.write(log)
    objs = [o for o, _ in results]
    out = lib_path()
    if not os.path.exists(out) or any(os.path.getmtime(o) > os.path.getmtime(out) for o in objs):
        cmd = [nvcc(), "-shared"] + ARCH + objs + ["-o", out]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return out


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas-info" in sys.argv))
