"""
Build libdifffea_b200.so, the C-ABI library of hand-written sm_100a kernels, in-tree.

    python differentiable-fea_b200/build.py [--force] [--verbose-ptxas]

Every CUDA source is compiled by nvcc for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``),
the host C++ by nvcc's host compiler, and the objects are linked into
``differentiable-fea_b200/difffea_b200/_lib/libdifffea_b200.so`` (static CUDA runtime, so the library
does not depend on the runtime version torch loads).  nvcc cross-compiles: no GPU is needed.
"""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
OUT_DIR = os.path.join(HERE, "difffea_b200", "_lib")
LIB = os.path.join(OUT_DIR, "libdifffea_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I" + INCLUDE, "-I" + CSRC]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False, quiet=False):
    """Compile every source and link the library; returns its path.  Raises on a compiler error."""
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = _nvcc()
    hdrs = headers()
    objs, jobs = [], []
    for src in sources():
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + hdrs + [os.path.abspath(__file__)]):
            continue
        cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas and src.endswith(".cu") else [])
        cmd += ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC, "-c", src, "-o", obj]
        jobs.append((src, cmd))

    def compile_one(job):
        src, cmd = job
        if not quiet:
            print(" ".join(cmd), flush=True)
        return src, subprocess.run(cmd, capture_output=True, text=True)

    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        results = list(pool.map(compile_one, jobs))
    for src, res in results:
        if verbose_ptxas or res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
    failed = [os.path.basename(src) for src, res in results if res.returncode != 0]
    if failed:
        raise RuntimeError(f"nvcc failed on {', '.join(failed)}")
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
        if not quiet:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link of libdifffea_b200.so failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))
