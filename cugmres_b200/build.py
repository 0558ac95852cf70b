"""Builds cugmres_b200/lib/libcugmres.so from cugmres_b200/csrc for sm_100a.

    python -m cugmres_b200.build            # incremental
    python -m cugmres_b200.build --force    # rebuild everything

Each source is compiled by nvcc in parallel into cugmres_b200/_build/ and the
objects are linked into one shared library (CUDA runtime linked statically),
so the library needs neither torch nor a JIT cache at run time.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcugmres.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["cg_matvec.cu", "cg_krylov.cu", "cg_dcgs2.cu", "cg_sstep.cu", "cg_api.cu", "cg_noalloc.cu", "cg_batch.cu", "cg_fno.cu", "cg_green_dev.cu",
           "cg_green.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-diag-suppress", "128"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src):
    heads = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    heads.append(os.path.join(INCLUDE, "cugmres.h"))
    return [os.path.join(CSRC, src)] + heads


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra, verbose):
    obj = os.path.join(BUILD, src + ".o")
    cmd = [nvcc()] + ARCH + NVFLAGS + extra + ["-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-c",
               os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr)
    return obj


def build(force=False, verbose=False, extra=None):
    extra = list(extra or [])
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    todo = [s for s in SOURCES if force or _stale(os.path.join(BUILD, s + ".o"), _deps(s))]
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        list(ex.map(lambda s: _compile(s, extra, verbose), todo))
    objs = [os.path.join(BUILD, s + ".o") for s in SOURCES]
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
