"""In-tree build of the native library ``pptk_b200/_lib/libpptkg.so``.

Every CUDA source under ``pptk_b200/csrc`` is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with nvcc, in parallel, and
linked into one shared library that exports the C ABI of
``include/pptkg.h``.  The library links the CUDA runtime statically and has
no dependency on torch or Python.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_lib", "obj")
LIB = os.path.join(PKG, "_lib", "libpptkg.so")
# the diagnostic build with every tree index of the query kernels checked
# (-DPPTKG_BOUNDS_CHECK); load it with PPTKG_LIBRARY=<path>
OBJ_CHECKED = os.path.join(PKG, "_lib", "obj_checked")
LIB_CHECKED = os.path.join(PKG, "_lib", "libpptkg_checked.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-I", INCLUDE, "-I", CSRC,
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _included_sources(src):
    """.cu files that `src` includes (query_d2.cu / query_d4.cu include
    query.cu to instantiate it for another dimension)."""
    with open(src) as f:
        text = f.read()
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith(".cu") and f'#include "{f}"' in text]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra_flags=(), bounds_check=False):
    """Compiles the library if any source changed; returns its path.
    bounds_check: the PPTKG_BOUNDS_CHECK build into libpptkg_checked.so."""
    obj_dir, lib_path = (OBJ_CHECKED, LIB_CHECKED) if bounds_check else (OBJ, LIB)
    if bounds_check:
        extra_flags = (*extra_flags, "-DPPTKG_BOUNDS_CHECK")
    os.makedirs(obj_dir, exist_ok=True)
    srcs = _sources()
    hdrs = _headers()
    cc = nvcc()
    jobs = []
    for s in srcs:
        o = os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o")
        if force or _stale(o, [s] + _included_sources(s) + hdrs + [__file__]):
            jobs.append((s, o))

    def compile_one(job):
        s, o = job
        cmd = [cc, *NVCC_FLAGS, *extra_flags, "-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n{r.stderr[-8000:]}")
        return r.stderr

    if jobs:
        with ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            for msg in ex.map(compile_one, jobs):
                if verbose and msg:
                    print(msg)
    objs = [os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    if force or jobs or _stale(lib_path, objs):
        cmd = [cc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", lib_path + ".tmp",
               "-Xcompiler", "-fPIC"]
        subprocess.check_call(cmd)
        os.replace(lib_path + ".tmp", lib_path)
    return lib_path


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, bounds_check="--bounds-check" in sys.argv))
