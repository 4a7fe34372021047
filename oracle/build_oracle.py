"""Build recipe for the oracle libraries (test infrastructure only).

* ``oracle/libpptk_port.so`` -- the CPU restatement in ``oracle/port.cpp``.
* ``oracle/_ref/libpptk_ref.so`` -- ``oracle/ref_harness.cpp`` compiled
  against the reference's own k-d tree headers where they lie
  (``<reference>/pptk/kdtree/src``).  Built only when the reference tree is
  present; nothing is copied out of it.

Flags follow the reference's release build (``CMakeLists.txt:4``: ``-O3
-DNDEBUG``) with no ``-march``, so x86-64 code has no FMA contraction, as in
the reference.  ``-std=c++14`` is needed for the harness's generic lambdas;
the reference headers compile unchanged under it.  OpenMP stands in for TBB,
which is not installed.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference source tree: $PPTK_REFERENCE, else a `reference` directory
# beside the repository
REF_SRC = os.environ.get("PPTK_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
FLAGS = ["-O3", "-DNDEBUG", "-std=c++14", "-fopenmp", "-shared", "-fPIC"]


def _newer(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_port(force=False):
    out = os.path.join(HERE, "libpptk_port.so")
    srcs = [os.path.join(HERE, "port.cpp"), os.path.join(HERE, "common.h")]
    if force or _newer(out, srcs):
        subprocess.check_call(["g++", *FLAGS, "-I", HERE, srcs[0], "-o", out])
    return out


def build_ref(force=False):
    """Returns the path of the reference harness, or None without the reference."""
    inc = os.path.join(REF_SRC, "pptk", "kdtree", "src")
    out_dir = os.path.join(HERE, "_ref")
    out = os.path.join(out_dir, "libpptk_ref.so")
    if not os.path.isdir(inc):
        return out if os.path.exists(out) else None
    os.makedirs(out_dir, exist_ok=True)
    srcs = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "common.h")]
    hdrs = [os.path.join(inc, f) for f in sorted(os.listdir(inc)) if f.endswith(".h")]
    if force or _newer(out, srcs + hdrs):
        subprocess.check_call(["g++", *FLAGS, "-I", HERE, "-I", inc, srcs[0], "-o", out])
    return out


def build_all(force=False):
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(2) as ex:
        a = ex.submit(build_port, force)
        b = ex.submit(build_ref, force)
        return a.result(), b.result()


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv))
