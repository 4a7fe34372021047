"""The PPTKG_BOUNDS_CHECK diagnostic build (libpptkg_checked.so): every
point-record, index-map and traversal-node index of the query kernels is
checked.  On valid trees it must give the product library's answers and no
check may fire (a fired check is an error of the call)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "pptk_b200", "_lib", "libpptkg_checked.so")

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from pptk_b200 import _native as N, kdtree, ragged, estimate_normals
assert N.lib().pptkg_bounds_checked() == {want}
rng = np.random.default_rng(3)
P = rng.random((60_000, 3)).astype(np.float32)
P[::97] = P[::89][: len(P[::97])]  # exact duplicates
P[5] = np.nan
t = kdtree._build(P)
idx, cnt = kdtree.knn(t, None, 16)
qi, qc = kdtree.knn(t, P[:500] + 1e-3, 8)
off, hits = kdtree.rnear(t, P[:300], 0.02)
ev = estimate_normals(P, 16, np.inf, verbose=False)
evr = estimate_normals(P, -1, 0.03, verbose=False)
coff = np.array([0, 20_000, 20_003, 60_000])
f = ragged.Forest(P, coff)
fi, fc, fn = f.knn_normals(12)
np.savez(sys.argv[2], idx=idx, cnt=cnt, qi=qi, qc=qc, off=off, hits=hits, ev=ev, evr=evr, fi=fi, fc=fc, fn=fn)
"""


def _run(tmp_path, lib, want, tag):
    env = dict(os.environ)
    if lib:
        env["PPTKG_LIBRARY"] = lib
    else:
        env.pop("PPTKG_LIBRARY", None)
    out = str(tmp_path / f"{tag}.npz")
    r = subprocess.run([sys.executable, "-c", CHILD.replace("{want}", str(want)), ROOT, out], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


def test_checked_build_matches_the_product_build(gpu, tmp_path):
    if not os.path.exists(CHECKED):
        pytest.skip("libpptkg_checked.so not built (python -m pptk_b200._build --bounds-check)")
    a = _run(tmp_path, None, 0, "product")
    b = _run(tmp_path, CHECKED, 1, "checked")
    for key in a.files:
        x, y = a[key], b[key]
        if x.dtype.kind == "f":
            assert np.array_equal(np.nan_to_num(x, nan=-9.0), np.nan_to_num(y, nan=-9.0)), key
        else:
            assert np.array_equal(x, y), key
