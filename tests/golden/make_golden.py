"""Generates the golden fixtures in this directory from the reference itself.

Run in a checkout where the reference source tree is available (the oracle
build compiles its k-d tree headers in place into oracle/_ref):

    python tests/golden/make_golden.py

Every fixture is a small .npz of seeded inputs and the reference's outputs:
the tree permutation (reverse_indices), the preorder node list, kNN results
(point and self queries), r-near results in the reference's order, and the
restated estimate_normals outputs on the collinear known-answer input of
tests/test_estimate_normals.py:38-138 of the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import build_oracle  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cloud(name):
    rng = np.random.default_rng(1234)
    if name == "f32_uniform":
        return rng.random((3000, 3), dtype=np.float32)
    if name == "f64_uniform":
        return rng.random((2000, 3))
    if name == "f32_nan_dups":
        p = rng.random((2500, 3), dtype=np.float32)
        p[::53] = np.nan
        p[7::61, 2] = np.inf
        p[100:160] = p[200]  # a pile of duplicates
        return p
    if name == "f32_grid":
        g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(6), indexing="ij"), -1)
        return g.reshape(-1, 3).astype(np.float32) * np.float32(0.5)
    if name == "f64_aniso":
        return rng.normal(size=(2500, 3)) * np.array([50.0, 1.0, 0.01]) + np.array([1e5, 1e5, 0.0])
    raise KeyError(name)


CASES = ["f32_uniform", "f64_uniform", "f32_nan_dups", "f32_grid", "f64_aniso"]


def make(name):
    P = cloud(name)
    t = O.RefTree(P)
    rng = np.random.default_rng(99)
    lo = np.nanmin(np.where(np.isfinite(P), P, np.nan), 0)
    hi = np.nanmax(np.where(np.isfinite(P), P, np.nan), 0)
    Q = (lo + (hi - lo) * rng.random((200, 3))).astype(P.dtype)
    k = 8
    kidx, kcnt = t.knn(Q, k)
    kidx_r, kcnt_r = t.knn(Q, k, dmax=float(np.float32(0.15 * (hi - lo).max())))
    nv = t.num_valid
    sidx = np.arange(min(nv, 500), dtype=np.int32)
    self_idx, self_cnt = t.knn_self(sidx, k)
    r = float(np.float32(0.08 * (hi - lo).max()))
    roff, rout = t.rnear(Q, r)
    soff, sout = t.rnear_self(sidx, r)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), points=P, reverse=t.reverse_indices(), nodes=t.nodes(),
                        queries=Q, k=k, knn_idx=kidx, knn_cnt=kcnt, knn_r_idx=kidx_r, knn_r_cnt=kcnt_r,
                        knn_r_dmax=np.float64(float(np.float32(0.15 * (hi - lo).max()))), self_q=sidx,
                        self_idx=self_idx, self_cnt=self_cnt, rnear_r=np.float64(r), rnear_off=roff,
                        rnear_idx=rout, rself_off=soff, rself_idx=sout)


def make_collinear():
    # estimate_normals known answer (reference tests/test_estimate_normals.py:38-47)
    y = np.zeros((10, 3), dtype=np.float64)
    y[:, 0] = np.arange(10)
    ev, ew, sz, _ = O.ref_estimate_normals(y, 4, 3.0, num_eigen=3)
    np.savez_compressed(os.path.join(HERE, "collinear_normals.npz"), points=y, k=4, r=3.0, evecs=ev, evals=ew,
                        sizes=sz)


if __name__ == "__main__":
    build_oracle.build_all()
    for c in CASES:
        make(c)
    make_collinear()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
