"""Shared checks for the parity tests (test infrastructure)."""
import numpy as np


def dist2(P, Q, idx):
    """Squared distances of result rows, computed as the reference does
    (kdtree-impl.h:331-339): per-axis (point - query) in the distance type
    (float32 for float32 and integer trees, float64 for float64), squared,
    summed in axis order with one rounding per operation.  -1 indices give
    inf."""
    dt = np.float64 if P.dtype == np.float64 else np.float32
    P = P.astype(dt, copy=False)
    Q = np.asarray(Q).astype(dt, copy=False)
    safe = np.where(idx >= 0, idx, 0)
    X = P[safe]  # m x k x d
    t = X - Q[:, None, :]
    s = t[..., 0] * t[..., 0]
    for d in range(1, P.shape[1]):
        s = s + t[..., d] * t[..., d]
    return np.where(idx >= 0, s, np.inf)


def canonical_rows(idx, d2):
    """Sorts each row by (dist2, point index); -1 entries stay last."""
    key = np.where(idx >= 0, idx, np.iinfo(np.int32).max).astype(np.int64)
    order = np.lexsort((key, d2), axis=-1)
    return np.take_along_axis(idx, order, -1), np.take_along_axis(d2, order, -1)


def brute_knn(P, Q, k, dmax=np.inf, exclude=None):
    """The specified kNN answer by exhaustive search: the k smallest
    (dist2, point index) pairs among the valid points with dist2 < dmax^2,
    dist2 in the reference's arithmetic.  exclude[i] (optional) is an index
    left out of row i (self queries).  NaN/inf rows of P are never answers.
    Returns (idx m x k, -1 padded; cnt m)."""
    P = np.asarray(P)
    Q = np.asarray(Q)
    m, n = len(Q), len(P)
    dt = np.float64 if P.dtype == np.float64 else np.float32
    r = dt(dmax)
    r2 = r * r
    valid = np.isfinite(P.astype(np.float64)).all(1)
    idx = np.full((m, k), -1, np.int32)
    cnt = np.zeros(m, np.int32)
    allidx = np.arange(n)[None, :]
    for i in range(m):
        d = dist2(P, Q[i:i + 1], allidx)[0]
        ok = valid & (d < r2)
        if exclude is not None and exclude[i] >= 0:
            ok[exclude[i]] = False
        cand = np.flatnonzero(ok)
        sel = cand[np.lexsort((cand, d[cand]))][:k]
        idx[i, :len(sel)] = sel
        cnt[i] = len(sel)
    return idx, cnt


def compare_knn(got, got_cnt, exp, exp_cnt, P, Q, k):
    """Compares a kNN result with the reference's, allowing only the
    reference's tie freedom.

    The reference keeps whichever equal-distance candidate its heap retains
    (kdtree-impl.h:360-373, 894-899), so its order inside a run of equal
    dist2, and its choice among points tied at the k-th distance, are
    arbitrary.  Both sides are canonicalised to (dist2, index) order and must
    then agree exactly, except inside the final run of equal dist2 of a full
    result, where both sides must hold points of that same distance.
    Returns (rows that differ beyond that, rows with a k-boundary tie choice
    that differs)."""
    got = np.asarray(got)
    exp = np.asarray(exp)
    if not np.array_equal(np.asarray(got_cnt), np.asarray(exp_cnt)):
        bad = np.flatnonzero(np.asarray(got_cnt) != np.asarray(exp_cnt))
        return len(bad), 0
    dg = dist2(P, Q, got)
    de = dist2(P, Q, exp)
    cg, dg = canonical_rows(got, dg)
    ce, de = canonical_rows(exp, de)
    same = (cg == ce).all(1)
    mism = 0
    ties = 0
    for i in np.flatnonzero(~same):
        if not np.array_equal(dg[i], de[i]):
            mism += 1
            continue
        c = int(got_cnt[i])
        last = dg[i, c - 1] if c else None
        run = dg[i, :c] == last
        if c == k and np.array_equal(cg[i, :c][~run], ce[i, :c][~run]):
            ties += 1
        else:
            mism += 1
    return mism, ties


def angle_error(a, b):
    """Angle (radians) between unit vectors a and b, sign-agnostic."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    na = np.linalg.norm(a, axis=-1)
    nb = np.linalg.norm(b, axis=-1)
    c = np.abs((a * b).sum(-1)) / np.maximum(na * nb, 1e-300)
    return np.arccos(np.clip(c, 0.0, 1.0))
