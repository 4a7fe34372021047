"""Shared checks for the parity tests (test infrastructure)."""
import numpy as np


def dist2(P, Q, idx):
    """Squared distances of result rows, computed as the reference does
    (kdtree-impl.h:331-339): per-axis (point - query) in the distance type
    (float32 for float32 trees, float64 for float64), squared, summed in
    axis order with one rounding per operation.  -1 indices give inf."""
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


def canonical_rows(idx, d2, pos_of):
    """Sorts each row by (dist2, tree position); -1 entries stay last."""
    pos = np.where(idx >= 0, pos_of[np.where(idx >= 0, idx, 0)], np.iinfo(np.int64).max)
    order = np.lexsort((pos, d2), axis=-1)
    return np.take_along_axis(idx, order, -1), np.take_along_axis(d2, order, -1)


def compare_knn(got, got_cnt, exp, exp_cnt, P, Q, pos_of, k):
    """Compares kNN results allowing only the reference's tie freedom.

    Both sides are canonicalised to (dist2, tree position) order.  They must
    agree exactly, except inside the final run of equal dist2 of a full
    result (a tie at the k-th distance), where the reference keeps whichever
    tied point its heap retained; there both sides must hold points of that
    same distance.  Returns (rows that differ beyond that, rows with a
    k-boundary tie choice that differs)."""
    got = np.asarray(got)
    exp = np.asarray(exp)
    if not np.array_equal(np.asarray(got_cnt), np.asarray(exp_cnt)):
        bad = np.flatnonzero(np.asarray(got_cnt) != np.asarray(exp_cnt))
        return len(bad), 0
    dg = dist2(P, Q, got)
    de = dist2(P, Q, exp)
    cg, dg = canonical_rows(got, dg, pos_of)
    ce, de = canonical_rows(exp, de, pos_of)
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
