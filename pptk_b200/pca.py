"""Batched symmetric 3x3 eigensolve on the GPU.

The B200 counterpart of the 3x3 case of ``vfuncs._eigh``
(pptk/vfuncs/vfuncs.cpp:1241-1293): eigenvalues ascending, eigenvectors as
the columns of each 3x3 block (``V[i][:, j]`` is the j-th eigenvector), as
the reference lays them out.  ``layout="rows"`` gives estimate_normals'
layout instead (``V[i, j, :]``).
"""
import numpy as np

from . import _native as N

_CODES = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}


def eigh3(A, layout="columns"):
    """A: (m, 3, 3) symmetric float32/float64 (numpy or CUDA torch).
    Returns (w (m, 3), V (m, 3, 3))."""
    lay = {"columns": 0, "rows": 1}[layout]
    if N.is_torch_cuda(A):
        import torch
        if A.dtype not in (torch.float32, torch.float64):
            raise TypeError("eigh3: float32 or float64 input required")
        a = A.reshape(-1, 9).contiguous()
        m = a.shape[0]
        w = torch.empty((m, 3), dtype=A.dtype, device=A.device)
        V = torch.empty((m, 3, 3), dtype=A.dtype, device=A.device)
        code = 0 if A.dtype == torch.float32 else 1
        N.call("pptkg_eigh3", N.ptr(a), m, code, N.MEM_DEVICE, N.ptr(w), N.ptr(V), lay, N.torch_stream(A.device))
        return w, V
    a = np.asarray(A)
    if a.dtype not in _CODES:
        raise TypeError("eigh3: float32 or float64 input required")
    a = np.ascontiguousarray(a.reshape(-1, 9))
    m = a.shape[0]
    w = np.empty((m, 3), a.dtype)
    V = np.empty((m, 3, 3), a.dtype)
    N.call("pptkg_eigh3", N.ptr(a), m, _CODES[a.dtype], N.MEM_HOST, N.ptr(w), N.ptr(V), lay, None)
    return w, V


def eigh_list(X):
    """The calling form of vfuncs ``_eigh`` (pptk/vfuncs/vfuncs.cpp:1241-1293)
    over the batched GPU solve: X is a non-empty list of square float32
    arrays; returns a list of (w, V) pairs, float32, w ascending and
    ``V[:, j]`` the j-th eigenvector (the reference copies Eigen's row-major
    eigenvector matrix element by element, :1285-1287).  As Eigen's
    SelfAdjointEigenSolver does, only the lower triangle of each matrix is
    read.  The GPU path solves 3 x 3 blocks (the neighbourhood covariances
    of the expression layer, pptk/points/expr.py:27-72); other sizes raise
    NotImplementedError."""
    if not isinstance(X, list):
        raise TypeError("eigh_list: a list of arrays is required")
    if not X:
        raise ValueError("eigh_list: the list must not be empty")
    blocks = np.empty((len(X), 3, 3), np.float32)
    for i, a in enumerate(X):
        if not isinstance(a, np.ndarray):
            raise TypeError(f"eigh_list: item {i} is not a numpy array")
        if a.dtype != np.float32:
            raise TypeError(f"eigh_list: item {i} must be float32")
        if a.ndim not in (1, 2):
            raise ValueError(f"eigh_list: item {i} must have 1 or 2 dimensions")
        rows, cols = (1, a.shape[0]) if a.ndim == 1 else a.shape
        if rows != cols:
            raise ValueError(f"eigh_list: item {i} is not square ({rows} x {cols})")
        if rows != 3:
            raise NotImplementedError(f"eigh_list: item {i} is {rows} x {rows}; the GPU path solves 3 x 3 blocks")
        low = np.tril(a)
        blocks[i] = low + np.tril(a, -1).T
    w, V = eigh3(blocks, layout="columns")
    return [(w[i].copy(), V[i].copy()) for i in range(len(X))]


def _csr(nbhds):
    """(offsets int64 m+1, indices int32) from a list of index arrays (the
    _query / Points.nbhds form), a (offsets, indices) pair, or a dense
    (indices m x k, counts m) pair from kdtree.knn."""
    if isinstance(nbhds, tuple) and len(nbhds) == 2:
        a, b = (np.asarray(x.cpu() if hasattr(x, "cpu") else x) for x in nbhds)
        if a.ndim == 2:  # dense kNN result: (indices m x k, counts m)
            cnt = b.astype(np.int64)
            off = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
            keep = np.arange(a.shape[1])[None, :] < cnt[:, None]
            return off, np.ascontiguousarray(a[keep], dtype=np.int32)
        return np.ascontiguousarray(a, dtype=np.int64), np.ascontiguousarray(b, dtype=np.int32)
    rows = [np.asarray(r, dtype=np.int64).reshape(-1) for r in nbhds]
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    idx = np.concatenate(rows).astype(np.int32) if rows else np.zeros(0, np.int32)
    return off, np.ascontiguousarray(idx)


def nbhd_covariance(points, nbhds):
    """Covariance Y^T Y / count of every neighbourhood (Y its points minus
    their mean): what pptk's expression layer builds per neighbourhood with
    MEAN / DOT / TRANSPOSE (pptk/points/expr.py:27-72).  points: n x 3
    float32/float64 numpy array; nbhds as for `nbhd_pca`.  Returns m x 3 x 3."""
    P = np.ascontiguousarray(np.asarray(points))
    if P.dtype not in _CODES or P.ndim != 2 or P.shape[1] != 3:
        raise TypeError("points must be an n x 3 float32 or float64 array")
    off, idx = _csr(nbhds)
    m = len(off) - 1
    C = np.empty((m, 3, 3), P.dtype)
    N.call("pptkg_nbhd_covariance", N.ptr(P), P.shape[0], _CODES[P.dtype], N.MEM_HOST, N.ptr(off), N.ptr(idx), m,
           N.ptr(C), None, where="nbhd_covariance()")
    return C


def nbhd_pca(points, nbhds):
    """PCA of every neighbourhood on the GPU: (w (m, 3) ascending, V (m, 3, 3)
    with V[i][:, j] the j-th eigenvector -- vfuncs `_eigh`'s layout).  nbhds:
    a list of index arrays (as returned by kdtree._query / Points.nbhds), an
    (offsets, indices) CSR pair, or kdtree.knn's (indices, counts)."""
    return eigh3(nbhd_covariance(points, nbhds), layout="columns")
