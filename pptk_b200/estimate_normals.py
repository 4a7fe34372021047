"""Drop-in for ``pptk.estimate_normals`` on the GPU.

Mirrors ``estimate_normals_wrapper`` (pptk/processing/estimate_normals/
estimate_normals.cpp:259-345): the same arguments, checks, exception types
and return layouts.  The whole computation -- tree build, neighbourhood
search and the per-point covariance eigensolve -- runs in one native call.
"""
import ctypes
import math
import sys
import time

import numpy as np

from . import _native as N
from ._args import as_points_2d, extract_indices

_FLOAT_CODES = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}
PRECISIONS = {"auto": N.PREC_AUTO, "fp32": N.PREC_FP32, "fp64": N.PREC_FP64}


def _alloc(like_torch, shape, dtype, device):
    if like_torch:
        import torch
        tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
               np.dtype(np.int32): torch.int32}[np.dtype(dtype)]
        return torch.empty(shape, dtype=tdt, device=device)
    return np.empty(shape, dtype)


def estimate_normals(points, k, r, subsample=None, output_eigenvalues=False, output_all_eigenvectors=False,
                     output_neighborhood_sizes=False, verbose=True, num_procs=-1, precision="auto"):
    """Estimates normals at all points using principal component analysis
    (PCA): eigenvectors of the covariance matrix of each point's local
    neighbourhood, C = 1/N sum (p_i - mu)(p_i - mu)^T.

    Parameters
    ----------
    points : n x 3 numpy array (or CUDA torch tensor) of float32 or float64
    k : int
        Number of neighbors to use (the point itself included).
        For pure r-near neighborhoods, set this to -1.
    r : float
        Use neighbors within r of query point.
        For pure k-nearest neighborhoods, set this to np.inf.
    subsample : 1-d array of bool or int, optional
        Estimate normals at the points selected by a boolean mask of length n
        or by integer indices. Default: None.
    output_eigenvalues, output_all_eigenvectors, output_neighborhood_sizes : bool
    verbose : bool
    num_procs : int
        Accepted for compatibility; the work runs on the GPU.
    precision : "auto" | "fp32" | "fp64"
        Covariance / eigensolve arithmetic.  "auto": float32 input uses the
        FP32 path (neighbourhood shifted to the query point, compensated
        sums, FP64 re-solve when the two smallest eigenvalues nearly
        coincide); float64 input uses FP64 throughout.

    Returns
    -------
    results : ndarray or tuple of ndarrays, as in the reference:
        m x 3 (or m x 3 x 3 with output_all_eigenvectors), and, when either
        output_eigenvalues or output_neighborhood_sizes is set, the tuple
        (eigenvectors, eigenvalues or None, sizes or None).
        The j-th eigenvector of the i-th result is [i, j, :]; eigenvectors are
        sorted by increasing eigenvalue.
    """
    # PyArg_ParseTupleAndKeywords "Oif|Oiiiii" (estimate_normals.cpp:270-279)
    try:
        if isinstance(k, float) or isinstance(k, (str, bytes)):
            raise TypeError("integer argument expected")
        k = int(k.__index__() if hasattr(k, "__index__") else k)
        r = float(np.float32(float(r)))
        output_eigenvalues = int(output_eigenvalues)
        output_all_eigenvectors = int(output_all_eigenvectors)
        output_neighborhood_sizes = int(output_neighborhood_sizes)
        verbose = int(verbose)
        num_procs = int(num_procs)
    except (TypeError, ValueError, AttributeError, OverflowError) as e:
        raise RuntimeError("Failed to parse inputs") from e
    if not (k >= -(2 ** 31) and k < 2 ** 31):
        raise RuntimeError("Failed to parse inputs")

    # argument checks (estimate_normals.cpp:283-293)
    if r <= 0.0:
        raise ValueError("r must be positive")
    if k == 0:
        raise ValueError("k cannot be zero")
    if k < 0 and r == math.inf:
        raise ValueError("invalid combo: r == inf and k < 0")
    if k < -1:
        raise ValueError("k must be positive, or -1 for r-near neighborhoods")

    try:
        arr, n, ncol = as_points_2d(points, "estimate_normals()")
    except TypeError:
        raise TypeError("points must be interpretable as 0, 1 or 2-d array")
    use_torch = N.is_torch_cuda(arr)
    if use_torch:
        import torch
        if arr.dtype not in (torch.float32, torch.float64):
            raise TypeError("points must be float32 or float64")
        arr = arr.contiguous()
        np_dtype = np.dtype(np.float32) if arr.dtype == torch.float32 else np.dtype(np.float64)
        mem, stream, device = N.MEM_DEVICE, N.torch_stream(arr.device), arr.device
    else:
        if arr.dtype not in _FLOAT_CODES:
            raise TypeError("points must be float32 or float64")
        arr = np.ascontiguousarray(arr)
        np_dtype = arr.dtype
        mem, stream, device = N.MEM_HOST, None, None
    if ncol != 3:
        raise ValueError(f"points must have 3 columns (got {ncol})")

    sub = None
    if subsample is not None:
        sub_obj = subsample.cpu().numpy() if N.is_torch_cuda(subsample) else subsample
        sub = extract_indices(sub_obj, n)
        if sub is None:
            raise TypeError("subsample must be interpretable as specifying a subset of points")
        if use_torch:
            import torch
            sub = torch.from_numpy(sub).to(device)
    m = n if sub is None else int(sub.shape[0])

    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    num_eigen = 3 if output_all_eigenvectors else 1
    evecs = _alloc(use_torch, (m, 3) if num_eigen == 1 else (m, 3, 3), np_dtype, device)
    evals = _alloc(use_torch, (m,) if num_eigen == 1 else (m, 3), np_dtype, device) if output_eigenvalues else None
    sizes = _alloc(use_torch, (m,), np.int32, device) if output_neighborhood_sizes else None

    if verbose:
        print("(estimate_normals) using the GPU", file=sys.stdout)
        print("(estimate_normals) neighborhood parameters: ", file=sys.stdout)
        print(f"  k = {k}", file=sys.stdout)
        print(f"  r = {r:g}", file=sys.stdout)
    t0 = time.perf_counter()
    N.call("pptkg_estimate_normals", N.ptr(arr), int(n), _FLOAT_CODES[np_dtype], mem, int(k), ctypes.c_float(r),
           N.ptr(sub), int(m), num_eigen, PRECISIONS[precision], N.ptr(evecs), N.ptr(evals), N.ptr(sizes), stream,
           where="estimate_normals()")
    if verbose:
        print(f"(estimate_normals) build + PCA time (s): {time.perf_counter() - t0}", file=sys.stdout)

    if evals is None and sizes is None:
        return evecs
    return (evecs, evals, sizes)
