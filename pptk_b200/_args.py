"""Argument conversion with the reference's rules and error types.

Restates the numpy-side helpers of ``pptk/include/python_util.h`` that the
hot path's Python boundary relies on: the 2-D array view
(``CheckAndExtractArray2D``, :252-352), the float rounding of ``dmax``
(``CastAsDouble``, :393-400) and index extraction from lists, integer arrays
and boolean masks with negative-index wrapping (``CheckAndExtractIndices``,
:576-610).
"""
import numbers

import numpy as np

from ._native import is_torch_cuda

_INT_KINDS = "iu"


def as_points_2d(data, where):
    """Returns (array_or_tensor, m, n) for a 0/1/2-d numeric array or scalar
    (CheckAndExtractArray2D): a 1-d array is one row, a scalar is 1 x 1."""
    if is_torch_cuda(data):
        t = data
        if t.dim() == 0:
            t = t.reshape(1, 1)
        elif t.dim() == 1:
            t = t.reshape(1, -1)
        elif t.dim() != 2:
            raise ValueError(f"{where}: only handles ndim of 0, 1 or 2; encountered ndim={data.dim()}")
        return t, int(t.shape[0]), int(t.shape[1])
    if isinstance(data, np.ndarray):
        a = data
    elif isinstance(data, (numbers.Number, np.generic)) and not isinstance(data, (str, bytes)):
        a = np.asarray(data)
    else:
        raise TypeError(f"{where}: points array type {type(data).__name__} unsupported")
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a.reshape(1, -1)
    elif a.ndim != 2:
        raise ValueError(f"ExtractArray2DFromPyArray(): only handles ndim of 0, 1 or 2; encountered ndim={a.ndim}")
    return a, a.shape[0], a.shape[1]


def cast_as_long(obj, what):
    """int(obj), as PyNumber_Long (python_util.h:354-369)."""
    try:
        return int(obj)
    except (TypeError, ValueError):
        raise
    except Exception as e:  # pragma: no cover - defensive
        raise RuntimeError(f"Query(): could not interpret {what} of type {type(obj).__name__} as C long.") from e


def cast_as_float_rounded(obj):
    """float(obj) rounded through float32, as CastAsDouble (python_util.h:393-400)."""
    return float(np.float32(float(obj)))


def _ints_from_list(obj):
    out = []
    for i, item in enumerate(obj):
        try:
            out.append(int(item.__index__()) if not isinstance(item, (bool, np.bool_)) else int(item))
        except (AttributeError, TypeError):
            raise TypeError(
                f"ExtractIndicesFromPyList(): Encountered non-index {type(item).__name__} object at the {i}-th item")
    return np.asarray(out, dtype=np.int64)


def extract_indices(obj, n):
    """Query / subsample indices as int32 in [0, n) (CheckAndExtractIndices).

    * list: every item must be an index (TypeError otherwise);
    * numpy bool array: a mask of length n (ValueError otherwise);
    * numpy integer array (0-d or 1-d): the indices themselves;
    * integer scalar: one index.
    Indices must lie in [-n, n-1] (RuntimeError otherwise); negatives wrap.
    Returns None when obj is of none of these kinds."""
    if isinstance(obj, list):
        idx = _ints_from_list(obj)
    elif isinstance(obj, np.ndarray):
        if obj.ndim > 1:
            raise ValueError(f"ExtractIndicesFromPyArray(): PyArray has dim = {obj.ndim} (expected dim = 0 or 1).")
        a = obj.reshape(-1)
        if a.dtype == np.bool_:
            if a.shape[0] != n:
                raise ValueError(
                    f"ExtractIndicesFromPyArray(): binary indexing mask has incorrect size {a.shape[0]} "
                    f"(expected {n}).")
            idx = np.flatnonzero(a).astype(np.int64)
        elif a.dtype.kind in _INT_KINDS:
            idx = a.astype(np.int64)
        else:
            raise ValueError(
                f"ExtractIndicesFromPyArray(): encountered unsupported type_num (dtype {a.dtype}) "
                "(expected boolean or integral type).")
    elif isinstance(obj, (bool, np.bool_)):
        idx = np.asarray([int(obj)], dtype=np.int64)
    elif isinstance(obj, (numbers.Integral, np.integer)):
        idx = np.asarray([int(obj)], dtype=np.int64)
    elif isinstance(obj, (numbers.Real, np.floating)):
        raise ValueError("CheckAndExtractIndices(): encountered non-integral scalar (float).")
    else:
        return None
    bad = np.flatnonzero((idx < -n) | (idx >= n))
    if bad.size:
        raise RuntimeError(f"CheckAndExtractIndices(): {int(bad[0])}-th query index is outside of [{-n},{n - 1}]")
    idx = np.where(idx < 0, idx + n, idx)
    return np.ascontiguousarray(idx, dtype=np.int32)
