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
