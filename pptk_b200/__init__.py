"""pptk_b200: pptk's point-processing hot path on NVIDIA B200.

``pptk_b200.kdtree._build`` / ``pptk_b200.kdtree._query`` and
``pptk_b200.estimate_normals`` are drop-ins for ``pptk.kdtree._build`` /
``pptk.kdtree._query`` and ``pptk.estimate_normals``; all work runs in
hand-written sm_100a CUDA kernels behind the C ABI of ``include/pptkg.h``.
"""
from . import kdtree
from .estimate_normals import estimate_normals
from .pca import eigh3, eigh_list, nbhd_pca
from .points import Points, points

__all__ = ["kdtree", "estimate_normals", "eigh3", "eigh_list", "nbhd_pca", "Points", "points"]
__version__ = "0.1.0"
