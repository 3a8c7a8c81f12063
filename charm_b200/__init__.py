"""charm_b200: CHarm's point spherical-harmonic synthesis and analysis on
NVIDIA B200 (sm_100a).

The C ABI lives in libcharm.so (include/charm_b200.h); this package exposes
it to Python with PyHarm's names (see charm_b200.pyharm).  Importing fails
loudly when libcharm.so has not been built.
"""
from .pyharm import (CHarmError, GRID, GRID_DH1, GRID_DH2, GRID_GL, SCATTERED,
                     PointGrid, PointGridDH1, PointGridDH2, PointGridGL,
                     PointSctr, Shc, sha_point, shs_point, shs_point_grad1,
                     shs_point_grad2, shs_point_guru)
from ._lib import LIB_PATH

__all__ = ["CHarmError", "GRID", "GRID_DH1", "GRID_DH2", "GRID_GL",
           "SCATTERED", "PointGrid", "PointGridDH1", "PointGridDH2",
           "PointGridGL", "PointSctr", "Shc", "sha_point", "shs_point",
           "shs_point_grad1", "shs_point_grad2", "shs_point_guru", "LIB_PATH"]
