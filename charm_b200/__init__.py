"""charm_b200: CHarm's point and cell (block-mean) spherical-harmonic
synthesis and analysis on NVIDIA B200 (sm_100a).

The C ABI lives in libcharm.so (include/charm_b200.h); this package exposes
it to Python with PyHarm's names (see charm_b200.pyharm).  The library is
loaded on first use of any of those names, and that fails loudly when
libcharm.so has not been built.  `charm_b200.workloads` (the seeded
synthetic inputs) needs no library.
"""
_PYHARM = ("CHarmError", "GRID", "GRID_DH1", "GRID_DH2", "GRID_GL",
           "SCATTERED", "PointGrid", "PointGridDH1", "PointGridDH2",
           "PointGridGL", "PointSctr", "Shc", "sha_point", "shs_point",
           "shs_point_grad1", "shs_point_grad2", "shs_point_guru",
           "CELL_GRID", "CELL_SCATTERED", "SHA_CELL_AQ", "CellGrid",
           "CellSctr", "shs_cell", "sha_cell", "gfm_global_density_3d",
           "gfm_global_density_lateral", "gfm_global_density_const")

__all__ = list(_PYHARM) + ["LIB_PATH"]


def __getattr__(name):
    if name in _PYHARM:
        from . import pyharm
        return getattr(pyharm, name)
    if name == "LIB_PATH":
        from ._lib import LIB_PATH
        return LIB_PATH
    raise AttributeError("module 'charm_b200' has no attribute %r" % name)
