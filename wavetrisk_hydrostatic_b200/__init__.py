"""B200-native implementation of WAVETRISK's data-parallel hot path.

TRiSK operators (src/ops.f90, src/multi_level.f90), wavelet lifting transforms
and threshold mask (src/wavelet.f90, src/mask.f90, src/adapt.f90) and the
multigrid free-surface solve (src/lin_solve.f90, src/barotropic_2d.f90) on the
padded lozenge layout, behind the C-ABI of include/wavetrisk_gpu.h.
"""
from .grid import Grid, LevelGeom, halo_edges, halo_nodes  # noqa: F401
from .cases import OceanParams, jet_state  # noqa: F401

__all__ = ["Grid", "LevelGeom", "OceanParams", "jet_state", "halo_nodes", "halo_edges"]
