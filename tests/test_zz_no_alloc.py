"""Allocation-free l2 norm entry point (wt_elliptic_l2_noalloc).

For hosts that cannot call cudaMalloc (a time loop running inside a memory
pool it does not control, or a code that must not grow its device footprint
after start-up): the caller passes device buffers it already owns and the
entry point uses a fixed device array for its partial sums.  Checked against
the handle-based wt_elliptic_l2 on two calls in a row, with the ghost remap
passed and with ghosts already filled on the host (nsrc = NULL), at level 5
and at level 8, the largest level the fixed array accepts."""
import ctypes as C

import numpy as np
import pytest

from wavetrisk_hydrostatic_b200 import Grid
from wavetrisk_hydrostatic_b200 import _native as N
from wavetrisk_hydrostatic_b200.cases import bathymetry
from wavetrisk_hydrostatic_b200.grid import halo_nodes
from wavetrisk_hydrostatic_b200.model import EllipticSolver


def _fn():
    f = N.lib().wt_elliptic_l2_noalloc
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_rejects_levels_beyond_the_fixed_scratch():
    # size check happens before any device work
    assert _fn()(9, 2, None, C.c_void_p(1), C.c_void_p(1), None) == N.WT_ERR_ARG


@pytest.fixture(scope="module")
def grids():
    g = Grid(4, 8, radius=6371e3)
    return {5: [g.level(4), g.level(5)], 8: [g.level(7), g.level(8)]}


@pytest.mark.gpu
@pytest.mark.parametrize("level", [5, 8])
@pytest.mark.parametrize("remap", [True, False], ids=["nsrc", "nsrc_null"])
def test_noalloc_l2_matches_handle_l2_twice(grids, level, remap):
    import torch

    levels = grids[level]
    topos = [bathymetry(lv, seed=4) for lv in levels]
    S = EllipticSolver(levels, topos)
    rng = np.random.default_rng(12 + level)
    f = np.concatenate([rng.standard_normal(lv.NN) for lv in levels])
    for q, lv in enumerate(levels):
        halo_nodes(lv, f[S.offsets[q]:S.offsets[q + 1]])
    fn = _fn()
    dev = torch.device("cuda", 0)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    lv = levels[1]
    nsrc_d = None
    if remap:
        nsrc = np.arange(lv.NN, dtype=np.int32)
        nsrc[lv.halo_node[:, 0]] = lv.halo_node[:, 1]
        nsrc_d = torch.from_numpy(nsrc).to(dev)
    for trial in range(2):
        f = f * (1.0 + trial)
        S.upload(f=f)
        ref = S.l2(level, which=1)
        seg = np.ascontiguousarray(f[S.offsets[1]:S.offsets[2]])
        if remap:
            # ghosts hold garbage: the remap alone must supply their values
            seg = seg.copy()
            seg[lv.halo_node[:, 0]] = 1e30
        seg_d = torch.from_numpy(seg).to(dev)
        rc = fn(level, 2, C.c_void_p(nsrc_d.data_ptr()) if remap else None, C.c_void_p(seg_d.data_ptr()),
                C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == N.WT_OK
        torch.cuda.synchronize(dev)
        got = float(out.item())
        assert abs(got / ref - 1) <= 1e-12, (level, remap, trial, got, ref)
    S.close()
