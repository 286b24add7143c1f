"""Allocation-free l2 norm entry point (wt_elliptic_l2_noalloc).

For hosts that cannot call cudaMalloc (a time loop running inside a memory
pool it does not control, or a code that must not grow its device footprint
after start-up): the caller passes device buffers it already owns and the
entry point uses a fixed device array for its partial sums.  Checked against
the handle-based wt_elliptic_l2 on two calls in a row."""
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


@pytest.mark.gpu
def test_noalloc_l2_matches_handle_l2_twice():
    import torch

    g = Grid(4, 5, radius=6371e3)
    levels = [g.level(4), g.level(5)]
    topos = [bathymetry(lv, seed=4) for lv in levels]
    S = EllipticSolver(levels, topos)
    rng = np.random.default_rng(12)
    f = np.concatenate([rng.standard_normal(lv.NN) for lv in levels])
    for q, lv in enumerate(levels):
        halo_nodes(lv, f[S.offsets[q]:S.offsets[q + 1]])
    fn = _fn()
    dev = torch.device("cuda", 0)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for trial in range(2):
        f = f * (1.0 + trial)
        S.upload(f=f)
        lv = levels[1]
        ref = S.l2(5, which=1)
        nsrc = np.arange(lv.NN, dtype=np.int32)
        nsrc[lv.halo_node[:, 0]] = lv.halo_node[:, 1]
        nsrc_d = torch.from_numpy(nsrc).to(dev)
        seg = torch.from_numpy(np.ascontiguousarray(f[S.offsets[1]:S.offsets[2]])).to(dev)
        rc = fn(5, 2, C.c_void_p(nsrc_d.data_ptr()), C.c_void_p(seg.data_ptr()), C.c_void_p(out.data_ptr()),
                C.c_void_p(stream.cuda_stream))
        assert rc == N.WT_OK
        torch.cuda.synchronize(dev)
        got = float(out.item())
        assert abs(got / ref - 1) <= 1e-12, (trial, got, ref)
    S.close()
