"""GPU parity of the wavelet transforms, threshold mask, compression and
WT_after_step (csrc/wt_wavelet.cu through the C-ABI) against the CPU oracle
(oracle/oracle_wavelet.cpp) on the same seeded inputs.

Fields are compared on owned nodes / edges ([0, n)^2 of every lozenge) of
every level, bit for bit (FP64, no FMA contraction); masks are compared
exactly."""
import numpy as np
import pytest

from oracle.wavelet import Hierarchy
from wavetrisk_hydrostatic_b200 import Grid
from wavetrisk_hydrostatic_b200.grid import halo_edges, halo_nodes
from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

pytestmark = pytest.mark.gpu
TOL = 0.0   # bit for bit: FP64 without FMA contraction, the oracle's operand order
NAMES = {"mass": "s_m", "temp": "s_t", "velo": "s_v", "wc_mass": "w_m", "wc_temp": "w_t", "wc_velo": "w_v"}


def _setup(lmin, lmax, nz):
    G = Grid(lmin, lmax)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    topos = [np.full(g.NN, -4000.0) for g in levels]
    return levels, Hierarchy(levels, nz), WaveletHierarchy(levels, topos, nz)


def _owned(g, name):
    own = np.nonzero(g.owned)[0]
    return np.concatenate([own, own + g.NN, own + 2 * g.NN]) if name.endswith("velo") else own


def _put(levels, orc, dev, level, name, a):
    orc.set(level, NAMES.get(name, name), a)
    dev.upload(level, name, a)


def _compare(levels, orc, dev, names):
    for g in levels:
        for name in names:
            o = orc.field(g.level, NAMES[name])
            d = dev.download(g.level, name)
            k = _owned(g, name)
            scale = max(np.abs(o[:, k]).max(), 1e-300)
            err = np.abs(d[:, k] - o[:, k]).max() / scale
            assert err <= TOL, (g.level, name, err)


def _random_fine(levels, orc, dev, nz, seed, smooth=False):
    g = levels[-1]
    rng = np.random.default_rng(seed)
    sm, st = rng.standard_normal((nz, g.NN)), rng.standard_normal((nz, g.NN))
    sv = rng.standard_normal((nz, 3 * g.NN))
    halo_nodes(g, sm)
    halo_nodes(g, st)
    halo_edges(g, sv)
    for name, a in (("mass", sm), ("temp", st), ("velo", sv)):
        _put(levels, orc, dev, g.level, name, a)


def _random_masks(levels, orc, dev, seed):
    rng = np.random.default_rng(seed)
    for g in levels:
        mn = rng.choice([0, 8, 12, 16, 32], size=g.NN, p=[0.1, 0.2, 0.1, 0.5, 0.1]).astype(np.int32)
        me = rng.choice([0, 8, 12, 16, 32], size=3 * g.NN, p=[0.1, 0.2, 0.1, 0.5, 0.1]).astype(np.int32)
        _put(levels, orc, dev, g.level, "mask_n", mn)
        _put(levels, orc, dev, g.level, "mask_e", me)


@pytest.mark.parametrize("lmin,lmax,nz", [(3, 5, 2), (4, 6, 1)])
def test_forward_transform_matches_oracle(lmin, lmax, nz):
    levels, orc, dev = _setup(lmin, lmax, nz)
    _random_fine(levels, orc, dev, nz, seed=lmax)
    orc.forward()
    dev.forward()
    _compare(levels, orc, dev, NAMES)
    dev.close()


def test_forward_transform_with_masks_matches_oracle():
    levels, orc, dev = _setup(3, 5, 2)
    _random_fine(levels, orc, dev, 2, seed=21)
    _random_masks(levels, orc, dev, seed=22)
    orc.forward()
    dev.forward()
    _compare(levels, orc, dev, NAMES)
    dev.close()


@pytest.mark.parametrize("masks", [False, True])
def test_inverse_transform_matches_oracle(masks):
    levels, orc, dev = _setup(3, 5, 2)
    rng = np.random.default_rng(31)
    for g in levels:
        for name in ("mass", "temp", "velo", "wc_mass", "wc_temp", "wc_velo"):
            a = rng.standard_normal((2, (3 if name.endswith("velo") else 1) * g.NN))
            if name.endswith("velo"):
                halo_edges(g, a)
            else:
                halo_nodes(g, a)
            _put(levels, orc, dev, g.level, name, a)
    if masks:
        _random_masks(levels, orc, dev, seed=32)
    orc.inverse()
    dev.inverse()
    _compare(levels, orc, dev, ("mass", "temp", "velo"))
    dev.close()


@pytest.mark.parametrize("level_fill", [0, 4])
def test_mask_tol_vars_matches_oracle_exactly(level_fill):
    levels, orc, dev = _setup(3, 5, 3)
    _random_fine(levels, orc, dev, 3, seed=41)
    _random_masks(levels, orc, dev, seed=42)
    orc.forward()
    dev.forward()
    thr = np.abs(np.random.default_rng(43).standard_normal((3, 3))) * 0.3
    orc.mask_tol(thr, level_fill)
    dev.mask_tol_vars(thr, level_fill)
    for g in levels:
        for name in ("mask_n", "mask_e"):
            assert np.array_equal(dev.download(g.level, name), orc.field(g.level, name)), (g.level, name)
    dev.close()


def test_compress_and_wt_after_step_match_oracle():
    levels, orc, dev = _setup(3, 5, 2)
    _random_fine(levels, orc, dev, 2, seed=51)
    orc.forward()
    dev.forward()
    thr = np.full((3, 2), 0.5)
    orc.mask_tol(thr, 0)
    dev.mask_tol_vars(thr, 0)
    orc.compress()
    dev.compress()
    _compare(levels, orc, dev, ("wc_mass", "wc_temp", "wc_velo"))
    orc.wt_after_step()
    dev.wt_after_step()
    _compare(levels, orc, dev, NAMES)
    assert dev.status() == 0
    dev.close()


def test_wt_after_step_after_wavelet_upload_matches_oracle():
    """WT_after_step starts from zeroed wavelets (zero_float): wavelets uploaded
    from the host into every slot (parent-coincident nodes and the coarsest
    level included) must not survive it, on the direct path nor in the graph
    of the adaptive step."""
    levels, orc, dev = _setup(3, 5, 2)
    _random_fine(levels, orc, dev, 2, seed=53)
    orc.forward()
    dev.forward()
    thr = np.full((3, 2), 0.5)
    orc.mask_tol(thr, 0)
    dev.mask_tol_vars(thr, 0)
    rng = np.random.default_rng(7)
    for g in levels:
        for name in ("wc_mass", "wc_temp", "wc_velo"):
            a = rng.standard_normal(orc.field(g.level, NAMES[name]).shape)
            orc.set(g.level, NAMES[name], a)
            dev.upload(g.level, name, a)
    orc.wt_after_step()
    dev.wt_after_step()
    _compare(levels, orc, dev, NAMES)
    for g in levels:  # parent-coincident slots and the coarsest level hold 0
        w = dev.download(g.level, "wc_mass")
        own = np.nonzero(g.owned)[0]
        d, r = np.divmod(own, g.P * g.P)
        j, i = np.divmod(r, g.P)
        even = own[((i - 2) % 2 == 0) & ((j - 2) % 2 == 0)]
        assert not np.any(w[:, even]), g.level
    orc.mask_tol(thr, 0)
    dev.mask_tol_vars(thr, 0)
    for g in levels:
        for name in ("mask_n", "mask_e"):
            assert np.array_equal(dev.download(g.level, name), orc.field(g.level, name)), (g.level, name)
    assert dev.status() == 0
    dev.close()


@pytest.mark.parametrize("level_fill,scale", [(3, 0.3), (0, 0.05), (4, 1.0)])
def test_mask_build_matches_oracle_exactly(level_fill, scale):
    """adapt's mask sequence: every node and edge mask of every level (ghost
    slots included) and every check_child_required flag equal the oracle's."""
    levels, orc, dev = _setup(3, 5, 2)
    _random_fine(levels, orc, dev, 2, seed=61)
    orc.forward()
    dev.forward()
    thr = np.full((3, 2), scale)
    rq_o = orc.mask_build(thr, level_fill, 6, patch_size=4)
    rq_d = dev.mask_build(thr, level_fill, 6, patch_size=4)
    for g in levels:
        for name in ("mask_n", "mask_e"):
            assert np.array_equal(dev.download(g.level, name), orc.field(g.level, name)), (g.level, name)
    assert np.array_equal(rq_d, rq_o)
    assert rq_o.sum() > 0
    dev.close()


def test_batched_transfers_match_single_field_transfers():
    """wt_upload_fields / wt_download_fields move the same bytes as the
    per-field calls, ghost copies included."""
    levels, orc, dev = _setup(3, 5, 2)
    _random_fine(levels, orc, dev, 2, seed=71)
    dev.forward()
    names = ("mass", "temp", "velo", "wc_mass", "wc_temp", "wc_velo", "mask_n", "mask_e")
    single = {(g.level, f): dev.download(g.level, f) for g in levels for f in names}
    outs = {k: np.empty_like(v) for k, v in single.items()}
    dev.download_many([(l, f, outs[(l, f)]) for (l, f) in outs])
    for k in single:
        assert np.array_equal(single[k], outs[k]), k
    rng = np.random.default_rng(5)
    new = {(g.level, f): rng.standard_normal(single[(g.level, f)].shape) for g in levels for f in ("mass", "velo")}
    dev.upload_many([(l, f, a) for (l, f), a in new.items()])
    for (l, f), a in new.items():
        own = np.nonzero(levels[l - levels[0].level].owned)[0]
        g = levels[l - levels[0].level]
        k = np.concatenate([own, own + g.NN, own + 2 * g.NN]) if f == "velo" else own
        assert np.array_equal(dev.download(l, f)[:, k], a[:, k]), (l, f)
    assert dev.status() == 0
    dev.close()
