"""CPU checks of adapt's mask sequence in the oracle (mask_build in
oracle/oracle_wavelet.cpp: src/adapt.f90:14-65 without tree surgery).

Every step of the sequence is a monotone max-update driven by
|wavelet| >= threshold, so the masks are monotone in the thresholds; with
infinite thresholds nothing above level_start becomes active; with zero
thresholds every child patch is required."""
import numpy as np

from oracle.wavelet import ADJZONE, TOLRNZ, Hierarchy
from oracle.grid import Grid
from wavetrisk_hydrostatic_b200.cases import jet_state

LS, LE, NZ, PS = 3, 5, 2, 4


def _hierarchy(seed=1):
    G = Grid(LS, LE)
    levels = [G.level(l) for l in range(LS, LE + 1)]
    H = Hierarchy(levels, NZ)
    g = levels[-1]
    st = jet_state(g, NZ, seed=seed)
    H.set(LE, "s_m", st["mass"] + 50.0 * np.random.default_rng(seed).standard_normal((NZ, g.NN)))
    H.set(LE, "s_t", st["temp"])
    H.set(LE, "s_v", st["velo"])
    H.forward()
    return levels, H


def _masks(levels, H):
    return [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]


def _reset(levels, H):
    for g in levels:
        H.set(g.level, "mask_n", TOLRNZ)
        H.set(g.level, "mask_e", TOLRNZ)


def test_masks_monotone_in_threshold():
    levels, H = _hierarchy()
    out = []
    for scale in (1e-2, 2e-3):      # velocity thresholds; mass and Theta never active
        _reset(levels, H)
        thr = np.array([[1e9] * NZ, [1e9] * NZ, [scale] * NZ])
        req = H.mask_build(thr, level_fill=LS, max_level=LE + 1, patch_size=PS)
        out.append((_masks(levels, H), req))
    (m_hi, r_hi), (m_lo, r_lo) = out
    grew = 0
    for (a_n, a_e), (b_n, b_e) in zip(m_hi, m_lo):
        assert (b_n >= a_n).all() and (b_e >= a_e).all()
        grew += int((b_n > a_n).sum())
    assert grew > 0
    assert (r_lo >= r_hi).all()


def test_infinite_threshold_leaves_finer_levels_inactive():
    levels, H = _hierarchy()
    _reset(levels, H)
    H.mask_build(np.full((3, NZ), np.inf), level_fill=0, max_level=LE + 1, patch_size=PS)
    for g in levels[1:]:
        assert (H.field(g.level, "mask_n") < ADJZONE).all()
        assert (H.field(g.level, "mask_e") < ADJZONE).all()


def test_zero_threshold_requires_every_child():
    levels, H = _hierarchy()
    _reset(levels, H)
    req = H.mask_build(np.zeros((3, NZ)), level_fill=0, max_level=LE + 1, patch_size=PS)
    assert req.all()
    g = levels[-1]
    assert (H.field(LE, "mask_n")[g.owned] == TOLRNZ).all()
