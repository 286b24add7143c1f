"""CPU checks of the wavelet oracle (oracle/oracle_wavelet.cpp) and of the
outer velocity weights I_u_wgt built by the grid builder.

The reference ships no golden vectors for these routines, so the oracle is
pinned by the properties its algorithm guarantees:
  * velocity: inverse(forward(u)) = u to round-off ("to ensure
    Restriction(Prolongation) = Identity", src/wavelet.f90:694,974), and the
    wavelets of a smooth field fall by 4x per level (second-order interpolation,
    which a wrong weight or stencil index would destroy);
  * scalars: inverse(forward(s)) differs from s at coarse-grid nodes by exactly
    the lifting term Prolong_scalar leaves out (src/wavelet.f90:593-605 sums 11
    of the 12 terms of Restrict_scalar);
  * mask_tol_vars agrees with a numpy statement of src/mask.f90:102-156.
"""
import numpy as np
import pytest

from oracle.wavelet import ADJZONE, FROZEN, TOLRNZ, Hierarchy
from oracle.grid import Grid
from wavetrisk_hydrostatic_b200.cases import edge_velocity, solid_body_rotation
from wavetrisk_hydrostatic_b200.grid import halo_edges, halo_nodes


def _random_state(H, g, nz, seed):
    rng = np.random.default_rng(seed)
    sm = rng.standard_normal((nz, g.NN))
    st = rng.standard_normal((nz, g.NN))
    sv = rng.standard_normal((nz, 3 * g.NN))
    halo_nodes(g, sm)
    halo_nodes(g, st)
    halo_edges(g, sv)
    return sm, st, sv


def _owned_edges(g):
    own = np.nonzero(g.owned)[0]
    return np.concatenate([own, own + g.NN, own + 2 * g.NN])


def test_velocity_round_trip_is_identity():
    G = Grid(4, 6)
    levels = [G.level(l) for l in (4, 5, 6)]
    nz = 2
    H = Hierarchy(levels, nz)
    g = levels[-1]
    sm, st, sv = _random_state(H, g, nz, 3)
    H.set(6, "s_m", sm)
    H.set(6, "s_t", st)
    H.set(6, "s_v", sv)
    H.forward()
    H.inverse()
    e = _owned_edges(g)
    err = np.abs(H.field(6, "s_v")[:, e] - sv[:, e]).max() / np.abs(sv[:, e]).max()
    assert err < 1e-13


def test_scalar_round_trip_misses_one_lifting_term():
    G = Grid(4, 5)
    levels = [G.level(4), G.level(5)]
    nz = 1
    H = Hierarchy(levels, nz)
    Pa, C = levels
    sm, st, sv = _random_state(H, C, nz, 5)
    H.set(5, "s_m", sm)
    H.set(5, "s_t", st)
    H.set(5, "s_v", sv)
    H.forward()
    wc = H.field(5, "w_m").copy()
    halo_nodes(C, wc)
    H.inverse()
    out = H.field(5, "s_m")
    # even child nodes (2ip, 2jp) of parents [0, n_par)^2: prolong - original = wc(id2NE) a4(id2NE) hex_inv_par
    d, ip, jp = np.meshgrid(np.arange(10), np.arange(Pa.n), np.arange(Pa.n), indexing="ij")
    d, ip, jp = d.ravel(), ip.ravel(), jp.ravel()
    kc = C.idx(d, 2 * ip, 2 * jp)
    k2 = C.idx(d, 2 * ip + 1, 2 * jp + 2)
    kp = Pa.idx(d, ip, jp)
    predicted = wc[0, k2] * C.overl_a[3, k2] * Pa.hex_inv[kp]
    diff = out[0, kc] - sm[0, kc]
    assert np.abs(predicted).max() > 1e-3                       # the term is not negligible
    assert np.abs(diff - predicted).max() < 1e-12 * np.abs(sm).max()


@pytest.mark.parametrize("lmax", [5, 6])
def test_smooth_velocity_wavelets_are_second_order(lmax):
    G = Grid(3, lmax)
    levels = [G.level(l) for l in range(3, lmax + 1)]
    H = Hierarchy(levels, 1)
    g = levels[-1]
    v = edge_velocity(g, solid_body_rotation(1.0))[None, :]
    H.set(lmax, "s_v", v)
    H.forward()
    peaks = []
    for q, l in enumerate(range(4, lmax + 1)):
        gl = levels[l - 3]
        peaks.append(np.abs(H.field(l, "w_v")[:, _owned_edges(gl)]).max())
    for a, b in zip(peaks[:-1], peaks[1:]):
        assert 3.5 < a / b < 4.5
    assert peaks[-1] < 5e-3


def _np_mask_tol(levels, wav, masks, thr, level_fill, nz):
    """numpy statement of mask_tol_vars over the mask_active ranges."""
    out = []
    le = levels[-1].level
    for g, (wm, wt, wv), (mn, me) in zip(levels, wav, masks):
        wm, wt, wv = wm.copy(), wt.copy(), wv.copy()
        halo_nodes(g, wm)
        halo_nodes(g, wt)
        halo_edges(g, wv)
        st, en = (0, 1) if g.level == le else (-1, 2)
        _, i, j = g.ij()
        sel = (i >= st) & (j >= st) & (i <= g.n - 1 + en) & (j <= g.n - 1 + en) & (mn != FROZEN)
        below = g.level < level_fill
        act = below | (np.abs(wm) >= thr[0][:, None]).any(0) | (np.abs(wt) >= thr[1][:, None]).any(0)
        mn2 = mn.copy()
        mn2[sel & act] = TOLRNZ
        mn2[sel & ~act & (mn > ADJZONE)] = ADJZONE
        me2 = me.copy().reshape(3, g.NN)
        wv3 = np.abs(wv).reshape(nz, 3, g.NN)
        for e in range(3):
            a = below | (wv3[:, e, :] >= thr[2][:, None]).any(0)
            m = me2[e]
            m[sel & a] = TOLRNZ
            m[sel & ~a & (m > ADJZONE)] = ADJZONE
        out.append((mn2, me2.ravel()))
    return out


@pytest.mark.parametrize("level_fill", [0, 5])
def test_mask_tol_vars_matches_numpy(level_fill):
    G = Grid(4, 6)
    levels = [G.level(l) for l in (4, 5, 6)]
    nz = 3
    H = Hierarchy(levels, nz)
    rng = np.random.default_rng(11)
    wav, masks = [], []
    for g in levels:
        w = (rng.standard_normal((nz, g.NN)) * 1e-2, rng.standard_normal((nz, g.NN)) * 1e-2,
             rng.standard_normal((nz, 3 * g.NN)) * 1e-2)
        m = (rng.choice([0, 8, 12, 16, 32], size=g.NN).astype(np.int32),
             rng.choice([0, 8, 12, 16, 32], size=3 * g.NN).astype(np.int32))
        for name, a in zip(("w_m", "w_t", "w_v", "mask_n", "mask_e"), w + m):
            H.set(g.level, name, a)
        wav.append(w)
        masks.append(m)
    thr = np.abs(rng.standard_normal((3, nz))) * 1e-2
    expect = _np_mask_tol(levels, wav, masks, thr, level_fill, nz)
    H.mask_tol(thr, level_fill)
    for g, (mn, me) in zip(levels, expect):
        assert np.array_equal(H.field(g.level, "mask_n"), mn)
        assert np.array_equal(H.field(g.level, "mask_e"), me)


def test_wt_after_step_on_active_grid_reproduces_velocity():
    G = Grid(4, 6)
    levels = [G.level(l) for l in (4, 5, 6)]
    nz = 1
    H = Hierarchy(levels, nz)
    g = levels[-1]
    sm, st, sv = _random_state(H, g, nz, 9)
    H.set(6, "s_m", sm)
    H.set(6, "s_t", st)
    H.set(6, "s_v", sv)
    H.forward()                      # coarse scaling consistent with the fine level
    H.wt_after_step()
    e = _owned_edges(g)
    assert np.abs(H.field(6, "s_v")[:, e] - sv[:, e]).max() < 1e-13 * np.abs(sv).max()


def test_outer_velocity_weights_cover_the_outer_child_edges():
    G = Grid(4, 5)
    g = G.level(5)
    d, i, j = g.ij()
    has = np.abs(g.iu_wgt).sum(0) > 0
    # RT weights at (odd, even), DG at (even, even), UP at (even, odd) children of parents [0, n/2)^2
    role = ((i % 2 == 1) & (j % 2 == 0)) | ((i % 2 == 0) & (j % 2 == 0)) | ((i % 2 == 0) & (j % 2 == 1))
    inside = (i >= 0) & (j >= 0) & (i < g.n) & (j < g.n)
    assert not has[~(role & inside)].any()
    assert has[role & inside].sum() >= 0.99 * (role & inside).sum()
    assert np.isfinite(g.iu_wgt).all() and np.abs(g.iu_wgt).max() < 0.1
