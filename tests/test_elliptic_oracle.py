"""CPU checks of the elliptic oracle: operator identities, conservative
restriction, prolongation of constants, and multigrid convergence."""
import numpy as np
import pytest

from oracle.elliptic import Hierarchy
from oracle.grid import Grid
from wavetrisk_hydrostatic_b200.cases import bathymetry, elliptic_rhs
from wavetrisk_hydrostatic_b200.grid import halo_nodes


@pytest.fixture(scope="module")
def setup():
    g = Grid(4, 6, radius=6371e3)
    levels = [g.level(l) for l in (4, 5, 6)]
    topos = [bathymetry(lv, seed=1) for lv in levels]
    return g, levels, topos


def ml(levels, fn):
    return np.concatenate([fn(lv) for lv in levels])


def area_sum(lv, x):
    own = lv.owned.copy()
    n, s = lv.pole_ids()
    own[n] = own[s] = True
    return (x[own] / lv.hex_inv[own]).sum()


def test_operator_of_constant_is_minus_constant(setup):
    g, levels, topos = setup
    H = Hierarchy(levels, topos)
    off = np.cumsum([0] + [lv.NN for lv in levels])
    q = np.full(off[-1], 2.5)
    out = H.apply(6, q)
    lv = levels[2]
    seg = out[off[2]:off[3]][lv.owned]
    assert np.allclose(seg, -2.5, rtol=1e-12, atol=1e-12)   # div(grad const) = 0


def test_divergence_form_conserves(setup):
    # sum over cells of area*(L q + q) = theta dt^2 * sum(area div F) = 0
    g, levels, topos = setup
    H = Hierarchy(levels, topos)
    off = np.cumsum([0] + [lv.NN for lv in levels])
    rng = np.random.default_rng(0)
    q = np.zeros(off[-1])
    lv = levels[2]
    seg = rng.standard_normal(lv.NN)
    halo_nodes(lv, seg)
    q[off[2]:off[3]] = seg
    out = H.apply(6, q)
    lq = out[off[2]:off[3]] + seg
    scale = np.abs(lq[lv.owned] / lv.hex_inv[lv.owned]).sum()
    assert abs(area_sum(lv, lq)) < 1e-12 * scale


def test_restriction_conserves_mass(setup):
    # Restrict_scalar lifts with overlap areas: the area integral is preserved
    # (the reference's check_m, src/wavelet.f90:1707)
    g, levels, topos = setup
    H = Hierarchy(levels, topos)
    off = np.cumsum([0] + [lv.NN for lv in levels])
    s = np.zeros(off[-1])
    s[off[2]:off[3]] = elliptic_rhs(levels[2], seed=3) + 1.0
    r = H.restrict_all(s)
    m6 = area_sum(levels[2], r[off[2]:off[3]])
    m5 = area_sum(levels[1], r[off[1]:off[2]])
    m4 = area_sum(levels[0], r[off[0]:off[1]])
    assert abs(m5 / m6 - 1) < 1e-3 and abs(m4 / m6 - 1) < 1e-3


def test_prolong_reproduces_constants(setup):
    g, levels, topos = setup
    H = Hierarchy(levels, topos)
    off = np.cumsum([0] + [lv.NN for lv in levels])
    s = np.zeros(off[-1])
    s[off[1]:off[2]] = 1.0
    p = H.prolong(6, s)
    seg = p[off[2]:off[3]][levels[2].owned]
    assert np.allclose(seg, 1.0, atol=2e-2)


@pytest.mark.parametrize("method", ["fmg", "srj"])
def test_solver_reaches_tolerance(setup, method):
    g, levels, topos = setup
    H = Hierarchy(levels, topos, fine_tol=1e-8, coarse_tol=1e-8, max_vcycle=30, coarse_iter=200, max_srj_iter=400)
    off = np.cumsum([0] + [lv.NN for lv in levels])
    f = np.zeros(off[-1])
    f[off[2]:off[3]] = elliptic_rhs(levels[2], seed=5)
    f = H.restrict_all(f)
    u, nrm, its = H.solve(np.zeros(off[-1]), f, method)
    assert nrm[-1, 1] <= 1e-8, (nrm, its)
