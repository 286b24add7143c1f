"""CPU checks of the compute-or-restrict oracle (oracle/oracle_restrict.cpp)
and of the flux-restriction weights R_F_wgt built with the grid.

The flux restriction is pinned by two properties of the reference's scheme
(src/multi_level.f90:394-659):
  * a divergence-free child flux (differences of a stream function at the
    circumcentres) restricts to a divergence-free parent flux, to rounding;
  * for a smooth potential flow the restricted parent flux converges to the
    parent flux computed directly, faster than first order (the dscalar terms
    of part_coarse_flux and coarse_flux carry the second-order correction).
The two writers of a shared R_F_wgt slot agree to rounding, and the scalar
and velocity-trend restrictions follow their masks."""
import numpy as np
import pytest

from oracle.restrict import ADJZONE, RESTRCT, Pair, _nodes, div
from oracle.grid import Grid
from wavetrisk_hydrostatic_b200.grid import halo_edges, halo_nodes


@pytest.fixture(scope="module")
def grid():
    return Grid(3, 6)


def _stream_flux(g):
    """(psi(t2) - psi(t1)) across every owned edge: discretely divergence free."""
    c = g.ccentre / 6.37e6
    psi = c[:, 0, :] + 0.3 * c[:, 2, :] * c[:, 1, :]
    NN, P = g.NN, g.P
    F = np.zeros((1, 3 * NN))
    ids = _nodes(g, 0, g.n)
    F[0, ids] = psi[0, ids] - psi[1, ids - P]
    F[0, NN + ids] = -(psi[1, ids] - psi[0, ids])
    F[0, 2 * NN + ids] = -(psi[1, ids] - psi[0, ids - 1])
    halo_edges(g, F)
    return F


def _potential_flux(g):
    """grad(phi) . n * pedlen of a smooth node potential (step1 itype 1)."""
    x = g.node / 6.37e6
    phi = x[0] + 0.5 * x[2] * x[1] + 0.2 * x[2] ** 2
    NN, P = g.NN, g.P
    F = np.zeros((1, 3 * NN))
    ids = _nodes(g, 0, g.n)
    F[0, ids] = (phi[ids + 1] - phi[ids]) / g.len[0, ids] * g.pedlen[0, ids]
    F[0, NN + ids] = (phi[ids] - phi[ids + P + 1]) / g.len[1, ids] * g.pedlen[1, ids]
    F[0, 2 * NN + ids] = (phi[ids + P] - phi[ids]) / g.len[2, ids] * g.pedlen[2, ids]
    halo_edges(g, F)
    return F


def _restrict(par, chd, F):
    pr = Pair(par, chd, 1)
    ds = -div(chd, F)  # scalar_trend: dscalar = -div(h_flux)
    halo_nodes(chd, ds)
    pr.field(1, "flux")[...] = F
    pr.field(1, "dscal")[...] = ds
    oob = pr.restrict_flux()
    Fp = pr.field(0, "flux").copy()
    halo_edges(par, Fp)
    return Fp, oob


def _owned_edges(g):
    own = np.nonzero(g.owned)[0]
    return own, np.concatenate([own, own + g.NN, own + 2 * g.NN])


def test_rf_weights_shared_slots_agree(grid):
    for l in range(3, 7):
        g = grid.level(l)
        assert g.rf_wgt is not None and np.count_nonzero(g.rf_wgt) > 0
        assert g.rf_conflict < 1e-13, (l, g.rf_conflict)
        assert np.abs(g.rf_wgt).max() < 1.0


@pytest.mark.parametrize("lc", [4, 5, 6])
def test_divergence_free_flux_restricts_divergence_free(grid, lc):
    par, chd = grid.level(lc - 1), grid.level(lc)
    F = _stream_flux(chd)
    own_c, _ = _owned_edges(chd)
    assert np.abs(div(chd, F)[:, own_c]).max() < 1e-12 * np.abs(F).max() * chd.hex_inv[own_c].max()
    Fp, oob = _restrict(par, chd, F)
    assert oob == 0
    own, _ = _owned_edges(par)
    dp = div(par, Fp)[:, own]
    assert np.abs(dp).max() < 1e-12 * np.abs(Fp).max() * par.hex_inv[own].max()


def test_potential_flow_restriction_converges(grid):
    err = []
    for lc in (4, 5, 6):
        par, chd = grid.level(lc - 1), grid.level(lc)
        Fp, oob = _restrict(par, chd, _potential_flux(chd))
        assert oob == 0
        Fd = _potential_flux(par)
        _, e = _owned_edges(par)
        err.append(np.abs(Fp[:, e] - Fd[:, e]).max() / np.abs(Fd).max())
    assert err[-1] < 1e-3, err
    assert err[0] / err[1] > 2.5 and err[1] / err[2] > 2.5, err


def test_scalar_and_u_source_restrictions_follow_masks(grid):
    par, chd = grid.level(4), grid.level(5)
    nz = 2
    pr = Pair(par, chd, nz)
    rng = np.random.default_rng(3)
    sc = rng.standard_normal((nz, chd.NN))
    dv = rng.standard_normal((nz, 3 * chd.NN))
    sp0 = rng.standard_normal((nz, par.NN))
    dp0 = rng.standard_normal((nz, 3 * par.NN))
    mn = rng.choice([0, 8, 12, 16], size=par.NN).astype(np.int32)
    me = rng.choice([0, 2, 8, 16], size=3 * chd.NN).astype(np.int32)
    pr.field(1, "scal")[...] = sc
    pr.field(1, "dvelo")[...] = dv
    pr.field(0, "scal")[...] = sp0
    pr.field(0, "dvelo")[...] = dp0
    pr.field(0, "mask_n")[...] = mn
    pr.field(1, "mask_e")[...] = me
    pr.restrict_scalar()
    pr.restrict_u_source()
    exp_s, exp_v = sp0.copy(), dp0.copy()
    Pp, Pc = par.P, chd.P
    for d in range(10):
        for jp in range(par.n + 1):
            for ip in range(par.n + 1):
                idp = (d * Pp + jp + 2) * Pp + ip + 2
                idc = (d * Pc + 2 * jp + 2) * Pc + 2 * ip + 2
                if mn[idp] >= RESTRCT:
                    exp_s[:, idp] = sc[:, idc]
                if ip == par.n or jp == par.n:
                    continue
                for e, nb in ((0, 1), (1, Pc + 1), (2, Pc)):
                    if me[e * chd.NN + idc] >= ADJZONE:
                        exp_v[:, e * par.NN + idp] = dv[:, e * chd.NN + idc] + dv[:, e * chd.NN + idc + nb]
    assert np.array_equal(pr.field(0, "scal"), exp_s)
    assert np.array_equal(pr.field(0, "dvelo"), exp_v)
