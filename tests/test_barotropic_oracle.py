"""CPU checks of the barotropic oracle (oracle/oracle_barotropic.cpp):
flux_divergence conserves the global mass (the area-weighted divergence of
the vertically summed flux sums to zero over the sphere: every edge flux
enters two hexagons with opposite signs), rhs_elliptic reduces to -eta at
dt = 0, and grad_eta of a uniform free surface is zero."""
import numpy as np

from oracle import barotropic as ob
from oracle.grid import Grid
from wavetrisk_hydrostatic_b200 import OceanParams, jet_state
from wavetrisk_hydrostatic_b200.grid import halo_nodes


def _case(level, nz, seed):
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=seed, ph=ph)
    rng = np.random.default_rng(seed)
    eta = rng.standard_normal(g.NN) * 0.1
    div_old = rng.standard_normal(g.NN) * 1e-6
    halo_nodes(g, eta)
    halo_nodes(g, div_old)
    return g, ph, st, eta, div_old


def _sphere(g):
    """owned nodes [0, n)^2 of every lozenge plus one copy of each pole"""
    k = np.nonzero(g.owned)[0]
    return np.concatenate([k, np.array(g.pole_ids())])


def test_flux_divergence_conserves_mass():
    g, ph, st, eta, div_old = _case(5, 3, 1)
    _, div, _ = ob.rhs_elliptic(g, 3, st["mass"], st["mean_m"], st["velo"], eta, div_old, 300.0, 1.0, ph.ref_density)
    k = _sphere(g)
    area_div = div[k] / g.hex_inv[k]
    assert np.abs(area_div).max() > 0
    assert abs(area_div.sum()) < 1e-11 * np.abs(area_div).sum()


def test_rhs_at_zero_dt_is_minus_eta():
    g, ph, st, eta, div_old = _case(4, 2, 2)
    _, _, rhs = ob.rhs_elliptic(g, 2, st["mass"], st["mean_m"], st["velo"], eta, div_old, 0.0, 1.0, ph.ref_density)
    _, i, j = g.ij()
    sel = (i >= 0) & (j >= 0) & (i <= g.n) & (j <= g.n)
    assert np.array_equal(rhs[sel], -eta[sel])


def test_grad_of_uniform_eta_is_zero():
    g, ph, st, _, _ = _case(4, 2, 3)
    eta = np.full(g.NN, 0.25)
    v, grad = ob.u_update(g, 2, ph.grav, eta, st["velo"], 300.0, 1.0)
    assert np.abs(grad).max() == 0.0
    assert np.array_equal(v, st["velo"])
