"""The vertical remap (remap_vertical_coordinates, src/remap.f90): the
oracle's column routines on their own (constants kept, column integrals
conserved, nothing moves when the grid does not), and the GPU kernel
(csrc/remap_kernels.cuh through wt_remap_vertical) against the oracle bit
for bit on a level over a seamount, for remap0, remap1 and remap2PPM.

remap1 keeps a reference behaviour: its harmonic-mean slope
2 FC(k) FC(k-1) / (FC(k) + FC(k-1)) is 0/0 where two neighbouring differences
are both zero (src/remap.f90:320-324 tests only for opposite signs), so a
column with a locally constant profile (a resting layer's velocity, uniform
buoyancy) comes out NaN, as in the reference; the comparison treats NaN as
equal there."""
import numpy as np
import pytest

from oracle import remap as R

TYPES = ("0", "1", "2PPM")


def _columns(nz, nc, seed):
    rng = np.random.default_rng(seed)
    h_old = 50.0 + 100.0 * rng.random((nz, nc))
    z_old = np.vstack([np.full((1, nc), -4000.0), -4000.0 + np.cumsum(h_old, axis=0)])
    top = z_old[-1]
    b = 1.0 - np.arange(nz + 1) / nz
    z_new = np.stack([(1.0 - b[k]) * top + b[k] * z_old[0] for k in range(nz + 1)])
    v = np.vstack([np.zeros((1, nc)), rng.standard_normal((nz, nc))])
    return z_new, z_old, v


@pytest.mark.parametrize("kind", TYPES)
def test_column_routines_conserve_and_keep_constants(kind):
    nz, nc = 12, 200
    z_new, z_old, v = _columns(nz, nc, 3)
    f = R.REMAP[kind]
    vn = f(nz, z_new, v, z_old)
    before = np.sum((z_old[1:] - z_old[:-1]) * v[1:], axis=0)
    after = np.sum((z_new[1:] - z_new[:-1]) * vn[1:], axis=0)
    assert np.abs(after - before).max() <= 1e-12 * np.abs((z_old[1:] - z_old[:-1]) * np.abs(v[1:])).sum(axis=0).max()
    c = np.vstack([np.zeros((1, nc)), np.full((nz, nc), 2.5)])
    with np.errstate(all="ignore"):
        vc = f(nz, z_new, c, z_old)[1:]
    if kind == "1":
        assert np.isnan(vc).all()       # the reference's 0/0 slope (module docstring)
    else:
        assert np.abs(vc - 2.5).max() <= 1e-13
    same = f(nz, z_old, v, z_old)
    assert np.abs(same[1:] - v[1:]).max() <= 1e-14 * np.abs(v).max()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", TYPES)
def test_remap_matches_oracle_bit_for_bit(kind):
    from wavetrisk_hydrostatic_b200 import Grid, OceanParams
    from wavetrisk_hydrostatic_b200.cases import bump_state, seamount_topography
    from wavetrisk_hydrostatic_b200.grid import halo_nodes
    from wavetrisk_hydrostatic_b200.model import TriskModel

    nz, level = 8, 5
    ph = OceanParams()
    g = Grid(level, level, radius=6371e3).level(level)
    st = bump_state(g, nz, seed=2, ph=ph, topo=seamount_topography(g, seed=2, radius=600e3))
    rng = np.random.default_rng(4)
    for k in range(nz):        # layers moved off the hybrid grid, as after Lagrangian steps
        st["mass"][k] += st["mean_m"][k] * 0.2 * (rng.random(g.NN) - 0.5)
        halo_nodes(g, st["mass"][k])
    b = 1.0 - np.arange(nz + 1) / nz
    a = 1.0 - b
    m = TriskModel(g, nz, st["topo"], ph)
    m.upload(st)
    m.remap_vertical(kind, a, b)
    out = m.download()
    assert m.status() == 0
    m.close()
    om, ot, ov = R.remap_level(g, nz, st, kind, a, b, ph.ref_density)
    d, i, j = g.ij()
    nodes = np.nonzero((i >= 0) & (j >= 0) & (i <= g.n) & (j <= g.n))[0]
    # the remapped nodes: those of [0, n]^2 that are their own source (owned
    # nodes and the pole slots); the download fills the ghost copies of the
    # others from their sources, which the oracle leaves as they were
    nsrc = np.arange(g.NN)
    nsrc[g.halo_node[:, 0]] = g.halo_node[:, 1]
    nodes = nodes[nsrc[nodes] == nodes]
    own = np.nonzero(g.owned)[0]
    edges = np.concatenate([own, own + g.NN, own + 2 * g.NN])
    assert np.array_equal(out["mass"][:, nodes], om[:, nodes], equal_nan=True)
    assert np.array_equal(out["temp"][:, nodes], ot[:, nodes], equal_nan=True)
    assert np.array_equal(out["velo"][:, edges], ov[:, edges], equal_nan=True)
    if kind != "1":
        assert np.isfinite(out["mass"][:, nodes]).all() and np.isfinite(out["velo"][:, edges]).all()
    assert np.abs(om[:, own] - st["mass"][:, own]).max() > 1.0      # the remap moved mass


@pytest.mark.gpu
def test_min_mass_matches_oracle():
    """cpt_min_mass on the device (wt_min_mass) against the oracle's
    cal_min_mass, exactly, on Lagrangian layers moved off the hybrid grid; and
    0 once a layer has collapsed."""
    from wavetrisk_hydrostatic_b200 import Grid, OceanParams
    from wavetrisk_hydrostatic_b200.cases import bump_state, seamount_topography
    from wavetrisk_hydrostatic_b200.grid import halo_nodes
    from wavetrisk_hydrostatic_b200.model import TriskModel

    nz, level = 8, 5
    ph = OceanParams()
    g = Grid(level, level, radius=6371e3).level(level)
    st = bump_state(g, nz, seed=3, ph=ph, topo=seamount_topography(g, seed=3, radius=600e3))
    rng = np.random.default_rng(5)
    for k in range(nz):
        st["mass"][k] += st["mean_m"][k] * 0.3 * (rng.random(g.NN) - 0.5)
        halo_nodes(g, st["mass"][k])
    b = 1.0 - np.arange(nz + 1) / nz
    m = TriskModel(g, nz, st["topo"], ph)
    m.upload(st)
    got = m.min_mass(b)
    want = R.min_mass_level(g, nz, st, b, ph.ref_density)
    assert got == want and 0.8 < got < 0.9
    own = np.nonzero(g.owned)[0]
    st["mass"][3, own[17]] = -st["mean_m"][3, own[17]] * 1.5   # a collapsed layer
    m.upload(st)
    assert m.min_mass(b) == 0.0 == R.min_mass_level(g, nz, st, b, ph.ref_density)
    assert m.status() == 0
    m.close()
