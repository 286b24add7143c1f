"""Seeded synthetic initial states for the benchmark and test workloads.

The reference builds initial conditions in its test-case modules
(test/seamount/test_case_module.f90: init_mean :381-412, init_sol :341-379):
sol_mean holds the layer mass rho0*dz and Theta = rho0*dz*(1 - rho/rho0);
sol holds the perturbation (the free surface rho0*eta in the top layer).
Velocities are edge-normal components of an analytic zonal jet
(proj_vel, src/sphere.f90:330).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .grid import DG, RT, UP, LevelGeom, halo_edges, halo_nodes


@dataclass
class OceanParams:
    grav: float = 9.80616          # grav_accel default, src/shared.f90:386
    ref_density: float = 1028.0    # ref_density_water, src/shared.f90:407
    p_top: float = 0.0
    depth: float = 4000.0


def _neighbours(g: LevelGeom):
    d, i, j = g.ij()
    ok = (i + 1 < g.n + 2) & (j + 1 < g.n + 2)
    E = np.where(ok, g.idx(d, np.minimum(i + 1, g.n + 1), j), 0)
    N = np.where(ok, g.idx(d, i, np.minimum(j + 1, g.n + 1)), 0)
    NE = np.where(ok, g.idx(d, np.minimum(i + 1, g.n + 1), np.minimum(j + 1, g.n + 1)), 0)
    return E, N, NE


def _proj_jet(p, q, u0, lat0, width):
    """Edge-normal velocity of u = u0 sech^2((lat-lat0)/width) along p->q at its midpoint."""
    m = p + q
    nrm = np.linalg.norm(m, axis=0)
    nrm = np.where(nrm == 0, 1.0, nrm)
    m = m / nrm
    lat = np.arcsin(np.clip(m[2], -1, 1))
    lon = np.arctan2(m[1], m[0])
    u = u0 / np.cosh((lat - lat0) / width) ** 2
    ez = np.stack([-np.sin(lon), np.cos(lon), np.zeros_like(lon)])
    v = q - p
    vn = np.linalg.norm(v, axis=0)
    vn = np.where(vn == 0, 1.0, vn)
    return u * np.einsum("ij,ij->j", ez, v / vn)


def seamount_topography(g: LevelGeom, seed: int = 0, depth: float = 4000.0, height: float = 2000.0,
                        radius: float = 50e3) -> np.ndarray:
    """Flat bottom at -depth with a Gaussian seamount of the given height and
    radius (m) centred at a seeded point of the sphere (the bathymetry of the
    reference's seamount case, test/seamount/test_case_module.f90, with a
    seeded centre): topography = -depth + height exp(-(r/radius)^2), r the
    great-circle distance, at every node of the level (ghosts from their own
    coordinates; padding slots without coordinates get the flat depth)."""
    rng = np.random.default_rng(20_000 + seed)
    c = rng.standard_normal(3)
    c /= np.linalg.norm(c)
    nrm = np.linalg.norm(g.node, axis=0)
    ok = nrm > 0
    R = float(nrm[g.owned][0])
    topo = np.full(g.NN, -depth)
    ang = np.arccos(np.clip(c @ (g.node[:, ok] / nrm[ok]), -1.0, 1.0))
    topo[ok] += height * np.exp(-((R * ang) / radius) ** 2)
    return topo


def jet_state(g: LevelGeom, nz: int, seed: int = 0, ph: OceanParams | None = None,
              u0: float = 1.0, eta_amp: float = 1e-3, rho_bottom: float = 1027.0, rho_top: float = 1024.0,
              topo: np.ndarray | None = None):
    """Uniform-level layered ocean state: flat bottom (or the given topography,
    layers of equal thickness H/nz following it as the reference's init_mean
    sets them with b_vert_mass = 1/nz), linear layer densities, zonal jet at
    45N in the top layer decaying linearly to 0 at the bottom, seeded white
    noise free surface.  Returns dict of float64 arrays in the C-ABI layout."""
    ph = ph or OceanParams()
    NN = g.NN
    rng = np.random.default_rng(seed)
    topo = np.full(NN, -ph.depth) if topo is None else np.asarray(topo, dtype=np.float64)
    dz = -topo / nz
    rho = rho_bottom + (rho_top - rho_bottom) * np.arange(nz) / max(nz - 1, 1)   # k=1 is the bottom layer
    mean_m = np.empty((nz, NN))
    mean_t = np.empty((nz, NN))
    for k in range(nz):
        mean_m[k] = ph.ref_density * dz
        mean_t[k] = mean_m[k] * (1.0 - rho[k] / ph.ref_density)
    eta = np.zeros(NN)
    own = g.owned
    eta[own] = eta_amp * rng.standard_normal(int(own.sum()))
    npole, spole = g.pole_ids()
    pole_eta = eta_amp * rng.standard_normal(2)
    d, i, j = g.ij()
    eta[(d >= 5) & (i == 0) & (j == g.n)] = pole_eta[0]
    eta[(d < 5) & (i == g.n) & (j == 0)] = pole_eta[1]
    halo_nodes(g, eta)
    mass = np.zeros((nz, NN))
    temp = np.zeros((nz, NN))
    mass[nz - 1] = ph.ref_density * eta
    velo = np.zeros((nz, 3 * NN))
    E, N, NE = _neighbours(g)
    p = g.node
    ujet = np.zeros(3 * NN)
    sel = own
    ujet[RT * NN:(RT + 1) * NN][sel] = _proj_jet(p[:, sel], p[:, E[sel]], u0, np.pi / 4, np.pi / 36)
    ujet[DG * NN:(DG + 1) * NN][sel] = _proj_jet(p[:, NE[sel]], p[:, sel], u0, np.pi / 4, np.pi / 36)
    ujet[UP * NN:(UP + 1) * NN][sel] = _proj_jet(p[:, sel], p[:, N[sel]], u0, np.pi / 4, np.pi / 36)
    for k in range(nz):
        velo[k] = ujet * (k / max(nz - 1, 1))
    for k in range(nz):
        halo_nodes(g, mass[k])
        halo_nodes(g, temp[k])
        halo_edges(g, velo[k])
    return dict(mass=mass, temp=temp, velo=velo, mean_m=mean_m, mean_t=mean_t, topo=topo)


def bump_state(g: LevelGeom, nz: int, seed: int = 0, ph: OceanParams | None = None, nbumps: int = 8,
               radius: float = 300e3, amp: float = 0.05, **jet_kw):
    """jet_state plus a seeded baroclinic perturbation: nbumps Gaussian bumps of
    the given radius (m) and amplitude (m) in the thickness of every layer, at
    seeded centres on the sphere (the same centres on every level).  The layer
    densities are unchanged, so Theta mass moves with the layer mass."""
    ph = ph or OceanParams()
    st = jet_state(g, nz, seed=seed, ph=ph, **jet_kw)
    rng = np.random.default_rng(10_000 + seed)
    c = rng.standard_normal((nbumps, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    nrm = np.linalg.norm(g.node, axis=0)
    ok = nrm > 0  # padding corners without coordinates keep dz = 0
    x = g.node[:, ok] / nrm[ok]
    R = float(nrm[g.owned][0])
    dz = np.zeros(g.NN)
    for q in range(nbumps):
        ang = np.arccos(np.clip(c[q] @ x, -1.0, 1.0))
        dz[ok] += amp * np.exp(-((R * ang) / radius) ** 2)
    halo_nodes(g, dz)
    for k in range(nz):
        dm = ph.ref_density * dz
        st["mass"][k] = st["mass"][k] + dm
        st["temp"][k] = st["temp"][k] + dm * (st["mean_t"][k] / st["mean_m"][k])
    return st


def bathymetry(g: LevelGeom, seed: int = 0, lmax: int = 32, nterms: int = 160,
               hmin: float = 500.0, hmax: float = 5000.0, _cache: dict = {}) -> np.ndarray:
    """Smooth seeded random depth H in [hmin, hmax] m: a sum of zonal harmonics
    P_l(x.a_q) of degree l <= lmax about random axes a_q with amplitude ~ l^-2
    (every term is a spherical harmonic of degree l).  Returns topography = -H
    at every node of the level (ghosts from their own coordinates)."""
    from scipy.special import eval_legendre

    key = (seed, lmax, nterms)
    if key not in _cache:
        rng = np.random.default_rng(seed)
        ax = rng.standard_normal((nterms, 3))
        ax /= np.linalg.norm(ax, axis=1, keepdims=True)
        deg = rng.integers(1, lmax + 1, nterms)
        amp = rng.standard_normal(nterms) / deg.astype(float) ** 2
        _cache[key] = (ax, deg, amp)
    ax, deg, amp = _cache[key]
    x = g.node
    r = np.linalg.norm(x, axis=0)
    ok = r > 0
    u = np.zeros_like(x)
    u[:, ok] = x[:, ok] / r[ok]
    h = np.zeros(g.NN)
    for a, l, c in zip(ax, deg, amp):
        h += c * eval_legendre(int(l), np.clip(a @ u, -1.0, 1.0))
    lo, hi = -sum(abs(amp)), sum(abs(amp))   # level-independent normalisation
    H = hmin + (hmax - hmin) * (h - lo) / (hi - lo)
    H[~ok] = hmin
    return -H


def elliptic_rhs(g: LevelGeom, seed: int = 0) -> np.ndarray:
    """Seeded N(0,1) right-hand side on the owned nodes and poles of level g,
    minus its area-weighted mean, copied to the ghosts."""
    rng = np.random.default_rng(seed)
    f = np.zeros(g.NN)
    own = g.owned.copy()
    npole, spole = g.pole_ids()
    d, i, j = g.ij()
    f[own] = rng.standard_normal(int(own.sum()))
    pv = rng.standard_normal(2)
    f[(d >= 5) & (i == 0) & (j == g.n)] = pv[0]
    f[(d < 5) & (i == g.n) & (j == 0)] = pv[1]
    area = np.where(g.hex_inv > 0, 1.0 / np.where(g.hex_inv > 0, g.hex_inv, 1.0), 0.0)
    sel = own.copy()
    sel[npole] = sel[spole] = True
    mean = (f[sel] * area[sel]).sum() / area[sel].sum()
    f[sel | ((d >= 5) & (i == 0) & (j == g.n)) | ((d < 5) & (i == g.n) & (j == 0))] -= mean
    halo_nodes(g, f)
    return f


def solid_body_rotation(u0: float = 1.0):
    """Tangent field of a rigid rotation about the polar axis, u0 at the equator:
    U(x) = u0 (-y, x, 0) / |x|, for x of shape (3, N)."""
    def U(x):
        r = np.linalg.norm(x, axis=0)
        r = np.where(r == 0, 1.0, r)
        return u0 * np.stack([-x[1], x[0], np.zeros_like(x[0])]) / r
    return U


def edge_velocity(g: LevelGeom, U) -> np.ndarray:
    """Velocity components of the tangent field U along every owned edge
    (endpoint 1 -> endpoint 2 of end_pt, src/shared.f90:287-292) at the edge
    midpoint, ghosts by the level's copy table; (3*NN,) in the C-ABI layout."""
    NN = g.NN
    E, N, NE = _neighbours(g)
    sel = g.owned
    ids = np.nonzero(sel)[0]
    p = g.node
    v = np.zeros(3 * NN)
    for e, (a, b) in ((RT, (ids, E[sel])), (DG, (NE[sel], ids)), (UP, (ids, N[sel]))):
        pa, pb = p[:, a], p[:, b]
        m = pa + pb
        m = m / np.linalg.norm(m, axis=0) * np.linalg.norm(pa, axis=0)
        t = pb - pa
        t = t / np.linalg.norm(t, axis=0)
        v[e * NN + ids] = np.einsum("ij,ij->j", U(m), t)
    halo_edges(g, v)
    return v
