"""GPU parity of the barotropic pieces of the mode-split step
(csrc/wt_barotropic.cu through the C-ABI) against the CPU oracle: flux
divergence and the free-surface right-hand side at nodes [0, n]^2, the
external pressure gradient and the updated velocity at owned edges.
Bit for bit (FP64, no FMA contraction)."""
import numpy as np
import pytest

from oracle import barotropic as ob
from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
from wavetrisk_hydrostatic_b200.grid import halo_edges, halo_nodes
from wavetrisk_hydrostatic_b200.model import TriskModel

pytestmark = pytest.mark.gpu
TOL = 0.0   # bit for bit: FP64 without FMA contraction, the oracle's operand order


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("level,nz", [(4, 2), (5, 4), (6, 3)])
def test_rhs_elliptic_and_u_update_match_oracle(level, nz):
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=level, ph=ph)
    rng = np.random.default_rng(level)
    eta = rng.standard_normal(g.NN) * 0.1
    div_old = rng.standard_normal(g.NN) * 1e-6
    halo_nodes(g, eta)
    halo_nodes(g, div_old)
    dt, th1, th2 = 600.0, 1.0, 0.75
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    model.barotropic_upload(eta, div_old)
    div, rhs = model.rhs_elliptic(dt, th2)
    _, odiv, orhs = ob.rhs_elliptic(g, nz, st["mass"], st["mean_m"], st["velo"], eta, div_old, dt, th2,
                                    ph.ref_density)
    _, i, j = g.ij()
    sel = (i >= 0) & (j >= 0) & (i <= g.n) & (j <= g.n)
    own = np.nonzero(g.owned)[0]
    # div at ghost nodes is read through the remap (the oracle holds the ghost copy there)
    assert rel(div[own], odiv[own]) <= TOL
    assert rel(rhs[sel], orhs[sel]) <= TOL
    grad = model.u_update(dt, th1)
    ov, ograd = ob.u_update(g, nz, ph.grav, eta, st["velo"], dt, th1)
    e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
    assert rel(grad[e], ograd[e]) <= TOL
    v = model.download()["velo"]
    halo_edges(g, ov)        # u_update leaves the ghosts stale; the next update_bdry copies them
    assert rel(v[:, e], ov[:, e]) <= TOL
    model.close()


@pytest.mark.parametrize("itype", [1, 5, 6, 7])
def test_step1_flux_itypes_match_oracle(itype):
    level, nz = 5, 2
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=9, ph=ph)
    s = np.random.default_rng(itype).standard_normal(g.NN)
    halo_nodes(g, s)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    k = nz - 1
    f = model.step1_flux(itype, k, s if itype in (1, 6) else None)
    of = ob.step1_flux(g, itype, st["velo"][k], st["mass"][k], st["mean_m"][k], s if itype in (1, 6) else None)
    own = np.nonzero(g.owned)[0]
    e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
    assert rel(f[e], of[e]) <= TOL
    model.close()


@pytest.mark.parametrize("level", [4, 6])
def test_step1_vorticity_matches_oracle_exactly(level):
    """itype 8 + post_vort: every triangle the reference's loop writes, the
    pentagon corners and the UPLT values written twice included, bit for bit."""
    nz = 2
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=level, ph=ph)
    st["velo"] = st["velo"] + np.random.default_rng(level).standard_normal(st["velo"].shape)
    halo_edges(g, st["velo"])
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    for k in range(nz):
        v = model.step1_vort(k)
        ov = ob.step1_vort(g, st["velo"][k])
        assert np.count_nonzero(ov) > 0
        assert np.array_equal(v, ov), (k, np.abs(v - ov).max())
    model.close()


@pytest.mark.parametrize("masks_kind", ["tolrnz", "built"])
def test_barotropic_pieces_on_the_hierarchy_match_oracle(masks_kind):
    """flux_divergence with cpt_or_restr_flux, rhs_elliptic, grad_eta with
    cpt_or_restr_eta and u_update on every level of a J3..J5 hierarchy."""
    from oracle.wavelet import Hierarchy
    from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

    lmin, lmax, nz, dt = 3, 5, 2, 300.0
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [jet_state(g, nz, seed=7 + q, ph=ph) for q, g in enumerate(levels)]
    rng = np.random.default_rng(5)
    etas, dolds = [], []
    for g in levels:
        e, d = rng.standard_normal(g.NN) * 0.1, rng.standard_normal(g.NN) * 1e-6
        halo_nodes(g, e)
        halo_nodes(g, d)
        etas.append(e)
        dolds.append(d)
    if masks_kind == "built":
        H = Hierarchy(levels, nz)
        for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
            H.set(lmax, key, states[-1][name])
        H.forward()
        H.mask_build(np.array([[5.0] * nz, [1e16] * nz, [0.05] * nz]), 0, lmax)
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
        assert np.count_nonzero(masks[1][0] >= 12) < np.count_nonzero(levels[1].owned)
    else:
        masks = [(np.full(g.NN, 16, np.int32), np.full(3 * g.NN, 16, np.int32)) for g in levels]
    dev = WaveletHierarchy(levels, [st["topo"] for st in states], nz, ph)
    for g, st, (mn, me), e, d in zip(levels, states, masks, etas, dolds):
        for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
            dev.upload(g.level, name, st[name])
        dev.upload(g.level, "mask_n", mn)
        dev.upload(g.level, "mask_e", me)
        dev.barotropic_upload(g.level, e, d)
    ro = ob.rhs_elliptic_multi(levels, nz, states, masks, etas, dolds, dt, 0.75, ph.ref_density)
    dev.rhs_elliptic_multi(dt, 0.75)
    uo = ob.u_update_multi(levels, nz, states, masks, etas, ph.grav, dt, 0.6)
    dev.u_update_multi(dt, 0.6)
    for q, g in enumerate(levels):
        div, rhs, grad = dev.barotropic_download(g.level)
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        assert rel(div[own], ro[q]["div"][own]) <= TOL, (g.level, "div")
        assert rel(rhs[own], ro[q]["rhs"][own]) <= TOL, (g.level, "rhs")
        assert rel(grad[e], uo[q]["grad"][e]) <= TOL, (g.level, "grad")
        v = dev.download(g.level, "velo")
        ov = uo[q]["velo"].copy()
        halo_edges(g, ov)
        assert rel(v[:, e], ov[:, e]) <= TOL, (g.level, "velo")
    assert dev.status() == 0
    dev.close()


def _split_case(masks_kind, lmin=3, lmax=5, nz=2):
    from oracle.wavelet import Hierarchy
    from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [jet_state(g, nz, seed=11 + q, ph=ph) for q, g in enumerate(levels)]
    rng = np.random.default_rng(9)
    etas = []
    for g in levels:
        e = rng.standard_normal(g.NN) * 0.1
        halo_nodes(g, e)
        etas.append(e)
    if masks_kind == "built":
        H = Hierarchy(levels, nz)
        for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
            H.set(lmax, key, states[-1][name])
        H.forward()
        H.mask_build(np.array([[5.0] * nz, [1e16] * nz, [0.05] * nz]), 0, lmax)
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
    else:
        masks = [(np.full(g.NN, 16, np.int32), np.full(3 * g.NN, 16, np.int32)) for g in levels]
    dev = WaveletHierarchy(levels, [st["topo"] for st in states], nz, ph)
    for g, st, (mn, me), e in zip(levels, states, masks, etas):
        for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
            dev.upload(g.level, name, st[name])
        dev.upload(g.level, "mask_n", mn)
        dev.upload(g.level, "mask_e", me)
        dev.barotropic_upload(g.level, e, None)
    return ph, levels, states, masks, etas, dev


def test_barotropic_correction_on_the_hierarchy_matches_oracle():
    """barotropic_correction with total_height on every level of J3..J5."""
    ph, levels, states, masks, etas, dev = _split_case("tolrnz")
    ref = ob.barotropic_correction_multi(levels, 2, ph, states, etas)
    dev.barotropic_correction()
    for (m, t), g in zip(ref, levels):
        own = np.nonzero(g.owned)[0]
        assert rel(dev.download(g.level, "mass")[:, own], m[:, own]) <= TOL, (g.level, "mass")
        assert rel(dev.download(g.level, "temp")[:, own], t[:, own]) <= TOL, (g.level, "temp")
    assert dev.status() == 0
    dev.close()


@pytest.mark.parametrize("masks_kind", ["tolrnz", "built"])
def test_rk4_split_explicit_matches_oracle(masks_kind):
    """RK4_split's four RK_split stages (barotropic_correction, trend_ml,
    scalar_star, u_star with grad_eta, WT_after_step) on J3..J5: every level's
    state on owned nodes and edges."""
    import oracle

    ph, levels, states, masks, etas, dev = _split_case(masks_kind)
    dt, theta1 = 150.0, 0.5
    ref = oracle.rk4_split_explicit(levels, 2, ph, states, masks, etas, dt, theta1)
    dev.rk4_split_explicit(dt, theta1)
    for (m, t, v), g in zip(ref, levels):
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        assert rel(dev.download(g.level, "mass")[:, own], m[:, own]) <= TOL, (g.level, "mass")
        assert rel(dev.download(g.level, "temp")[:, own], t[:, own]) <= TOL, (g.level, "temp")
        assert rel(dev.download(g.level, "velo")[:, e], v[:, e]) <= TOL, (g.level, "velo")
    assert dev.status() == 0
    dev.close()
