"""GPU parity of trend_ml over a whole hierarchy (csrc/wt_trend_ml.cu,
csrc/trisk_ml.cuh through wt_trend_multi) against the CPU oracle's
multi-level trend (oracle_trisk.cpp: orc_trend_multi) on the same seeded
per-level states, layer means and masks.

Scalar trends are compared at nodes [0, n]^2 of every lozenge, velocity
trends on the owned edges, of every level, bit for bit (FP64, reference
operand order, no FMA contraction)."""
import numpy as np
import pytest

import oracle
from oracle.wavelet import Hierarchy
from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
from wavetrisk_hydrostatic_b200.grid import halo_edges, halo_nodes
from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

pytestmark = pytest.mark.gpu
TOL = 0.0   # bit for bit: FP64 without FMA contraction, the oracle's operand order


def _nodes0n(g):
    i = np.arange(0, g.n + 1)
    ii, jj = np.meshgrid(i, i, indexing="xy")
    return np.concatenate([((d * g.P + jj + 2) * g.P + ii + 2).ravel() for d in range(10)])


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("lmin,lmax,nz,masks", [(3, 5, 2, "tolrnz"), (3, 5, 2, "random"), (4, 6, 1, "built")])
def test_trend_multi_matches_oracle(lmin, lmax, nz, masks):
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = []
    for q, g in enumerate(levels):
        st = jet_state(g, nz, seed=10 + q, ph=ph)
        rng = np.random.default_rng(20 + q)
        st["velo"] = st["velo"] + 0.05 * rng.standard_normal(st["velo"].shape)
        halo_edges(g, st["velo"])
        states.append(st)
    dev = WaveletHierarchy(levels, [st["topo"] for st in states], nz, ph)
    for g, st in zip(levels, states):
        for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
            dev.upload(g.level, name, st[name])
    rng = np.random.default_rng(7)
    if masks == "built":
        orc_h = Hierarchy(levels, nz)
        for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
            orc_h.set(levels[-1].level, key, states[-1][name])
        orc_h.forward()
        dev.forward()
        thr = np.full((3, nz), 0.12)  # velocity and Theta
        thr[0] = 5.0                  # mass: partially refined masks at every level
        orc_h.mask_build(thr, 0, lmax + 1)
        mk = [(orc_h.field(g.level, "mask_n").copy(), orc_h.field(g.level, "mask_e").copy()) for g in levels]
        # the forward transform restricted the scaling fields: use them on both sides
        for q, g in enumerate(levels[:-1]):
            for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
                states[q][name] = orc_h.field(g.level, key).copy()
                dev.upload(g.level, name, states[q][name])
    elif masks == "random":
        mk = [(rng.choice([0, 2, 8, 12, 16], size=g.NN).astype(np.int32),
               rng.choice([0, 2, 8, 12, 16], size=3 * g.NN).astype(np.int32)) for g in levels]
    else:
        mk = [(np.full(g.NN, 16, np.int32), np.full(3 * g.NN, 16, np.int32)) for g in levels]
    for g, (mn, me) in zip(levels, mk):
        dev.upload(g.level, "mask_n", mn)
        dev.upload(g.level, "mask_e", me)
    if masks == "built":
        assert np.count_nonzero(mk[-1][0] == 0) > 0 and np.count_nonzero(mk[-1][0] == 8) > 0
    out = oracle.trend_multi(levels, nz, ph, states, mk)
    dev.trend_multi()
    for q, g in enumerate(levels):
        dm, dt, dv = dev.download_trend(g.level)
        odm, odt, odv, _ = out[q]
        nodes = _nodes0n(g)
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        assert _rel(dm[:, nodes], odm[:, nodes]) <= TOL, (g.level, "dmass")
        assert _rel(dt[:, nodes], odt[:, nodes]) <= TOL, (g.level, "dtemp")
        assert _rel(dv[:, e], odv[:, e]) <= TOL, (g.level, "dvelo")
        assert np.abs(odv[:, e]).max() > 0
    assert dev.status() == 0
    dev.close()


def test_rk4_multi_matches_oracle():
    """Two RK4 steps of the whole hierarchy (trend_ml on every level, RK
    sub-step on every level, WT_after_step per stage) with adapt-built masks."""
    ph = OceanParams()
    lmin, lmax, nz, dt = 3, 5, 2, 300.0
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    top = jet_state(levels[-1], nz, seed=3, ph=ph)
    top["velo"] = top["velo"] + 0.05 * np.random.default_rng(4).standard_normal(top["velo"].shape)
    halo_edges(levels[-1], top["velo"])
    orc_h = Hierarchy(levels, nz)
    for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
        orc_h.set(lmax, key, top[name])
    orc_h.forward()
    thr = np.full((3, nz), 0.12)
    thr[0] = 5.0
    orc_h.mask_build(thr, 0, lmax + 1)
    masks = [(orc_h.field(g.level, "mask_n").copy(), orc_h.field(g.level, "mask_e").copy()) for g in levels]
    states = []
    for g in levels:
        st = jet_state(g, nz, seed=3, ph=ph)  # means and topography of the level
        for name, key in (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v")):
            st[name] = orc_h.field(g.level, key).copy()
        states.append(st)
    dev = WaveletHierarchy(levels, [st["topo"] for st in states], nz, ph)
    for g, st, (mn, me) in zip(levels, states, masks):
        for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
            dev.upload(g.level, name, st[name])
        dev.upload(g.level, "mask_n", mn)
        dev.upload(g.level, "mask_e", me)
    ref = oracle.rk4_multi(levels, nz, ph, states, masks, dt, nsteps=2)
    dev.rk4_multi(dt, 2)
    for q, g in enumerate(levels):
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        for name, o, k in (("mass", ref[q][0], own), ("temp", ref[q][1], own), ("velo", ref[q][2], e)):
            d = dev.download(g.level, name)
            assert _rel(d[:, k], o[:, k]) <= TOL, (g.level, name, _rel(d[:, k], o[:, k]))
    assert dev.status() == 0
    dev.close()


@pytest.mark.parametrize("order", ["inf", "min", "1", "2"])
def test_lnorm_matches_numpy(order):
    from oracle.wavelet import lnorm
    ph = OceanParams()
    nz = 2
    G = Grid(3, 5, radius=6371e3)
    levels = [G.level(l) for l in range(3, 6)]
    dev = WaveletHierarchy(levels, [np.full(g.NN, -4000.0) for g in levels], nz, ph)
    rng = np.random.default_rng(5)
    fields, masks = [], []
    for g in levels:
        st = jet_state(g, nz, seed=g.level, ph=ph)
        st["velo"] = st["velo"] + rng.standard_normal(st["velo"].shape)
        f = {k: st[k] for k in ("mass", "temp", "velo", "mean_m", "mean_t")}
        for k, a in f.items():
            dev.upload(g.level, k, a)
        mn = rng.choice([0, 2, 8, 12, 16], size=g.NN).astype(np.int32)
        me = np.full(3 * g.NN, 16, np.int32)
        dev.upload(g.level, "mask_n", mn)
        dev.upload(g.level, "mask_e", me)
        fields.append(f)
        masks.append((mn, me))
    got = dev.lnorm(order)
    ref = lnorm(levels, masks, fields, order)
    if order in ("inf", "min"):
        assert np.array_equal(got, ref)
    else:
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    dev.close()


def test_rk4_multi_tma_step1_matches_plain(monkeypatch):
    """The finest level's step1 runs TMA-staged in the multi-level RK4 when the
    handle selects it (J6 and up, or WAVETRISK_TREND_KERNEL=tma); the hierarchy
    then steps to the same bits as with the L1 step1."""
    ph = OceanParams()
    lmin, lmax, nz = 3, 5, 2
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [jet_state(g, nz, seed=2 + q, ph=ph) for q, g in enumerate(levels)]
    outs = []
    for variant in ("tma", "plain"):
        monkeypatch.setenv("WAVETRISK_TREND_KERNEL", variant)
        dev = WaveletHierarchy(levels, [st["topo"] for st in states], nz, ph)
        for g, st in zip(levels, states):
            for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
                dev.upload(g.level, name, st[name])
        dev.rk4_multi(150.0, 2)
        outs.append([[dev.download(g.level, name) for name in ("mass", "temp", "velo")] for g in levels])
        assert dev.status() == 0
        dev.close()
    for a, b in zip(outs[0], outs[1]):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
