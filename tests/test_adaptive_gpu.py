"""GPU parity of the adaptive time step on a fully refined hierarchy
(wavetrisk_hydrostatic_b200.adaptive.AdaptiveOcean: RK4 of the hierarchy with
WT_after_step per stage, adapt's mask sequence with compression, inverse
transform) against the same sequence of CPU oracle calls.

Masks of every level are compared exactly after the initial adapt and after
every step; the scaling fields of every level on owned nodes and edges bit
for bit (FP64 without FMA contraction, the oracle's operand order)."""
import numpy as np
import pytest

import oracle
from oracle.wavelet import Hierarchy
from wavetrisk_hydrostatic_b200 import Grid, OceanParams
from wavetrisk_hydrostatic_b200.adaptive import AdaptiveOcean
from wavetrisk_hydrostatic_b200.cases import bump_state

pytestmark = pytest.mark.gpu
KEYS = (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v"))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("lmin,lmax,nz,tol,upload", [(3, 5, 2, 5e-3, False), (3, 6, 2, 1e-2, False),
                                                      (3, 5, 2, 5e-3, True)])
def test_adaptive_steps_match_oracle(lmin, lmax, nz, tol, upload):
    """upload: random wavelets are uploaded into every slot of every level
    between the steps; the step's first WT_after_step zeroes them (zero_float),
    so the replayed graph must give the oracle's step all the same."""
    ph = OceanParams()
    dt, nsteps = 300.0, 2
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [bump_state(g, nz, seed=1, ph=ph) for g in levels]
    model = AdaptiveOcean(G, lmin, lmax, nz, states, ph, tol=tol, init="dense")
    # oracle: the same sequence of calls
    H = Hierarchy(levels, nz)
    for name, key in KEYS:
        H.set(lmax, key, states[-1][name])
    H.forward()
    thr = model.threshold_def
    H.mask_build(thr, 0, lmax)
    H.compress()
    H.inverse()

    def check_masks(tag):
        for g, (mn, me) in zip(levels, model.masks()):
            assert np.array_equal(mn, H.field(g.level, "mask_n")), (tag, g.level, "mask_n")
            assert np.array_equal(me, H.field(g.level, "mask_e")), (tag, g.level, "mask_e")

    check_masks("init")
    act = np.count_nonzero(H.field(lmax, "mask_e") >= 16)
    assert 0 < act < 3 * np.count_nonzero(levels[-1].owned)  # partially refined finest level
    for s in range(nsteps):
        cur = [dict(states[q], **{n: H.field(g.level, k).copy() for n, k in KEYS}) for q, g in enumerate(levels)]
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
        oracle.rk4_multi(levels, nz, ph, cur, masks, dt, 1, H=H)
        H.mask_build(thr, 0, lmax)
        H.compress()
        H.inverse()
        model.step(dt)
        check_masks(f"step {s}")
        if upload:
            rng = np.random.default_rng(s)
            for g in levels:
                for name in ("wc_mass", "wc_temp", "wc_velo"):
                    n = 3 * g.NN if name == "wc_velo" else g.NN
                    model.dev.upload(g.level, name, rng.standard_normal((nz, n)))
    for g in levels:
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        for name, key in KEYS:
            k = e if name == "velo" else own
            d, o = model.dev.download(g.level, name), H.field(g.level, key)
            assert _rel(d[:, k], o[:, k]) == 0.0, (g.level, name, _rel(d[:, k], o[:, k]))
    assert model.dev.status() == 0
    model.close()


@pytest.mark.parametrize("lmin,lmax,nz,dt,nsteps", [(3, 5, 2, 300.0, 50), (4, 6, 4, 150.0, 10)])
def test_adaptive_long_run_masks_every_step(lmin, lmax, nz, dt, nsteps):
    """The adaptive run of the headline workload's kind (jet + Gaussian bumps,
    tol 5e-3 thresholds) over many steps: every mask of every level equal to
    the oracle's after every step, the masks changing during the run, and the
    scaling fields of every level within 1e-12 at the end."""
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [bump_state(g, nz, seed=2, ph=ph) for g in levels]
    model = AdaptiveOcean(G, lmin, lmax, nz, states, ph, tol=5e-3, init="dense")
    H = Hierarchy(levels, nz)
    for name, key in KEYS:
        H.set(lmax, key, states[-1][name])
    thr = model.threshold_def
    H.forward()
    H.mask_build(thr, 0, lmax)
    H.compress()
    H.inverse()
    first = [H.field(g.level, "mask_e").copy() for g in levels]
    changed = False
    for s in range(nsteps):
        cur = [dict(states[q], **{n: H.field(g.level, k).copy() for n, k in KEYS}) for q, g in enumerate(levels)]
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
        oracle.rk4_multi(levels, nz, ph, cur, masks, dt, 1, H=H)
        H.mask_build(thr, 0, lmax)
        H.compress()
        H.inverse()
        model.step(dt)
        for g, (mn, me) in zip(levels, model.masks()):
            assert np.array_equal(mn, H.field(g.level, "mask_n")), (s, g.level, "mask_n")
            assert np.array_equal(me, H.field(g.level, "mask_e")), (s, g.level, "mask_e")
        changed = changed or any(not np.array_equal(f, H.field(g.level, "mask_e")) for f, g in zip(first, levels))
    assert changed
    for g in levels:
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        for name, key in KEYS:
            k = e if name == "velo" else own
            d, o = model.dev.download(g.level, name), H.field(g.level, key)
            assert _rel(d[:, k], o[:, k]) == 0.0, (g.level, name, _rel(d[:, k], o[:, k]))
    assert model.dev.status() == 0
    model.close()


@pytest.mark.parametrize("lmin,lmax,nz,dt,nsteps", [(4, 7, 4, 150.0, 6), (3, 6, 2, 300.0, 20)])
def test_skipping_inactive_nodes_changes_nothing(lmin, lmax, nz, dt, nsteps):
    """The finest level's step1 and trend leave out the nodes outside the
    needed-node map (WT_TUNE_SKIP_INACTIVE, the default): every mask and every
    owned value of every level must equal, bit for bit, those of the same run
    computing every node, after every step (graph-replayed adaptive steps, the
    finest level J7 in the first case)."""
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [bump_state(g, nz, seed=3, ph=ph) for g in levels]
    a = AdaptiveOcean(G, lmin, lmax, nz, states, ph, tol=5e-3, init="dense")
    b = AdaptiveOcean(G, lmin, lmax, nz, states, ph, tol=5e-3, init="dense")
    b.dev.skip_inactive(False)
    for s in range(nsteps):
        a.step(dt)
        b.step(dt)
        for g, (ma, mb) in zip(levels, zip(a.masks(), b.masks())):
            assert np.array_equal(ma[0], mb[0]) and np.array_equal(ma[1], mb[1]), (s, g.level)
        for g in levels:
            own = np.nonzero(g.owned)[0]
            e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
            for name in ("mass", "temp", "velo"):
                k = e if name == "velo" else own
                da, db = a.dev.download(g.level, name)[:, k], b.dev.download(g.level, name)[:, k]
                assert np.array_equal(da, db), (s, g.level, name, np.abs(da - db).max())
    assert a.dev.status() == 0 and b.dev.status() == 0
    a.close()
    b.close()
