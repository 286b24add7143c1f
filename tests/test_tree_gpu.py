"""GPU parity of the partially refined hierarchy: the reference's initial
refinement (initialize, src/main.f90:36-135) and adaptive steps whose adapt
refines the patch tree (refine, src/refine_patch.f90:12-49), against the
oracle's restatement (oracle/tree.py) on the same seeded inputs.

After the initialisation and after every step: the tree (every level's patch
bytes), its level_end, every mask of every level bit for bit; the scaling
fields of every level bit for bit on the nodes of existing patches and their
edges (the device limits its work to the tree, so the state is complete
there, as the reference's is); and no mask that is not ZERO outside the tree
(the reference has no node there)."""
import numpy as np
import pytest

import oracle
from oracle.tree import ReferenceInit, adapt
from wavetrisk_hydrostatic_b200 import Grid, OceanParams
from wavetrisk_hydrostatic_b200._native import WtError
from wavetrisk_hydrostatic_b200.adaptive import AdaptiveOcean, patch_size_for
from wavetrisk_hydrostatic_b200.cases import bump_state, seamount_topography

pytestmark = pytest.mark.gpu
KEYS = (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v"))


def _owned(g, tree=None):
    """Owned nodes (those of existing patches with a tree: after a step the
    state is complete there, as the reference's is) and their edges."""
    sel = g.owned if tree is None else g.owned & tree.node_map(g)
    own = np.nonzero(sel)[0]
    return own, np.concatenate([own, own + g.NN, own + 2 * g.NN])


def _pair(lmin, lmax, nz, make, ph, tol=5e-3):
    G = Grid(lmin, lmax, radius=6371e3)
    root = G.level(lmin - 1)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    ics = {g.level: make(g) for g in [root] + levels}
    model = AdaptiveOcean(G, lmin, lmax, nz, [ics[g.level] for g in levels], ph, tol=tol, root_state=ics[root.level])
    RI = ReferenceInit(root, levels, nz, ics, model.threshold_def, lmax, ps=patch_size_for(lmin)).run()
    return G, levels, ics, model, RI


def _check(levels, model, RI, tag, fields=True):
    H, tree = RI.H, RI.tree
    assert model.level_end() == tree.level_end, tag
    for g in levels:
        assert np.array_equal(model.patches(g.level), tree.exist[g.level]), (tag, g.level, "tree")
        mn, me = model.dev.download(g.level, "mask_n"), model.dev.download(g.level, "mask_e")
        assert np.array_equal(mn, H.field(g.level, "mask_n")), (tag, g.level, "mask_n")
        assert np.array_equal(me, H.field(g.level, "mask_e")), (tag, g.level, "mask_e")
        assert model.dev.tree_stats(g.level)[2] == 0, (tag, g.level, "mask outside the tree")
        if fields:
            own, edges = _owned(g, tree)
            for name, key in KEYS:
                k = edges if name == "velo" else own
                d, o = model.dev.download(g.level, name)[:, k], H.field(g.level, key)[:, k]
                assert np.array_equal(d, o), (tag, g.level, name, float(np.abs(d - o).max()))


def _steps(levels, ics, model, RI, nz, ph, dt, nsteps):
    H, tree, lmax = RI.H, RI.tree, levels[-1].level
    base = [{k: v for k, v in ics[g.level].items() if k not in ("mass", "temp", "velo")} for g in levels]
    grew = False
    for s in range(nsteps):
        cur = [dict(base[q], **{n: H.field(g.level, k).copy() for n, k in KEYS}) for q, g in enumerate(levels)]
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
        oracle.rk4_multi(levels, nz, ph, cur, masks, dt, 1, H=H)
        grew = adapt(H, tree, model.threshold_def, lmax) or grew
        H.inverse()
        model.step(dt)
        _check(levels, model, RI, f"step {s}", fields=(s == nsteps - 1))
    assert model.dev.status() == 0
    return grew


@pytest.mark.parametrize("lmin,lmax,nz", [(3, 5, 2), (4, 6, 4)])
def test_reference_init_matches_oracle(lmin, lmax, nz):
    """The initial grid: refinement level by level from level_start + 1, the
    root level's wavelets, count_active's stopping rule."""
    oracle.set_threads(8)
    ph = OceanParams()
    G, levels, ics, model, RI = _pair(lmin, lmax, nz, lambda g: bump_state(g, nz, seed=2, ph=ph), ph)
    assert model.init_log == [(le, nn, ne) for le, nn, ne in RI.log]
    _check(levels, model, RI, "init")
    own, edges = _owned(levels[-1])
    for key, name in (("w_m", "wc_mass"), ("w_v", "wc_velo")):
        k = edges if name == "wc_velo" else own
        assert np.array_equal(model.dev.download(levels[-1].level, name)[:, k], RI.H.field(levels[-1].level, key)[:, k])
    model.close()


@pytest.mark.parametrize("lmin,lmax,nz,dt,nsteps,tol", [(3, 5, 2, 300.0, 12, 5e-3), (4, 6, 4, 150.0, 8, 5e-3),
                                                         (3, 6, 2, 300.0, 6, 0.2)])
def test_tree_grows_as_the_oracle_every_step(lmin, lmax, nz, dt, nsteps, tol):
    """Adaptive steps after the reference's initialisation: refine() inside the
    device step graph (or, at tol 0.2 where the initial grid stops at J5 below
    the top J6, the unfused step) gives the oracle's tree, masks and fields
    after every step."""
    oracle.set_threads(8)
    ph = OceanParams()
    G, levels, ics, model, RI = _pair(lmin, lmax, nz, lambda g: bump_state(g, nz, seed=2, ph=ph), ph, tol=tol)
    if tol > 0.1:
        assert RI.tree.level_end < lmax
    _steps(levels, ics, model, RI, nz, ph, dt, nsteps)
    model.close()


def test_grid_sync_round_trip():
    """wt_grid_sync uploads a host tree: the device then holds it and its
    level_end; level_start must be complete."""
    ph = OceanParams()
    nz = 2
    G, levels, ics, model, RI = _pair(3, 5, nz, lambda g: bump_state(g, nz, seed=2, ph=ph), ph)
    ps = model.patch_size
    rng = np.random.default_rng(0)
    ex = [np.ones((10, g.n // ps, g.n // ps), dtype=bool) if q == 0 else rng.random((10, g.n // ps, g.n // ps)) < 0.3
          for q, g in enumerate(levels)]
    model.dev.grid_sync(ex, levels[-1].level)
    assert model.level_end() == levels[-1].level
    for q, g in enumerate(levels):
        assert np.array_equal(model.patches(g.level), ex[q])
    bad = [e.copy() for e in ex]
    bad[0][0, 0, 0] = False
    with pytest.raises(WtError):
        model.dev.grid_sync(bad, levels[-1].level)
    model.close()


def test_packed_tree_state_round_trip():
    """wt_download_tree_state gives level_end's state on its existing patches,
    patch by patch in lozenge-major order; wt_upload_tree_state writes packed
    values back to exactly those nodes."""
    ph = OceanParams()
    nz = 3
    G, levels, ics, model, RI = _pair(3, 5, nz, lambda g: bump_state(g, nz, seed=2, ph=ph), ph)
    model.step(300.0)
    g, ps = levels[-1], model.patch_size
    bufs = model.dev.tree_state_buffers()
    n = model.dev.download_tree_state(bufs)
    ex = model.patches(g.level)
    assert n == int(ex.sum()) > 0
    full = {k: model.dev.download(g.level, k) for k in ("mass", "temp", "velo")}
    d, pj, pi = np.nonzero(ex)
    s = np.arange(ps * ps)
    ii = (pi[:, None] * ps + s[None, :] % ps)
    jj = (pj[:, None] * ps + s[None, :] // ps)
    x = g.idx(d[:, None], ii, jj)                       # [patch][node]
    assert np.array_equal(bufs[0][:n], full["mass"][:, x].transpose(1, 0, 2))
    assert np.array_equal(bufs[1][:n], full["temp"][:, x].transpose(1, 0, 2))
    v = full["velo"].reshape(nz, 3, g.NN)[:, :, x]      # [nz][3][patch][node]
    assert np.array_equal(bufs[2][:n], v.transpose(2, 0, 1, 3))
    # upload changed values: only the patch nodes change
    new = tuple(b.copy() for b in bufs)
    for b in new:
        b[:n] += 1.0
    model.dev.upload_tree_state(new, n)
    after = {k: model.dev.download(g.level, k) for k in ("mass", "temp", "velo")}
    mask = np.zeros(g.NN, dtype=bool)
    mask[x.ravel()] = True
    own = g.owned
    assert np.array_equal(after["mass"][:, mask], full["mass"][:, mask] + 1.0)
    assert np.array_equal(after["mass"][:, own & ~mask], full["mass"][:, own & ~mask])
    with pytest.raises(WtError):
        model.dev.upload_tree_state(new, n + 1)
    model.close()


def test_checkpoint_exact_resume(tmp_path):
    """AdaptiveOcean.save / load: a run resumed from a checkpoint on a fresh
    handle takes the same steps as the run that was saved: the patch tree,
    every mask and every field of every level bit for bit."""
    ph = OceanParams()
    nz = 3
    G, levels, ics, a, RI = _pair(3, 5, nz, lambda g: bump_state(g, nz, seed=2, ph=ph), ph)
    for _ in range(3):
        a.step(300.0)
    path = str(tmp_path / "run.npz")
    a.save(path)
    b = AdaptiveOcean.load(path, G)
    assert b.istep == a.istep and b.level_end() == a.level_end()
    for _ in range(3):
        a.step(300.0)
        b.step(300.0)
    for g in levels:
        assert np.array_equal(a.patches(g.level), b.patches(g.level)), g.level
        for name in ("mask_n", "mask_e", "mass", "temp", "velo"):
            assert np.array_equal(a.dev.download(g.level, name), b.dev.download(g.level, name)), (g.level, name)
    assert a.dev.status() == 0 and b.dev.status() == 0
    a.close()
    b.close()
