"""GPU parity against the CPU oracle at the sizes of the benchmark
configurations, through the C-ABI.

* Plain method (uniform J5, 8 layers, jet + white-noise free surface, RK4
  dt 300 s): the state after every one of 100 steps, bit for bit.
* Adaptive J4..J7, 16 layers (jet + 8 Gaussian bumps, tol 5e-3, dt 150 s),
  the initial grid refined level by level as the reference's initialize
  does: the patch tree and every mask of every level after every one of 20
  steps, bit for bit; the scaling fields of every level at the end, bit for
  bit.
* Elliptic: the operator at J7 and J8, restriction J8 -> J5 and prolongation
  into J7 and J8 on the hierarchy J5..J8; FMG and SRJ at J7 with the oracle's
  iteration counts.
* The benchmark's adaptive workload at J5..J8, 32 layers (seamount, jet and
  bumps, dt 75 s, the reference's initial refinement): tree and masks after
  every one of 3 steps bit for bit, fields at the end bit for bit.

The FP64 kernels are compiled without FMA contraction and follow the oracle's
operand order, so their results are compared with np.array_equal; the
solvers' reductions are summed in a different order (1e-9 on the solution,
exact iteration counts)."""
import numpy as np
import pytest

import oracle
from oracle.elliptic import Hierarchy as EHier
from oracle.tree import ReferenceInit, adapt
from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
from wavetrisk_hydrostatic_b200.adaptive import AdaptiveOcean, patch_size_for
from wavetrisk_hydrostatic_b200.cases import bathymetry, bump_state, elliptic_rhs, seamount_topography
from wavetrisk_hydrostatic_b200.grid import halo_nodes
from wavetrisk_hydrostatic_b200.model import EllipticSolver, TriskModel, solver_opts

pytestmark = pytest.mark.gpu
KEYS = (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v"))


def _owned_idx(g):
    own = np.nonzero(g.owned)[0]
    return own, np.concatenate([own, own + g.NN, own + 2 * g.NN])


def test_plain_method_j5x8_100_steps_every_step():
    oracle.set_threads(8)
    g = Grid(5, 5, radius=6371e3).level(5)
    ph = OceanParams()
    nz, dt = 8, 300.0
    st = jet_state(g, nz, seed=0, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    cur = dict(st)
    own, edges = _owned_idx(g)
    for s in range(100):
        model.rk4(dt, 1)
        out = model.download()
        m, t, v = oracle.rk4(g, nz, ph, cur, dt, 1)
        cur = dict(cur, mass=m, temp=t, velo=v)
        assert np.array_equal(out["mass"][:, own], m[:, own]), s
        assert np.array_equal(out["temp"][:, own], t[:, own]), s
        assert np.array_equal(out["velo"][:, edges], v[:, edges]), s
    model.close()


def _adaptive_pair(lmin, lmax, nz, make, ph):
    """The device model and the oracle hierarchy after the reference's initial
    refinement (the patch tree grown level by level from level_start + 1),
    and the per-level inputs the oracle's steps need besides the state."""
    G = Grid(lmin, lmax, radius=6371e3)
    root = G.level(lmin - 1)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    ics = {g.level: make(g) for g in [root] + levels}
    states = [ics[g.level] for g in levels]
    model = AdaptiveOcean(G, lmin, lmax, nz, states, ph, tol=5e-3, root_state=ics[root.level])
    RI = ReferenceInit(root, levels, nz, ics, model.threshold_def, lmax, ps=patch_size_for(lmin)).run()
    base = [{k: v for k, v in st.items() if k not in ("mass", "temp", "velo")} for st in states]
    return levels, model, RI, base


def _run_adaptive(levels, model, RI, nz, ph, dt, nsteps, base):
    lmax = levels[-1].level
    H, tree = RI.H, RI.tree
    for s in range(nsteps):
        cur = [dict(base[q], **{n: H.field(g.level, k).copy() for n, k in KEYS}) for q, g in enumerate(levels)]
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
        oracle.rk4_multi(levels, nz, ph, cur, masks, dt, 1, H=H)
        adapt(H, tree, model.threshold_def, lmax)
        H.inverse()
        model.step(dt)
        assert model.level_end() == tree.level_end, s
        for g, (mn, me) in zip(levels, model.masks()):
            assert np.array_equal(model.patches(g.level), tree.exist[g.level]), (s, g.level, "tree")
            assert np.array_equal(mn, H.field(g.level, "mask_n")), (s, g.level, "mask_n")
            assert np.array_equal(me, H.field(g.level, "mask_e")), (s, g.level, "mask_e")
    for g in levels:  # on the nodes of existing patches, where the state after a step is complete
        own = np.nonzero(g.owned & tree.node_map(g))[0]
        edges = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        for name, key in KEYS:
            k = edges if name == "velo" else own
            d, o = model.dev.download(g.level, name)[:, k], H.field(g.level, key)[:, k]
            assert np.array_equal(d, o), (g.level, name, float(np.abs(d - o).max()))
    assert model.dev.status() == 0


def test_adaptive_j4_j7_x16_20_steps_masks_every_step():
    oracle.set_threads(10)
    ph = OceanParams()
    nz = 16
    levels, model, RI, base = _adaptive_pair(4, 7, nz, lambda g: bump_state(g, nz, seed=1, ph=ph), ph)
    _run_adaptive(levels, model, RI, nz, ph, 150.0, 20, base)
    model.close()


def test_benchmark_workload_j5_j8_x32_3_steps():
    oracle.set_threads(10)
    ph = OceanParams()
    nz = 32
    make = lambda g: bump_state(g, nz, seed=1, ph=ph, topo=seamount_topography(g, seed=1))
    levels, model, RI, base = _adaptive_pair(5, 8, nz, make, ph)
    _run_adaptive(levels, model, RI, nz, ph, 75.0, 3, base)
    model.close()


@pytest.fixture(scope="module")
def ehier():
    g = Grid(5, 8, radius=6371e3)
    levels = [g.level(l) for l in range(5, 9)]
    topos = [bathymetry(lv, seed=2) for lv in levels]
    off = np.cumsum([0] + [lv.NN for lv in levels])
    return levels, topos, off


def _owned_nodes(levels):
    m = []
    for lv in levels:
        o = lv.owned.copy()
        n, s = lv.pole_ids()
        o[n] = o[s] = True
        m.append(o)
    return np.concatenate(m)


def test_elliptic_operator_transfer_at_j7_j8(ehier):
    levels, topos, off = ehier
    S = EllipticSolver(levels, topos)
    H = EHier(levels, topos)
    rng = np.random.default_rng(3)
    q = []
    for lv in levels:
        x = rng.standard_normal(lv.NN)
        halo_nodes(lv, x)
        q.append(x)
    q = np.concatenate(q)
    own = _owned_nodes(levels)
    for level in (7, 8):
        S.upload(u=q)
        S.apply(level)
        _, out = S.download()
        ref = H.apply(level, q)
        k = level - 5
        sl = slice(off[k], off[k + 1])
        assert np.array_equal(out[sl][own[sl]], ref[sl][own[sl]]), level
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=9)
    S.upload(f=f)
    S.restrict()
    _, fg = S.download()
    assert np.array_equal(fg[own], H.restrict_all(f)[own])
    for fine in (7, 8):
        S.upload(u=q)
        S.prolong(fine)
        ug, _ = S.download()
        uo = H.prolong(fine, q)
        k = fine - 5
        sl = slice(off[k], off[k + 1])
        assert np.array_equal(ug[sl][own[sl]], uo[sl][own[sl]]), fine
    S.close()


@pytest.mark.parametrize("method", ["fmg", "srj"])
def test_elliptic_solvers_at_j7_iteration_counts(method):
    g = Grid(5, 7, radius=6371e3)
    levels = [g.level(l) for l in range(5, 8)]
    topos = [bathymetry(lv, seed=2) for lv in levels]
    off = np.cumsum([0] + [lv.NN for lv in levels])
    tol = 1e-8
    kw = dict(max_vcycle=30, coarse_iter=200, max_srj_iter=800)
    S = EllipticSolver(levels, topos)
    H = EHier(levels, topos, fine_tol=tol, coarse_tol=tol, **kw)
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=5)
    f = H.restrict_all(f)
    S.upload(u=np.zeros(off[-1]), f=f)
    rep = S.solve(solver_opts(method, tol, **kw))
    ug, _ = S.download()
    uo, nrm, its = H.solve(np.zeros(off[-1]), f, method)
    assert rep.true_rel_residual <= tol * 1.01
    assert list(rep.iterations)[:3] == its
    own = _owned_nodes(levels)[off[-2]:off[-1]]
    a, b = ug[off[-2]:off[-1]][own], uo[off[-2]:off[-1]][own]
    assert np.abs(a - b).max() / np.abs(b).max() <= 1e-9
    S.close()
