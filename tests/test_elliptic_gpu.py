"""GPU parity of the elliptic operator, wavelet restriction/prolongation and
the multigrid solvers against the CPU oracle, through the C-ABI.  Operator and
transforms: bit for bit (FP64, no contraction).  Solves: both reach the
tolerance with the same iteration counts; solutions agree to 1e-9 relative
(reductions are summed in a different order)."""
import numpy as np
import pytest

from oracle.elliptic import Hierarchy
from wavetrisk_hydrostatic_b200 import Grid
from wavetrisk_hydrostatic_b200.cases import bathymetry, elliptic_rhs
from wavetrisk_hydrostatic_b200.grid import halo_nodes
from wavetrisk_hydrostatic_b200.model import EllipticSolver, solver_opts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hier():
    g = Grid(4, 6, radius=6371e3)
    levels = [g.level(l) for l in (4, 5, 6)]
    topos = [bathymetry(lv, seed=2) for lv in levels]
    off = np.cumsum([0] + [lv.NN for lv in levels])
    return levels, topos, off


def owned_mask(levels):
    m = []
    for lv in levels:
        o = lv.owned.copy()
        n, s = lv.pole_ids()
        o[n] = o[s] = True
        m.append(o)
    return np.concatenate(m)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def random_ml(levels, seed):
    rng = np.random.default_rng(seed)
    out = []
    for lv in levels:
        x = rng.standard_normal(lv.NN)
        halo_nodes(lv, x)
        out.append(x)
    return np.concatenate(out)


@pytest.mark.parametrize("level", [4, 5, 6])
def test_operator_matches_oracle(hier, level):
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    H = Hierarchy(levels, topos)
    q = random_ml(levels, level)
    S.upload(u=q)
    S.apply(level)
    _, out = S.download()
    ref = H.apply(level, q)
    q_ = level - 4
    own = owned_mask(levels)[off[q_]:off[q_ + 1]]
    assert rel(out[off[q_]:off[q_ + 1]][own], ref[off[q_]:off[q_ + 1]][own]) == 0.0
    S.close()


def test_restriction_matches_oracle(hier):
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    H = Hierarchy(levels, topos)
    f = np.zeros(off[-1])
    f[off[2]:off[3]] = elliptic_rhs(levels[2], seed=9)
    S.upload(f=f)
    S.restrict()
    _, fg = S.download()
    fo = H.restrict_all(f)
    own = owned_mask(levels)
    assert rel(fg[own], fo[own]) == 0.0
    S.close()


def test_prolongation_matches_oracle(hier):
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    H = Hierarchy(levels, topos)
    u = random_ml(levels, 4)
    S.upload(u=u)
    S.prolong(6)
    ug, _ = S.download()
    uo = H.prolong(6, u)
    own = owned_mask(levels)[off[2]:off[3]]
    assert rel(ug[off[2]:off[3]][own], uo[off[2]:off[3]][own]) == 0.0
    S.close()


def test_l2_matches_oracle(hier):
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    H = Hierarchy(levels, topos)
    f = random_ml(levels, 8)
    S.upload(f=f)
    for l in (4, 5, 6):
        assert abs(S.l2(l) / H.l2(l, f) - 1) < 1e-13
    S.close()


@pytest.mark.parametrize("method", ["fmg", "srj"])
def test_solver_matches_oracle(hier, method):
    levels, topos, off = hier
    tol = 1e-8
    S = EllipticSolver(levels, topos)
    H = Hierarchy(levels, topos, fine_tol=tol, coarse_tol=tol, max_vcycle=30, coarse_iter=200, max_srj_iter=400)
    f = np.zeros(off[-1])
    f[off[2]:off[3]] = elliptic_rhs(levels[2], seed=5)
    f = H.restrict_all(f)
    S.upload(u=np.zeros(off[-1]), f=f)
    rep = S.solve(solver_opts(method, tol, max_vcycle=30, coarse_iter=200, max_srj_iter=400))
    ug, _ = S.download()
    uo, nrm, its = H.solve(np.zeros(off[-1]), f, method)
    assert rep.true_rel_residual <= tol * 1.01
    assert list(rep.iterations)[:3] == its
    own = owned_mask(levels)[off[2]:off[3]]
    assert rel(ug[off[2]:off[3]][own], uo[off[2]:off[3]][own]) <= 1e-9
    S.close()


def test_mixed_precision_reaches_1e_10(hier):
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    H = Hierarchy(levels, topos)
    f = np.zeros(off[-1])
    f[off[2]:off[3]] = elliptic_rhs(levels[2], seed=6)
    f = H.restrict_all(f)
    S.upload(u=np.zeros(off[-1]), f=f)
    rep = S.solve(solver_opts("mixed", 1e-10, down_iter=2, up_iter=2, coarse_iter=20))
    assert rep.status == 0 and rep.true_rel_residual <= 1e-10, (rep.true_rel_residual, rep.outer_iterations)
    S.close()


def test_solvers_interleaved_keep_converging(hier):
    """The reference-path FMG/SRJ swap work buffers between calls; the mixed and
    FP64 refinement solves (whose V-cycle is a captured graph) and the learned
    FCG must converge whatever ran before them on the same handle."""
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=5)
    S.upload(f=f)
    S.restrict()
    _, fr = S.download()
    S.learned_setup(1)
    S.learned_train(n_rhs=2, cycles=2, epochs=2)
    kw = dict(down_iter=2, up_iter=2, coarse_iter=20)
    seq = [("mg64", kw), ("fmg", dict(max_vcycle=50, coarse_iter=300)), ("mg64", kw), ("mixed", kw),
           ("fmg", dict(max_vcycle=50, coarse_iter=300)), ("srj", dict(max_srj_iter=4000, coarse_iter=300)),
           ("mixed", kw), ("mg64", kw), ("fcg_learned", kw), ("fmg", dict(max_vcycle=50, coarse_iter=300)),
           ("mg64", kw), ("fcg_mg", kw)]
    for name, k in seq:
        S.upload(u=np.zeros(off[-1]), f=fr)
        rep = S.solve(solver_opts(name, 1e-10, **k))
        assert rep.true_rel_residual <= 1e-9, (name, rep.true_rel_residual)
        if name in ("mg64", "mixed", "fcg_learned", "fcg_mg"):
            assert rep.status == 0 and rep.true_rel_residual <= 1e-10, name
    S.close()


def test_graph_solvers_after_odd_reference_sweeps(hier):
    """FMG with one pre-sweep (an odd number of u/tmp swaps on every level
    above level_start) and SRJ stopped after an odd sweep count leave the
    solver's u, tmp, res and au pointers rotated.  Every captured-graph solver
    run after them, twice each and with odd V-cycle sweep counts, must give
    the same solution as on a handle that never ran the reference path."""
    levels, topos, off = hier
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=6)
    kw = dict(down_iter=3, up_iter=3, coarse_iter=5)
    graph_methods = ("mixed", "mg64", "fcg_mg", "fcg_learned")

    def fresh(params=None):
        S = EllipticSolver(levels, topos)
        S.upload(f=f)
        S.restrict()
        _, fr = S.download()
        S.learned_setup(1)
        if params is None:
            S.learned_train(n_rhs=2, cycles=2, epochs=2, down_iter=3, up_iter=3, coarse_iter=5)
        else:
            S.learned_params(set_to=params)     # the same network on both handles
        return S, fr

    S0, fr = fresh()
    params = S0.learned_params()
    clean = {}
    for name in graph_methods:
        S0.upload(u=np.zeros(off[-1]), f=fr)
        rep = S0.solve(solver_opts(name, 1e-10, **kw))
        assert rep.status == 0 and rep.true_rel_residual <= 1e-10, name
        clean[name] = S0.download()[0][off[-2]:off[-1]].copy()
    S0.close()

    S, fr = fresh(params)
    disturb = [("fmg", dict(pre_iter=1, post_iter=2, max_vcycle=50, coarse_iter=300)),
               ("srj", dict(max_srj_iter=7, coarse_iter=300))]
    for dname, dk in disturb:
        S.upload(u=np.zeros(off[-1]), f=fr)
        S.solve(solver_opts(dname, 1e-10, **dk))
        for name in graph_methods:
            for _ in range(2):
                S.upload(u=np.zeros(off[-1]), f=fr)
                rep = S.solve(solver_opts(name, 1e-10, **kw))
                assert rep.status == 0 and rep.true_rel_residual <= 1e-10, (dname, name, rep.true_rel_residual)
                u = S.download()[0][off[-2]:off[-1]]
                assert np.array_equal(u, clean[name]), (dname, name, rel(u, clean[name]))
    S.close()


def test_autotune_picks_a_converging_candidate_and_keeps_u_f(hier):
    levels, topos, off = hier
    S = EllipticSolver(levels, topos)
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=6)
    S.upload(f=f)
    S.restrict()
    u0 = random_ml(levels, 3) * 1e-3
    _, fr = S.download()
    S.upload(u=u0, f=fr)
    cands = [(2, 2, 20), (2, 2, 6), (1, 1, 6)]
    best, ms = S.autotune("mg64", 1e-10, candidates=cands, repeats=2)
    assert (best.down_iter, best.up_iter, best.coarse_iter) in cands and best.method == 3 and ms > 0
    u1, f1 = S.download()
    assert np.array_equal(u1, u0) and np.array_equal(f1, fr)
    rep = S.solve(best)
    assert rep.status == 0 and rep.true_rel_residual <= 1e-10
    S.close()
