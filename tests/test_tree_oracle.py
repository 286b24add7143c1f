"""The oracle's patch tree (refine, src/refine_patch.f90:12-49) and initial
refinement (initialize, src/main.f90:36-135) on the CPU: refine's rules on
hand-made flags, and the property the partially refined hierarchy rests on:
no mask outside the tree is ever set (the reference has no node there), after
the initialisation and after adaptive steps."""
import numpy as np
import pytest

import oracle
from oracle.tree import QUADRANTS, PatchTree, ReferenceInit, adapt
from wavetrisk_hydrostatic_b200 import Grid, OceanParams
from wavetrisk_hydrostatic_b200.adaptive import patch_size_for
from wavetrisk_hydrostatic_b200.cases import bump_state


def _flags(tree, max_level, marks):
    """check_child_required flags with the given (level, d, pj, pi, c) set."""
    out = []
    for l in range(tree.ls, tree.flag_levels(max_level) + 1):
        npp = 2 ** l // tree.ps
        f = np.zeros((10, npp, npp, 4), dtype=np.uint8)
        for (ml, d, pj, pi, c) in marks:
            if ml == l:
                f[d, pj, pi, c] = 1
        out.append(f.ravel())
    return np.concatenate(out) if out else np.zeros(0, dtype=np.uint8)


def test_patch_size_follows_the_parameter_files():
    assert [patch_size_for(l) for l in (3, 4, 5, 6, 7, 8)] == [4, 4, 4, 4, 16, 32]


def test_refine_rules():
    T = PatchTree(3, 5, 4)
    assert T.level_end == 3 and T.exist[3].all() and not T.exist[4].any()
    # quadrant c of parent patch (d, pj, pi) -> child patch (d, 2 pj + oy, 2 pi + ox)
    assert T.refine(_flags(T, 5, [(3, 2, 1, 0, 0), (3, 7, 0, 1, 2)]), 5)
    assert T.level_end == 4
    ox, oy = QUADRANTS[0]
    assert T.exist[4][2, 2 + oy, 0 + ox] and T.exist[4][7, 0, 2] and T.exist[4].sum() == 2
    assert np.array_equal(T.new[4], T.exist[4])
    # flags under a missing parent make nothing; one under an existing one
    # makes a level-5 patch and raises level_end; a repeated flag adds nothing
    assert T.refine(_flags(T, 5, [(4, 0, 0, 0, 0), (4, 2, 3, 1, 2), (3, 2, 1, 0, 0)]), 5)
    assert T.level_end == 5 and T.exist[5].sum() == 1 and T.exist[5][2, 6, 2]
    assert T.new[4].sum() == 0 and T.new[5].sum() == 1
    assert not T.refine(_flags(T, 5, [(4, 2, 3, 1, 2)]), 5)
    # max_level caps the parent levels refine visits
    T2 = PatchTree(3, 5, 4)
    assert not T2.refine(_flags(T2, 3, []), 3) and T2.level_end == 3


def _outside(H, tree, levels):
    bad = 0
    for g in levels:
        ex = tree.node_map(g)
        own = g.owned
        me = H.field(g.level, "mask_e").reshape(3, g.NN)
        bad += np.count_nonzero((H.field(g.level, "mask_n") != 0) & own & ~ex)
        bad += np.count_nonzero(((me != 0).any(axis=0)) & own & ~ex)
    return bad


@pytest.mark.parametrize("lmin,lmax,nz,tol,nsteps", [(3, 5, 2, 5e-3, 4), (3, 6, 2, 0.2, 2), (4, 6, 2, 5e-3, 2)])
def test_masks_stay_inside_the_tree(lmin, lmax, nz, tol, nsteps):
    oracle.set_threads(4)
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    root = G.level(lmin - 1)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    ics = {g.level: bump_state(g, nz, seed=2, ph=ph) for g in [root] + levels}
    dz = np.full(nz, ph.depth / nz)
    thr = tol * np.stack([ph.ref_density * dz, np.full(nz, 1e16), np.full(nz, 1.0)])
    RI = ReferenceInit(root, levels, nz, ics, thr, lmax, ps=patch_size_for(lmin)).run()
    H, tree = RI.H, RI.tree
    assert tree.level_end > lmin and RI.log
    # refinement went on while the new patches held significant wavelets
    assert all(nn + ne > 0 for _, nn, ne in RI.log[:-1])
    assert _outside(H, tree, levels) == 0
    # levels above level_end have no mask at all
    for g in levels:
        if g.level > tree.level_end:
            assert not H.field(g.level, "mask_n").any() and not H.field(g.level, "mask_e").any()
    keys = (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v"))
    base = [{k: v for k, v in ics[g.level].items() if k not in ("mass", "temp", "velo")} for g in levels]
    for _ in range(nsteps):
        cur = [dict(base[q], **{n: H.field(g.level, k).copy() for n, k in keys}) for q, g in enumerate(levels)]
        masks = [(H.field(g.level, "mask_n").copy(), H.field(g.level, "mask_e").copy()) for g in levels]
        oracle.rk4_multi(levels, nz, ph, cur, masks, 300.0, 1, H=H)
        adapt(H, tree, thr, lmax)
        H.inverse()
        assert _outside(H, tree, levels) == 0
