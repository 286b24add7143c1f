"""ORACLE (test infrastructure only): the reference's patch tree and its
initial refinement, on the oracle's wavelet hierarchy.

`PatchTree` restates refine() (src/refine_patch.f90:12-49) on patch-existence
maps: level l holds 10 x (n_l/ps)^2 patches of ps x ps nodes (ps =
PATCH_SIZE = 2^PATCH_LEVEL, src/patch.f90:6, src/shared.f90:33; 4 for min
levels 3..6).  Level level_start is complete (add_second_level,
src/refine_patch.f90:247-268); a child patch is created where
check_child_required (src/refine_patch.f90:289-327) flags its parent patch's
quadrant, the parent exists and its level is below max_level; refine visits
the patches that exist when it starts (the Fortran loop bound is fixed at
entry), so one refine adds at most one level; level_end rises when a patch of
level level_end+1 is created (refine_patch1, :51-75); patches are never
removed.

`reference_init` restates initialize (src/main.f90:36-135) for an explicit
run with fixed thresholds: init_structures (level_end = level_start, masks
TOLRNZ on the root level min_level-1, add_second_level, mask_adj_child of the
root: src/main.f90:482-524, src/mask.f90:704-720), then count_active
(initial conditions on every level, forward_wavelet_transform from
level_end down to the root, src/main.f90:137-172) and adapt (src/adapt.f90:14-65)
until level_end reaches max_level or the patches the last adapt created hold
no significant wavelet, then one more adapt and count_active.

The hierarchy's levels above the tree's level_end hold ZERO masks, so the
mask-tested wavelet and restriction routines leave them out exactly as the
reference, which has no such level, does.
"""
from __future__ import annotations

import numpy as np

from .wavelet import TOLRNZ, ZERO, Hierarchy

# check_child_required's quadrants c = 0 NE, 1 SE, 2 SW, 3 NW (chd_offs,
# src/domain.f90:119) as (x, y) offsets of half a patch
QUADRANTS = ((1, 1), (1, 0), (0, 0), (0, 1))


class PatchTree:
    """Patch existence of levels ls .. lmax (bool arrays [10][n/ps][n/ps],
    index [lozenge, patch row j, patch column i])."""

    def __init__(self, ls: int, lmax: int, ps: int):
        self.ls, self.lmax, self.ps = ls, lmax, ps
        self.exist = {l: np.zeros((10, 2 ** l // ps, 2 ** l // ps), dtype=bool) for l in range(ls, lmax + 1)}
        self.exist[ls][...] = True  # add_second_level
        self.new = {l: np.zeros_like(e) for l, e in self.exist.items()}
        self.level_end = ls

    def flag_levels(self, max_level: int) -> int:
        """Top parent level whose patches refine() can refine."""
        return min(self.level_end, max_level - 1)

    def refine(self, flags: np.ndarray, max_level: int) -> bool:
        """refine(): flags are check_child_required of parent levels
        ls .. flag_levels(max_level), 4 quadrants a patch, lozenge-major.
        Returns whether a patch was created; self.new marks the new patches."""
        ps = self.ps
        snap = {l: e.copy() for l, e in self.exist.items()}
        for e in self.new.values():
            e[...] = False
        did = False
        o = 0
        for l in range(self.ls, self.flag_levels(max_level) + 1):
            npp = 2 ** l // ps
            f = flags[o:o + 10 * npp * npp * 4].reshape(10, npp, npp, 4).astype(bool)
            o += 10 * npp * npp * 4
            f &= snap[l][..., None]
            ch = np.zeros((10, 2 * npp, 2 * npp), dtype=bool)
            for c, (ox, oy) in enumerate(QUADRANTS):
                ch[:, oy::2, ox::2] |= f[..., c]
            new = ch & ~self.exist[l + 1]
            if new.any():
                did = True
                self.exist[l + 1] |= new
                self.new[l + 1] |= new
                if l == self.level_end:
                    self.level_end = l + 1
        if o != len(flags):
            raise ValueError("refine: flag count does not match the tree's levels")
        return did

    def node_map(self, g, which: str = "exist") -> np.ndarray:
        """Per padded node of level g: True where the owned node [0, n)^2 lies in
        an existing (or, which="new", a newly created) patch."""
        src = (self.exist if which == "exist" else self.new)[g.level]
        d, i, j = g.ij()
        own = (i >= 0) & (j >= 0) & (i < g.n) & (j < g.n)
        out = np.zeros(g.NN, dtype=bool)
        out[own] = src[d[own], j[own] // self.ps, i[own] // self.ps]
        return out

    def count_patches(self):
        return {l: int(e.sum()) for l, e in self.exist.items()}


def count_active_new(H: Hierarchy, tree: PatchTree, levels, threshold) -> tuple[int, int]:
    """count_active's counts over the nodes of the patches the last refine
    created: node wavelets (mass, Theta) and edge wavelets (velocity, the three
    edges a node holds) with |w| >= threshold(v, k)."""
    nz = H.nz
    thr = np.asarray(threshold).reshape(3, nz)
    nn = ne = 0
    for g in levels:
        if g.level <= tree.ls:
            continue
        sel = tree.node_map(g, "new")
        if not sel.any():
            continue
        for v, key in ((0, "w_m"), (1, "w_t")):
            w = H.field(g.level, key)[:, sel]
            nn += int(np.count_nonzero(np.abs(w) >= thr[v][:, None]))
        wv = H.field(g.level, "w_v").reshape(nz, 3, g.NN)[:, :, sel]
        ne += int(np.count_nonzero(np.abs(wv) >= thr[2][:, None, None]))
    return nn, ne


def adapt(H: Hierarchy, tree: PatchTree, threshold, max_level: int, level_fill: int = 0) -> bool:
    """adapt (src/adapt.f90:14-65) with refine() between the two halves of the
    mask sequence, then compress_wavelets on the levels refine left."""
    flags = H.mask_phase1(threshold, level_fill, max_level, tree.ps, tree.level_end, tree.flag_levels(max_level))
    did = tree.refine(flags, max_level)
    H.mask_phase2(tree.level_end)
    H.compress(le=tree.level_end)
    return did


class ReferenceInit:
    """initialize() of an explicit run with fixed thresholds on an oracle
    hierarchy of levels ls .. lmax (root = level ls-1 from the same grid).

    ics[l]: dict of mass, temp, velo (the initial conditions evaluated on level
    l, every level ls-1 .. lmax).  After run(), H holds the reference's state
    at the start of the time loop: scaling fields (initial conditions,
    restricted where children exist), wavelets of the last count_active, masks,
    and tree the patch tree."""

    KEYS = (("mass", "s_m"), ("temp", "s_t"), ("velo", "s_v"))

    def __init__(self, root, levels, nz, ics, threshold, max_level, ps=4, level_fill=0):
        self.root, self.levels, self.nz, self.ics = root, levels, nz, ics
        self.threshold = np.asarray(threshold, dtype=np.float64).reshape(3, nz)
        self.max_level, self.ps, self.level_fill = max_level, ps, level_fill
        self.ls = levels[0].level
        self.H = Hierarchy(levels, nz)
        self.R = Hierarchy([root, levels[0]], nz)
        self.tree = PatchTree(self.ls, levels[-1].level, ps)
        self.log = []

    def _init_masks(self):
        """init_masks (every root node and edge TOLRNZ), add_second_level
        (level_start ZERO), then mask_adj_child of the root (child nodes and
        edges of active root nodes and edges to ADJZONE); every finer level
        ZERO."""
        H, R = self.H, self.R
        for lv in self.levels:
            H.field(lv.level, "mask_n")[...] = ZERO
            H.field(lv.level, "mask_e")[...] = ZERO
        R.field(self.root.level, "mask_n")[...] = TOLRNZ
        R.field(self.root.level, "mask_e")[...] = TOLRNZ
        R.field(self.ls, "mask_n")[...] = ZERO
        R.field(self.ls, "mask_e")[...] = ZERO
        R.mask_adj_child(self.root.level)
        H.set(self.ls, "mask_n", R.field(self.ls, "mask_n"))
        H.set(self.ls, "mask_e", R.field(self.ls, "mask_e"))

    def count_active(self):
        """Initial conditions on every level, then forward_wavelet_transform
        from level_end down to the root (the root step on the two-level
        hierarchy: wavelets of level_start relative to the root)."""
        H, R, le = self.H, self.R, self.tree.level_end
        for lv in self.levels:
            for name, key in self.KEYS:
                H.set(lv.level, key, self.ics[lv.level][name])
        H.forward(le=le)
        for key in ("s_m", "s_t", "s_v"):
            R.set(self.ls, key, H.field(self.ls, key))
        for name, key in self.KEYS:
            R.set(self.root.level, key, self.ics[self.root.level][name])
        R.set(self.ls, "mask_n", H.field(self.ls, "mask_n"))
        R.set(self.ls, "mask_e", H.field(self.ls, "mask_e"))
        R.forward()
        for key in ("w_m", "w_t", "w_v"):
            H.set(self.ls, key, R.field(self.ls, key))

    def adapt(self):
        return adapt(self.H, self.tree, self.threshold, self.max_level, self.level_fill)

    def run(self, max_iter: int = 32):
        self._init_masks()
        self.count_active()
        it = 0
        while self.tree.level_end < self.max_level and it < max_iter:
            it += 1
            self.adapt()
            self.count_active()
            nn, ne = count_active_new(self.H, self.tree, self.levels, self.threshold)
            self.log.append((self.tree.level_end, nn, ne))
            if nn == 0 and ne == 0:
                break
        self.adapt()
        self.count_active()
        return self
