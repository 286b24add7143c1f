"""Host driver of the adaptive ocean time step on a hierarchy of levels whose
patch tree is partially refined.

It mirrors the reference's explicit (non-mode-split) incompressible run:
initialize (src/main.f90:36-135) builds the initial grid level by level
(count_active, adapt with refine(), until level_end reaches max_level or the
patches just made hold no significant wavelet), then time_step
(src/main.f90:405-444) does

    dt_step (RK4 with trend_ml and WT_after_step per stage)
    adapt (set_thresholds, the mask sequence with refine(), compress_wavelets)
    inverse_wavelet_transform (wav_coeff, sol)

Every level's fields are allocated on the device; the patch tree (one byte
per PATCH_SIZE^2 patch, refined on the device, include/wavetrisk_gpu.h) says
which patches exist, and the levels above its level_end hold ZERO masks.  The
thresholds follow initialize_thresholds_case and set_thresholds_case of the
reference's ocean test cases (test/seamount/test_case_module.f90:554-608): tol *
(rho0 dz_k, 1e16, Udim) by default, or tol * cal_lnorm("inf") with the same
floors and the 1 % / 99 % blending after step 10 when dynamic.  Everything
below runs on the device through the C-ABI; this class only sequences it.

init="dense" keeps the earlier start-up instead: the initial condition on the
finest level, its wavelets on every level at once, one adapt and the inverse
transform, with every patch present.
"""
from __future__ import annotations

import json

import numpy as np

from .cases import OceanParams
from .grid import Grid, halo_nodes
from .model import WaveletHierarchy, solver_opts

TOLRNZ, ZERO = 16, 0


def patch_size_for(min_level: int) -> int:
    """PATCH_SIZE = 2^PATCH_LEVEL with PATCH_LEVEL = MIN_LEVEL - DOMAIN_LEVEL - 1
    (src/shared.f90:33) and DOMAIN_LEVEL from the reference's parameter files
    (src/param_J3.f90 .. param_J9.f90: 0, 1, 2, 3 for MIN_LEVEL 3..6, then 2)."""
    domain_level = {3: 0, 4: 1, 5: 2, 6: 3}.get(min_level, 2)
    return 2 ** (min_level - domain_level - 1)


class AdaptiveOcean:
    def __init__(self, grid: Grid, min_level: int, max_level: int, nz: int, states: list[dict],
                 ph: OceanParams | None = None, tol: float = 5e-3, udim: float = 1.0, level_fill: int = 0,
                 dynamic_thresholds: bool = False, init: str = "reference", root_state: dict | None = None):
        """states[q]: dict of mass, temp, velo, mean_m, mean_t, topo of level
        min_level + q, the initial condition evaluated on that level;
        root_state the same on level min_level - 1 (init="reference": the
        reference keeps that level below level_start, and its forward transform
        takes level_start's wavelets from it).  init="dense": only the finest
        level's scaling fields are read."""
        self.ph = ph or OceanParams()
        self.levels = [grid.level(l) for l in range(min_level, max_level + 1)]
        self.nz, self.tol, self.udim = nz, tol, udim
        self.min_level, self.max_level, self.level_fill = min_level, max_level, level_fill
        self.dynamic = dynamic_thresholds
        self.topos = [np.asarray(st["topo"], dtype=np.float64) for st in states]
        self.dev = WaveletHierarchy(self.levels, self.topos, nz, self.ph)
        for g, st in zip(self.levels, states):
            for name in ("mean_m", "mean_t"):
                self.dev.upload(g.level, name, st[name])
        top = states[-1]
        for name in ("mass", "temp", "velo"):
            self.dev.upload(max_level, name, top[name])
        # initialize_thresholds_case: the mass scale of layer k is rho0 dz_k with
        # dz_k from the maximum depth (equal layers), whatever the bathymetry
        dz = np.full(nz, self.ph.depth / nz)
        lnorm = np.stack([self.ph.ref_density * dz, np.full(nz, 1e16), np.full(nz, udim)])
        self.threshold_def = tol * lnorm
        self.threshold = self.threshold_def.copy()
        self.istep = 0
        self.patch_size = patch_size_for(min_level)
        self.tree = False
        self.init_log = []
        if init == "reference":
            if root_state is None:
                raise ValueError("init='reference' needs root_state: the initial condition on level min_level-1")
            self._reference_init(grid, states, root_state)
        elif init == "dense":
            # initial grid: wavelets of the initial condition, masks, compression, inverse transform
            self.dev.forward()
            self.adapt()
            self.dev.inverse()
        else:
            raise ValueError(f"unknown init {init!r}")

    def _reference_init(self, grid: Grid, states: list[dict], root_state: dict) -> None:
        """initialize (src/main.f90:36-135) for fixed thresholds.

        init_structures (src/main.f90:482-524): masks TOLRNZ on the root level
        (init_masks, src/mask.f90:704-720), level_start's patches made
        (add_second_level), mask_adj_child of the root; level_end =
        level_start.  Then count_active (the initial condition on every level
        and forward_wavelet_transform down to the root, src/main.f90:137-172)
        and adapt until level_end reaches max_level or the patches the last
        adapt made hold no significant wavelet; then adapt and count_active
        once more.  The root level lives in a second two-level hierarchy
        (root, level_start) that gives level_start its wavelets."""
        ls, nz, dev = self.min_level, self.nz, self.dev
        root = grid.level(ls - 1)
        R = WaveletHierarchy([root, self.levels[0]], [root_state["topo"], states[0]["topo"]], nz, self.ph)
        try:
            for g in self.levels:
                dev.upload(g.level, "mask_n", ZERO)
                dev.upload(g.level, "mask_e", ZERO)
            R.upload(root.level, "mask_n", TOLRNZ)
            R.upload(root.level, "mask_e", TOLRNZ)
            R.upload(ls, "mask_n", ZERO)
            R.upload(ls, "mask_e", ZERO)
            R.mask_adj_child(root.level)
            dev.upload(ls, "mask_n", R.download(ls, "mask_n"))
            dev.upload(ls, "mask_e", R.download(ls, "mask_e"))
            dev.tree_init(self.patch_size)
            self.tree = True

            def count_active():
                dev.upload_many([(g.level, name, st[name]) for g, st in zip(self.levels, states)
                                 for name in ("mass", "temp", "velo")])
                dev.forward()
                R.upload_many([(ls, name, dev.download(ls, name)) for name in ("mass", "temp", "velo", "mask_n",
                                                                               "mask_e")]
                              + [(root.level, name, root_state[name]) for name in ("mass", "temp", "velo")])
                R.forward()
                dev.upload_many([(ls, name, R.download(ls, name)) for name in ("wc_mass", "wc_temp", "wc_velo")])

            count_active()
            while dev.tree_level_end() < self.max_level:
                self.set_thresholds()
                le, _ = dev.adapt(self.threshold, self.level_fill, self.max_level)
                count_active()
                nn, ne = dev.count_active(self.threshold)
                self.init_log.append((le, nn, ne))
                if nn == 0 and ne == 0:
                    break
            self.set_thresholds()
            dev.adapt(self.threshold, self.level_fill, self.max_level)
            count_active()
        finally:
            R.close()

    def level_end(self) -> int:
        """The patch tree's level_end (the hierarchy's top without a tree)."""
        return self.dev.tree_level_end() if self.tree else self.max_level

    def patches(self, level: int):
        """Patch existence of `level` ([10][n/ps][n/ps] bool), or None without a tree."""
        return self.dev.tree(level, self.patch_size)[0] if self.tree else None

    def set_thresholds(self) -> None:
        """set_thresholds_case (test/seamount/test_case_module.f90:554-581)."""
        if not self.dynamic:
            new = self.threshold_def
        else:
            new = self.tol * self.dev.lnorm("inf")
            floor = self.threshold_def / 10
            new = np.where(new < floor, self.threshold_def, new)
        self.threshold = 0.01 * new + 0.99 * self.threshold if self.istep >= 10 else new.copy()

    def adapt(self, patch_size: int = 0):
        """adapt (src/adapt.f90:14-65): with a patch tree the mask sequence with
        refine() inside and compression (returns None); without one the mask
        sequence on the whole hierarchy, returning the check_child_required
        flags when patch_size > 0."""
        self.set_thresholds()
        if self.tree:
            self.dev.adapt(self.threshold, self.level_fill, self.max_level)
            return None
        req = self.dev.mask_build(self.threshold, self.level_fill, self.max_level, patch_size)
        self.dev.compress()
        return req

    def step(self, dt: float) -> None:
        """One time step: RK4 of the hierarchy, adapt, inverse transform.  With
        fixed thresholds the whole step is one graph replay on the device
        (wt_adaptive_step); dynamic thresholds need cal_lnorm of the new state
        on the host between the RK4 and the mask sequence."""
        if not self.dynamic and (not self.tree or self.dev.tree_level_end() == self.max_level):
            # the step graph refines the tree on the device while its level_end is the top
            self.set_thresholds()
            self.dev.adaptive_step(dt, self.threshold, self.level_fill, self.max_level)
        else:
            self.dev.rk4_multi(dt, 1)
            self.adapt()
            if self.tree:   # as the graph's inverse: the parents the next step reads and the tree's
                self.dev.inverse_tree()
            else:
                self.dev.inverse()
        self.istep += 1

    def masks(self):
        return [(self.dev.download(g.level, "mask_n"), self.dev.download(g.level, "mask_e")) for g in self.levels]

    # every device field the next step reads (the RK stage buffers and the maps are rebuilt from these)
    CHECKPOINT_FIELDS = ("mass", "temp", "velo", "wc_mass", "wc_temp", "wc_velo", "mask_n", "mask_e", "mean_m",
                         "mean_t")

    def save(self, path: str) -> None:
        """Checkpoint for an exact resume: every level's scaling fields, wavelets, masks and layer means, the
        patch tree, the topography, the thresholds and the step count, in one .npz file.  A run resumed by
        load() takes the same steps, bit for bit, as the run that was saved.  (The reference's
        dump_adapt_mpi, src/io.f90:792-935, stores a pruned tree and the wavelets only and rebuilds the rest
        on restart; its file format is not this one.)"""
        arrays = {}
        for g in self.levels:
            for name in self.CHECKPOINT_FIELDS:
                arrays[f"L{g.level}_{name}"] = self.dev.download(g.level, name)
            arrays[f"L{g.level}_topo"] = self.topos[g.level - self.min_level]
            if self.tree:
                arrays[f"L{g.level}_patches"] = self.dev.tree(g.level, self.patch_size)[0].astype(np.uint8)
        meta = {"kind": "AdaptiveOcean", "min_level": self.min_level, "max_level": self.max_level, "nz": self.nz,
                "tol": self.tol, "udim": self.udim, "level_fill": self.level_fill, "dynamic": self.dynamic,
                "istep": self.istep, "tree": self.tree, "patch_size": self.patch_size,
                "level_end": self.level_end(), "threshold": self.threshold.tolist(),
                "threshold_def": self.threshold_def.tolist(), "ph": vars(self.ph)}
        np.savez(path, meta=np.array(json.dumps(meta)), **arrays)

    @classmethod
    def load(cls, path: str, grid: Grid) -> "AdaptiveOcean":
        """A model resumed from save()'s file on the grid it was made on."""
        z = np.load(path, allow_pickle=False)
        meta = json.loads(str(z["meta"]))
        if meta.get("kind") != "AdaptiveOcean":
            raise ValueError(f"{path}: not an AdaptiveOcean checkpoint")
        self = cls.__new__(cls)
        self.ph = OceanParams(**meta["ph"])
        self.min_level, self.max_level, self.nz = meta["min_level"], meta["max_level"], meta["nz"]
        self.tol, self.udim, self.level_fill = meta["tol"], meta["udim"], meta["level_fill"]
        self.dynamic, self.istep = meta["dynamic"], meta["istep"]
        self.patch_size, self.tree, self.init_log = meta["patch_size"], False, []
        self.levels = [grid.level(l) for l in range(self.min_level, self.max_level + 1)]
        self.topos = [z[f"L{g.level}_topo"] for g in self.levels]
        self.dev = WaveletHierarchy(self.levels, self.topos, self.nz, self.ph)
        self.threshold = np.array(meta["threshold"])
        self.threshold_def = np.array(meta["threshold_def"])
        for g in self.levels:
            for name in self.CHECKPOINT_FIELDS:
                self.dev.upload(g.level, name, z[f"L{g.level}_{name}"])
        if meta["tree"]:
            self.dev.tree_init(self.patch_size)
            self.dev.grid_sync([z[f"L{g.level}_patches"] for g in self.levels], meta["level_end"])
            self.tree = True
        return self

    def close(self) -> None:
        self.dev.close()


class ModeSplitOcean(AdaptiveOcean):
    """The adaptive time step with mode splitting (dt_step => RK4_split,
    src/time_integr.f90:360-382; free_surface_update :465-478) on the fully
    refined hierarchy: per step wt_rk4_split (the four RK_split stages with
    WT_after_step, then the implicit free-surface solve with coefficients from
    the old free surface, barotropic_correction, u_update and the free
    surface's own WT_after_step), then adapt (masks from the layers' mass,
    Theta and velocity thresholds, as mask_tol_vars tests layers 1..zlevels
    only; compression) and the inverse transform, both also of the free
    surface (layer zlevels+1 of sol, wt_free_surface_adapt).  The initial free
    surface of every level is the sum of its layers' mass perturbations over
    rho0, so layers and free surface start consistent.

    remap ('0', '1' or '2PPM'; None turns it off): after each step, as the
    reference's time_step does by default (remap = .true., src/main.f90:
    447-454), the Lagrangian layers are remapped to the hybrid grid
    z_k = a_k eta + b_k z_s of the initial layers (a_k = k/nz, b_k = 1 - a_k
    from the bottom) when the smallest relative layer mass (cpt_min_mass) is
    below min_mass_remap.  The default 2PPM stands in for the reference's
    default PPR reconstruction, which is not built."""

    def __init__(self, grid: Grid, min_level: int, max_level: int, nz: int, states: list[dict], dt: float,
                 ph: OceanParams | None = None, theta1: float = 1.0, theta2: float = 1.0, solver=None,
                 remap: str | None = "2PPM", min_mass_remap: float = 0.9, **kw):
        ph = ph or OceanParams()
        super().__init__(grid, min_level, max_level, nz, states, ph, **kw)
        self.dt, self.theta1, self.theta2 = float(dt), float(theta1), float(theta2)
        self.remap, self.min_mass_remap, self.remaps = remap, float(min_mass_remap), 0
        self.b_vert = 1.0 - np.arange(nz + 1) / nz
        self.a_vert = 1.0 - self.b_vert
        self.min_mass = None
        self.solver = solver if solver is not None else solver_opts("mixed", 1e-9, down_iter=2, up_iter=2,
                                                                     coarse_iter=6)
        for g, st in zip(self.levels, states):
            eta = st["mass"].sum(axis=0) / ph.ref_density
            halo_nodes(g, eta)
            self.dev.barotropic_upload(g.level, eta, None)
        self.dev.elliptic_setup(self.dt, self.theta1, self.theta2, domain_level=grid.domain_level)
        self.last_report = None

    def step(self, dt: float | None = None):
        """One mode-split time step; returns the free-surface solve's report."""
        if dt is not None and float(dt) != self.dt:
            raise ValueError("the free-surface solver is set up for dt = %g" % self.dt)
        self.set_thresholds()
        rep = self.dev.rk4_split(self.dt, self.theta1, self.theta2, self.solver)
        if self.tree:
            self.dev.adapt(self.threshold, self.level_fill, self.max_level)
            self.dev.inverse_tree()
        else:
            self.dev.mask_build(self.threshold, self.level_fill, self.max_level, 0)
            self.dev.compress()
            self.dev.inverse()
        self.dev.free_surface_adapt()
        if self.remap:
            self.min_mass = self.dev.min_mass(self.b_vert)
            if self.min_mass < self.min_mass_remap:
                self.dev.remap_vertical(self.remap, self.a_vert, self.b_vert)
                self.remaps += 1
        self.istep += 1
        self.last_report = rep
        return rep
