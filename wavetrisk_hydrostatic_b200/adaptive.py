"""Host driver of the adaptive ocean time step on a fully refined hierarchy.

It mirrors the reference's time loop for an explicit (non-mode-split)
incompressible run, time_step in src/main.f90:405-444:

    dt_step (RK4 with trend_ml and WT_after_step per stage)
    adapt (set_thresholds, the mask sequence, compress_wavelets)
    inverse_wavelet_transform (wav_coeff, sol)

on levels [min_level, max_level] with every patch present: refine() has no
patch to create, so adapt reduces to its mask sequence (check_child_required
is still returned).  The thresholds follow initialize_thresholds_case and
set_thresholds_case of the reference's ocean test cases
(test/seamount/test_case_module.f90:554-608): tol * (rho0 dz_k, 1e16, Udim)
by default, or tol * cal_lnorm("inf") with the same floors and the 1 % / 99 %
blending after step 10 when dynamic.  Everything below runs on the device
through the C-ABI (include/wavetrisk_gpu.h); this class only sequences it.
"""
from __future__ import annotations

import numpy as np

from .cases import OceanParams
from .grid import Grid, halo_nodes
from .model import WaveletHierarchy, solver_opts


class AdaptiveOcean:
    def __init__(self, grid: Grid, min_level: int, max_level: int, nz: int, states: list[dict],
                 ph: OceanParams | None = None, tol: float = 5e-3, udim: float = 1.0, level_fill: int = 0,
                 dynamic_thresholds: bool = False):
        """states[q]: dict of mass, temp, velo, mean_m, mean_t, topo of level
        min_level + q; the scaling fields of the finest level are the initial
        condition, the coarser ones are recomputed by the forward transform."""
        self.ph = ph or OceanParams()
        self.levels = [grid.level(l) for l in range(min_level, max_level + 1)]
        self.nz, self.tol, self.udim = nz, tol, udim
        self.min_level, self.max_level, self.level_fill = min_level, max_level, level_fill
        self.dynamic = dynamic_thresholds
        self.dev = WaveletHierarchy(self.levels, [st["topo"] for st in states], nz, self.ph)
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
        # initial grid: wavelets of the initial condition, masks, compression, inverse transform
        self.dev.forward()
        self.adapt()
        self.dev.inverse()

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
        """adapt (src/adapt.f90:14-65) on the dense hierarchy; returns the
        check_child_required flags when patch_size > 0."""
        self.set_thresholds()
        req = self.dev.mask_build(self.threshold, self.level_fill, self.max_level, patch_size)
        self.dev.compress()
        return req

    def step(self, dt: float) -> None:
        """One time step: RK4 of the hierarchy, adapt, inverse transform.  With
        fixed thresholds the whole step is one graph replay on the device
        (wt_adaptive_step); dynamic thresholds need cal_lnorm of the new state
        on the host between the RK4 and the mask sequence."""
        if not self.dynamic:
            self.set_thresholds()
            self.dev.adaptive_step(dt, self.threshold, self.level_fill, self.max_level)
        else:
            self.dev.rk4_multi(dt, 1)
            self.adapt()
            self.dev.inverse()
        self.istep += 1

    def masks(self):
        return [(self.dev.download(g.level, "mask_n"), self.dev.download(g.level, "mask_e")) for g in self.levels]

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
    rho0, so layers and free surface start consistent."""

    def __init__(self, grid: Grid, min_level: int, max_level: int, nz: int, states: list[dict], dt: float,
                 ph: OceanParams | None = None, theta1: float = 1.0, theta2: float = 1.0, solver=None, **kw):
        ph = ph or OceanParams()
        super().__init__(grid, min_level, max_level, nz, states, ph, **kw)
        self.dt, self.theta1, self.theta2 = float(dt), float(theta1), float(theta2)
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
        req = self.dev.mask_build(self.threshold, self.level_fill, self.max_level, 0)
        del req
        self.dev.compress()
        self.dev.inverse()
        self.dev.free_surface_adapt()
        self.istep += 1
        self.last_report = rep
        return rep
