"""GPU parity of the mode-split time step with its implicit free surface
(RK4_split, src/time_integr.f90:360-382, and free_surface_update, :465-478)
against the CPU oracle on the hierarchy J3..J5, 2 layers, over a seamount:
the four RK_split stages, then eta_update (rhs_elliptic on every level, the
elliptic operator's coefficients rebuilt from the old free surface, FMG to
1e-10 from the old surface), barotropic_correction, u_update and
WT_after_step.  The solver's per-level iteration counts must equal the
oracle's; the free surface and the state of every level agree to 1e-9
relative (the solver's reductions are summed in another order)."""
import numpy as np
import pytest

import oracle
from wavetrisk_hydrostatic_b200 import Grid, OceanParams
from wavetrisk_hydrostatic_b200.cases import bump_state, seamount_topography
from wavetrisk_hydrostatic_b200.grid import halo_nodes
from wavetrisk_hydrostatic_b200.model import WaveletHierarchy, solver_opts

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("masks_kind", ["tolrnz", "built"])
def test_rk4_split_with_free_surface_matches_oracle(masks_kind):
    from oracle.wavelet import Hierarchy

    ph = OceanParams()
    lmin, lmax, nz = 3, 5, 2
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [bump_state(g, nz, seed=4, ph=ph, topo=seamount_topography(g, seed=4, radius=600e3)) for g in levels]
    rng = np.random.default_rng(5)
    etas = []
    for g in levels:
        e = rng.standard_normal(g.NN) * 0.05
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
    dt, theta1, theta2 = 600.0, 0.5, 1.0
    solver = dict(fine_tol=1e-10, coarse_tol=1e-10, max_vcycle=50, coarse_iter=300)
    dev = WaveletHierarchy(levels, [st["topo"] for st in states], nz, ph)
    for g, st, (mn, me), e in zip(levels, states, masks, etas):
        for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
            dev.upload(g.level, name, st[name])
        dev.upload(g.level, "mask_n", mn)
        dev.upload(g.level, "mask_e", me)
        dev.barotropic_upload(g.level, e, None)
    dev.elliptic_setup(dt, theta1, theta2, domain_level=G.domain_level)
    rep = dev.rk4_split(dt, theta1, theta2, solver_opts("fmg", 1e-10, max_vcycle=50, coarse_iter=300))
    assert rep.status == 0
    ref, ref_eta, its, He = oracle.rk4_split(levels, nz, ph, states, masks, etas, dt, theta1, theta2,
                                             domain_level=G.domain_level, keep_eta_hierarchy=True, **solver)
    assert list(rep.iterations)[:len(levels)] == its
    for q, g in enumerate(levels):
        own = np.nonzero(g.owned)[0]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        m, t, v = ref[q]
        assert _rel(dev.free_surface(g.level)[own], ref_eta[q][own]) <= 1e-9, (g.level, "eta")
        assert _rel(dev.download(g.level, "mass")[:, own], m[:, own]) <= 1e-9, (g.level, "mass")
        assert _rel(dev.download(g.level, "temp")[:, own], t[:, own]) <= 1e-9, (g.level, "temp")
        assert _rel(dev.download(g.level, "velo")[:, e], v[:, e]) <= 1e-9, (g.level, "velo")
    # the free surface moved: the solve is not a no-op
    assert _rel(ref_eta[-1], etas[-1]) > 1e-3
    # adapt: new masks from the layers, then the free surface compressed under
    # them and rebuilt (wt_free_surface_adapt against the oracle's)
    dev.mask_build(np.array([[2.0] * nz, [1e16] * nz, [0.02] * nz]), 0, lmax)
    new_masks = [(dev.download(g.level, "mask_n"), dev.download(g.level, "mask_e")) for g in levels]
    dev.free_surface_adapt()
    ref_eta2 = oracle.free_surface_adapt(levels, He, new_masks)
    for q, g in enumerate(levels):
        own = np.nonzero(g.owned)[0]
        assert _rel(dev.free_surface(g.level)[own], ref_eta2[q][own]) <= 1e-9, (g.level, "eta after adapt")
    assert dev.status() == 0
    dev.close()


def test_free_surface_update_refuses_a_mismatched_solver_setup():
    from wavetrisk_hydrostatic_b200 import _native as N

    ph = OceanParams()
    G = Grid(3, 4, radius=6371e3)
    levels = [G.level(3), G.level(4)]
    dev = WaveletHierarchy(levels, [np.full(g.NN, -4000.0) for g in levels], 2, ph)
    opts = solver_opts("fmg", 1e-8)
    rep = N.wt_solver_report()
    import ctypes as C
    assert N.lib().wt_free_surface_update(dev.h, 600.0, 1.0, 1.0, C.byref(opts), C.byref(rep)) == N.WT_ERR_STATE
    dev.elliptic_setup(300.0, 1.0, 1.0)
    assert N.lib().wt_free_surface_update(dev.h, 600.0, 1.0, 1.0, C.byref(opts), C.byref(rep)) == N.WT_ERR_STATE
    dev.close()


@pytest.mark.parametrize("init", ["dense", "reference"])
def test_mode_split_adaptive_steps_run(init):
    """ModeSplitOcean (RK4_split + adapt + inverse transform, the ensemble's
    member step) on J3..J5 x 2 over a seamount, from the dense start and from
    the reference's initial refinement (patch tree refined by adapt): every
    step's free-surface solve converges and the state and free surface stay
    finite and bounded."""
    from wavetrisk_hydrostatic_b200.adaptive import ModeSplitOcean

    ph = OceanParams()
    G = Grid(3, 5, radius=6371e3)
    levels = [G.level(l) for l in range(2, 6)]
    states = [bump_state(g, 2, seed=6, ph=ph, topo=seamount_topography(g, seed=6, radius=600e3)) for g in levels]
    root, states, levels = states[0], states[1:], levels[1:]
    model = ModeSplitOcean(G, 3, 5, 2, states, 1200.0, ph, tol=5e-3, init=init,
                           root_state=root if init == "reference" else None)
    for _ in range(5):
        rep = model.step()
        assert rep.status == 0 and rep.true_rel_residual <= 1e-8
    assert model.dev.status() == 0
    for name in ("mass", "temp", "velo"):
        assert np.isfinite(model.dev.download(5, name)).all()
    eta = model.dev.free_surface(5)
    assert np.isfinite(eta).all() and np.abs(eta).max() < 10.0
    for (mn, me), g in zip(model.masks(), levels):   # every mask entry is one of adapt's values
        assert mn.min() >= 0 and mn.max() <= 16 and me.min() >= 0 and me.max() <= 16
    model.close()


def test_mode_split_remaps_below_min_mass():
    """The reference's remap trigger in the mode-split step (min_mass <
    min_mass_remap, src/main.f90:447-454): with the threshold above every
    relative layer mass each step remaps, and the layers' total mass stays
    what the free surface says (the remap moves mass only within columns)."""
    from wavetrisk_hydrostatic_b200.adaptive import ModeSplitOcean

    ph = OceanParams()
    G = Grid(3, 5, radius=6371e3)
    levels = [G.level(l) for l in range(2, 6)]
    states = [bump_state(g, 4, seed=8, ph=ph, topo=seamount_topography(g, seed=8, radius=600e3)) for g in levels]
    root, states, levels = states[0], states[1:], levels[1:]
    g = levels[-1]
    own = np.nonzero(g.owned)[0]
    area = 1.0 / g.hex_inv[own]
    model = ModeSplitOcean(G, 3, 5, 4, states, 1200.0, ph, tol=5e-3, root_state=root, min_mass_remap=2.0)
    mean = model.dev.download(5, "mean_m")[:, own]
    m0 = float(np.sum((mean + states[-1]["mass"][:, own]) * area))
    for s in range(3):
        rep = model.step()
        assert rep.status == 0
        assert model.remaps == s + 1 and 0.5 < model.min_mass < 2.0
    assert model.dev.status() == 0
    mass = model.dev.download(5, "mass")
    assert np.isfinite(mass).all() and np.isfinite(model.dev.download(5, "velo")).all()
    assert abs(float(np.sum((mean + mass[:, own]) * area)) - m0) <= 1e-7 * m0
    model.close()
