"""FP32 TRiSK flux stencils inside the FP64 single-level step
(WT_TUNE_FLUX_PRECISION = 32, csrc/trisk_mixed.cuh) against the FP64 oracle
on the plain-method configuration: uniform J5, 8 Boussinesq layers, jet and
white-noise free surface, RK4 with dt 300 s, 100 steps.

Reported per step (printed with -s): the largest error of the layer mass,
Theta mass and velocity relative to each field's largest magnitude, and the
relative change of the total mass.  Measured on B200: one trend 4.3e-5
(mass tendency: the divergence is a difference of six fluxes of 1e9, each
rounded to FP32) and 1.0e-7 (velocity tendency); the state stays within
3e-5 of the FP64 oracle's every step (2e-7 after 100 steps) and the total
mass of every layer is conserved to 4e-15 (the FP64 divergence of shared FP32
fluxes telescopes).  Bounds: 1e-4 for one trend and for the state after
every step, 1e-6 after 100 steps, 1e-13 for the total mass."""
import numpy as np
import pytest

import oracle
from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
from wavetrisk_hydrostatic_b200.model import TriskModel

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _total_mass(g, mass):
    own = np.nonzero(g.owned)[0]
    area = 1.0 / g.hex_inv[own]
    n, s = g.pole_ids()
    return mass[:, own] @ area + mass[:, n] / g.hex_inv[n] + mass[:, s] / g.hex_inv[s]


def test_mixed_trend_within_fp32_rounding_of_fp64():
    g = Grid(5, 5, radius=6371e3).level(5)
    ph = OceanParams()
    nz = 8
    st = jet_state(g, nz, seed=0, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    d64 = model.trend_ml()
    model.flux_precision(32)
    d32 = model.trend_ml()
    own = np.nonzero(g.owned)[0]
    edges = np.concatenate([own, own + g.NN, own + 2 * g.NN])
    errs = [_rel(d32[0][:, own], d64[0][:, own]), _rel(d32[2][:, edges], d64[2][:, edges])]
    print("one trend, FP32 fluxes vs FP64: dmass", errs[0], "dvelo", errs[1])
    assert max(errs) < 1e-4 and max(errs) > 0   # the mass divergence: differences of O(1e9) FP32 fluxes
    model.close()


def test_mixed_plain_method_100_steps_against_fp64_oracle():
    oracle.set_threads(8)
    g = Grid(5, 5, radius=6371e3).level(5)
    ph = OceanParams()
    nz, dt = 8, 300.0
    st = jet_state(g, nz, seed=0, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    model.flux_precision(32)
    own = np.nonzero(g.owned)[0]
    edges = np.concatenate([own, own + g.NN, own + 2 * g.NN])
    cur = dict(st)
    m0 = _total_mass(g, st["mass"] + st["mean_m"])
    worst = 0.0
    for s in range(100):
        model.rk4(dt, 1)
        out = model.download()
        m, t, v = oracle.rk4(g, nz, ph, cur, dt, 1)
        cur = dict(cur, mass=m, temp=t, velo=v)
        e = (_rel(out["mass"][:, own], m[:, own]), _rel(out["temp"][:, own], t[:, own]),
             _rel(out["velo"][:, edges], v[:, edges]))
        dmass = float(np.abs(_total_mass(g, out["mass"] + st["mean_m"]) / m0 - 1).max())
        if s % 10 == 9 or s == 0:
            print(f"step {s + 1:3d}: rel err mass {e[0]:.2e} temp {e[1]:.2e} velo {e[2]:.2e}, "
                  f"total mass change {dmass:.1e}")
        worst = max(worst, *e)
        assert dmass < 1e-13, (s, dmass)
    assert worst < 1e-4, worst
    assert max(e) < 1e-6, e     # after 100 steps
    model.close()


def test_hierarchy_steps_refuse_fp32_fluxes():
    from wavetrisk_hydrostatic_b200 import _native as N
    from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

    G = Grid(3, 4, radius=6371e3)
    levels = [G.level(3), G.level(4)]
    H = WaveletHierarchy(levels, [np.full(g.NN, -4000.0) for g in levels], 2)
    N.check("wt_tune", N.lib().wt_tune(H.h, 3, 32))
    assert N.lib().wt_rk4_multi(H.h, 100.0, 1) == N.WT_ERR_STATE
    N.check("wt_tune", N.lib().wt_tune(H.h, 3, 64))
    H.close()
