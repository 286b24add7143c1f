"""GPU parity of the TRiSK trend and RK4 stepper against the CPU oracle,
through the C-ABI (libwtgpu.so).  Compared bit for bit (relative error 0):
the FP64 kernels are built without FMA contraction and follow the oracle's
operand order."""
import numpy as np
import pytest

import oracle
from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
from wavetrisk_hydrostatic_b200.model import TriskModel

pytestmark = pytest.mark.gpu
TOL = 0.0   # bit for bit: FP64 without FMA contraction, the oracle's operand order


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("level,nz", [(4, 1), (4, 4), (5, 8), (6, 3)])
def test_trend_matches_oracle(level, nz):
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=level * 10 + nz, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    dm, dt, dv = model.trend_ml()
    om, ot, ov, _ = oracle.trend(g, nz, ph, st)
    assert rel(dm, om) <= TOL
    assert rel(dv, ov) <= TOL
    assert np.array_equal(dt == 0, ot == 0)
    model.close()


@pytest.mark.parametrize("level,nz,steps", [(4, 2, 3), (5, 8, 2)])
def test_rk4_matches_oracle(level, nz, steps):
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=7, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    model.rk4(300.0, steps)
    out = model.download()
    m, t, v = oracle.rk4(g, nz, ph, st, 300.0, steps)
    assert rel(out["mass"], m) <= TOL
    assert rel(out["velo"], v) <= TOL
    assert rel(out["temp"], t) <= TOL if np.abs(t).max() > 0 else np.abs(out["temp"]).max() == 0
    model.close()


def test_rk4_host_buffers_match_resident_path():
    g = Grid(4, 4, radius=6371e3).level(4)
    nz = 3
    ph = OceanParams()
    st = jet_state(g, nz, seed=11, ph=ph)
    a = TriskModel(g, nz, st["topo"], ph)
    a.upload(st)
    a.rk4(300.0, 2)
    ref = a.download()
    b = TriskModel(g, nz, st["topo"], ph)
    b.upload(st)
    m, t, v = st["mass"].copy(), st["temp"].copy(), st["velo"].copy()
    b.rk4_host(300.0, 2, m, t, v)
    assert np.array_equal(m, ref["mass"]) and np.array_equal(v, ref["velo"])
    a.close(); b.close()


def test_mass_conserved_over_steps():
    g = Grid(5, 5, radius=6371e3).level(5)
    nz = 4
    ph = OceanParams()
    st = jet_state(g, nz, seed=5, ph=ph)
    model = TriskModel(g, nz, st["topo"], ph)
    model.upload(st)
    area = np.where(g.hex_inv > 0, 1 / np.where(g.hex_inv > 0, g.hex_inv, 1), 0)
    own = g.owned.copy()
    npole, spole = g.pole_ids()
    own[npole] = own[spole] = True

    def total(m):
        return sum(((m[k] + st["mean_m"][k]) * area)[own].sum() for k in range(nz))

    m0 = total(st["mass"])
    model.rk4(300.0, 20)
    out = model.download()
    assert abs(total(out["mass"]) / m0 - 1) < 1e-13
    assert np.isfinite(out["velo"]).all()
    model.close()


def test_rk4_is_deterministic():
    # a stage never writes the array it reads at neighbouring nodes
    g = Grid(4, 4, radius=6371e3).level(4)
    nz = 3
    ph = OceanParams()
    st = jet_state(g, nz, seed=11, ph=ph)
    outs = []
    for _ in range(3):
        m = TriskModel(g, nz, st["topo"], ph)
        m.upload(st)
        m.rk4(300.0, 3)
        outs.append(m.download())
        m.close()
    for o in outs[1:]:
        for k in ("mass", "temp", "velo"):
            assert np.array_equal(o[k], outs[0][k])


@pytest.mark.parametrize("level,nz", [(4, 2), (5, 8), (7, 2)])
def test_trend_kernel_variants_agree(level, nz, monkeypatch):
    """The TMA-staged trend kernel (default) and the L1 variant
    (WAVETRISK_TREND_KERNEL=plain) give identical RK4 states, and both match
    the oracle."""
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=3 + level, ph=ph)
    outs = []
    for variant in ("tma", "plain"):
        monkeypatch.setenv("WAVETRISK_TREND_KERNEL", variant)
        model = TriskModel(g, nz, st["topo"], ph)
        model.upload(st)
        model.rk4(300.0, 2)
        outs.append(model.download())
        assert model.status() == 0
        model.close()
    for key in ("mass", "temp", "velo"):
        assert np.array_equal(outs[0][key], outs[1][key])
    m, t, v = oracle.rk4(g, nz, ph, st, 300.0, 2)
    assert rel(outs[0]["mass"], m) <= TOL
    assert rel(outs[0]["velo"], v) <= TOL
