"""The wait-timeout path of the TMA-staged kernels (k_step1_tma, k_trend_tma
in csrc/trisk_tma.cuh), made to run without a fault: WT_TUNE_TEST_TMA_TIMEOUT
has every block declare more bytes than its copies deliver, so its bounded
mbarrier wait gives up after 20 us; the block then retires the extra bytes,
waits for its own copies and returns.  The handle reports WT_ERR_TIMEOUT,
stays usable, and after wt_clear_status the next step is bit-identical to a
clean one."""
import numpy as np
import pytest

from wavetrisk_hydrostatic_b200 import Grid, OceanParams, jet_state
from wavetrisk_hydrostatic_b200.model import TriskModel

pytestmark = pytest.mark.gpu
WT_ERR_TIMEOUT = -6


def test_tma_wait_timeout_is_reported_and_the_handle_recovers():
    level, nz, dt = 6, 2, 300.0          # level 6: n = 64, the TMA stepper
    g = Grid(level, level, radius=6371e3).level(level)
    ph = OceanParams()
    st = jet_state(g, nz, seed=3, ph=ph)
    m = TriskModel(g, nz, st["topo"], ph)
    m.upload(st)
    m.rk4(dt, 2)
    assert m.status() == 0
    clean = m.download()

    m.upload(st)
    m.test_tma_timeout(True)
    m.rk4(dt, 1)
    assert m.status() == WT_ERR_TIMEOUT
    assert m.status() == WT_ERR_TIMEOUT  # sticky until acknowledged
    m.test_tma_timeout(False)
    m.clear_status()
    assert m.status() == 0

    m.upload(st)
    m.rk4(dt, 2)
    assert m.status() == 0
    again = m.download()
    for k in ("mass", "temp", "velo"):
        assert np.array_equal(again[k], clean[k]), k
    m.close()


def test_tma_wait_timeout_on_the_hierarchy_step():
    """The finest level's k_step1_tma / k_trend_tma<MODE_ML> inside the
    hierarchy's captured RK4 graph (wt_rk4_multi) on J5..J6, with the
    needed-node maps off: with them the levels run persistent kernels over
    their work lists, and the TMA-staged kernels only without."""
    from wavetrisk_hydrostatic_b200.model import WaveletHierarchy

    lmin, lmax, nz, dt = 5, 6, 2, 300.0
    ph = OceanParams()
    G = Grid(lmin, lmax, radius=6371e3)
    levels = [G.level(l) for l in range(lmin, lmax + 1)]
    states = [jet_state(g, nz, seed=5 + q, ph=ph) for q, g in enumerate(levels)]
    dev = WaveletHierarchy(levels, [s["topo"] for s in states], nz, ph)
    dev.skip_inactive(False)

    def load():
        for g, s in zip(levels, states):
            for name in ("mass", "temp", "velo", "mean_m", "mean_t"):
                dev.upload(g.level, name, s[name])
            dev.upload(g.level, "mask_n", np.full(g.NN, 16, np.int32))
            dev.upload(g.level, "mask_e", np.full(3 * g.NN, 16, np.int32))

    load()
    dev.rk4_multi(dt)
    assert dev.status() == 0
    clean = [dev.download(lmax, k) for k in ("mass", "temp", "velo")]
    load()
    dev.test_tma_timeout(True)
    dev.rk4_multi(dt)
    assert dev.status() == WT_ERR_TIMEOUT
    dev.test_tma_timeout(False)
    dev.clear_status()
    load()
    dev.rk4_multi(dt)
    assert dev.status() == 0
    for a, b in zip([dev.download(lmax, k) for k in ("mass", "temp", "velo")], clean):
        assert np.array_equal(a, b)
    dev.close()
