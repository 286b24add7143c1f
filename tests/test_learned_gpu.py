"""The learned free-surface preconditioner on the GPU, through the C-ABI:
its node layout, the preconditioner and the gradient of the training loss
against the CPU oracle (float64 from the same BF16-rounded weights; the GPU
accumulates in FP32 and stores BF16 activations, so a hidden activation can
land one BF16 step away where the accumulation order moves it across a
rounding boundary: 2e-3 relative in the 2-norm on the output and the
gradient), the tensor-core layer exactly (operands whose sums are exact in
FP32, so any order gives the oracle's bits), training on residual/error pairs
from the FP64 multigrid, streamed in batches, and flexible CG preconditioned
by a V-cycle plus the trained network's correction: it reaches the true FP64
residual 1e-10 in fewer iterations than flexible CG with the V-cycle alone,
and the V-cycle alone takes over when the network fails to contract."""
import numpy as np
import pytest

from oracle import learned as LO
from oracle.elliptic import Hierarchy
from wavetrisk_hydrostatic_b200 import Grid
from wavetrisk_hydrostatic_b200.cases import bathymetry, elliptic_rhs
from wavetrisk_hydrostatic_b200.grid import halo_nodes
from wavetrisk_hydrostatic_b200.model import EllipticSolver, solver_opts

pytestmark = pytest.mark.gpu


def make(lmin, lmax, seed=1):
    g = Grid(lmin, lmax, radius=6371e3)
    levels = [g.level(l) for l in range(lmin, lmax + 1)]
    topos = [bathymetry(lv, seed=seed) for lv in levels]
    return levels, topos, EllipticSolver(levels, topos)


@pytest.fixture(scope="module")
def small():
    levels, topos, S = make(4, 5)
    S.learned_setup(3)
    slot, tap = LO.layout(levels[-1])
    yield S, levels, topos, slot, tap
    S.close()


def small_own(small):
    _, levels, _, slot, _ = small
    return levels[-1].owned[slot].astype(np.float64)


def test_layout_matches_oracle(small):
    S, _, _, slot, tap = small
    ns, s_gpu, t_gpu = S.learned_layout(full=True)
    assert ns == slot.size
    assert np.array_equal(s_gpu, slot) and np.array_equal(t_gpu, tap)


def nrel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("slope", [1.0, 0.25])
def test_infer_matches_oracle(small, slope):
    S, _, topos, slot, tap = small
    theta = LO.init_params(11)
    S.learned_params(theta)
    S.learned_activation(slope)
    assert np.array_equal(S.learned_params(), theta)
    rng = np.random.default_rng(2)
    r = rng.standard_normal(slot.size) * 3e-4
    z = S.learned_infer(r)
    S.learned_activation(1.0)
    ref = LO.infer(theta, r, topos[-1][slot], tap, small_own(small), slope)
    assert nrel(z, ref) <= 2e-3, nrel(z, ref)
    assert np.abs(z - ref).max() <= 2e-2 * np.abs(ref).max()


def test_tensor_core_layer_is_exact():
    """Depth 4125 m (feature 0.5), residual +-1 (rms 1), dyadic weights and
    slope 1/4: every sum up to the stored second hidden layer is exact in FP32,
    so the tcgen05 layer must reproduce the oracle's BF16 activations bit for
    bit; the last layer's FP32 sum then leaves 1e-6 at most.  A wrong operand
    layout, descriptor or accumulator read-back shows as an O(1) error."""
    levels, _, _ = make(4, 5)
    topos = [np.full(lv.NN, -4125.0) for lv in levels]
    S = EllipticSolver(levels, topos)
    try:
        S.learned_setup(3)
        slot, tap = LO.layout(levels[-1])
        rng = np.random.default_rng(8)
        theta = (rng.integers(-8, 9, LO.NPARAMS) / 16.0).astype(np.float32)
        S.learned_params(theta)
        own = levels[-1].owned[slot].astype(np.float64)
        for tc in (True, False):
            S.learned_tensor_cores(tc)
            S.learned_activation(0.25)
            r = rng.choice([-1.0, 1.0], slot.size)
            z = S.learned_infer(r)
            ref = LO.infer(theta, r, topos[-1][slot], tap, own, 0.25)
            assert np.abs(ref).max() > 1.0
            assert np.abs(z - ref).max() <= 1e-6 * np.abs(ref).max(), (tc, np.abs(z - ref).max())
        assert S.status() == 0
    finally:
        S.close()


def test_tensor_cores_match_cuda_cores(small):
    S, _, _, slot, _ = small
    S.learned_params(LO.init_params(13))
    S.learned_activation(0.25)
    r = np.random.default_rng(6).standard_normal(slot.size)
    S.learned_tensor_cores(False)
    z0 = S.learned_infer(r)
    S.learned_tensor_cores(True)
    z1 = S.learned_infer(r)
    S.learned_activation(1.0)
    assert nrel(z1, z0) <= 2e-3, nrel(z1, z0)


@pytest.mark.parametrize("slope", [1.0, 0.25])
def test_gradient_matches_oracle(small, slope):
    S, levels, topos, slot, tap = small
    theta = LO.init_params(12)
    S.learned_params(theta)
    S.learned_activation(slope)
    rng = np.random.default_rng(4)
    r, e = rng.standard_normal(slot.size), rng.standard_normal(slot.size) * 0.3
    loss, g = S.learned_grad(r, e)
    S.learned_activation(1.0)
    H = Hierarchy(levels, topos)
    lv, off = levels[-1], S.offsets

    def apply_L(d):
        x = d.copy()
        halo_nodes(lv, x)
        full = np.zeros(off[-1])
        full[off[-2]:] = x
        return H.apply(lv.level, full)[off[-2]:]

    loss_o, g_o = LO.energy_loss_and_grad(theta, r, e, topos[-1][slot], tap, slot, lv.hex_inv, lv.NN, apply_L,
                                          small_own(small), slope)
    assert abs(loss - loss_o) <= 1e-3 * loss_o, (loss, loss_o)
    o = 0
    for name, shp in LO.SHAPES:                      # every parameter block on its own scale
        k = int(np.prod(shp))
        a, b = g[o:o + k].astype(np.float64), g_o[o:o + k]
        assert nrel(a, b) <= 2e-3, (name, nrel(a, b))
        o += k


@pytest.fixture(scope="module")
def trained():
    levels, topos, S = make(4, 6)
    S.learned_setup(1)
    rep = S.learned_train(n_rhs=8, cycles=4, epochs=15, lr=2e-3, seed=1)
    off = S.offsets
    f = np.zeros(off[-1])
    f[off[-2]:off[-1]] = elliptic_rhs(levels[-1], seed=2)
    slot, _ = LO.layout(levels[-1])
    yield S, rep, f, off[-2] + slot                  # the finest level's nodes in the multi-level arrays
    S.close()


def run(S, f, method, **kw):
    S.upload(u=np.zeros_like(f), f=f)
    rep = S.solve(solver_opts(method, 1e-10, down_iter=2, up_iter=2, coarse_iter=20, ir_max=400, **kw))
    u, _ = S.download()
    return rep, u


def test_training_reduces_loss(trained):
    _, rep, _, _ = trained
    assert rep.pairs == 32 and rep.steps == 32 * 15
    assert rep.loss_last_epoch < 0.5 * rep.loss_first_epoch


def test_streamed_training_reduces_loss():
    """Pairs generated and trained two right-hand sides at a time."""
    levels, topos, S = make(4, 5)
    try:
        S.learned_setup(2)
        S.learned_activation(0.25)
        rep = S.learned_train(n_rhs=8, cycles=2, epochs=3, lr=2e-3, seed=3, batch_rhs=2)
        assert rep.pairs == 16 and rep.steps == 16 * 3
        assert rep.loss_last_epoch < 0.7 * rep.loss_first_epoch, (rep.loss_first_epoch, rep.loss_last_epoch)
        assert S.status() == 0
    finally:
        S.close()


def test_learned_fcg_beats_fcg_without_network(trained):
    """The method without the network is FCG preconditioned by the V-cycle
    alone; the trained network's correction must save iterations over it."""
    S, _, f, nodes = trained
    r_net, u_net = run(S, f, "fcg_learned")
    r_v, _ = run(S, f, "fcg_mg")
    r_mg, u_mg = run(S, f, "mg64")
    assert r_net.status == 0 and r_v.status == 0 and r_mg.status == 0
    assert r_net.true_rel_residual <= 1e-10 and r_v.true_rel_residual <= 1e-10
    assert r_net.precond_fallback == 0
    q = len(S.offsets) - 2
    assert r_net.iterations[q] < r_v.iterations[q], (r_net.iterations[q], r_v.iterations[q])
    assert np.abs(u_net[nodes] - u_mg[nodes]).max() <= 1e-8 * np.abs(u_mg[nodes]).max()


def test_fallback_when_network_fails(trained):
    S, _, f, _ = trained
    keep = S.learned_params()
    bad = np.random.default_rng(0).standard_normal(keep.size).astype(np.float32)
    S.learned_params(bad)                            # an untrained network adding noise to the V-cycle
    try:
        rep, _ = run(S, f, "fcg_learned")
    finally:
        S.learned_params(keep)
    assert rep.status == 0 and rep.true_rel_residual <= 1e-10
    assert rep.precond_fallback > 0


def test_fcg_with_vcycle_matches_mg(trained):
    S, _, f, nodes = trained
    rep, u = run(S, f, "fcg_mg")
    _, u_mg = run(S, f, "mg64")
    assert rep.status == 0 and rep.true_rel_residual <= 1e-10
    assert np.abs(u[nodes] - u_mg[nodes]).max() <= 1e-8 * np.abs(u_mg[nodes]).max()
