"""CPU checks of the learned-preconditioner oracle: BF16 rounding against
torch's conversion, the node layout, and the oracle's parameter gradient
against central finite differences (float64, unrounded weights)."""
import numpy as np
import pytest
import torch

from oracle import learned as LO
from oracle.grid import Grid
from wavetrisk_hydrostatic_b200.cases import bathymetry


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(0)
    w = np.concatenate([rng.standard_normal(4096).astype(np.float32),
                        np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5e-3, 0.0], np.float32)])
    ref = torch.from_numpy(w).to(torch.bfloat16).float().numpy()
    assert np.array_equal(LO.bf16_round(w), ref)


def test_layout_is_every_node_once():
    g = Grid(3, 4, radius=6371e3)
    lv = g.level(4)
    slot, tap = LO.layout(lv)
    assert slot.size == 10 * lv.n ** 2 + 10          # the 10 n^2 + 2 nodes and 8 pole copies
    assert np.array_equal(tap[0], np.arange(slot.size))
    assert np.unique(slot).size == slot.size
    d, i, j = lv.ij()
    own = lv.owned[slot]
    pent = own & (i[slot] == 0) & (j[slot] == 0)     # the lozenges' (0, 0) corners are pentagons
    assert (tap[:, own & ~pent] >= 0).all()          # every other owned node has six neighbours
    assert pent.sum() == 10 and (tap[5, pent] < 0).all() and (np.delete(tap[:, pent], 5, 0) >= 0).all()


@pytest.mark.parametrize("slope", [1.0, 0.25])
def test_oracle_gradient_finite_differences(slope):
    g = Grid(3, 3, radius=6371e3)
    lv = g.level(3)
    slot, tap = LO.layout(lv)
    depth = bathymetry(lv, seed=3)[slot]
    rng = np.random.default_rng(5)
    r, e = rng.standard_normal(slot.size), rng.standard_normal(slot.size)
    theta = LO.init_params(7).astype(np.float64)

    def f(th):
        return LO.loss_and_grad(th, r, e, depth, tap, round_weights=False, slope=slope)

    loss, grad = f(theta)
    idx = rng.choice(LO.NPARAMS, 24, replace=False)
    h = 1e-6
    for k in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (f(tp)[0] - f(tm)[0]) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(grad).max()), (k, fd, grad[k])
    assert loss > 0


def test_infer_homogeneity_and_linearity():
    g = Grid(3, 3, radius=6371e3)
    lv = g.level(3)
    slot, tap = LO.layout(lv)
    depth = bathymetry(lv, seed=3)[slot]
    theta = LO.init_params(9)
    own = lv.owned[slot].astype(np.float64)
    r = np.random.default_rng(1).standard_normal(slot.size)
    for slope in (1.0, 0.25):
        z = LO.infer(theta, r, depth, tap, own, slope)
        # positively homogeneous, exactly: 4 r has the same r / rms(r)
        assert np.array_equal(LO.infer(theta, 4.0 * r, depth, tap, own, slope), 4.0 * z)
        zm = LO.infer(theta, -r, depth, tap, own, slope)
        if slope == 1.0:
            assert np.array_equal(zm, -z)                # identity activations: odd
        else:
            assert np.abs(zm + z).max() > 1e-3 * np.abs(z).max()
        assert (z[own == 0] == 0).all() and own.sum() == 10 * lv.n ** 2
    # identity activations, unrounded: linear up to the FP32 rounding of the inputs
    r2 = np.random.default_rng(2).standard_normal(slot.size)

    def y(rr):
        A = LO.forward(theta, rr, depth, tap, round_weights=False)
        return A["rs"] * A["y"]

    y12 = y(r + r2)
    assert np.abs(y12 - y(r) - y(r2)).max() <= 1e-5 * np.abs(y12).max()
