"""Host grid builder: geometric invariants of the restated reference grid."""
import math

import numpy as np
import pytest

from wavetrisk_hydrostatic_b200 import Grid


@pytest.fixture(scope="module", params=[(4, 1), (5, 2)])
def grid(request):
    minl, dl = request.param
    return Grid(minl, minl + 1, domain_level=dl)


def total_area(lv):
    own = lv.owned
    npole, spole = lv.pole_ids()
    return (1 / lv.hex_inv[own]).sum() + 1 / lv.hex_inv[npole] + 1 / lv.hex_inv[spole]


def test_node_count(grid):
    for l in (grid.min_level, grid.min_level + 1):
        lv = grid.level(l)
        assert int(lv.owned.sum()) + 2 == 10 * 4 ** l + 2 - 2 + 2  # N_l = 10*4^l + 2 (src/shared.f90:448)


def test_hexagons_tile_the_sphere(grid):
    for l in (grid.min_level, grid.min_level + 1):
        lv = grid.level(l)
        assert abs(total_area(lv) / (4 * math.pi * grid.radius ** 2) - 1) < 1e-13


def test_dual_triangles_tile_the_sphere(grid):
    lv = grid.level(grid.min_level)
    own = lv.owned
    s = lv.triarea[0][own].sum() + lv.triarea[1][own].sum()
    assert abs(s / (4 * math.pi * grid.radius ** 2) - 1) < 1e-12


def test_lengths_positive_and_regular(grid):
    lv = grid.level(grid.min_level)
    own = lv.owned
    h = math.sqrt(4 * math.pi * grid.radius ** 2 / (10 * 4 ** lv.level))
    for e in range(3):
        le = lv.len[e][own]
        assert le.min() > 0.5 * h and le.max() < 1.6 * h
        pe = lv.pedlen[e][own]
        assert pe.min() > 0.25 * h and pe.max() < 1.0 * h


def test_poles_are_poles(grid):
    lv = grid.level(grid.min_level)
    npole, spole = lv.pole_ids()
    assert np.allclose(lv.node[:, npole] / grid.radius, [0, 0, 1], atol=1e-12)
    assert np.allclose(lv.node[:, spole] / grid.radius, [0, 0, -1], atol=1e-12)


def test_ghost_coordinates_match_sources_off_the_corners(grid):
    lv = grid.level(grid.min_level + 1)
    hn = lv.halo_node
    d, i, j = lv.ij()
    dst = hn[:, 0]
    corner = ((i[dst] < 0) | (i[dst] >= lv.n)) & ((j[dst] < 0) | (j[dst] >= lv.n))
    diff = np.abs(lv.node[:, dst] - lv.node[:, hn[:, 1]]).max(axis=0)
    assert diff[~corner].max() < 1e-6 * grid.radius


def test_overlap_weights_sum_to_hexagon(grid):
    # Interp_node (src/wavelet.f90:1487) is a convex combination: the four overlap
    # areas of a new fine node add up to about its hexagon area.
    lv = grid.level(grid.min_level + 1)
    d, i, j = lv.ij()
    odd = lv.owned & ((i % 2 == 1) | (j % 2 == 1))
    s = lv.overl_a[:, odd].sum(axis=0) * lv.hex_inv[odd]
    assert np.all(s > 0.9) and np.all(s < 1.1)
