"""The oracle's grid builder (oracle/oracle_grid.cpp) against the product's
(csrc/grid.cpp): two restatements of the reference's host set-up, written
separately, must give bit-identical tables on every level -- coordinates,
circumcentres, lengths, dual lengths, hexagon area parts, 1/area, triangle
areas, Coriolis, overlap areas and splits, I_u_wgt, R_F_wgt and the ghost
tables.  Plus geometric checks of the ghost tables that neither builder's
code path enters: a ghost node sits where its source node sits, and a ghost
edge joins the same two points as its source edge, with the sign giving
their relative orientation."""
import numpy as np
import pytest

from oracle.grid import Grid as OGrid
from wavetrisk_hydrostatic_b200 import Grid

TABLES = ("node", "ccentre", "len", "pedlen", "part", "hex_inv", "triarea", "coriolis", "overl_a", "overl_split",
          "iu_wgt", "rf_wgt", "halo_node", "halo_edge")


@pytest.fixture(scope="module", params=[(3, 5, 0), (4, 7, 1), (5, 7, 2)], ids=["J2-J5", "J3-J7", "J4-J7"])
def pair(request):
    lmin, lmax, dl = request.param
    return (lmin, lmax, Grid(lmin, lmax, domain_level=dl, radius=6371e3),
            OGrid(lmin, lmax, domain_level=dl, radius=6371e3))


def test_every_table_bit_identical(pair):
    lmin, lmax, P, O = pair
    for l in range(lmin - 1, lmax + 1):
        p, o = P.level(l), O.level(l)
        assert (p.n, p.P, p.NN) == (o.n, o.P, o.NN)
        for name in TABLES:
            a, b = getattr(p, name), getattr(o, name)
            if a is None or b is None:
                assert a is None and b is None, (l, name)
                continue
            assert a.shape == b.shape, (l, name)
            assert np.array_equal(a, b), (l, name, int(np.count_nonzero(a != b)))


def _corner_block(g, k):
    d, i, j = g.ij()
    out_i = (i[k] < 0) | (i[k] >= g.n)
    out_j = (j[k] < 0) | (j[k] >= g.n)
    return out_i & out_j


def test_ghost_nodes_copy_the_node_at_their_position(pair):
    """Root level: ghost coordinates are copies, so every entry is exact.
    Finer levels: the ghosts' coordinates are built from the parent's ghost
    midpoints, so outside the four corner blocks of a lozenge every entry
    joins two slots that agree to rounding (1e-14 of the radius).  Entries into a corner block
    are the pentagon and pole special cases of create_comm/create_comm_pole
    (comm.f90:395-530); there are at most 30 per level."""
    lmin, lmax, P, O = pair
    for l in range(lmin - 1, lmax + 1):
        g = O.level(l)
        hn = g.halo_node
        dist = np.linalg.norm(g.node[:, hn[:, 0]] - g.node[:, hn[:, 1]], axis=0)
        if l == lmin - 1:
            assert np.all(dist == 0.0), l
            continue
        corner = _corner_block(g, hn[:, 0])
        tol = 1e-14 * 6371e3
        assert np.all(dist[~corner] <= tol), (l, float(dist[~corner].max()))
        assert np.count_nonzero(dist[corner] > tol) <= 30, l


def test_ghost_edges_join_the_same_points(pair):
    """Edge e of slot x joins node(x) + end_pt(1, e) and node(x) + end_pt(2, e)
    (shared.f90:287-292: RT x -> x+E, DG x+NE -> x, UP x -> x+N).  Outside the
    corner blocks a ghost edge and its source join the same two points, in the
    same order when the sign is +1 and in reverse when it is -1."""
    lmin, lmax, P, O = pair
    for l in range(lmin - 1, lmax + 1):
        g = O.level(l)
        he = g.halo_edge
        NN, Pp = g.NN, g.P
        offs = {0: ((0, 0), (1, 0)), 1: ((1, 1), (0, 0)), 2: ((0, 0), (0, 1))}

        def ends(code):
            e, x = code // NN, code % NN
            a = np.zeros((3, code.size))
            b = np.zeros((3, code.size))
            for ee, ((i1, j1), (i2, j2)) in offs.items():
                s = e == ee
                a[:, s] = g.node[:, x[s] + i1 + Pp * j1]
                b[:, s] = g.node[:, x[s] + i2 + Pp * j2]
            return a, b

        d, i, j = g.ij()
        x = he[:, 0] % NN
        inside = (i[x] >= -1) & (j[x] >= -1) & (i[x] <= g.n) & (j[x] <= g.n) & ~_corner_block(g, x)
        he = he[inside]
        da, db = ends(he[:, 0])
        sa, sb = ends(he[:, 1])
        fwd = np.maximum(np.linalg.norm(da - sa, axis=0), np.linalg.norm(db - sb, axis=0))
        rev = np.maximum(np.linalg.norm(da - sb, axis=0), np.linalg.norm(db - sa, axis=0))
        plus = he[:, 2] > 0
        assert np.all(fwd[plus] <= 1e-6), (l, float(fwd[plus].max()))
        assert np.all(rev[~plus] <= 1e-6), (l, float(rev[~plus].max()))
