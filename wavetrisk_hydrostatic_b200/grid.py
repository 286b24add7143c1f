"""Host-side grid: per-level geometry and ghost tables on the padded lozenge layout.

This is the role the Fortran host plays in the reference (init_grid,
precompute_geometry, refine_patch2: src/init.f90, src/refine_patch.f90); the
tables come from the native builder ``wt_grid_build`` (C++, host only).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

RT, DG, UP = 0, 1, 2
LORT, UPLT = 0, 1
HALO = 2


@dataclass
class LevelGeom:
    level: int
    n: int
    P: int
    NN: int
    node: np.ndarray          # (3, NN)
    len: np.ndarray           # (3, NN)
    pedlen: np.ndarray        # (3, NN)
    part: np.ndarray          # (6, NN)
    hex_inv: np.ndarray       # (NN,)
    triarea: np.ndarray       # (2, NN)
    coriolis: np.ndarray      # (2, NN)
    overl_a: np.ndarray       # (4, NN)
    overl_split: np.ndarray   # (2, NN)
    ccentre: np.ndarray       # (2, 3, NN)
    halo_node: np.ndarray     # (n_halo_node, 2) int64
    halo_edge: np.ndarray     # (n_halo_edge, 3) int64
    iu_wgt: np.ndarray | None = None   # (9, NN) outer velocity weights I_u_wgt (levels above min_level-1)
    rf_wgt: np.ndarray | None = None   # (3, NN) flux-restriction weights R_F_wgt (levels above min_level-1)
    rf_conflict: float = 0.0           # largest difference between two writers of one R_F_wgt slot
    grid_spec: tuple | None = None     # (min_level, max_level, domain_level, radius, omega) of the grid
    _owned: np.ndarray | None = field(default=None, repr=False)

    def idx(self, d, i, j):
        """Flat node index of (lozenge d, i, j); i, j in [-2, n+1]."""
        return (np.asarray(d) * self.P + (np.asarray(j) + HALO)) * self.P + (np.asarray(i) + HALO)

    def ij(self):
        """(d, i, j) of every node of the level, each an (NN,) int array."""
        k = np.arange(self.NN)
        d = k // (self.P * self.P)
        r = k % (self.P * self.P)
        return d, r % self.P - HALO, r // self.P - HALO

    @property
    def owned(self) -> np.ndarray:
        """Boolean (NN,) mask of owned nodes: (i, j) in [0, n)^2 of every lozenge."""
        if self._owned is None:
            _, i, j = self.ij()
            self._owned = (i >= 0) & (j >= 0) & (i < self.n) & (j < self.n)
        return self._owned

    def pole_ids(self):
        """Node indices of the north pole (in lozenge 5) and south pole (in lozenge 0)."""
        return int(self.idx(5, 0, self.n)), int(self.idx(0, self.n, 0))


class Grid:
    """Uniform icosahedral grid, levels min_level-1 .. max_level."""

    def __init__(self, min_level: int, max_level: int, domain_level: int | None = None,
                 radius: float = 6371.22e3, omega: float = 7.292e-5):
        if domain_level is None:
            # param_J4: DOMAIN_LEVEL 1; param_J5..J9: DOMAIN_LEVEL 2 (src/param_J*.f90)
            domain_level = {3: 0, 4: 1}.get(min_level, 2)
        self.min_level, self.max_level, self.domain_level = min_level, max_level, domain_level
        self.radius, self.omega = radius, omega
        L = N.lib()
        h = C.c_void_p()
        N.check("wt_grid_build", L.wt_grid_build(min_level, max_level, domain_level, radius, omega, C.byref(h)))
        self._h = h
        self._levels: dict[int, LevelGeom] = {}

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.lib().wt_grid_free(self._h)
                self._h = None
        except Exception:
            pass

    def level(self, l: int) -> LevelGeom:
        if l in self._levels:
            return self._levels[l]
        L = N.lib()
        dims = N.wt_level_dims()
        N.check("wt_grid_level_dims", L.wt_grid_level_dims(self._h, l, C.byref(dims)))
        NN = dims.NN

        def get(name, shape, dtype=np.float64):
            a = np.zeros(shape, dtype=dtype)
            N.check(f"wt_grid_copy({name})", L.wt_grid_copy(self._h, l, name.encode(), a.ctypes.data_as(C.c_void_p)))
            return a

        g = LevelGeom(
            level=l, n=dims.n, P=dims.P, NN=NN,
            node=get("node", (3, NN)), len=get("len", (3, NN)), pedlen=get("pedlen", (3, NN)),
            part=get("part", (6, NN)), hex_inv=get("hex_inv", (NN,)), triarea=get("triarea", (2, NN)),
            coriolis=get("coriolis", (2, NN)), overl_a=get("overl_a", (4, NN)),
            overl_split=get("overl_split", (2, NN)), ccentre=get("ccentre", (2, 3, NN)),
            halo_node=get("halo_node", (dims.n_halo_node, 2), np.int64),
            halo_edge=get("halo_edge", (dims.n_halo_edge, 3), np.int64),
            iu_wgt=get("iu_wgt", (9, NN)) if l > self.min_level - 1 else None,
            rf_wgt=get("rf_wgt", (3, NN)) if l > self.min_level - 1 else None,
            rf_conflict=float(get("rf_conflict", (1,))[0]) if l > self.min_level - 1 else 0.0,
            grid_spec=(self.min_level, self.max_level, self.domain_level, self.radius, self.omega),
        )
        self._levels[l] = g
        return g


def halo_nodes(g: LevelGeom, f: np.ndarray) -> None:
    """In-place ghost copy of a node field (cp_bdry_inside, src/comm.f90:785)."""
    f[..., g.halo_node[:, 0]] = f[..., g.halo_node[:, 1]]


def halo_edges(g: LevelGeom, f: np.ndarray) -> None:
    """In-place ghost copy of an edge field laid out as (..., 3*NN) with sign flips."""
    v = f[..., g.halo_edge[:, 1]]
    f[..., g.halo_edge[:, 0]] = np.where(g.halo_edge[:, 2] < 0, -v, v)
