"""ORACLE -- test infrastructure only.

The oracle's own grid (oracle_grid.cpp in liboracle.so): geometry and ghost
tables of every level, restated from the reference's host set-up
(src/init.f90, src/sphere.f90, src/refine_patch.f90, src/comm.f90, the weight
builders of src/wavelet.f90).  The oracle and the timed CPU baseline take
their geometry from here, never from the product's builder; the tests compare
the two table by table.

A level object has the attributes the oracle's routines read (the same names
and layouts as the product's level descriptors, because both describe the same
padded lozenge arrays): n, P, NN, node (3, NN), len, pedlen (3, NN), part
(6, NN), hex_inv, triarea, coriolis (2, NN), overl_a (4, NN), overl_split
(2, NN), ccentre (2, 3, NN), halo_node (m, 2), halo_edge (m, 3), iu_wgt (9, NN)
and rf_wgt (3, NN) above level min_level-1.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import lib

HALO = 2


@dataclass
class Level:
    level: int
    n: int
    P: int
    NN: int
    node: np.ndarray
    len: np.ndarray
    pedlen: np.ndarray
    part: np.ndarray
    hex_inv: np.ndarray
    triarea: np.ndarray
    coriolis: np.ndarray
    overl_a: np.ndarray
    overl_split: np.ndarray
    ccentre: np.ndarray
    halo_node: np.ndarray
    halo_edge: np.ndarray
    iu_wgt: np.ndarray | None = None
    rf_wgt: np.ndarray | None = None
    rf_conflict: float = 0.0
    _owned: np.ndarray | None = field(default=None, repr=False)

    def idx(self, d, i, j):
        return (np.asarray(d) * self.P + (np.asarray(j) + HALO)) * self.P + (np.asarray(i) + HALO)

    def ij(self):
        k = np.arange(self.NN)
        d = k // (self.P * self.P)
        r = k % (self.P * self.P)
        return d, r % self.P - HALO, r // self.P - HALO

    @property
    def owned(self) -> np.ndarray:
        if self._owned is None:
            _, i, j = self.ij()
            self._owned = (i >= 0) & (j >= 0) & (i < self.n) & (j < self.n)
        return self._owned

    def pole_ids(self):
        """North pole slot (lozenge 5, (0, n)) and south pole slot (lozenge 0, (n, 0))."""
        return int(self.idx(5, 0, self.n)), int(self.idx(0, self.n, 0))


def _bind():
    L = lib()
    if not getattr(L, "_grid_bound", False):
        L.orc_grid_build.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_grid_build.restype = C.c_void_p
        L.orc_grid_free.argtypes = [C.c_void_p]
        L.orc_grid_free.restype = None
        L.orc_grid_dims.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]
        L.orc_grid_dims.restype = C.c_int
        L.orc_grid_copy.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_void_p]
        L.orc_grid_copy.restype = C.c_int
        L._grid_bound = True
    return L


class Grid:
    """Uniform grid, levels min_level-1 .. max_level, one domain per lozenge."""

    def __init__(self, min_level: int, max_level: int, domain_level: int | None = None,
                 radius: float = 6371.22e3, omega: float = 7.292e-5):
        if domain_level is None:
            # param_J4: DOMAIN_LEVEL 1; param_J5..J9: DOMAIN_LEVEL 2 (src/param_J*.f90)
            domain_level = {3: 0, 4: 1}.get(min_level, 2)
        self.min_level, self.max_level, self.domain_level = min_level, max_level, domain_level
        self.radius, self.omega = radius, omega
        L = _bind()
        h = L.orc_grid_build(min_level, max_level, domain_level, radius, omega)
        if not h:
            raise RuntimeError("orc_grid_build failed")
        self._h = h
        self._levels: dict[int, Level] = {}

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _bind().orc_grid_free(self._h)
                self._h = None
        except Exception:
            pass

    def level(self, l: int) -> Level:
        if l in self._levels:
            return self._levels[l]
        L = _bind()
        dims = (C.c_int64 * 5)()
        if L.orc_grid_dims(self._h, l, dims) != 0:
            raise ValueError(f"level {l} outside {self.min_level - 1}..{self.max_level}")
        n, P, NN, nhn, nhe = (int(x) for x in dims)

        def get(name, shape, dtype=np.float64):
            a = np.zeros(shape, dtype=dtype)
            if L.orc_grid_copy(self._h, l, name.encode(), a.ctypes.data_as(C.c_void_p)) != 0:
                raise RuntimeError(f"orc_grid_copy({name})")
            return a

        above = l > self.min_level - 1
        g = Level(level=l, n=n, P=P, NN=NN, node=get("node", (3, NN)), len=get("len", (3, NN)),
                  pedlen=get("pedlen", (3, NN)), part=get("part", (6, NN)), hex_inv=get("hex_inv", (NN,)),
                  triarea=get("triarea", (2, NN)), coriolis=get("coriolis", (2, NN)),
                  overl_a=get("overl_a", (4, NN)), overl_split=get("overl_split", (2, NN)),
                  ccentre=get("ccentre", (2, 3, NN)), halo_node=get("halo_node", (nhn, 2), np.int64),
                  halo_edge=get("halo_edge", (nhe, 3), np.int64),
                  iu_wgt=get("iu_wgt", (9, NN)) if above else None,
                  rf_wgt=get("rf_wgt", (3, NN)) if above else None)
        self._levels[l] = g
        return g


_GRIDS: dict = {}


def own(g):
    """The oracle's own level for a level object of any builder: the level of
    the same number from the oracle's grid with the same parameters
    (min_level, max_level, domain_level, radius, omega).  Oracle routines call
    this on every level they are given and read no geometry from the caller's
    object, so a product level only names which grid and level is meant."""
    if isinstance(g, Level):
        return g
    spec = getattr(g, "grid_spec", None)
    if spec is None:
        raise TypeError("level object without grid parameters (grid_spec)")
    G = _GRIDS.get(spec)
    if G is None:
        if len(_GRIDS) >= 4:
            _GRIDS.clear()
        lmin, lmax, dl, radius, omega = spec
        G = _GRIDS[spec] = Grid(lmin, lmax, domain_level=dl, radius=radius, omega=omega)
    return G.level(g.level)
