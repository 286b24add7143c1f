"""ORACLE (test infrastructure only): bindings of oracle_elliptic.cpp."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _d, _dp, _ip, lib


class orc_elevel(C.Structure):
    _fields_ = [("level", C.c_int), ("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64),
                ("len", _dp), ("pedlen", _dp), ("hex_inv", _dp), ("overl_a", _dp), ("topo", _dp),
                ("halo_node", _ip), ("n_halo_node", C.c_int64), ("halo_edge", _ip), ("n_halo_edge", C.c_int64),
                ("eta_old", _dp)]


class orc_eparams(C.Structure):
    _fields_ = [("grav", C.c_double), ("dt", C.c_double), ("theta1", C.c_double), ("theta2", C.c_double),
                ("domain_level", C.c_int), ("coarse_iter", C.c_int), ("max_vcycle", C.c_int),
                ("pre_iter", C.c_int), ("down_iter", C.c_int), ("up_iter", C.c_int), ("post_iter", C.c_int),
                ("max_srj_iter", C.c_int), ("fine_tol", C.c_double), ("coarse_tol", C.c_double)]


def _bind():
    L = lib()
    E, P = C.POINTER(orc_elevel), C.POINTER(orc_eparams)
    L.orc_elliptic_apply.argtypes = [E, C.c_int, P, C.c_int, _dp, _dp]
    L.orc_restrict_all.argtypes = [E, C.c_int, P, _dp]
    L.orc_prolong.argtypes = [E, C.c_int, P, C.c_int, _dp]
    L.orc_l2.argtypes = [E, C.c_int, P, C.c_int, _dp]
    L.orc_l2.restype = C.c_double
    L.orc_elliptic_solve.argtypes = [E, C.c_int, P, C.c_int, _dp, _dp, _dp, C.POINTER(C.c_int)]
    return L


class Hierarchy:
    """Keeps the per-level numpy buffers alive behind an orc_elevel array."""

    def __init__(self, levels, topos, grav=9.80616, dt=600.0, theta1=1.0, theta2=1.0, domain_level=2, eta_old=None,
                 **solver):
        """eta_old: per level the old free surface of eta_update (ghosts holding
        their copies), which enters the operator's coefficients
        g (|H| + eta_old) and its diagonal; None for 0."""
        from .grid import own
        levels = [own(g) for g in levels]
        self.L = _bind()
        self.keep = []
        self.arr = (orc_elevel * len(levels))()
        for q, (g, topo) in enumerate(zip(levels, topos)):
            b = [np.ascontiguousarray(x, dtype=np.float64) for x in (g.len, g.pedlen, g.hex_inv, g.overl_a, topo)]
            hn = np.ascontiguousarray(g.halo_node, dtype=np.int64)
            he = np.ascontiguousarray(g.halo_edge, dtype=np.int64)
            eo = None if eta_old is None else np.ascontiguousarray(eta_old[q], dtype=np.float64)
            self.keep += b + [hn, he] + ([eo] if eo is not None else [])
            self.arr[q] = orc_elevel(g.level, g.n, g.P, g.NN, *[_d(x) for x in b], hn.ctypes.data_as(_ip), len(hn),
                                     he.ctypes.data_as(_ip), len(he), None if eo is None else _d(eo))
        d = dict(coarse_iter=50, max_vcycle=3, pre_iter=2, down_iter=2, up_iter=2, post_iter=4, max_srj_iter=200,
                 fine_tol=1e-3, coarse_tol=1e-3)
        d.update(solver)
        self.p = orc_eparams(grav, dt, theta1, theta2, domain_level, d["coarse_iter"], d["max_vcycle"],
                             d["pre_iter"], d["down_iter"], d["up_iter"], d["post_iter"], d["max_srj_iter"],
                             d["fine_tol"], d["coarse_tol"])
        self.nlev = len(levels)
        self.ls = levels[0].level

    def apply(self, level, q):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        out = np.zeros_like(q)
        self.L.orc_elliptic_apply(self.arr, self.nlev, C.byref(self.p), level, _d(q), _d(out))
        return out

    def restrict_all(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).copy()
        self.L.orc_restrict_all(self.arr, self.nlev, C.byref(self.p), _d(s))
        return s

    def prolong(self, fine, s):
        s = np.ascontiguousarray(s, dtype=np.float64).copy()
        self.L.orc_prolong(self.arr, self.nlev, C.byref(self.p), fine, _d(s))
        return s

    def l2(self, level, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        return self.L.orc_l2(self.arr, self.nlev, C.byref(self.p), level, _d(s))

    def solve(self, u, f, method="fmg"):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        nrm = np.zeros(2 * self.nlev)
        its = (C.c_int * self.nlev)()
        self.L.orc_elliptic_solve(self.arr, self.nlev, C.byref(self.p), {"fmg": 0, "srj": 1}[method], _d(u), _d(f),
                                  _d(nrm), its)
        return u, nrm.reshape(self.nlev, 2), list(its)
