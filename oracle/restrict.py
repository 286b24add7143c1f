"""ORACLE (test infrastructure only): bindings of oracle_restrict.cpp.

`Pair` holds, for a parent level and its child level of a uniform hierarchy,
the multi-level trend's work fields (node scalar, scalar trend, horizontal
flux and velocity trend, every layer) and masks as numpy arrays in the padded
lozenge layout, and runs the reference's compute-or-restrict operators on them
in place (src/multi_level.f90:311-659).  `div` and `restrict_fwr` restate the
divergence (src/ops.f90:1340-1355) and full-weighting restriction
(src/wavelet.f90:839-882) used by the conservation checks."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _dp, _ip, lib

TOLRNZ, RESTRCT, ADJZONE = 16, 12, 8
_i32p = C.POINTER(C.c_int32)


class orc_rlevel(C.Structure):
    _fields_ = [("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64),
                ("hex_inv", _dp), ("overl_a", _dp), ("overl_split", _dp), ("rf_wgt", _dp),
                ("halo_node", _ip), ("n_halo_node", C.c_int64), ("halo_edge", _ip), ("n_halo_edge", C.c_int64),
                ("mask_n", _i32p), ("mask_e", _i32p),
                ("scal", _dp), ("dscal", _dp), ("flux", _dp), ("dvelo", _dp)]


def _bind():
    L = lib()
    P = C.POINTER(orc_rlevel)
    L.orc_restrict_scalar.argtypes = [P, P, C.c_int]
    L.orc_restrict_u_source.argtypes = [P, P, C.c_int]
    L.orc_restrict_flux.argtypes = [P, P, C.c_int]
    L.orc_restrict_flux.restype = C.c_int64
    return L


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Pair:
    """Parent level `par` and child level `chd` (LevelGeom) with nz layers.
    Fields: scal, dscal (nz, NN), flux, dvelo (nz, 3*NN); masks mask_n (NN),
    mask_e (3*NN), initialised to TOLRNZ."""

    FIELDS = ("scal", "dscal", "flux", "dvelo")

    def __init__(self, par, chd, nz):
        from .grid import own
        par, chd = own(par), own(chd)
        self.L = _bind()
        self.nz = nz
        self.geo = (par, chd)
        self.f = []
        self.s = []
        self.keep = []
        for g in (par, chd):
            rf = g.rf_wgt if g.rf_wgt is not None else np.zeros((3, g.NN))
            geo = [np.ascontiguousarray(x, dtype=np.float64) for x in (g.hex_inv, g.overl_a, g.overl_split, rf)]
            hn = np.ascontiguousarray(g.halo_node, dtype=np.int64)
            he = np.ascontiguousarray(g.halo_edge, dtype=np.int64)
            fl = {"mask_n": np.full(g.NN, TOLRNZ, dtype=np.int32), "mask_e": np.full(3 * g.NN, TOLRNZ, dtype=np.int32),
                  "scal": np.zeros((nz, g.NN)), "dscal": np.zeros((nz, g.NN)),
                  "flux": np.zeros((nz, 3 * g.NN)), "dvelo": np.zeros((nz, 3 * g.NN))}
            self.keep += geo + [hn, he]
            self.f.append(fl)
            self.s.append(orc_rlevel(g.n, g.P, g.NN, *[_p(x) for x in geo], _p(hn, _ip), len(hn), _p(he, _ip), len(he),
                                     _p(fl["mask_n"], _i32p), _p(fl["mask_e"], _i32p),
                                     *[_p(fl[k]) for k in self.FIELDS]))

    def field(self, which, name):
        """Array `name` of the parent (which=0) or child (which=1), by reference."""
        return self.f[which][name]

    def restrict_scalar(self):
        self.L.orc_restrict_scalar(C.byref(self.s[0]), C.byref(self.s[1]), self.nz)

    def restrict_flux(self):
        """Returns the number of non-zero-weighted child dscalar reads outside the padded level."""
        return int(self.L.orc_restrict_flux(C.byref(self.s[0]), C.byref(self.s[1]), self.nz))

    def restrict_u_source(self):
        self.L.orc_restrict_u_source(C.byref(self.s[0]), C.byref(self.s[1]), self.nz)


def div(g, flux):
    """Flux divergence at every node (i, j) in [0, n]^2 of every lozenge
    (div, src/ops.f90:1340-1355); other nodes 0.  flux: (..., 3*NN), ghost-copied."""
    from .grid import own
    g = own(g)
    NN, P = g.NN, g.P
    f = flux.reshape(flux.shape[:-1] + (3, NN))
    out = np.zeros(flux.shape[:-1] + (NN,))
    ids = _nodes(g, 0, g.n + 1)
    out[..., ids] = (f[..., 0, ids] - f[..., 0, ids - 1] + f[..., 1, ids - P - 1] - f[..., 1, ids]
                     + f[..., 2, ids] - f[..., 2, ids - P]) * g.hex_inv[ids]
    return out


def restrict_fwr(par, chd, s):
    """Restrict_fwr of the child node field s (..., NN_chd), ghost-copied, to
    the owned parents [0, n_par)^2 (other parent nodes 0)."""
    out = np.zeros(s.shape[:-1] + (par.NN,))
    a = chd.overl_a
    Pc = chd.P
    for d in range(10):
        for jp in range(par.n):
            for ip in range(par.n):
                ic, jc = 2 * ip, 2 * jp

                def c(i, j):
                    return (d * Pc + jc + j + 2) * Pc + ic + i + 2
                t = s[..., c(0, 0)] / chd.hex_inv[c(0, 0)]
                for (i, j, k) in ((1, 0, 0), (1, 1, 1), (2, 1, 2), (1, 2, 3), (0, 1, 0), (-1, 0, 1), (-1, 1, 2),
                                  (-2, -1, 3), (-1, -1, 0), (0, -1, 1), (-1, -2, 2), (1, -1, 3)):
                    t = t + s[..., c(i, j)] * a[k, c(i, j)]
                idp = (d * par.P + jp + 2) * par.P + ip + 2
                out[..., idp] = t * par.hex_inv[idp]
    return out


def _nodes(g, lo, hi):
    i = np.arange(lo, hi)
    ii, jj = np.meshgrid(i, i, indexing="xy")
    return np.concatenate([((d * g.P + jj + 2) * g.P + ii + 2).ravel() for d in range(10)])
