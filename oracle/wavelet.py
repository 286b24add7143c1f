"""ORACLE (test infrastructure only): bindings of oracle_wavelet.cpp.

`Hierarchy` holds, for every level of a uniform hierarchy, the scaling and
wavelet fields of layer mass, potential temperature and velocity (all layers)
and the node/edge masks, as numpy arrays in the padded lozenge layout, and runs
the reference's forward/inverse wavelet transforms, mask_tol_vars, compression
and WT_after_step on them in place."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _dp, _ip, lib

FROZEN, TOLRNZ, ADJZONE, ZERO = 32, 16, 8, 0
_i32p = C.POINTER(C.c_int32)


class orc_wlevel(C.Structure):
    _fields_ = [("level", C.c_int), ("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64),
                ("len", _dp), ("triarea", _dp), ("hex_inv", _dp), ("overl_a", _dp), ("iu_wgt", _dp),
                ("halo_node", _ip), ("n_halo_node", C.c_int64), ("halo_edge", _ip), ("n_halo_edge", C.c_int64),
                ("mask_n", _i32p), ("mask_e", _i32p),
                ("s_m", _dp), ("s_t", _dp), ("s_v", _dp), ("w_m", _dp), ("w_t", _dp), ("w_v", _dp)]


def _bind():
    L = lib()
    P = C.POINTER(orc_wlevel)
    for name in ("orc_wt_forward", "orc_wt_inverse", "orc_compress", "orc_wt_after_step"):
        getattr(L, name).argtypes = [P, C.c_int, C.c_int, C.c_int]
    L.orc_mask_tol.argtypes = [P, C.c_int, C.c_int, C.c_int, _dp, C.c_int]
    L.orc_mask_build.argtypes = [P, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int, C.c_void_p]
    L.orc_mask_phase1.argtypes = [P, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int]
    L.orc_mask_phase2.argtypes = [P, C.c_int, C.c_int, C.c_int]
    L.orc_mask_adj_child.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int]
    return L


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Hierarchy:
    """Fields of levels levels[0].level .. levels[-1].level with nz layers."""

    FIELDS = ("s_m", "s_t", "s_v", "w_m", "w_t", "w_v")

    def __init__(self, levels, nz):
        from .grid import own
        levels = [own(g) for g in levels]
        self.L = _bind()
        self.levels = levels
        self.nz = nz
        self.ls, self.le = levels[0].level, levels[-1].level
        self.arr = (orc_wlevel * len(levels))()
        self.keep = []
        self.f = []
        for q, g in enumerate(levels):
            geo = [np.ascontiguousarray(x, dtype=np.float64) for x in (g.len, g.triarea, g.hex_inv, g.overl_a)]
            iu = np.ascontiguousarray(g.iu_wgt if g.iu_wgt is not None else np.zeros((9, g.NN)), dtype=np.float64)
            hn = np.ascontiguousarray(g.halo_node, dtype=np.int64)
            he = np.ascontiguousarray(g.halo_edge, dtype=np.int64)
            fl = {
                "mask_n": np.full(g.NN, TOLRNZ, dtype=np.int32),
                "mask_e": np.full(3 * g.NN, TOLRNZ, dtype=np.int32),
                "s_m": np.zeros((nz, g.NN)), "s_t": np.zeros((nz, g.NN)), "s_v": np.zeros((nz, 3 * g.NN)),
                "w_m": np.zeros((nz, g.NN)), "w_t": np.zeros((nz, g.NN)), "w_v": np.zeros((nz, 3 * g.NN)),
            }
            self.keep += geo + [iu, hn, he]
            self.f.append(fl)
            self.arr[q] = orc_wlevel(g.level, g.n, g.P, g.NN, *[_p(x) for x in geo], _p(iu),
                                     _p(hn, _ip), len(hn), _p(he, _ip), len(he),
                                     _p(fl["mask_n"], _i32p), _p(fl["mask_e"], _i32p),
                                     *[_p(fl[k]) for k in self.FIELDS])

    def field(self, level, name):
        """The numpy array of `name` (s_m, s_t, s_v, w_m, w_t, w_v, mask_n, mask_e) at `level`, by reference."""
        return self.f[level - self.ls][name]

    def set(self, level, name, value):
        self.f[level - self.ls][name][...] = value

    def forward(self, le=None):
        """forward_wavelet_transform over levels ls .. le (default: the top)."""
        self.L.orc_wt_forward(self.arr, self.ls, self.le if le is None else le, self.nz)

    def inverse(self, le=None):
        self.L.orc_wt_inverse(self.arr, self.ls, self.le if le is None else le, self.nz)

    def mask_tol(self, threshold, level_fill):
        thr = np.ascontiguousarray(threshold, dtype=np.float64).reshape(3, self.nz)
        self.L.orc_mask_tol(self.arr, self.ls, self.le, self.nz, _p(thr), int(level_fill))

    def mask_build(self, threshold, level_fill, max_level, patch_size=0):
        thr = np.ascontiguousarray(threshold, dtype=np.float64).reshape(3, self.nz)
        out = None
        if patch_size > 0:
            n = sum(10 * (g.n // patch_size) ** 2 * 4 for g in self.levels[:-1])
            out = np.zeros(n, dtype=np.uint8)
        self.L.orc_mask_build(self.arr, self.ls, self.le, self.nz, _p(thr), int(level_fill), int(max_level),
                              int(patch_size), None if out is None else out.ctypes.data)
        return out

    def mask_phase1(self, threshold, level_fill, max_level, patch_size, le, req_hi):
        """adapt's mask sequence up to refine() on levels ls .. le; returns the
        check_child_required flags of parent levels ls .. req_hi (uint8, level
        by level, lozenge-major, 4 quadrants a parent patch)."""
        thr = np.ascontiguousarray(threshold, dtype=np.float64).reshape(3, self.nz)
        n = sum(10 * (g.n // patch_size) ** 2 * 4 for g in self.levels[:req_hi - self.ls + 1])
        out = np.zeros(max(n, 1), dtype=np.uint8)
        self.L.orc_mask_phase1(self.arr, self.ls, int(le), self.nz, _p(thr), int(level_fill), int(max_level),
                               int(patch_size), out.ctypes.data, int(req_hi))
        return out[:n]

    def mask_phase2(self, le):
        """adapt's mask sequence after refine() on levels ls .. le."""
        self.L.orc_mask_phase2(self.arr, self.ls, int(le), self.nz)

    def mask_adj_child(self, level):
        """mask_adj_child of the parents of `level` alone."""
        if self.L.orc_mask_adj_child(self.arr, self.ls, self.le, self.nz, int(level)):
            raise ValueError("mask_adj_child: level out of range")

    def compress(self, le=None):
        self.L.orc_compress(self.arr, self.ls, self.le if le is None else le, self.nz)

    def wt_after_step(self):
        self.L.orc_wt_after_step(self.arr, self.ls, self.le, self.nz)


def lnorm(levels, masks, fields, order="inf"):
    """cal_lnorm (src/lnorms.f90:7-58) over the hierarchy in numpy: (3, nz)
    for mass, Theta, velocity.  fields[q]: dict of mass, temp, velo, mean_m,
    mean_t of levels[q]; masks[q]: (mask_n, mask_e).  Scalars are mean +
    perturbation at nodes [0, n]^2, velocities the edges of nodes [0, n)^2,
    where mask_n >= ADJZONE; "1" and "2" divide by the count of nodes
    [-1, n+1]^2 with mask_n >= ADJZONE."""
    nz = fields[0]["mass"].shape[0]
    init = 1e16 if order == "min" else 0.0
    out = np.full((3, nz), init)
    count = 0

    def sel(g, lo, hi):
        i = np.arange(lo, hi)
        ii, jj = np.meshgrid(i, i, indexing="xy")
        return np.concatenate([((d * g.P + jj + 2) * g.P + ii + 2).ravel() for d in range(10)])

    for g, (mn, _), f in zip(levels, masks, fields):
        count += int(np.count_nonzero(mn[sel(g, -1, g.n + 2)] >= ADJZONE))
        ids = sel(g, 0, g.n + 1)
        ids = ids[mn[ids] >= ADJZONE]
        own = sel(g, 0, g.n)
        own = own[mn[own] >= ADJZONE]
        e = np.concatenate([own, own + g.NN, own + 2 * g.NN])
        for v, x in enumerate((f["mean_m"] + f["mass"], f["mean_t"] + f["temp"])):
            a = x[:, ids]
            out[v] = _red(order, out[v], a)
        out[2] = _red(order, out[2], f["velo"][:, e])
    if order == "1":
        out = out / count
    elif order == "2":
        out = np.sqrt(out / count)
    return out


def _red(order, acc, a):
    if a.shape[1] == 0:
        return acc
    if order == "inf":
        return np.maximum(acc, np.abs(a).max(axis=1))
    if order == "min":
        return np.minimum(acc, a.min(axis=1))
    if order == "1":
        return acc + np.abs(a).sum(axis=1)
    return acc + (a * a).sum(axis=1)
