"""ORACLE (test infrastructure only): bindings of oracle_barotropic.cpp."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _dp, _ip, lib


class orc_blevel(C.Structure):
    _fields_ = [("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64), ("len", _dp), ("pedlen", _dp), ("hex_inv", _dp),
                ("halo_node", _ip), ("n_halo_node", C.c_int64), ("halo_edge", _ip), ("n_halo_edge", C.c_int64)]


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class _Level:
    def __init__(self, g):
        from .grid import own
        g = own(g)
        self.keep = [_c(g.len), _c(g.pedlen), _c(g.hex_inv), np.ascontiguousarray(g.halo_node, dtype=np.int64),
                     np.ascontiguousarray(g.halo_edge, dtype=np.int64)]
        ln, pl, hi, hn, he = self.keep
        self.s = orc_blevel(g.n, g.P, g.NN, _p(ln), _p(pl), _p(hi), _p(hn, _ip), len(hn), _p(he, _ip), len(he))


def rhs_elliptic(g, nz, mass, mean_m, velo, eta, div_old, dt, theta2, rho0):
    """flux_divergence + rhs_elliptic on one level: returns (hflux, div, rhs)."""
    L = lib()
    lv = _Level(g)
    hflux, div, rhs = np.zeros(3 * g.NN), np.zeros(g.NN), np.zeros(g.NN)
    bufs = [_c(mass), _c(mean_m), _c(velo), _c(eta), _c(div_old)]
    L.orc_rhs_elliptic.argtypes = [C.POINTER(orc_blevel), C.c_int] + [_dp] * 5 + [C.c_double] * 3 + [_dp] * 3
    L.orc_rhs_elliptic(C.byref(lv.s), nz, *[_p(b) for b in bufs], dt, theta2, rho0, _p(hflux), _p(div), _p(rhs))
    return hflux, div, rhs


def u_update(g, nz, grav, eta, velo, dt, theta1):
    """grad_eta + u_update on one level: returns (velo, grad)."""
    L = lib()
    lv = _Level(g)
    v = _c(velo).copy()
    grad = np.zeros(3 * g.NN)
    e = _c(eta)
    L.orc_u_update.argtypes = [C.POINTER(orc_blevel), C.c_int, C.c_double, _dp, C.c_double, C.c_double, _dp, _dp]
    L.orc_u_update(C.byref(lv.s), nz, grav, _p(e), dt, theta1, _p(v), _p(grad))
    return v, grad


def step1_flux(g, itype, velo, mass, mean_m, scalar=None):
    """step1 itype 1, 5, 6 or 7 on one layer: returns the edge flux (3*NN)."""
    L = lib()
    lv = _Level(g)
    flux = np.zeros(3 * g.NN)
    bufs = [None if scalar is None else _c(scalar), _c(velo), _c(mass), _c(mean_m)]
    L.orc_step1_flux.argtypes = [C.POINTER(orc_blevel), C.c_int, _dp, _dp, _dp, _dp, _dp]
    L.orc_step1_flux.restype = C.c_int
    rc = L.orc_step1_flux(C.byref(lv.s), int(itype), *[None if b is None else _p(b) for b in bufs], _p(flux))
    assert rc == 0
    return flux


def step1_vort(g, velo):
    """step1 itype 8 + post_vort on one layer's velocity: vorticity (2*NN, LORT then UPLT)."""
    from .grid import own
    g = own(g)
    L = lib()
    lv = _Level(g)
    vort = np.zeros(2 * g.NN)
    tri = _c(g.triarea)
    L.orc_step1_vort.argtypes = [C.POINTER(orc_blevel), _dp, _dp, _dp]
    L.orc_step1_vort.restype = C.c_int
    rc = L.orc_step1_vort(C.byref(lv.s), _p(tri), _p(_c(velo)), _p(vort))
    assert rc == 0
    return vort


def _multi(levels, nz, states, masks, etas, div_olds):
    from .grid import own
    from .restrict import orc_rlevel
    levels = [own(g) for g in levels]
    i32 = C.POINTER(C.c_int32)

    class orc_bml(C.Structure):
        _fields_ = [("b", orc_blevel), ("r", orc_rlevel), ("mass", _dp), ("mean_m", _dp), ("velo", _dp),
                    ("eta", _dp), ("div_old", _dp), ("div", _dp), ("rhs", _dp), ("grad", _dp)]

    arr = (orc_bml * len(levels))()
    keep, outs = [], []
    for q, g in enumerate(levels):
        lv = _Level(g)
        rf = g.rf_wgt if (q > 0 and g.rf_wgt is not None) else np.zeros((3, g.NN))
        geo = [_c(x) for x in (g.hex_inv, g.overl_a, g.overl_split, rf)]
        hn = np.ascontiguousarray(g.halo_node, dtype=np.int64)
        he = np.ascontiguousarray(g.halo_edge, dtype=np.int64)
        mn, me = (np.ascontiguousarray(x, dtype=np.int32) for x in masks[q])
        r = orc_rlevel(g.n, g.P, g.NN, *[_p(x) for x in geo], _p(hn, _ip), len(hn), _p(he, _ip), len(he),
                       mn.ctypes.data_as(i32), me.ctypes.data_as(i32), None, None, None, None)
        m, mm = _c(states[q]["mass"]), _c(states[q]["mean_m"])
        v = _c(states[q]["velo"]).copy()
        e, do = _c(etas[q]), _c(div_olds[q])
        div, rhs, grad = np.zeros(g.NN), np.zeros(g.NN), np.zeros(3 * g.NN)
        keep += [lv, geo, hn, he, mn, me, m, mm, v, e, do]
        outs.append(dict(div=div, rhs=rhs, grad=grad, velo=v))
        arr[q] = orc_bml(lv.s, r, _p(m), _p(mm), _p(v), _p(e), _p(do), _p(div), _p(rhs), _p(grad))
    return arr, keep, outs


def rhs_elliptic_multi(levels, nz, states, masks, etas, div_olds, dt, theta2, rho0):
    """flux_divergence (with cpt_or_restr_flux) + rhs_elliptic over the hierarchy:
    per level dict(div, rhs)."""
    L = lib()
    arr, keep, outs = _multi(levels, nz, states, masks, etas, div_olds)
    L.orc_rhs_elliptic_multi.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
    L.orc_rhs_elliptic_multi.restype = C.c_int
    assert L.orc_rhs_elliptic_multi(C.addressof(arr), len(levels), nz, dt, theta2, rho0) == 0
    return outs


def u_update_multi(levels, nz, states, masks, etas, grav, dt, theta1):
    """grad_eta (with cpt_or_restr_eta) + u_update over the hierarchy: per level dict(grad, velo)."""
    L = lib()
    arr, keep, outs = _multi(levels, nz, states, masks, etas, [np.zeros(g.NN) for g in levels])
    L.orc_u_update_multi.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
    L.orc_u_update_multi.restype = C.c_int
    assert L.orc_u_update_multi(C.addressof(arr), len(levels), nz, grav, dt, theta1) == 0
    return outs


def barotropic_correction_multi(levels, nz, ph, states, etas):
    """barotropic_correction (src/barotropic_2d.f90:52-116) on every level:
    total_height/cal_height (:368-412) summed over the layers from 0, then the
    layer-dilation correction cal_barotropic_correction (:85-116) of each
    layer's mass and mass-weighted buoyancy from the free surface eta, porosity
    1.  Element by element with the reference's operand order; returns per
    level (mass, temp).  Slots whose column is empty come out non-finite and are
    not compared."""
    out = []
    rho0 = ph.ref_density
    for q, g in enumerate(levels):
        st = states[q]
        mass = np.array(st["mass"], dtype=np.float64).copy()
        temp = np.array(st["temp"], dtype=np.float64).copy()
        mm, mt, topo = st["mean_m"], st["mean_t"], st["topo"]
        with np.errstate(all="ignore"):
            height = np.zeros(g.NN)
            for k in range(nz):
                height = height + (mm[k] + mass[k]) / (rho0 * 1.0)
            e = np.asarray(etas[q], dtype=np.float64) / 1.0
            for k in range(nz):
                rho_dz = mm[k] + mass[k]
                theta = (mt[k] + temp[k]) / rho_dz
                mass[k] = (e - topo) / height * rho_dz - mm[k]
                rho_dz = mm[k] + mass[k]
                temp[k] = rho_dz * theta - mt[k]
        out.append((mass, temp))
    return out
