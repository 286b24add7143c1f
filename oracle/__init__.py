"""ORACLE -- test infrastructure only.

CPU FP64 restatement of the reference's hot-path operators (see the header of
oracle_trisk.cpp and oracle_elliptic.cpp for the reference routines followed,
file:line).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this package, and only as the checker.  The product library never
links or calls it.

Geometry: every routine takes its geometry and ghost tables from the oracle's
own grid builder (oracle_grid.cpp through grid.own), never from the level
objects it is given; a product level only names the grid parameters and the
level number.

Parity status: not pinned against a reference binary (the reference is
Fortran, and neither the build container nor the GPU host has a Fortran
compiler).  Pinned instead by its own grid builder, bit-identical to the
product's separate restatement (tests/test_oracle_grid.py), by known answers
(the analytic elliptic problem's second-order convergence, div curl = 0, the
energy-neutral Coriolis term, Restrict(Prolong) = I: tests/test_known_answers.py)
and by the properties the reference relies on (conservation, identities:
tests/test_*_oracle.py, tests/test_grid.py).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)


class orc_level(C.Structure):
    _fields_ = [("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64),
                ("len", _dp), ("pedlen", _dp), ("part", _dp), ("hex_inv", _dp), ("triarea", _dp), ("coriolis", _dp),
                ("halo_node", _ip), ("n_halo_node", C.c_int64), ("halo_edge", _ip), ("n_halo_edge", C.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing; run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        L.orc_trend.argtypes = [C.POINTER(orc_level), C.c_int, C.c_double, C.c_double, C.c_double] + [_dp] * 9
        L.orc_trend.restype = C.c_int
        L.orc_rk4.argtypes = [C.POINTER(orc_level), C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_int] + [_dp] * 6
        L.orc_rk4.restype = C.c_int
        if hasattr(L, "orc_elliptic_apply"):
            from . import elliptic as _e  # noqa: F401  (binds its own signatures)
        _lib = L
    return _lib


def _d(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class _Level:
    """Keeps the numpy arrays alive for the lifetime of the ctypes struct."""

    def __init__(self, g):
        from .grid import own
        g = own(g)
        self.keep = [np.ascontiguousarray(x) for x in
                     (g.len, g.pedlen, g.part, g.hex_inv, g.triarea, g.coriolis)]
        self.hn = np.ascontiguousarray(g.halo_node, dtype=np.int64)
        self.he = np.ascontiguousarray(g.halo_edge, dtype=np.int64)
        k = self.keep
        self.s = orc_level(g.n, g.P, g.NN, _d(k[0]), _d(k[1]), _d(k[2]), _d(k[3]), _d(k[4]), _d(k[5]),
                           self.hn.ctypes.data_as(_ip), len(self.hn), self.he.ctypes.data_as(_ip), len(self.he))


def trend(g, nz, ph, state):
    """One evaluation of trend_ml on a uniform level.  Returns (dmass, dtemp, dvelo, state_after_halo)."""
    lv = _Level(g)
    m, t, v = (np.ascontiguousarray(state[k]).copy() for k in ("mass", "temp", "velo"))
    dm, dt, dv = np.zeros_like(m), np.zeros_like(t), np.zeros_like(v)
    rc = lib().orc_trend(C.byref(lv.s), nz, ph.grav, ph.ref_density, ph.p_top, _d(m), _d(t), _d(v),
                         _d(np.ascontiguousarray(state["mean_m"])), _d(np.ascontiguousarray(state["mean_t"])),
                         _d(np.ascontiguousarray(state["topo"])), _d(dm), _d(dt), _d(dv))
    assert rc == 0
    return dm, dt, dv, dict(mass=m, temp=t, velo=v)


def rk4(g, nz, ph, state, dt, nsteps):
    """nsteps RK4 steps on a uniform level; returns the new (mass, temp, velo)."""
    lv = _Level(g)
    m, t, v = (np.ascontiguousarray(state[k]).copy() for k in ("mass", "temp", "velo"))
    rc = lib().orc_rk4(C.byref(lv.s), nz, ph.grav, ph.ref_density, ph.p_top, float(dt), int(nsteps), _d(m), _d(t),
                       _d(v), _d(np.ascontiguousarray(state["mean_m"])), _d(np.ascontiguousarray(state["mean_t"])),
                       _d(np.ascontiguousarray(state["topo"])))
    assert rc == 0
    return m, t, v


def set_threads(n: int) -> None:
    """Worker threads of the oracle (parallel over the 10 lozenge domains)."""
    L = lib()
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_set_threads.restype = None
    L.orc_set_threads(int(n))


def get_threads() -> int:
    L = lib()
    L.orc_get_threads.restype = C.c_int
    return int(L.orc_get_threads())


class orc_mlevel(C.Structure):
    _fields_ = [("geo", orc_level), ("overl_a", _dp), ("overl_split", _dp), ("rf_wgt", _dp),
                ("mask_n", C.POINTER(C.c_int32)), ("mask_e", C.POINTER(C.c_int32)),
                ("mass", _dp), ("temp", _dp), ("velo", _dp), ("mean_m", _dp), ("mean_t", _dp), ("topo", _dp),
                ("dmass", _dp), ("dtemp", _dp), ("dvelo", _dp)]


def trend_multi(levels, nz, ph, states, masks):
    """trend_ml over the hierarchy levels[0] .. levels[-1] (level_start ..
    level_end), every level present.  states[q]: dict of mass, temp, velo,
    mean_m, mean_t, topo of levels[q]; masks[q]: (mask_n, mask_e) int32.
    Returns per level (dmass, dtemp, dvelo, state_after_halo)."""
    from .grid import own
    levels = [own(g) for g in levels]
    L = lib()
    L.orc_trend_multi.argtypes = [C.POINTER(orc_mlevel), C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
    L.orc_trend_multi.restype = C.c_int
    arr = (orc_mlevel * len(levels))()
    keep, out = [], []
    i32 = C.POINTER(C.c_int32)
    for q, g in enumerate(levels):
        lv = _Level(g)
        st = states[q]
        m, t, v = (np.ascontiguousarray(st[k], dtype=np.float64).copy() for k in ("mass", "temp", "velo"))
        mm, mt, tp = (np.ascontiguousarray(st[k], dtype=np.float64) for k in ("mean_m", "mean_t", "topo"))
        geo = [np.ascontiguousarray(x, dtype=np.float64) for x in (g.overl_a, g.overl_split)]
        rf = None if (q == 0 or g.rf_wgt is None) else np.ascontiguousarray(g.rf_wgt, dtype=np.float64)
        mn, me = (np.ascontiguousarray(x, dtype=np.int32) for x in masks[q])
        dm, dt, dv = np.zeros_like(m), np.zeros_like(t), np.zeros_like(v)
        keep += [lv, m, t, v, mm, mt, tp, mn, me, dm, dt, dv, rf] + geo
        arr[q] = orc_mlevel(lv.s, _d(geo[0]), _d(geo[1]), None if rf is None else _d(rf),
                            mn.ctypes.data_as(i32), me.ctypes.data_as(i32), _d(m), _d(t), _d(v), _d(mm), _d(mt),
                            _d(tp), _d(dm), _d(dt), _d(dv))
        out.append((dm, dt, dv, dict(mass=m, temp=t, velo=v)))
    rc = L.orc_trend_multi(arr, len(levels), nz, ph.grav, ph.ref_density, ph.p_top)
    assert rc == 0
    return out


def rk4_multi(levels, nz, ph, states, masks, dt, nsteps=1, H=None):
    """RK4 (src/time_integr.f90:78-103) over the hierarchy: per stage
    trend_multi on every level, RK_sub_step on every level, then
    WT_after_step (src/adapt.f90:186-237) of the stage state with the masks
    held fixed.  Returns per level the new (mass, temp, velo).  H (an
    oracle.wavelet.Hierarchy, optional) receives the masks and is left holding
    the final state and its compressed wavelets, as adapt needs them."""
    from .wavelet import Hierarchy
    if H is None:
        H = Hierarchy(levels, nz)
    for g, (mn, me) in zip(levels, masks):
        H.set(g.level, "mask_n", mn)
        H.set(g.level, "mask_e", me)
    keys = ("mass", "temp", "velo")
    q = [{k: np.array(st[k], dtype=np.float64) for k in keys} for st in states]
    hs = (dt / 4.0, dt / 3.0, dt / 2.0, dt)
    for _ in range(nsteps):
        q1 = None
        for stage in range(4):
            src = q if stage == 0 else q1
            st = [dict(states[i], **src[i]) for i in range(len(levels))]
            tr = trend_multi(levels, nz, ph, st, masks)
            dest = [{k: q[i][k] + hs[stage] * tr[i][j] for j, k in enumerate(keys)} for i in range(len(levels))]
            for i, g in enumerate(levels):
                for k, f in zip(keys, ("s_m", "s_t", "s_v")):
                    H.set(g.level, f, dest[i][k])
            H.wt_after_step()
            dest = [{k: H.field(g.level, f).copy() for k, f in zip(keys, ("s_m", "s_t", "s_v"))}
                    for g in levels]
            if stage < 3:
                q1 = dest
            else:
                q = dest
    return [(x["mass"], x["temp"], x["velo"]) for x in q]


def rk4_split_explicit(levels, nz, ph, states, masks, etas, dt, theta1, H=None):
    """The four RK_split calls of RK4_split (src/time_integr.f90:360-382,
    444-463) over the hierarchy, without free_surface_update: per stage
    barotropic_correction of the stage's source state (in place, so the first
    stage corrects the solution itself), trend_ml, scalar_star and u_star
    (src/barotropic_2d.f90:9-50: the base is the solution, the velocity adds
    theta1 times grad_eta of each level's free surface) and WT_after_step.
    Returns per level the new (mass, temp, velo)."""
    from .barotropic import barotropic_correction_multi, u_update_multi
    from .wavelet import Hierarchy
    if H is None:
        H = Hierarchy(levels, nz)
    for g, (mn, me) in zip(levels, masks):
        H.set(g.level, "mask_n", mn)
        H.set(g.level, "mask_e", me)
    keys = ("mass", "temp", "velo")
    q = [{k: np.array(st[k], dtype=np.float64) for k in keys} for st in states]
    hs = (dt / 4.0, dt / 3.0, dt / 2.0, dt)
    q1 = None
    for stage in range(4):
        src = q if stage == 0 else q1
        st = [dict(states[i], **src[i]) for i in range(len(levels))]
        for i, (m, t) in enumerate(barotropic_correction_multi(levels, nz, ph, st, etas)):
            src[i]["mass"], src[i]["temp"] = m, t
        st = [dict(states[i], **src[i]) for i in range(len(levels))]
        tr = trend_multi(levels, nz, ph, st, masks)
        grad = [o["grad"] for o in u_update_multi(levels, nz, st, masks, etas, ph.grav, 0.0, 0.0)]
        dest = []
        for i in range(len(levels)):
            d = {"mass": q[i]["mass"] + hs[stage] * tr[i][0], "temp": q[i]["temp"] + hs[stage] * tr[i][1],
                 "velo": q[i]["velo"] + hs[stage] * (tr[i][2] + theta1 * grad[i][None, :])}
            dest.append(d)
        for i, g in enumerate(levels):
            for k, f in zip(keys, ("s_m", "s_t", "s_v")):
                H.set(g.level, f, dest[i][k])
        H.wt_after_step()
        dest = [{k: H.field(g.level, f).copy() for k, f in zip(keys, ("s_m", "s_t", "s_v"))} for g in levels]
        if stage < 3:
            q1 = dest
        else:
            q = dest
    return [(x["mass"], x["temp"], x["velo"]) for x in q]



def free_surface_update(levels, nz, ph, states, masks, etas, div_olds, dt, theta1, theta2, H, method="fmg",
                        domain_level=2, keep_eta_hierarchy=False, **solver):
    """free_surface_update (src/time_integr.f90:465-478) over the hierarchy:
    eta_update (src/barotropic_2d.f90:118-129: rhs_elliptic on every level, the
    solve with the operator's coefficients from the old free surface, starting
    from it), barotropic_correction, u_update and WT_after_step (with the
    masks H holds).  states[q]: the level's mass, temp, velo, mean_m, mean_t,
    topo.  Returns per level (mass, temp, velo), the new free surfaces and the
    solver's per-level iteration counts (and, with keep_eta_hierarchy, the
    one-layer wavelet hierarchy holding the free surface and its wavelets,
    for free_surface_adapt)."""
    from .barotropic import barotropic_correction_multi, rhs_elliptic_multi, u_update_multi
    from .elliptic import Hierarchy as EH
    from .grid import own

    ol = [own(g) for g in levels]
    ro = rhs_elliptic_multi(levels, nz, states, masks, etas, div_olds, dt, theta2, ph.ref_density)
    eo = []
    for g, e in zip(ol, etas):
        x = np.array(e, dtype=np.float64).copy()
        x[g.halo_node[:, 0]] = x[g.halo_node[:, 1]]   # Laplacian_scalar(S_TEMP) after update_bdry
        eo.append(x)
    E = EH(levels, [st["topo"] for st in states], grav=ph.grav, dt=dt, theta1=theta1, theta2=theta2,
           domain_level=domain_level, eta_old=eo, **solver)
    u, _, its = E.solve(np.concatenate([np.asarray(e, dtype=np.float64) for e in etas]),
                        np.concatenate([r["rhs"] for r in ro]), method)
    off = np.cumsum([0] + [g.NN for g in ol])
    new_etas = [u[off[q]:off[q + 1]].copy() for q in range(len(ol))]
    mt = barotropic_correction_multi(levels, nz, ph, states, new_etas)
    st2 = [dict(states[q], mass=m, temp=t) for q, (m, t) in enumerate(mt)]
    uo = u_update_multi(levels, nz, st2, masks, new_etas, ph.grav, dt, theta1)
    for q, g in enumerate(ol):
        H.set(g.level, "s_m", st2[q]["mass"])
        H.set(g.level, "s_t", st2[q]["temp"])
        H.set(g.level, "s_v", uo[q]["velo"])
    H.wt_after_step()
    out = [(H.field(g.level, "s_m").copy(), H.field(g.level, "s_t").copy(), H.field(g.level, "s_v").copy())
           for g in ol]
    # the free surface goes through the same WT_after_step (it is layer
    # zlevels+1 of sol): a one-layer hierarchy with the same masks
    from .wavelet import Hierarchy
    He = Hierarchy(levels, 1)
    for q, g in enumerate(ol):
        He.set(g.level, "mask_n", H.field(g.level, "mask_n"))
        He.set(g.level, "mask_e", H.field(g.level, "mask_e"))
        He.set(g.level, "s_m", new_etas[q][None, :])
    He.wt_after_step()
    new_etas = [He.field(g.level, "s_m")[0].copy() for g in ol]
    if keep_eta_hierarchy:
        return out, new_etas, its, He
    return out, new_etas, its


def free_surface_adapt(levels, He, masks):
    """The free surface's part of adapt (src/adapt.f90:79-103 compress_wavelets
    and the inverse transform after it, src/main.f90:441): the wavelets He kept
    from free_surface_update, compressed under the new masks, then the inverse
    transform.  Returns the new free surface of every level."""
    for g, (mn, me) in zip(levels, masks):
        He.set(g.level, "mask_n", mn)
        He.set(g.level, "mask_e", me)
    He.compress()
    He.inverse()
    return [He.field(g.level, "s_m")[0].copy() for g in levels]


def rk4_split(levels, nz, ph, states, masks, etas, dt, theta1, theta2, method="fmg", domain_level=2,
              keep_eta_hierarchy=False, **solver):
    """RK4_split (src/time_integr.f90:360-382) over the hierarchy with theta2 = 1
    (no previous flux divergence): the four RK_split stages, then
    free_surface_update.  Returns what free_surface_update returns."""
    from .wavelet import Hierarchy

    assert theta2 == 1.0
    H = Hierarchy(levels, nz)
    q = rk4_split_explicit(levels, nz, ph, states, masks, etas, dt, theta1, H=H)
    st = [dict(states[i], mass=m, temp=t, velo=v) for i, (m, t, v) in enumerate(q)]
    zero = [np.zeros(g.NN) for g in levels]
    return free_surface_update(levels, nz, ph, st, masks, etas, zero, dt, theta1, theta2, H, method=method,
                               domain_level=domain_level, keep_eta_hierarchy=keep_eta_hierarchy, **solver)
