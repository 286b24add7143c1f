"""Host-side mirror of the reference's operator interface for this path.

The reference plugs its operators into the time stepper through Fortran
interfaces (src/time_integr.f90:7-31): ``trend_fun(q, dq)`` and
``dt_step(q, wav, trend_fun, h)`` (RK4, :78-103).  ``TriskModel`` exposes the
same two operations over the C-ABI of libwtgpu.so, on device-resident state:

    model = TriskModel(grid_level, nz, params)
    model.upload(state)                   # sol, sol_mean
    dq = model.trend_ml()                 # trend_fun(sol, trend)
    model.rk4(dt, nsteps)                 # dt_step => RK4
    state = model.download()

There is no fallback: if the CUDA library or a device is missing every call
raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .cases import OceanParams
from .grid import LevelGeom


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _LevelDescs:
    """wt_level_desc array + the numpy buffers it points into."""

    def __init__(self, levels: list[LevelGeom], topos: list[np.ndarray]):
        self.keep = []
        arr = (N.wt_level_desc * len(levels))()
        for q, (g, topo) in enumerate(zip(levels, topos)):
            bufs = [_c(x) for x in (g.len, g.pedlen, g.part, g.hex_inv, g.triarea, g.coriolis, g.overl_a, topo)]
            hn = np.ascontiguousarray(g.halo_node, dtype=np.int64)
            he = np.ascontiguousarray(g.halo_edge, dtype=np.int64)
            self.keep += bufs + [hn, he]
            iu = _c(g.iu_wgt) if (g.iu_wgt is not None and q > 0) else None
            rf = _c(g.rf_wgt) if (getattr(g, "rf_wgt", None) is not None and q > 0) else None
            sp = _c(g.overl_split)
            self.keep += [x for x in (iu, rf, sp) if x is not None]
            arr[q] = N.wt_level_desc(g.level, g.n, g.P, g.NN, *[N.dptr(b) for b in bufs],
                                     N.iptr(hn), len(hn), N.iptr(he), len(he), N.dptr(iu), N.dptr(sp), N.dptr(rf))
        self.arr = arr


class DeviceGrid:
    """Owns one wt_handle: geometry of levels [level_start, level_end] on the GPU."""

    def __init__(self, levels: list[LevelGeom], topos: list[np.ndarray], nz: int, ph: OceanParams | None = None):
        ph = ph or OceanParams()
        self.levels = levels
        self.nz = nz
        self.ph = ph
        descs = _LevelDescs(levels, topos)
        desc = N.wt_grid_desc(levels[0].level, levels[-1].level, nz, ph.grav, ph.ref_density, ph.p_top, descs.arr)
        h = C.c_void_p()
        N.check("wt_create", N.lib().wt_create(C.byref(desc), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            N.lib().wt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return N.lib().wt_stream(self.h) or 0

    def status(self) -> int:
        return N.lib().wt_status(self.h)

    def remap_vertical(self, remap_type: str, a_vert: np.ndarray, b_vert: np.ndarray) -> None:
        """remap_vertical_coordinates of every layered level (wt_remap_vertical):
        remap_type '0', '1' or '2PPM'; a_vert, b_vert the nz + 1 hybrid
        coefficients from the bottom."""
        code = {"0": 0, "1": 1, "2PPM": 2}[remap_type]
        a = np.ascontiguousarray(a_vert, dtype=np.float64)
        b = np.ascontiguousarray(b_vert, dtype=np.float64)
        N.check("wt_remap_vertical", N.lib().wt_remap_vertical(self.h, code, N.dptr(a), N.dptr(b)))

    def min_mass(self, b_vert: np.ndarray) -> float:
        """cpt_min_mass (wt_min_mass): the smallest relative layer mass against the
        zero-perturbation grid b_vert z_s, over the nodes the masks keep."""
        b = np.ascontiguousarray(b_vert, dtype=np.float64)
        out = np.zeros(1)
        N.check("wt_min_mass", N.lib().wt_min_mass(self.h, N.dptr(b), N.dptr(out)))
        return float(out[0])

    def clear_status(self) -> None:
        """Acknowledge a device-side error: flag and sticky status back to 0."""
        N.check("wt_clear_status", N.lib().wt_clear_status(self.h))

    def test_tma_timeout(self, on: bool) -> None:
        """WT_TUNE_TEST_TMA_TIMEOUT (test only): the TMA-staged kernels take
        their wait-timeout path while on."""
        N.check("wt_tune", N.lib().wt_tune(self.h, 4, 1 if on else 0))


class TriskModel(DeviceGrid):
    """Uniform-level layered ocean model (incompressible, explicit RK4)."""

    def __init__(self, g: LevelGeom, nz: int, topo: np.ndarray, ph: OceanParams | None = None):
        super().__init__([g], [topo], nz, ph)
        self.g = g

    def upload(self, state: dict) -> None:
        N.check("wt_upload_state", N.lib().wt_upload_state(
            self.h, N.dptr(_c(state["mass"])), N.dptr(_c(state["temp"])), N.dptr(_c(state["velo"])),
            N.dptr(_c(state["mean_m"])), N.dptr(_c(state["mean_t"]))))

    def download(self) -> dict:
        nz, NN = self.nz, self.g.NN
        m, t, v = np.empty((nz, NN)), np.empty((nz, NN)), np.empty((nz, 3 * NN))
        N.check("wt_download_state", N.lib().wt_download_state(self.h, N.dptr(m), N.dptr(t), N.dptr(v)))
        return dict(mass=m, temp=t, velo=v)

    def trend_ml(self):
        """trend_fun(sol, trend): returns (dmass, dtemp, dvelo) of the resident state."""
        N.check("wt_trend", N.lib().wt_trend(self.h))
        nz, NN = self.nz, self.g.NN
        dm, dt, dv = np.empty((nz, NN)), np.empty((nz, NN)), np.empty((nz, 3 * NN))
        N.check("wt_download_trend", N.lib().wt_download_trend(self.h, N.dptr(dm), N.dptr(dt), N.dptr(dv)))
        return dm, dt, dv

    def rk4(self, dt: float, nsteps: int = 1) -> None:
        """dt_step => RK4 on the resident state (asynchronous on the handle's stream)."""
        N.check("wt_rk4_step", N.lib().wt_rk4_step(self.h, float(dt), int(nsteps)))

    def rk4_host(self, dt: float, nsteps: int, mass: np.ndarray, temp: np.ndarray, velo: np.ndarray) -> None:
        """RK4 through host buffers (uploaded, stepped, downloaded in place)."""
        N.check("wt_rk4_step_host", N.lib().wt_rk4_step_host(
            self.h, float(dt), int(nsteps), N.dptr(mass), N.dptr(temp), N.dptr(velo)))

    def synchronize(self) -> None:
        N.check("wt_synchronize", N.lib().wt_synchronize(self.h))

    def flux_precision(self, bits: int) -> None:
        """WT_TUNE_FLUX_PRECISION: 32 runs step1's flux stencils in FP32 (FP64
        trends, conservation and RK accumulation); 64 is the FP64 path."""
        N.check("wt_tune", N.lib().wt_tune(self.h, 3, int(bits)))

    # -- barotropic pieces of the mode-split step (src/barotropic_2d.f90) --
    def barotropic_upload(self, eta: np.ndarray | None = None, div_old: np.ndarray | None = None) -> None:
        N.check("wt_barotropic_upload", N.lib().wt_barotropic_upload(
            self.h, N.dptr(None if eta is None else _c(eta)), N.dptr(None if div_old is None else _c(div_old))))

    def rhs_elliptic(self, dt: float, theta2: float = 1.0):
        """flux_divergence + rhs_elliptic of the resident state: returns (div_flux, rhs)."""
        N.check("wt_rhs_elliptic", N.lib().wt_rhs_elliptic(self.h, float(dt), float(theta2)))
        div, rhs = np.empty(self.g.NN), np.empty(self.g.NN)
        N.check("wt_barotropic_download", N.lib().wt_barotropic_download(self.h, N.dptr(div), N.dptr(rhs), None))
        return div, rhs

    def u_update(self, dt: float, theta1: float = 1.0) -> np.ndarray:
        """grad_eta + u_update on the resident velocity: returns grad eta (3*NN)."""
        N.check("wt_u_update", N.lib().wt_u_update(self.h, float(dt), float(theta1)))
        grad = np.empty(3 * self.g.NN)
        N.check("wt_barotropic_download", N.lib().wt_barotropic_download(self.h, None, None, N.dptr(grad)))
        return grad


def _step1_flux(model, itype: int, layer: int = 0, scalar: np.ndarray | None = None) -> np.ndarray:
    flux = np.empty(3 * model.g.NN)
    N.check("wt_step1_flux", N.lib().wt_step1_flux(model.h, int(itype), int(layer),
                                                   N.dptr(None if scalar is None else _c(scalar)), N.dptr(flux)))
    return flux


def _step1_vort(model, layer: int = 0) -> np.ndarray:
    vort = np.empty(2 * model.g.NN)
    N.check("wt_step1_vort", N.lib().wt_step1_vort(model.h, int(layer), N.dptr(vort)))
    return vort


TriskModel.step1_flux = _step1_flux
TriskModel.step1_flux.__doc__ = """step1 itype 1, 5, 6 or 7 on one layer of the resident state: edge flux (3*NN)."""
TriskModel.step1_vort = _step1_vort
TriskModel.step1_vort.__doc__ = """step1 itype 8 + post_vort on one layer of the resident velocity: vorticity (2*NN)."""


class WaveletHierarchy(DeviceGrid):
    """Layer mass, potential temperature and velocity on every level of a
    uniform hierarchy, their wavelet coefficients and the node/edge masks, with
    the reference's forward_wavelet_transform, inverse_wavelet_transform,
    mask_tol_vars, compress_wavelets and WT_after_step (src/wavelet.f90,
    src/mask.f90, src/adapt.f90), and the multi-level trend's work fields
    (scalar, dscalar, flux, dvelo) with its compute-or-restrict operators
    (src/multi_level.f90:311-659).  Level level_end's scaling fields are the
    stepper's state."""

    FIELDS = {"mass": 0, "temp": 1, "velo": 2, "wc_mass": 3, "wc_temp": 4, "wc_velo": 5, "mask_n": 6, "mask_e": 7,
              "scalar": 8, "dscalar": 9, "flux": 10, "dvelo": 11, "mean_m": 12, "mean_t": 13}

    def __init__(self, levels: list[LevelGeom], topos: list[np.ndarray], nz: int, ph: OceanParams | None = None):
        super().__init__(levels, topos, nz, ph)
        self.ls, self.le = levels[0].level, levels[-1].level
        N.check("wt_wavelet_setup", N.lib().wt_wavelet_setup(self.h))

    def _shape(self, level, name):
        NN = self.levels[level - self.ls].NN
        if name == "mask_n":
            return (NN,), np.int32
        if name == "mask_e":
            return (3 * NN,), np.int32
        edge = name.endswith("velo") or name == "flux"
        return (self.nz, (3 if edge else 1) * NN), np.float64

    def upload(self, level: int, name: str, a: np.ndarray) -> None:
        shape, dt = self._shape(level, name)
        buf = np.ascontiguousarray(np.broadcast_to(a, shape), dtype=dt)
        N.check("wt_upload_field", N.lib().wt_upload_field(self.h, level, self.FIELDS[name], buf.ctypes.data))

    def download(self, level: int, name: str) -> np.ndarray:
        shape, dt = self._shape(level, name)
        buf = np.empty(shape, dtype=dt)
        N.check("wt_download_field", N.lib().wt_download_field(self.h, level, self.FIELDS[name], buf.ctypes.data))
        return buf

    def _batch(self, items):
        n = len(items)
        lv = (N.C.c_int * n)(*[int(l) for l, _, _ in items])
        fd = (N.C.c_int * n)(*[self.FIELDS[f] for _, f, _ in items])
        return n, lv, fd

    def upload_many(self, items) -> None:
        """items: (level, name, array) triples, copied in one batch (wt_upload_fields)."""
        bufs = []
        for l, f, a in items:
            shape, dt = self._shape(l, f)
            bufs.append(np.ascontiguousarray(np.broadcast_to(a, shape), dtype=dt))
        n, lv, fd = self._batch(items)
        ptr = (N.C.c_void_p * n)(*[b.ctypes.data for b in bufs])
        N.check("wt_upload_fields", N.lib().wt_upload_fields(self.h, n, lv, fd, ptr))

    def download_many(self, items) -> None:
        """items: (level, name, out) triples; out arrays of the field's shape and
        dtype, C-contiguous, filled in one batch (wt_download_fields)."""
        for l, f, out in items:
            shape, dt = self._shape(l, f)
            if out.shape != shape or out.dtype != dt or not out.flags["C_CONTIGUOUS"]:
                raise ValueError(f"download_many: {f} of level {l} needs a C-contiguous {dt} array {shape}")
        n, lv, fd = self._batch(items)
        ptr = (N.C.c_void_p * n)(*[o.ctypes.data for _, _, o in items])
        N.check("wt_download_fields", N.lib().wt_download_fields(self.h, n, lv, fd, ptr))

    def forward(self) -> None:
        N.check("wt_forward_wt", N.lib().wt_forward_wt(self.h))

    def inverse(self) -> None:
        N.check("wt_inverse_wt", N.lib().wt_inverse_wt(self.h))

    def inverse_tree(self) -> None:
        """The inverse transform after adapt on the patch tree (wt_inverse_tree):
        the parents the next step reads and those of the tree's nodes."""
        N.check("wt_inverse_tree", N.lib().wt_inverse_tree(self.h))

    def mask_tol_vars(self, threshold: np.ndarray, level_fill: int) -> None:
        thr = _c(np.asarray(threshold).reshape(3, self.nz))
        N.check("wt_mask_tol_vars", N.lib().wt_mask_tol_vars(self.h, N.dptr(thr), int(level_fill)))

    def mask_build(self, threshold: np.ndarray, level_fill: int, max_level: int, patch_size: int = 0):
        """adapt's mask sequence; returns the check_child_required flags (uint8)
        of every parent patch and child quadrant when patch_size > 0."""
        thr = _c(np.asarray(threshold).reshape(3, self.nz))
        out = None
        if patch_size > 0:
            n = sum(10 * (g.n // patch_size) ** 2 * 4 for g in self.levels[:-1])
            out = np.zeros(n, dtype=np.uint8)
        N.check("wt_mask_build", N.lib().wt_mask_build(self.h, N.dptr(thr), int(level_fill), int(max_level),
                                                       int(patch_size), None if out is None else out.ctypes.data))
        return out

    def compress(self) -> None:
        N.check("wt_compress", N.lib().wt_compress(self.h))

    # ---- patch tree (src/refine_patch.f90)
    def tree_init(self, patch_size: int) -> None:
        N.check("wt_tree_init", N.lib().wt_tree_init(self.h, int(patch_size)))
        self.patch_size = int(patch_size)

    def tree_state_buffers(self, alloc=np.empty):
        """Packed arrays of level_end's state for every patch of the level
        (mass, temp [patches][nz][ps*ps], velo [patches][nz][3][ps*ps]);
        alloc(shape) makes each (e.g. pinned host memory)."""
        ps, g = self.patch_size, self.levels[-1]
        npatch = 10 * (g.n // ps) ** 2
        return (alloc((npatch, self.nz, ps * ps)), alloc((npatch, self.nz, ps * ps)),
                alloc((npatch, self.nz, 3, ps * ps)))

    def download_tree_state(self, bufs) -> int:
        """level_end's state on its existing patches into the packed arrays
        bufs (tree_state_buffers); returns the patch count (the arrays' first
        that many rows)."""
        m, t, v = bufs
        n = C.c_longlong(0)
        N.check("wt_download_tree_state", N.lib().wt_download_tree_state(
            self.h, N.dptr(m), N.dptr(t), N.dptr(v), m.shape[0], C.byref(n)))
        return n.value

    def upload_tree_state(self, bufs, n_patches: int) -> None:
        m, t, v = bufs
        N.check("wt_upload_tree_state", N.lib().wt_upload_tree_state(self.h, N.dptr(m), N.dptr(t), N.dptr(v),
                                                                     int(n_patches)))

    def tree_level_end(self) -> int:
        le = C.c_int(0)
        N.check("wt_tree_level_end", N.lib().wt_tree_level_end(self.h, C.byref(le)))
        return le.value

    def tree(self, level: int, patch_size: int):
        """(exist, fresh) patch bytes of `level` as bool arrays [10][n/ps][n/ps]."""
        npp = self.levels[level - self.ls].n // patch_size
        ex = np.empty((10, npp, npp), dtype=np.uint8)
        fr = np.empty_like(ex)
        N.check("wt_tree_download", N.lib().wt_tree_download(self.h, int(level), ex.ctypes.data, fr.ctypes.data))
        return ex.astype(bool), fr.astype(bool)

    def grid_sync(self, exist_levels, level_end: int) -> None:
        """Upload a host tree: exist_levels[q] the patch bytes of level ls + q."""
        buf = np.ascontiguousarray(np.concatenate([np.asarray(e, dtype=np.uint8).ravel() for e in exist_levels]))
        N.check("wt_grid_sync", N.lib().wt_grid_sync(self.h, buf.ctypes.data, int(level_end)))

    def adapt(self, threshold: np.ndarray, level_fill: int, max_level: int):
        """adapt on the tree (mask sequence with refine() inside, compression);
        returns (level_end, refined)."""
        thr = _c(np.asarray(threshold).reshape(3, self.nz))
        le, rf = C.c_int(0), C.c_int(0)
        N.check("wt_adapt", N.lib().wt_adapt(self.h, N.dptr(thr), int(level_fill), int(max_level), C.byref(le),
                                             C.byref(rf)))
        return le.value, bool(rf.value)

    def count_active(self, threshold: np.ndarray):
        """count_active over the patches the last refine made: (node, edge) counts."""
        thr = _c(np.asarray(threshold).reshape(3, self.nz))
        out = (C.c_longlong * 2)()
        N.check("wt_count_active", N.lib().wt_count_active(self.h, N.dptr(thr), out))
        return int(out[0]), int(out[1])

    def tree_stats(self, level: int):
        """(patches, patches made by the last refine, owned nodes outside the
        tree with a mask that is not ZERO, owned nodes in the needed-node map
        or -1) of `level`."""
        out = (C.c_longlong * 4)()
        N.check("wt_tree_stats", N.lib().wt_tree_stats(self.h, int(level), out))
        return tuple(int(x) for x in out)

    def mask_adj_child(self, level: int) -> None:
        N.check("wt_mask_adj_child", N.lib().wt_mask_adj_child(self.h, int(level)))

    def wt_after_step(self) -> None:
        N.check("wt_wt_after_step", N.lib().wt_wt_after_step(self.h))

    def trend_multi(self) -> None:
        """trend_ml over every level of the hierarchy (scaling fields, layer means and masks as uploaded)."""
        N.check("wt_trend_multi", N.lib().wt_trend_multi(self.h))

    def adaptive_step(self, dt: float, threshold: np.ndarray, level_fill: int, max_level: int,
                      nsteps: int = 1) -> None:
        """nsteps adaptive time steps (RK4 of the hierarchy, adapt's masks and compression,
        inverse transform) replayed as one CUDA graph per step."""
        thr = _c(np.asarray(threshold).reshape(3, self.nz))
        N.check("wt_adaptive_step", N.lib().wt_adaptive_step(self.h, float(dt), N.dptr(thr), int(level_fill),
                                                             int(max_level), int(nsteps)))

    def barotropic_upload(self, level: int, eta=None, div_old=None) -> None:
        """Free surface and previous flux divergence of one level (NN each; either may be None)."""
        N.check("wt_barotropic_upload_level", N.lib().wt_barotropic_upload_level(
            self.h, int(level), N.dptr(None if eta is None else _c(eta)),
            N.dptr(None if div_old is None else _c(div_old))))

    def rhs_elliptic_multi(self, dt: float, theta2: float = 1.0) -> None:
        """flux_divergence with its compute-or-restrict and rhs_elliptic on every level."""
        N.check("wt_rhs_elliptic_multi", N.lib().wt_rhs_elliptic_multi(self.h, float(dt), float(theta2)))

    def u_update_multi(self, dt: float, theta1: float = 1.0) -> None:
        """grad_eta with cpt_or_restr_eta and u_update on every level."""
        N.check("wt_u_update_multi", N.lib().wt_u_update_multi(self.h, float(dt), float(theta1)))

    def barotropic_download(self, level: int):
        """(div_flux, rhs, grad_eta) of one level."""
        NN = self.levels[level - self.ls].NN
        div, rhs, grad = np.empty(NN), np.empty(NN), np.empty(3 * NN)
        N.check("wt_barotropic_download_level", N.lib().wt_barotropic_download_level(
            self.h, int(level), N.dptr(div), N.dptr(rhs), N.dptr(grad)))
        return div, rhs, grad

    def lnorm(self, order: str = "inf") -> np.ndarray:
        """cal_lnorm of the scaling fields: (3, nz) for mass, Theta, velocity; order "inf", "1", "2" or "min"."""
        out = np.empty((3, self.nz))
        code = {"inf": 0, "1": 1, "2": 2, "min": 3}[order]
        N.check("wt_lnorm", N.lib().wt_lnorm(self.h, code, N.dptr(out)))
        return out

    def rk4_split_explicit(self, dt: float, theta1: float) -> None:
        """RK4_split's four RK_split stages (barotropic_correction, trend_ml,
        scalar_star, u_star, WT_after_step) with each level's free surface."""
        N.check("wt_rk4_split_explicit", N.lib().wt_rk4_split_explicit(self.h, float(dt), float(theta1)))

    def barotropic_correction(self) -> None:
        """barotropic_correction of every level's scaling fields from its free surface."""
        N.check("wt_barotropic_correction_multi", N.lib().wt_barotropic_correction_multi(self.h))

    def elliptic_setup(self, dt: float, theta1: float = 1.0, theta2: float = 1.0, domain_level: int = 2) -> None:
        """The free-surface solver of this hierarchy (wt_elliptic_setup)."""
        N.check("wt_elliptic_setup", N.lib().wt_elliptic_setup(self.h, float(dt), float(theta1), float(theta2),
                                                               int(domain_level)))

    def _solve_call(self, name, dt, theta1, theta2, opts):
        rep = N.wt_solver_report()
        rc = getattr(N.lib(), name)(self.h, float(dt), float(theta1), float(theta2), C.byref(opts), C.byref(rep))
        if rc not in (N.WT_OK, N.WT_ERR_NOT_CONVERGED):
            N.check(name, rc)
        rep.status = rc
        return rep

    def free_surface_update(self, dt: float, theta1: float, theta2: float, opts) -> "N.wt_solver_report":
        """free_surface_update: eta_update (rhs, coefficients from the old free
        surface, solve), barotropic_correction, u_update, WT_after_step."""
        return self._solve_call("wt_free_surface_update", dt, theta1, theta2, opts)

    def rk4_split(self, dt: float, theta1: float, theta2: float, opts) -> "N.wt_solver_report":
        """One mode-split time step, RK4_split: RK_split x 4 and free_surface_update."""
        return self._solve_call("wt_rk4_split", dt, theta1, theta2, opts)

    def free_surface_adapt(self) -> None:
        """The free surface's compression under the current masks and its
        inverse transform (adapt's part for layer zlevels+1 of sol)."""
        N.check("wt_free_surface_adapt", N.lib().wt_free_surface_adapt(self.h))

    def free_surface(self, level: int) -> np.ndarray:
        """The free surface of `level` (sol(S_MASS, zlevels+1)), NN doubles."""
        eta = np.empty(self.levels[level - self.ls].NN)
        N.check("wt_free_surface_download", N.lib().wt_free_surface_download(self.h, int(level), N.dptr(eta)))
        return eta

    def skip_inactive(self, on: bool) -> None:
        """WT_TUNE_SKIP_INACTIVE: let the RK stages leave out the finest level's
        nodes whose step1 and trend results cannot reach the state after
        WT_after_step (on by default; the states and masks are the same)."""
        N.check("wt_tune", N.lib().wt_tune(self.h, 2, 1 if on else 0))

    def rk4_multi(self, dt: float, nsteps: int = 1) -> None:
        """nsteps RK4 steps of the whole hierarchy with WT_after_step per stage (masks fixed)."""
        N.check("wt_rk4_multi", N.lib().wt_rk4_multi(self.h, float(dt), int(nsteps)))

    def download_trend(self, level: int):
        """(dmass, dtemp, dvelo) of `level` from the last trend_multi."""
        NN = self.levels[level - self.ls].NN
        dm, dt, dv = np.empty((self.nz, NN)), np.empty((self.nz, NN)), np.empty((self.nz, 3 * NN))
        N.check("wt_download_trend_level", N.lib().wt_download_trend_level(self.h, int(level), N.dptr(dm),
                                                                           N.dptr(dt), N.dptr(dv)))
        return dm, dt, dv

    def restrict_scalar(self, level: int) -> None:
        """scalar_cpt_restr of the work scalar from level+1 to level."""
        N.check("wt_restrict_scalar", N.lib().wt_restrict_scalar(self.h, int(level)))

    def restrict_flux(self, level: int) -> None:
        """flux_cpt_restr of the work flux from level+1's flux and dscalar."""
        N.check("wt_restrict_flux", N.lib().wt_restrict_flux(self.h, int(level)))

    def restrict_u_source(self, level: int) -> None:
        """The restriction of u_source_cpt_restr on the work dvelo."""
        N.check("wt_restrict_u_source", N.lib().wt_restrict_u_source(self.h, int(level)))


def solver_opts(method: str = "fmg", tol: float = 1e-10, **kw):
    """wt_solver_opts with the reference's defaults (src/lin_solve.f90:11-26),
    tolerances set to tol.  method: 'fmg', 'srj' (the reference's solvers),
    'mixed' (FP32 V-cycles in FP64 refinement), 'mg64' (same cycle in FP64),
    'fcg_learned' (flexible CG preconditioned by the learned network, the FP64
    V-cycle as fallback), 'fcg' (flexible CG without a preconditioner) or
    'fcg_mg' (flexible CG preconditioned by the FP64 V-cycle); ir_tol/ir_max
    bound every iterative method after the reference's two."""
    o = N.wt_solver_opts()
    o.method = {"fmg": 0, "srj": 1, "mixed": 2, "mg64": 3, "fcg_learned": 4, "fcg": 5, "fcg_mg": 6}[method]
    o.coarse_iter, o.max_vcycle = 50, 3
    o.pre_iter, o.down_iter, o.up_iter, o.post_iter = 2, 2, 2, 4
    o.max_srj_iter = 200
    o.fine_tol = o.coarse_tol = tol
    o.ir_tol, o.ir_max = tol, 60
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class EllipticSolver(DeviceGrid):
    """Barotropic free-surface solve on a uniform hierarchy (elliptic_solver)."""

    def __init__(self, levels: list[LevelGeom], topos: list[np.ndarray], ph: OceanParams | None = None,
                 dt: float = 600.0, theta1: float = 1.0, theta2: float = 1.0, domain_level: int = 2):
        super().__init__(levels, topos, 1, ph)
        self.offsets = np.cumsum([0] + [g.NN for g in levels])
        N.check("wt_elliptic_setup", N.lib().wt_elliptic_setup(self.h, dt, theta1, theta2, domain_level))

    def field(self) -> np.ndarray:
        return np.zeros(int(self.offsets[-1]))

    def level_view(self, a: np.ndarray, q: int) -> np.ndarray:
        return a[self.offsets[q]:self.offsets[q + 1]]

    def upload(self, u=None, f=None):
        N.check("wt_elliptic_upload", N.lib().wt_elliptic_upload(self.h, N.dptr(u), N.dptr(f)))

    def download(self):
        u, f = self.field(), self.field()
        N.check("wt_elliptic_download", N.lib().wt_elliptic_download(self.h, N.dptr(u), N.dptr(f)))
        return u, f

    def apply(self, level: int) -> None:
        N.check("wt_elliptic_apply", N.lib().wt_elliptic_apply(self.h, level))

    def restrict(self) -> None:
        N.check("wt_elliptic_restrict", N.lib().wt_elliptic_restrict(self.h))

    def prolong(self, fine: int) -> None:
        N.check("wt_elliptic_prolong", N.lib().wt_elliptic_prolong(self.h, fine))

    def l2(self, level: int, which: int = 1) -> float:
        v = C.c_double()
        N.check("wt_elliptic_l2", N.lib().wt_elliptic_l2(self.h, level, which, C.byref(v)))
        return v.value

    def autotune(self, method: str, tol: float = 1e-10, candidates=None, repeats: int = 3, **kw):
        """Fastest V-cycle schedule (down_iter, up_iter, coarse_iter) of `method`
        on the resident problem (wt_elliptic_autotune): (opts, best ms).
        candidates: iterable of (down, up, coarse), or None for the built-in set."""
        base = solver_opts(method, tol, **kw)
        cand, n = None, 0
        if candidates is not None:
            arr = np.ascontiguousarray(np.asarray(list(candidates), dtype=np.int32).reshape(-1, 3))
            n = arr.shape[0]
            cand = arr.ctypes.data_as(C.POINTER(C.c_int))
        best = N.wt_solver_opts()
        ms = C.c_double()
        N.check("wt_elliptic_autotune", N.lib().wt_elliptic_autotune(self.h, C.byref(base), cand, n, int(repeats),
                                                                     C.byref(best), C.byref(ms)))
        return best, ms.value

    # ---- learned preconditioner (network on level_end) ----
    def learned_setup(self, seed: int = 1) -> int:
        """He-initialised network; returns its node count ns."""
        N.check("wt_learned_setup", N.lib().wt_learned_setup(self.h, int(seed)))
        return self.learned_layout()[0]

    def learned_layout(self, full: bool = False):
        ns = C.c_int()
        N.check("wt_learned_layout", N.lib().wt_learned_layout(self.h, C.byref(ns), None, None))
        if not full:
            return ns.value, None, None
        slot = np.zeros(ns.value, np.int32)
        tap = np.zeros((7, ns.value), np.int32)
        N.check("wt_learned_layout", N.lib().wt_learned_layout(
            self.h, C.byref(ns), slot.ctypes.data_as(C.POINTER(C.c_int)), tap.ctypes.data_as(C.POINTER(C.c_int))))
        return ns.value, slot, tap

    def learned_params(self, set_to: np.ndarray | None = None) -> np.ndarray:
        """FP32 master parameters (after setting them to set_to, if given)."""
        out = np.zeros(N.lib().wt_learned_num_params(), np.float32)
        src = None
        if set_to is not None:
            src = np.ascontiguousarray(set_to, dtype=np.float32)
            assert src.size == out.size
            src = src.ctypes.data_as(C.POINTER(C.c_float))
        N.check("wt_learned_params", N.lib().wt_learned_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), src))
        return out

    def learned_infer(self, r: np.ndarray) -> np.ndarray:
        """The preconditioner applied to a compact residual r (ns,)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        N.check("wt_learned_infer", N.lib().wt_learned_infer(self.h, N.dptr(r), N.dptr(z)))
        return z

    def learned_grad(self, r: np.ndarray, e: np.ndarray):
        """(loss, parameter gradient) of the training loss for one pair."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        e = np.ascontiguousarray(e, dtype=np.float64)
        loss = np.zeros(1)
        g = np.zeros(N.lib().wt_learned_num_params(), np.float32)
        N.check("wt_learned_grad", N.lib().wt_learned_grad(self.h, N.dptr(r), N.dptr(e), N.dptr(loss),
                                                           g.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss[0]), g

    def learned_activation(self, slope: float) -> None:
        """Hidden activation slope in (0, 1] (1: identity)."""
        N.check("wt_learned_activation", N.lib().wt_learned_activation(self.h, float(slope)))

    def learned_tensor_cores(self, on: bool) -> None:
        """The 32 -> 32 layer on the tensor cores (default) or the CUDA cores."""
        N.check("wt_learned_tensor_cores", N.lib().wt_learned_tensor_cores(self.h, 1 if on else 0))

    def learned_layer_times(self, reps: int = 20) -> list[float]:
        """Mean device ms of the forward pass's three layers (wt_learned_layer_times)."""
        ms = (C.c_float * 3)()
        N.check("wt_learned_layer_times", N.lib().wt_learned_layer_times(self.h, int(reps), ms))
        return [float(v) for v in ms]

    def learned_train(self, n_rhs: int = 16, cycles: int = 4, epochs: int = 40, lr: float = 2e-3, seed: int = 1,
                      down_iter: int = 2, up_iter: int = 2, coarse_iter: int = 6,
                      batch_rhs: int = 0) -> "N.wt_learn_report":
        """Pairs from the FP64 multigrid, batch_rhs right-hand sides at a time
        (0: all), each batch trained with Adam on the GPU (wt_learned_train)."""
        o = N.wt_learn_opts(n_rhs, cycles, epochs, lr, seed, down_iter, up_iter, coarse_iter, batch_rhs)
        rep = N.wt_learn_report()
        N.check("wt_learned_train", N.lib().wt_learned_train(self.h, C.byref(o), C.byref(rep)))
        return rep

    def solve(self, opts) -> "N.wt_solver_report":
        rep = N.wt_solver_report()
        rc = N.lib().wt_elliptic_solve(self.h, C.byref(opts), C.byref(rep))
        if rc not in (N.WT_OK, N.WT_ERR_NOT_CONVERGED):
            N.check("wt_elliptic_solve", rc)
        rep.status = rc
        return rep
