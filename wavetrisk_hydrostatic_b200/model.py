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
            arr[q] = N.wt_level_desc(g.level, g.n, g.P, g.NN, *[N.dptr(b) for b in bufs],
                                     N.iptr(hn), len(hn), N.iptr(he), len(he))
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
