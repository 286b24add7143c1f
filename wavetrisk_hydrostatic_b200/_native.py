"""ctypes bindings of libwtgpu.so (the C-ABI declared in include/wavetrisk_gpu.h).

The shared library is built in-tree by ``wavetrisk_hydrostatic_b200.build``.
Loading fails loudly when it is missing: there is no Python or CPU fallback
for any device entry point.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwtgpu.so")

WT_OK = 0
WT_ERR_ARG = -1
WT_ERR_CUDA = -2
WT_ERR_ALLOC = -3
WT_ERR_NONFINITE = -4
WT_ERR_NOT_CONVERGED = -5
WT_ERR_TIMEOUT = -6
WT_ERR_STATE = -7
WT_ERR_NO_DEVICE = -8

STATUS_NAMES = {
    WT_OK: "WT_OK", WT_ERR_ARG: "WT_ERR_ARG", WT_ERR_CUDA: "WT_ERR_CUDA", WT_ERR_ALLOC: "WT_ERR_ALLOC",
    WT_ERR_NONFINITE: "WT_ERR_NONFINITE", WT_ERR_NOT_CONVERGED: "WT_ERR_NOT_CONVERGED",
    WT_ERR_TIMEOUT: "WT_ERR_TIMEOUT", WT_ERR_STATE: "WT_ERR_STATE", WT_ERR_NO_DEVICE: "WT_ERR_NO_DEVICE",
}


class WtError(RuntimeError):
    def __init__(self, where: str, code: int):
        super().__init__(f"{where} failed: {STATUS_NAMES.get(code, code)}")
        self.code = code


class wt_level_dims(C.Structure):
    _fields_ = [("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64),
                ("n_halo_node", C.c_int64), ("n_halo_edge", C.c_int64)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)


class wt_level_desc(C.Structure):
    _fields_ = [("level", C.c_int), ("n", C.c_int), ("P", C.c_int), ("NN", C.c_int64),
                ("len", _dp), ("pedlen", _dp), ("part", _dp), ("hex_inv", _dp), ("triarea", _dp),
                ("coriolis", _dp), ("overl_a", _dp), ("topo", _dp),
                ("halo_node", _ip), ("n_halo_node", C.c_int64),
                ("halo_edge", _ip), ("n_halo_edge", C.c_int64), ("iu_wgt", _dp),
                ("overl_split", _dp), ("rf_wgt", _dp)]


class wt_grid_desc(C.Structure):
    _fields_ = [("level_start", C.c_int), ("level_end", C.c_int), ("nz", C.c_int),
                ("grav", C.c_double), ("ref_density", C.c_double), ("p_top", C.c_double),
                ("levels", C.POINTER(wt_level_desc))]


class wt_solver_opts(C.Structure):
    _fields_ = [("method", C.c_int), ("coarse_iter", C.c_int), ("max_vcycle", C.c_int), ("pre_iter", C.c_int),
                ("down_iter", C.c_int), ("up_iter", C.c_int), ("post_iter", C.c_int), ("max_srj_iter", C.c_int),
                ("fine_tol", C.c_double), ("coarse_tol", C.c_double), ("ir_tol", C.c_double), ("ir_max", C.c_int)]


class wt_solver_report(C.Structure):
    _fields_ = [("nrm_res_init", C.c_double * 16), ("nrm_res_final", C.c_double * 16), ("iterations", C.c_int * 16),
                ("outer_iterations", C.c_int), ("true_rel_residual", C.c_double), ("ms", C.c_double),
                ("precond_fallback", C.c_int), ("restarts", C.c_int)]


class wt_learn_opts(C.Structure):
    _fields_ = [("n_rhs", C.c_int), ("cycles", C.c_int), ("epochs", C.c_int), ("lr", C.c_float),
                ("seed", C.c_ulonglong), ("down_iter", C.c_int), ("up_iter", C.c_int), ("coarse_iter", C.c_int),
                ("batch_rhs", C.c_int)]


class wt_learn_report(C.Structure):
    _fields_ = [("pairs", C.c_int), ("steps", C.c_int), ("loss_first_epoch", C.c_double),
                ("loss_last_epoch", C.c_double), ("ms_generate", C.c_double), ("ms_train", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """Load libwtgpu.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; run wavetrisk_hydrostatic_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.wt_grid_build.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(vp)]
        L.wt_grid_build.restype = C.c_int
        L.wt_grid_free.argtypes = [vp]
        L.wt_grid_free.restype = None
        L.wt_grid_level_dims.argtypes = [vp, C.c_int, C.POINTER(wt_level_dims)]
        L.wt_grid_level_dims.restype = C.c_int
        L.wt_grid_copy.argtypes = [vp, C.c_int, C.c_char_p, vp]
        L.wt_grid_copy.restype = C.c_int
        for name, args in _DEVICE_SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.wt_stream.argtypes = [vp]
        L.wt_stream.restype = vp
        _lib = L
    return _lib


_vp = C.c_void_p
_DEVICE_SIGS = {
    "wt_create": [C.POINTER(wt_grid_desc), C.POINTER(_vp)],
    "wt_destroy": [_vp],
    "wt_status": [_vp],
    "wt_clear_status": [_vp],
    "wt_synchronize": [_vp],
    "wt_upload_state": [_vp, _dp, _dp, _dp, _dp, _dp],
    "wt_download_state": [_vp, _dp, _dp, _dp],
    "wt_trend": [_vp],
    "wt_download_trend": [_vp, _dp, _dp, _dp],
    "wt_rk4_step": [_vp, C.c_double, C.c_int],
    "wt_rk4_step_host": [_vp, C.c_double, C.c_int, _dp, _dp, _dp],
    "wt_profile_rk4": [_vp, C.c_double, C.c_int, _dp, C.POINTER(C.c_int)],
    "wt_elliptic_setup": [_vp, C.c_double, C.c_double, C.c_double, C.c_int],
    "wt_elliptic_upload": [_vp, _dp, _dp],
    "wt_elliptic_download": [_vp, _dp, _dp],
    "wt_elliptic_apply": [_vp, C.c_int],
    "wt_elliptic_restrict": [_vp],
    "wt_elliptic_prolong": [_vp, C.c_int],
    "wt_elliptic_l2": [_vp, C.c_int, C.c_int, _dp],
    "wt_elliptic_solve": [_vp, C.POINTER(wt_solver_opts), C.POINTER(wt_solver_report)],
    "wt_free_surface_update": [_vp, C.c_double, C.c_double, C.c_double, C.POINTER(wt_solver_opts),
                               C.POINTER(wt_solver_report)],
    "wt_rk4_split": [_vp, C.c_double, C.c_double, C.c_double, C.POINTER(wt_solver_opts),
                     C.POINTER(wt_solver_report)],
    "wt_free_surface_download": [_vp, C.c_int, _dp],
    "wt_elliptic_autotune": [_vp, C.POINTER(wt_solver_opts), C.POINTER(C.c_int), C.c_int, C.c_int,
                             C.POINTER(wt_solver_opts), _dp],
    "wt_learned_setup": [_vp, C.c_ulonglong],
    "wt_learned_num_params": [],
    "wt_learned_params": [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float)],
    "wt_learned_layout": [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "wt_learned_infer": [_vp, _dp, _dp],
    "wt_learned_grad": [_vp, _dp, _dp, _dp, C.POINTER(C.c_float)],
    "wt_learned_train": [_vp, C.POINTER(wt_learn_opts), C.POINTER(wt_learn_report)],
    "wt_learned_activation": [_vp, C.c_float],
    "wt_remap_vertical": [_vp, C.c_int, _dp, _dp],
    "wt_min_mass": [_vp, _dp, _dp],
    "wt_free_surface_adapt": [_vp],
    "wt_learned_tensor_cores": [_vp, C.c_int],
    "wt_learned_layer_times": [_vp, C.c_int, C.POINTER(C.c_float)],
    "wt_wavelet_setup": [_vp],
    "wt_upload_field": [_vp, C.c_int, C.c_int, _vp],
    "wt_download_field": [_vp, C.c_int, C.c_int, _vp],
    "wt_rk4_split_explicit": [_vp, C.c_double, C.c_double],
    "wt_barotropic_correction_multi": [_vp],
    "wt_upload_fields": [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(_vp)],
    "wt_download_fields": [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(_vp)],
    "wt_forward_wt": [_vp],
    "wt_inverse_wt": [_vp],
    "wt_inverse_tree": [_vp],
    "wt_mask_tol_vars": [_vp, _dp, C.c_int],
    "wt_compress": [_vp],
    "wt_mask_build": [_vp, _dp, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "wt_tree_init": [_vp, C.c_int],
    "wt_tree_level_end": [_vp, C.POINTER(C.c_int)],
    "wt_tree_download": [_vp, C.c_int, C.c_void_p, C.c_void_p],
    "wt_grid_sync": [_vp, C.c_void_p, C.c_int],
    "wt_adapt": [_vp, _dp, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "wt_count_active": [_vp, _dp, C.POINTER(C.c_longlong)],
    "wt_tree_stats": [_vp, C.c_int, C.POINTER(C.c_longlong)],
    "wt_mask_adj_child": [_vp, C.c_int],
    "wt_download_tree_state": [_vp, _dp, _dp, _dp, C.c_longlong, C.POINTER(C.c_longlong)],
    "wt_upload_tree_state": [_vp, _dp, _dp, _dp, C.c_longlong],
    "wt_wt_after_step": [_vp],
    "wt_step1_vort": [_vp, C.c_int, _dp],
    "wt_barotropic_upload_level": [_vp, C.c_int, _dp, _dp],
    "wt_rhs_elliptic_multi": [_vp, C.c_double, C.c_double],
    "wt_u_update_multi": [_vp, C.c_double, C.c_double],
    "wt_barotropic_download_level": [_vp, C.c_int, _dp, _dp, _dp],
    "wt_trend_multi": [_vp],
    "wt_rk4_multi": [_vp, C.c_double, C.c_int],
    "wt_adaptive_step": [_vp, C.c_double, _dp, C.c_int, C.c_int, C.c_int],
    "wt_profile_rk4_multi": [_vp, C.c_double, C.c_int, _dp, C.POINTER(C.c_int)],
    "wt_lnorm": [_vp, C.c_int, _dp],
    "wt_tune": [_vp, C.c_int, C.c_int],
    "wt_download_trend_level": [_vp, C.c_int, _dp, _dp, _dp],
    "wt_restrict_scalar": [_vp, C.c_int],
    "wt_restrict_flux": [_vp, C.c_int],
    "wt_restrict_u_source": [_vp, C.c_int],
    "wt_barotropic_upload": [_vp, _dp, _dp],
    "wt_rhs_elliptic": [_vp, C.c_double, C.c_double],
    "wt_u_update": [_vp, C.c_double, C.c_double],
    "wt_barotropic_download": [_vp, _dp, _dp, _dp],
    "wt_step1_flux": [_vp, C.c_int, C.c_int, _dp, _dp],
}


def check(where: str, code: int) -> None:
    if code != WT_OK:
        raise WtError(where, code)


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array (or NULL for None)."""
    if a is None:
        return C.cast(None, _dp)
    assert a.dtype.kind == "f" and a.dtype.itemsize == 8 and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return C.cast(None, _ip)
    assert a.dtype.kind == "i" and a.dtype.itemsize == 8 and a.flags["C_CONTIGUOUS"], "need contiguous int64"
    return a.ctypes.data_as(_ip)
