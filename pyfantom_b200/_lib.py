"""ctypes binding of libpyfantom_b200.so (the C ABI in include/pyfantom_b200.h).

The library is built in-tree by ``pyfantom_b200._build``.  There is no fallback: if the
shared library cannot be loaded, or no CUDA device is present, every call raises.
Pointers passed to the library come from torch CUDA tensors (``tensor.data_ptr()``); the
stream is torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes
import os

import torch

from . import _build

PF_OK, PF_NOT_CONVERGED, PF_BREAKDOWN, PF_NONFINITE, PF_TIMEOUT = 0, 1, 2, 3, 4
PF_BAD_ARG, PF_CUDA_ERROR, PF_NO_MEMORY, PF_UNSUPPORTED, PF_FACTOR_FAILED = 5, 6, 7, 8, 9

STATUS_NAMES = {0: "PF_OK", 1: "PF_NOT_CONVERGED", 2: "PF_BREAKDOWN", 3: "PF_NONFINITE", 4: "PF_TIMEOUT",
                5: "PF_BAD_ARG", 6: "PF_CUDA_ERROR", 7: "PF_NO_MEMORY", 8: "PF_UNSUPPORTED",
                9: "PF_FACTOR_FAILED"}


class PFError(RuntimeError):
    """A library call returned a failure status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class pf_grid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nel", ctypes.c_int * 3)]


class pf_mg_config(ctypes.Structure):
    _fields_ = [("n_level", ctypes.c_int), ("n_smooth", ctypes.c_int), ("omega", ctypes.c_double),
                ("min_omega", ctypes.c_double), ("omega_boost", ctypes.c_double), ("coarse_beta", ctypes.c_double),
                ("precision", ctypes.c_int), ("check_every", ctypes.c_int), ("coarse_op", ctypes.c_int),
                ("w_mask", ctypes.c_uint), ("omega_fixed", ctypes.c_double)]


class pf_solve_info(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("status", ctypes.c_int), ("residual", ctypes.c_double),
                ("setup_ms", ctypes.c_double), ("solve_ms", ctypes.c_double)]


class pf_simp_params(ctypes.Structure):
    _fields_ = [("penalty", ctypes.c_double), ("void_value", ctypes.c_double), ("E_mul", ctypes.c_double),
                ("beta", ctypes.c_double), ("eta", ctypes.c_double), ("heavyside", ctypes.c_int)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong
_D = ctypes.c_double
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); every exported symbol of include/pyfantom_b200.h
SIGNATURES = {
    "pf_version": (_I, []),
    "pf_launch_count": (ctypes.c_ulonglong, []),
    "pf_mg_set_profiling": (_I, [_P, _I]),
    "pf_mg_profile": (_I, [_P, ctypes.POINTER(_D), ctypes.POINTER(_LL), ctypes.POINTER(_D)]),
    "pf_mg_profile_select": (_I, [_P, _I]),
    "pf_mg_level_matvec": (_I, [_P, _I, _P, _P, _P]),
    "pf_mg_level_info": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "pf_mg_set_deflation": (_I, [_P, _P, _P]),
    "pf_last_error": (ctypes.c_char_p, []),
    "pf_status_string": (ctypes.c_char_p, [_I]),
    "pf_op_create": (_I, [ctypes.POINTER(pf_grid), _P, ctypes.POINTER(_P)]),
    "pf_op_destroy": (_I, [_P]),
    "pf_op_set_variant": (_I, [_P, _I]),
    "pf_pack_mask": (_I, [_P, _P, _P, _P]),
    "pf_csr_nnz": (_LL, [_P]),
    "pf_construct_csr_f64": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "pf_matvec_f64": (_I, [_P, _P, _P, _P, _P, _P]),
    "pf_matvec_f32": (_I, [_P, _P, _P, _P, _P, _P]),
    "pf_matvec_f32_bf16": (_I, [_P, _P, _P, _P, _P, _P]),
    "pf_diagonal_f64": (_I, [_P, _P, _P, _P, _P]),
    "pf_sensitivity_f64": (_I, [_P, _P, _P, _P]),
    "pf_restrict_f64": (_I, [ctypes.POINTER(pf_grid), _P, _P, _P]),
    "pf_prolong_f64": (_I, [ctypes.POINTER(pf_grid), _P, _P, _P]),
    "pf_galerkin_l0_f64": (_I, [_P, _P, _P, _P, _P]),
    "pf_galerkin_l1p_f64": (_I, [ctypes.POINTER(pf_grid), _P, _P, _P]),
    "pf_stencil_matvec_f64": (_I, [ctypes.POINTER(pf_grid), _P, _P, _P, _P]),
    "pf_stencil_size": (_SZ, [ctypes.POINTER(pf_grid)]),
    "pf_mg_create": (_I, [_P, ctypes.POINTER(pf_mg_config), ctypes.POINTER(_P)]),
    "pf_mg_destroy": (_I, [_P]),
    "pf_mg_setup": (_I, [_P, _P, _P, _P]),
    "pf_mg_vcycle": (_I, [_P, _P, _P, _D, _P]),
    "pf_mg_solve": (_I, [_P, _P, _P, _I, _D, _I, ctypes.POINTER(pf_solve_info), _P]),
    "pf_cg_workspace_size": (_SZ, [_P]),
    "pf_cg_solve": (_I, [_P, _P, _P, _P, _P, _I, _D, _I, _P, ctypes.POINTER(pf_solve_info), _P]),
    "pf_filter_create": (_I, [ctypes.POINTER(pf_grid), _I, _P, _P, ctypes.POINTER(_P)]),
    "pf_filter_destroy": (_I, [_P]),
    "pf_filter_normalizer_f64": (_I, [_P, _P, _P]),
    "pf_filter_fwd_f64": (_I, [_P, _P, _P, _P]),
    "pf_filter_adj_f64": (_I, [_P, _P, _P, _P]),
    "pf_penalize_f64": (_I, [_LL, _P, ctypes.POINTER(pf_simp_params), _P, _P, _P]),
    "pf_mul_f64": (_I, [_LL, _P, _P, _P, _P]),
    "pf_adjoint_f64": (_I, [_P, _P, _P, ctypes.POINTER(pf_simp_params), _D, _P, _P]),
    "pf_dot_workspace_size": (_SZ, [_LL]),
    "pf_dot_f64": (_I, [_LL, _P, _P, _P, _P, _P]),
    "pf_oc_workspace_size": (_SZ, [_LL]),
    "pf_oc_update_f64": (_I, [_LL, _P, _P, _P, _D, _D, _P, _P, _P, _P]),
    "pf_oc_update_noalloc_f64": (_I, [_LL, _P, _P, _P, _D, _D, _P, _P, _P]),
    "pf_direct_create": (_I, [_P, ctypes.POINTER(_P)]),
    "pf_direct_destroy": (_I, [_P]),
    "pf_direct_solve_f64": (_I, [_P, _P, _P, _P, _I, _P, _P, _P]),
    "pf_penalize_multi_f64": (_I, [_LL, _I, _P, ctypes.POINTER(pf_simp_params), _P, _P, _P, _P]),
    "pf_oc_multi_workspace_size": (_SZ, [_LL, _I]),
    "pf_oc_update_multi_f64": (_I, [_LL, _I, _P, _P, _P, _P, _D, _P, _P, _P, _P]),
    "pf_pgd_workspace_size": (_SZ, [_LL]),
    "pf_pgd_stats_f64": (_I, [_LL, _P, _P, _P, _P, _P, _P, _P]),
    "pf_pgd_step_f64": (_I, [_LL, _P, _P, _P, _D, _D, _P, _P, _P]),
    "pf_pgd_project_f64": (_I, [_LL, _P, _P, _D, _D, _D, _D, _P, _P, _P, _P]),
    "pf_pgd_multi_workspace_size": (_SZ, [_LL, _I]),
    "pf_pgd_project_multi_f64": (_I, [_LL, _I, _P, _P, _P, _D, _D, _D, _P, _P, _P, _P]),
    "pf_cnn_conv3d_fwd_f32": (_I, [_P, _I, _I, _I, _I, _I, _P, _P, _I, _I, _I, _P, _P]),
    "pf_cnn_conv3d_bwd_data_f32": (_I, [_P, _I, _I, _I, _I, _I, _P, _I, _I, _I, _P, _P]),
    "pf_cnn_conv3d_fwd_tc": (_I, [_P, _I, _I, _I, _I, _I, _P, _P, _I, _I, _I, _P, _P, _P]),
    "pf_cnn_conv3d_bwd_data_tc": (_I, [_P, _I, _I, _I, _I, _I, _P, _I, _I, _I, _P, _P, _P]),
    "pf_cnn_conv3d_bwd_weight_tc_workspace": (_SZ, [_I, _I, _I, _I, _I, _I, _I]),
    "pf_cnn_conv3d_bwd_weight_tc": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "pf_cnn_conv3d_bwd_weight_workspace": (_SZ, [_I, _I]),
    "pf_cnn_conv3d_bwd_weight_f32": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P]),
    "pf_cnn_relu_bwd_f32": (_I, [_LL, _P, _P, _P]),
    "pf_cnn_upsample2_f32": (_I, [_I, _I, _I, _I, _P, _P, _I, _P]),
    "pf_cnn_copy_channels_f32": (_I, [_I, _I, _LL, _P, _I, _I, _I, _I, _P, _P]),
    "pf_cnn_channel_sum_f32": (_I, [_I, _I, _LL, _P, _I, _I, ctypes.c_float, _P, _P]),
    "pf_cnn_channel_bcast_f32": (_I, [_I, _I, _LL, _P, ctypes.c_float, _I, _I, _I, _P, _P]),
    "pf_cnn_cell2node_f32": (_I, [_I, _I, _I, _I, _P, _P, _I, _P]),
    "pf_cnn_mse_workspace": (_SZ, [_LL]),
    "pf_cnn_mse_f32": (_I, [_LL, _P, _P, _P, _P, _P, _P]),
    "pf_cnn_adam_f32": (_I, [_LL, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                             _I, _P]),
    "pf_cnn_features_f32": (_I, [ctypes.POINTER(pf_grid), _I, _P, _P, _P, _P, _P, _P]),
    "pf_cnn_guess_f64": (_I, [ctypes.POINTER(pf_grid), _I, _P, _P, _P, _P]),
    "pf_cnn_energy_scale_workspace": (_SZ, []),
    "pf_cnn_energy_scale_f64": (_I, [_LL, _P, _P, _P, _P, _P]),
    "pf_cnn_guess_select_workspace": (_SZ, []),
    "pf_cnn_guess_select_f64": (_I, [_LL, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pf_cnn_energy_loss_workspace": (_SZ, []),
    "pf_cnn_energy_loss_f64": (_I, [_LL, _P, _P, _P, _D, _P, _P, _P, _P]),
}

_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load (building first if needed and possible) and return the ctypes library."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_missing and _build.needs_build():
        try:
            _build.build()
        except Exception as exc:  # a stale but present library is still usable
            if not os.path.exists(path):
                raise RuntimeError(f"libpyfantom_b200.so is missing and could not be built: {exc}") from exc
    if not os.path.exists(path):
        raise RuntimeError(f"libpyfantom_b200.so not found at {path}; run `python -m pyfantom_b200._build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != PF_OK:
        msg = load().pf_last_error()
        raise PFError(status, msg.decode() if msg else "")
    return status


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("pyfantom_b200 needs a CUDA device (sm_100a); none is available")


def stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t: torch.Tensor | None, dtype: torch.dtype | None = None) -> ctypes.c_void_p:
    """Device pointer of a contiguous CUDA tensor (None -> NULL)."""
    if t is None:
        return ctypes.c_void_p(0)
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"expected dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def make_grid(nel) -> pf_grid:
    g = pf_grid()
    g.dim = len(nel)
    for a in range(3):
        g.nel[a] = int(nel[a]) if a < len(nel) else 0
    return g
