"""ctypes binding of ``libvtem_b200.so`` (the C ABI in ``include/vtem_b200.h``).

There is no fallback: if the library is missing, importing a compute function
raises, and every call on a tensor that is not on a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libvtem_b200.so")

VTB_OK = 0
VTB_BAD_ARG = 1
VTB_OVERFLOW = 2
VTB_OOM = 3
VTB_TIMEOUT = 4
VTB_CUDA_ERR = 5
VTB_NOT_CONVERGED = 6
VTB_NO_DATA = 7
VTB_BLOCK_LIMIT = 8

P = ctypes.c_void_p
I = ctypes.c_int
L = ctypes.c_int64
D = ctypes.c_double

# name -> argtypes (restype int)
SIGNATURES = {
    "vtb_version": [],
    "vtb_last_cuda_error": [],
    "vtb_set_wait_limit": [L, P],
    "vtb_rf_gabor": [P, P, P, P, P, P, I, I, I, D, D, D, D, D, P, L, P],
    "vtb_rf_cs": [P, P, P, P, I, I, I, D, D, D, D, D, D, P, L, P],
    "vtb_rf_filter": [P, I, I, L, P, I, L, D, P, L, L, P],
    "vtb_gemm_f64": [I, I, I, P, L, L, P, L, L, P, L, L, D, D, P],
    "vtb_iaf_encode": [P, L, L, I, I, I, D, P, P, P, P, P, P, L, L, L, I, P, P, P, P, P, I, P, D, P, D, P],
    "vtb_spike_pairs": [P, P, P, I, I, I, D, D, D, P, P, P, P, P, P],
    "vtb_dirichlet_coeffs": [P, I, I, I, L, I, I, D, P, P],
    "vtb_dirich_space": [P, I, I, I, I, I, I, I, P, P],
    "vtb_dsw": [P, I, I, P, P, L, P],
    "vtb_compute_q": [P, P, P, I, P, P, P, P, P, P],
    "vtb_compute_G": [P, P, P, I, D, I, P, L, D, I, P, L, P],
    "vtb_solve_eq_sym_workspace": [I, P],
    "vtb_solve_eq_sym": [P, L, P, P, I, D, P, L, P, P],
    "vtb_rnn": [P, L, P, P, P, P, I, D, I, P, I, P],
    "vtb_reconstruct_workspace": [I, I, I, P],
    "vtb_reconstruct": [P, I, I, P, P, P, P, P, I, P, I, I, D, P, P, L, P],
    "vtb_coeff_pack": [P, I, I, P, I, P, P, P],
    "vtb_coeff_temporal_gram": [P, P, P, I, I, P, P, P, P, I, D, P, P, P],
    "vtb_coeff_gram": [P, I, I, P, P, I, P, L, P, P],
    "vtb_herm_solve_workspace": [I, I, P],
    "vtb_herm_solve": [P, L, P, P, I, D, I, I, P, L, P, P, P],
    "vtb_coeff_synthesize": [P, P, I, I, I, I, D, D, D, I, I, I, I, I, P, P, I, P],
    "vtb_coeff_basis": [P, P, I, I, I, I, I, I, I, I, P, I, P],
    "vtb_synth_harmonics": [P, I, I, I, D, D, D, I, P, I, P],
    "vtb_coeff_synth_rank": [P, P, I, I, I, I, I, I, I, I, P, I, D, D, D, I, P, I, P],
    "vtb_coeff_synthesize_noalloc": [P, P, I, I, I, I, D, D, D, I, I, I, I, I, P, I, P],
    "vtb_split_bf16x3": [P, I, I, I, L, L, D, I, P, P],
    "vtb_tc_gemm_bf16": [P, I, P, I, I, P, L, L, I, D, I, P, P],
    "vtb_tc_gemm_bf16_bn": [P, I, P, I, I, P, L, L, I, D, I, P, I, P],
    "vtb_tc_gemm_bf16x3_bn": [P, I, P, I, I, P, L, L, I, D, I, P, I, P],
    "vtb_split_bf16x2": [P, I, I, I, L, L, D, P, P],
    "vtb_coeff_lhs_sym": [P, I, I, P, P, I, P, P],
    "vtb_coeff_wn_sym": [P, I, I, P, P],
    "vtb_coeff_rhs": [P, I, I, P, I, P, P],
    "vtb_coeff_residual": [P, P, P, I, I, P, P, P, P, I, D, P, I, P, P, P, P],
    "vtb_herm_potrs": [P, L, P, I, P, L, P],
    "vtb_zadd": [P, P, I, P],
    "vtb_herm_chol_batched": [P, L, P, I, I, D, P, P, P],
    "vtb_coeff_from_spike_weights": [P, P, P, I, I, P, I, D, P, I, P, P, P],
    "vtb_herm_pinv_batched_workspace": [I, I, P],
    "vtb_herm_pinv_batched": [P, P, P, I, I, D, P, L, P, P, P],
    "vtb_coeff_real_scatter": [P, L, I, I, P, L, I, P],
    "vtb_coeff_realify": [P, L, I, P, L, I, P],
    "vtb_coeff_realify_vec": [P, I, I, P, P],
    "vtb_coeff_unrealify_vec": [P, I, I, P, I, P],
    "vtb_sym_workspace": [I, I, P],
    "vtb_sym_factor": [P, L, I, I, D, P, L, P, P, P],
    "vtb_sym_potrs": [P, L, P, I, I, P, L, P],
    "vtb_sym_dinv": [P, L, I, P, P],
    "vtb_sym_potrs_flags_bytes": [I],  # restype int64, set in lib()
    "vtb_sym_potrs_flags": [P, L, P, I, P, P, L, P, P],
    "vtb_norm_ratio": [P, P, I, P, P],
    "vtb_daxpy1": [P, P, I, P],
    "vtb_sym_pinv": [P, L, P, P, I, D, P, L, P, P, P],
    "vtb_sym_factor_batched": [P, L, I, I, D, P, P, P, P, P],
    "vtb_sym_potrs_batched": [P, I, I, P],
    "vtb_sym_pinv_batched_workspace": [I, I, P],
    "vtb_sym_pinv_batched": [P, P, P, I, I, D, P, L, P, P, P],
    "vtb_rnn_coeff": [P, L, P, P, P, I, D, I, P, P],
    "vtb_tc_group_bytes": [I],  # restype int64, set in lib()
    "vtb_tc_group_build": [P, I, P, P, P, P, P, P, P, P, I, P],
    "vtb_tc_gemm_grouped": [P, I, I, I, P],
    "vtb_tc_group_build_x3": [P, I, P, P, P, P, P, P, P, P, I, P],
    "vtb_tc_gemm_grouped_x3": [P, I, I, I, P],
    "vtb_sym_dinv_floats": [I],  # restype int64, set in lib()
    "vtb_chol_dinv_floats": [I],  # restype int64, set in lib()
    "vtb_chol_work_bytes": [I],  # restype int64, set in lib()
    "vtb_chol_factor": [P, L, I, P, P, L, P, P, D, P],
    "vtb_chol_solve": [P, L, P, I, P, P],
    "vtb_chol_solve_cluster": [],
    "vtb_chol_inverse_floats": [I],  # restype int64, set in lib()
    "vtb_chol_factor_inverse": [P, L, I, P, P, P, L, P, P, D, P],
    "vtb_chol_solve_inverse_bytes": [I],  # restype int64, set in lib()
    "vtb_chol_solve_inverse": [P, I, P, P, L, P],
}

_lib = None


class VtbError(RuntimeError):
    def __init__(self, fn, status):
        self.status = status
        msg = "%s failed: %s (status %d)" % (fn, status_string(status), status)
        if status == VTB_CUDA_ERR and _lib is not None:
            msg += ", cudaError %d" % _lib.vtb_last_cuda_error()
        super().__init__(msg)


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "vtem_b200 CUDA library not built (%s); run `python -m vtem_b200.build`" % LIB_PATH)
        l = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(l, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        for name in ("vtb_sym_dinv_floats", "vtb_tc_group_bytes", "vtb_sym_potrs_flags_bytes", "vtb_chol_dinv_floats",
                     "vtb_chol_work_bytes", "vtb_chol_inverse_floats", "vtb_chol_solve_inverse_bytes"):
            getattr(l, name).argtypes = [ctypes.c_int]
            getattr(l, name).restype = ctypes.c_int64
        l.vtb_status_string.argtypes = [ctypes.c_int]
        l.vtb_status_string.restype = ctypes.c_char_p
        _lib = l
    return _lib


def status_string(status: int) -> str:
    return lib().vtb_status_string(int(status)).decode()


def call(name, *args):
    """Call ``name`` and raise :class:`VtbError` on a nonzero status."""
    st = getattr(lib(), name)(*args)
    if st != VTB_OK:
        raise VtbError(name, st)
    return st


class wait_limit(object):
    """Context manager: inside it, every bounded device wait of the kernels
    launched (by any thread) gives up after ``polls`` polls and reports
    VTB_TIMEOUT (vtb_set_wait_limit); the previous limit is restored on exit."""

    def __init__(self, polls):
        self.polls = int(polls)

    def __enter__(self):
        import numpy as np
        prev = np.zeros(1, np.int64)
        call("vtb_set_wait_limit", self.polls, prev.ctypes.data)
        self.prev = int(prev[0])
        return self

    def __exit__(self, *exc):
        call("vtb_set_wait_limit", self.prev, None)
        return False


def stream_ptr(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def dptr(t: torch.Tensor | None, dtype=None):
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("vtem_b200 kernels take CUDA tensors (got a %s tensor)" % t.device)
    if dtype is not None and t.dtype != dtype:
        raise TypeError("expected %s, got %s" % (dtype, t.dtype))
    return t.data_ptr()
