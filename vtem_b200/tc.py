"""Split-bf16 products on the sm_100a tensor cores (csrc/tc_gemm.cu).

``gemm_split_bf16(A, B)`` returns alpha * A @ B.T for float64/float32 CUDA
matrices, computed as hi*hi + hi*lo + lo*hi bf16 products accumulated in
fp32 by tcgen05.mma (relative error ~1e-5 of the result's scale), from
[hi | lo] operands whose shared-memory tiles serve all three products.
"""
from __future__ import annotations

import torch

from . import autotune
from ._abi import VtbError, call, dptr, stream_ptr

KB = 64


def padded_k(K):
    return -(-K // KB) * KB


def split_bf16x3(X, pattern, scale=1.0, out=None):
    """(rows, K) float64/float32 -> (rows, 3*Kp) bf16 split operand."""
    if X.dim() != 2 or X.stride(1) != 1:
        raise ValueError("expected a row-major 2-D matrix")
    rows, K = X.shape
    Kp = padded_k(K)
    if out is None:
        out = torch.empty((rows, 3 * Kp), dtype=torch.bfloat16, device=X.device)
    call("vtb_split_bf16x3", dptr(X), int(X.dtype == torch.float32), rows, K, X.stride(0), 1, float(scale),
         int(pattern), dptr(out), stream_ptr())
    return out


def split_bf16x2(X, scale=1.0, out=None):
    """(rows, K) float64/float32 -> (rows, 2*Kp) bf16 [hi | lo] operand of
    the three-product mode."""
    if X.dim() != 2 or X.stride(1) != 1:
        raise ValueError("expected a row-major 2-D matrix")
    rows, K = X.shape
    Kp = padded_k(K)
    if out is None:
        out = torch.empty((rows, 2 * Kp), dtype=torch.bfloat16, device=X.device)
    call("vtb_split_bf16x2", dptr(X), int(X.dtype == torch.float32), rows, K, X.stride(0), 1, float(scale), dptr(out),
         stream_ptr())
    return out


def gemm_bf16x3(A2, B2, out, alpha=1.0, accumulate=False, out_layout="row"):
    """out = alpha * (A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T) on the tensor
    cores from [hi | lo] operands (split_bf16x2): the products of gemm_bf16
    on the three-part layout, with two thirds of its operand bytes."""
    M, K2 = A2.shape
    N = B2.shape[0]
    err = torch.zeros(1, dtype=torch.int32, device=A2.device)
    if out_layout == "row":
        cm, cn = out.stride(0), out.stride(1)
    else:
        cm, cn = out.stride(1), out.stride(0)
    autotune.gemm_bf16_tuned(dptr(A2), M, dptr(B2), N, K2 // 2, dptr(out), cm, cn, out.dtype == torch.float64, alpha,
                             bool(accumulate), dptr(err), stream_ptr(), x3=True)
    return out, err


def gemm_bf16(A3, B3, out, alpha=1.0, accumulate=False, out_layout="row"):
    """out = alpha * A3 @ B3.T on the tensor cores (A3, B3 bf16, K-major).
    out_layout "row": out[m, n]; "col": out is (N, M) and receives the
    transpose (out[n, m])."""
    M, K = A3.shape
    N = B3.shape[0]
    err = torch.zeros(1, dtype=torch.int32, device=A3.device)
    if out_layout == "row":
        cm, cn = out.stride(0), out.stride(1)
    else:
        cm, cn = out.stride(1), out.stride(0)
    autotune.gemm_bf16_tuned(dptr(A3), M, dptr(B3), N, K, dptr(out), cm, cn, out.dtype == torch.float64, alpha,
                             bool(accumulate), dptr(err), stream_ptr())
    return out, err


def gemm_split_bf16(A, B, alpha=1.0, out=None, out_dtype=torch.float64, out_layout="row", check=True):
    """alpha * A @ B.T via split-bf16 tensor-core products."""
    M, K = A.shape
    N, K2 = B.shape
    if K != K2:
        raise ValueError("inner dimensions differ")
    A2 = split_bf16x2(A)
    B2 = split_bf16x2(B)
    if out is None:
        shape = (M, N) if out_layout == "row" else (N, M)
        out = torch.empty(shape, dtype=out_dtype, device=A.device)
    out, err = gemm_bf16x3(A2, B2, out, alpha=alpha, out_layout=out_layout)
    if check and int(err.item()) != 0:
        raise VtbError("vtb_tc_gemm_bf16", int(err.item()))
    return out
