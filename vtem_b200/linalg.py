"""Linear algebra of the decode path (reference: ``vtem/utils/linalg.py``)."""
from __future__ import annotations

import numpy as np
import torch

from . import _abi
from ._abi import call, dptr, stream_ptr

F64 = torch.float64


def solve_eq_sym(G, q, rcond=1e-8, return_kept=False):
    """Solve G c = q for symmetric G by pseudoinversion, dropping singular
    values at or below ``rcond * s_0`` (linalg.py:591-631).  As in the
    reference, G is destroyed (it holds the eigenvectors afterwards).  Only
    G's lower triangle is read."""
    if not isinstance(G, torch.Tensor) or not isinstance(q, torch.Tensor):
        raise TypeError("G, q must be CUDA tensors")
    if G.dtype != q.dtype:
        raise TypeError("G,q must be of the same dtype")
    if G.dtype != F64:
        raise TypeError("the plain solve runs in float64")
    if G.dim() != 2 or G.shape[0] != G.shape[1]:
        raise ValueError("G must be square matrix")
    n = G.shape[0]
    if q.numel() != n:
        raise ValueError("number of columns of G must be the same of size of q")
    if not G.is_contiguous():
        raise ValueError("G must be contiguous")
    nbytes = np.zeros(1, np.int64)
    call("vtb_solve_eq_sym_workspace", n, nbytes.ctypes.data)
    work = torch.empty(int(nbytes[0]), dtype=torch.uint8, device=G.device)
    qv = q.reshape(-1).contiguous()
    c = torch.empty_like(qv)
    kept = torch.zeros(1, dtype=torch.int32, device=G.device)
    call("vtb_solve_eq_sym", dptr(G), n, dptr(qv), dptr(c), n, float(rcond), dptr(work), int(nbytes[0]),
         dptr(kept), stream_ptr())
    c = c.reshape(q.shape)
    if return_kept:
        return c, int(kept.item())
    return c


def norm(A):
    """2-norm of a vector (linalg.py:341-364)."""
    return float(torch.linalg.vector_norm(A.reshape(-1)).item())
