"""RNN (gradient-flow) decoder (reference: ``vtem/neural_network.py``)."""
from __future__ import annotations

import numpy as np
import torch

from ._abi import call, dptr, stream_ptr

F64 = torch.float64


def rnn3(G, q, dt=1e-6, alpha=5000, steps=4000, XOUTPUTSTEPS=None, return_trace=False):
    """Run c <- c + dt*alpha*(q - G c) from c = 0, steps+1 times
    (neural_network.py:15-99).  G must be real and positive semidefinite.
    The squared residual norm is recorded every steps/min(20, steps) steps
    (the reference prints it); ``return_trace`` returns it."""
    if G.dtype != q.dtype:
        raise TypeError("matrix multiplication must have same dtype")
    if torch.is_complex(G):
        raise TypeError("RNN currently only solves real types")
    if G.dim() != 2 or q.dim() != 2:
        raise TypeError("G, q must both be matrices")
    if G.dtype != F64:
        raise TypeError("the RNN decoder runs in float64")
    n = G.shape[0]
    every = max(1, steps // max(1, min(20, steps)))
    ntrace = steps // every + 1
    c = torch.empty((n,), dtype=F64, device=G.device)
    y = torch.empty((n,), dtype=F64, device=G.device)
    tmp = torch.empty((n,), dtype=F64, device=G.device)
    trace = torch.zeros((ntrace,), dtype=F64, device=G.device)
    Gc = G if G.is_contiguous() else G.contiguous()
    call("vtb_rnn", dptr(Gc), n, dptr(q.reshape(-1).contiguous()), dptr(c), dptr(y), dptr(tmp), n,
         float(dt) * float(alpha), int(steps), dptr(trace), every, stream_ptr())
    c = c.reshape(q.shape)
    if return_trace:
        return c, torch.sqrt(trace)
    return c
