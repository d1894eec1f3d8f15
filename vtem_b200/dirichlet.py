"""Dirichlet-kernel decoder of IAF-encoded video (plain float64 path).

Same class and methods as the reference's ``vtem/dirichlet.py``
(``dirichlet`` :15-198).  File arguments (``Dswfilename``,
``dirichfilename``) accept either a path written by
:func:`vtem_b200.simpleio.write_memory_to_file` or the array itself.
"""
from __future__ import annotations

import numpy as np
import torch

from ._abi import call, dptr, stream_ptr
from . import simpleio

F64 = torch.float64


def _dev(a, dtype=F64):
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _load(x):
    if isinstance(x, str):
        return simpleio.read_file(x)
    return x


def sort_by_neuron(tk1, tk2, neuron_ind):
    """Stable sort of a spike-interval list by neuron index (the order the
    reference's reader produces, spike_store.py:345-348).  Returns the
    permutation (or None when already sorted) and the sorted arrays."""
    ind = _dev(neuron_ind, torch.int32)
    if ind.numel() < 2 or bool((ind[1:] >= ind[:-1]).all()):
        return None, _dev(tk1), _dev(tk2), ind
    perm = torch.sort(ind, stable=True).indices
    return perm, _dev(tk1)[perm].contiguous(), _dev(tk2)[perm].contiguous(), ind[perm].contiguous()


class dirichlet(object):
    def __init__(self, decode_neuron, tk1, tk2, neuron_ind, kappa, delta, bias, norm, Wt, Mt, dtype=np.float64):
        """Decoder state for spike intervals (tk1[j], tk2[j]) of neuron
        neuron_ind[j] (dirichlet.py:16-53)."""
        self.size = int(np.asarray(tk1).size if not isinstance(tk1, torch.Tensor) else tk1.numel())
        if self.size == 0:
            raise ValueError("no spikes to decode")
        self.Wt = float(Wt)
        self.Mt = int(Mt)
        self.dtype = np.dtype(dtype)
        if self.dtype != np.float64:
            raise TypeError("the plain decoder computes in float64")
        self.decode_neuron = int(decode_neuron)
        self.d_tk1 = _dev(tk1)
        self.d_tk2 = _dev(tk2)
        self.d_neuron_ind = _dev(neuron_ind, torch.int32)
        self.d_kappa = _dev(kappa)
        self.d_delta = _dev(delta)
        self.d_bias = _dev(bias)
        self.d_norm = _dev(norm)

    def compute_q(self):
        """q (size, 1) (dirichlet.py:55-60)."""
        self.d_q = torch.empty((self.size, 1), dtype=F64, device="cuda")
        call("vtb_compute_q", dptr(self.d_tk1), dptr(self.d_tk2), dptr(self.d_neuron_ind), self.size,
             dptr(self.d_kappa), dptr(self.d_delta), dptr(self.d_bias), dptr(self.d_norm), dptr(self.d_q),
             stream_ptr())

    def compute_G(self, Dswfilename, lamb=0.0, lower_only=False):
        """Analytic Gram from the RF cross-weights (dirichlet.py:62-85).
        ``lower_only`` (extension) fills only the lower triangle, which is
        all the pseudoinverse solve reads."""
        Dsw = _dev(_load(Dswfilename))
        self.d_G = torch.empty((self.size, self.size), dtype=F64, device="cuda")
        call("vtb_compute_G", dptr(self.d_tk1), dptr(self.d_tk2), dptr(self.d_neuron_ind), self.size, self.Wt,
             self.Mt, dptr(Dsw), Dsw.shape[1], float(lamb), int(bool(lower_only)), dptr(self.d_G), self.size,
             stream_ptr())

    def compute_Gb(self, Dsfilename, lamb=0.0, lower_only=False):
        """Gram from the Dirichlet coefficients (dirichlet.py:87-126): the
        cross-weights Re(Ds Ds^H) with this decoder's norm, then compute_G."""
        Ds = _load(Dsfilename)
        Ds = _dev(Ds, torch.complex128) if not isinstance(Ds, torch.Tensor) else Ds.to("cuda", torch.complex128)
        N = Ds.shape[0]
        Ks = Ds[0].numel()
        W = torch.empty((N, N), dtype=F64, device="cuda")
        call("vtb_dsw", dptr(Ds.contiguous()), N, Ks, dptr(self.d_norm), dptr(W), N, stream_ptr())
        self.compute_G(W, lamb, lower_only)

    def store_Gq(self):
        """Move G, q to host memory (dirichlet.py:129-136)."""
        self.G = self.d_G.cpu().numpy()
        self.q = self.d_q.cpu().numpy()
        del self.d_G
        del self.d_q

    def restore_Gq(self):
        """dirichlet.py:151-155."""
        self.d_G = _dev(self.G)
        self.d_q = _dev(self.q)

    def store_others(self):
        """dirichlet.py:138-149."""
        self.tk1 = self.d_tk1.cpu().numpy()
        self.tk2 = self.d_tk2.cpu().numpy()
        self.neuron_ind = self.d_neuron_ind.cpu().numpy()
        self.norm = self.d_norm.cpu().numpy()
        del self.d_tk1, self.d_tk2, self.d_neuron_ind, self.d_norm

    def restore_others(self):
        """dirichlet.py:157-162."""
        self.d_tk1 = _dev(self.tk1)
        self.d_tk2 = _dev(self.tk2)
        self.d_neuron_ind = _dev(self.neuron_ind, torch.int32)
        self.d_norm = _dev(self.norm)

    def reconstruct(self, dirichfilename, time_frame, dt):
        """Video (len(t), Py, Px) float64 on the device from the solution c
        held in ``self.d_q``, at t = arange(time_frame[0], time_frame[1], dt)
        (dirichlet.py:165-189)."""
        t = np.arange(time_frame[0], time_frame[1], dt)
        d_t = _dev(t)
        dirich = _dev(_load(dirichfilename))
        N, Py, Px = dirich.shape
        c = self.d_q.reshape(-1).contiguous()
        perm, tk1, tk2, ind = sort_by_neuron(self.d_tk1, self.d_tk2, self.d_neuron_ind)
        if perm is not None:
            c = c[perm].contiguous()
        nbytes = np.zeros(1, np.int64)
        from . import _abi
        _abi.lib().vtb_reconstruct_workspace(N, len(t), self.Mt, nbytes.ctypes.data)
        work = torch.empty(int(nbytes[0]), dtype=torch.uint8, device="cuda")
        u = torch.empty((len(t), Py, Px), dtype=F64, device="cuda")
        call("vtb_reconstruct", dptr(dirich), N, Py * Px, dptr(tk1), dptr(tk2), dptr(c), dptr(ind),
             dptr(self.d_norm), self.size, dptr(d_t), len(t), self.Mt, self.Wt / self.Mt, dptr(u), dptr(work),
             int(nbytes[0]), stream_ptr())
        return u

    def freeG(self):
        """Drop G (dirichlet.py:191-197)."""
        self.d_G = None
        self.G = None
