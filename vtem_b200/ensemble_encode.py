"""Population encoding with ideal IAF neurons on the B200.

Same classes and methods as the reference's ``vtem/ensemble_encode.py``
(``IAF_encode`` :21-172, ``IAF_encode_rt`` :175-333).  ``encode`` keeps the
reference's contract (inputs (samples, neurons), returns a list of
per-neuron spike-time arrays and the int32 counts, raises ValueError when a
neuron overflows its ``ceil(samples/avg_rate)`` slots).  ``encode_blocks``
(extension) runs VTEM_IAF's whole block loop in one launch and keeps the
spikes on the device.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from ._abi import VTB_BLOCK_LIMIT, VTB_OVERFLOW, VtbError, call, dptr, stream_ptr

F64 = torch.float64


def _dev(a, dtype=F64):
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


# First-try spike buffer of encode_blocks: one slot per this many samples
# (plus 64) per neuron, i.e. up to 625 spikes/s at dt = 1e-4.
SMALL_CAP_STRIDE = 16


@dataclass
class DeviceSpikes:
    """Spikes of one encode launch, on the device.

    ``time[n, j]`` is the block-relative spike time (the reference stores
    times relative to their refresh interval, spike_store.py:37-38),
    ``step[n, j]`` the global sample index of the interval holding the
    crossing, ``count[n]`` the number of valid entries of row n.
    """
    time: torch.Tensor
    step: torch.Tensor
    count: torch.Tensor
    block_frames: int
    dt: float
    near_threshold: int = 0

    @property
    def refresh_interval(self):
        return (self.block_frames - 1) * self.dt

    def to_host_lists(self):
        cnt = self.count.cpu().numpy()
        t = self.time.cpu().numpy()
        s = self.step.cpu().numpy()
        return [t[i, :cnt[i]].copy() for i in range(len(cnt))], [s[i, :cnt[i]].copy() for i in range(len(cnt))], cnt


class pop_encode(object):
    """Population encoding (ensemble_encode.py:10-15)."""

    def __init__(self, num_neurons, dt, dtype=np.float64):
        self.num_neurons = int(num_neurons)
        self.dtype = np.dtype(dtype)
        if self.dtype != np.float64:
            raise TypeError("the IAF encoder computes in float64 only")
        self.dt = float(self.dtype.type(dt))


class IAF_encode(pop_encode):
    """IAF neurons with deterministic thresholds (ensemble_encode.py:21-172)."""

    random_thresholds = False

    def set_time_count(self):
        """time_count = 0 (ensemble_encode.py:42-44)."""
        self.h_time_count = np.zeros(self.num_neurons, np.float64)

    def set_parameters(self):
        """Defaults kappa = 1, delta = 0.03, bias = 0.8 (ensemble_encode.py:46-59)."""
        self.h_kappa = np.zeros(self.num_neurons) + 1.0
        self.h_delta = np.zeros(self.num_neurons) + 0.03
        self.h_bias = np.zeros(self.num_neurons) + 0.8
        self.h_sigma = np.zeros(self.num_neurons)

    def set_initial_value(self):
        """v0 ~ U(0, 1) * delta (ensemble_encode.py:61-65; unseeded, as there)."""
        self.h_v0 = np.random.uniform(0, 1, self.num_neurons).astype(np.float64) * self.h_delta

    def load_parameters(self, h_kappa=None, h_bias=None, h_delta=None, h_sigma=None, h_time_count=None,
                        h_v0=None):
        """Load encoding parameters to the GPU (ensemble_encode.py:67-103)."""
        if h_kappa is None:
            self.set_parameters()
        else:
            self.h_kappa = np.asarray(h_kappa, np.float64)
            self.h_delta = np.asarray(h_delta, np.float64)
            self.h_bias = np.asarray(h_bias, np.float64)
            self.h_sigma = np.zeros(self.h_kappa.shape)
        if h_time_count is None:
            self.set_time_count()
        else:
            self.h_time_count = np.asarray(h_time_count, np.float64).reshape(-1)
        if h_v0 is None:
            self.set_initial_value()
        else:
            self.h_v0 = np.asarray(h_v0, np.float64)
        self.d_kappa = _dev(self.h_kappa)
        self.d_delta = _dev(self.h_delta)
        self.d_bias = _dev(self.h_bias)
        self.d_v0 = _dev(self.h_v0)
        self.d_time_count = _dev(self.h_time_count)

    def reset_timer(self):
        """time_count = 0 on the device (ensemble_encode.py:170-172)."""
        self.d_time_count.zero_()

    # ------------------------------------------------------------------
    def _launch(self, x, ts, ns, N, F, block_frames, cap, startbias, randn=None, block_cap=0,
                near_eps=1e-12, block_rate=0.0):
        sl = slice(startbias, startbias + N)
        st = torch.empty((N, cap), dtype=F64, device=x.device)
        ss = torch.empty((N, cap), dtype=torch.int32, device=x.device)
        cnt = torch.empty(N, dtype=torch.int32, device=x.device)
        # one buffer for the near-threshold count (int64) and the status word
        # (int32 in the low half of the second word): one read returns both
        flags = torch.zeros(2, dtype=torch.int64, device=x.device)
        near = flags[0:1]
        status = flags[1:2].view(torch.int32)[0:1]
        self._flags = flags
        if randn is not None:
            rb, rs, rn = randn.stride()
            rargs = (dptr(randn), rb, rs, rn, block_cap, dptr(self.d_sigma[sl]), dptr(self.d_delta_value[sl]))
        else:
            rargs = (None, 0, 0, 0, 0, None, None)
        call("vtb_iaf_encode", dptr(x), ts, ns, N, F, block_frames, self.dt, dptr(self.d_kappa[sl]),
             dptr(self.d_bias[sl]), dptr(self.d_delta[sl]), dptr(self.d_v0[sl]), dptr(self.d_time_count[sl]),
             *rargs, dptr(st), dptr(ss), dptr(cnt), cap, dptr(near), near_eps, dptr(status), float(block_rate),
             stream_ptr())
        return st, ss, cnt, near, status

    @staticmethod
    def _as_input(neural_inputs, layout):
        x = _dev(neural_inputs)
        if x.dim() != 2:
            raise ValueError("neural inputs must be a 2-D (samples, neurons) array")
        if layout == "time":
            F, N = x.shape
            return x, N, 1, N, F
        N, F = x.shape
        return x, 1, F, N, F

    def encode(self, neural_inputs, startbias=0, avg_rate=0.1, layout="time"):
        """Encode (samples, neurons) inputs; returns (list of per-neuron
        spike times, int32 counts) like ensemble_encode.py:106-168."""
        x, ts, ns, N, F = self._as_input(neural_inputs, layout)
        if startbias == 0 and self.num_neurons != N:
            raise ValueError("input size should match number of neurons")
        if startbias + N > self.num_neurons:
            raise ValueError("input size should match number of neurons")
        cap = int(np.ceil(F / avg_rate))
        randn = self._draw_randn(1, cap, N)
        st, ss, cnt, near, status = self._launch(x, ts, ns, N, F, max(F, 1), cap, startbias, randn=randn,
                                                 block_cap=cap)
        cnt_h = cnt.cpu().numpy()
        if status.item() == VTB_OVERFLOW or (cnt_h.size and cnt_h.max() >= cap):
            raise ValueError("number of spikes exceeded the limit of buffer")
        self.last_near_threshold = int(near.item())
        t = st.cpu().numpy()
        return [t[i, :cnt_h[i]].copy() for i in range(N)], cnt_h

    def encode_blocks(self, neural_inputs, block_frames=101, avg_rate=0.1, layout="time", cap=None,
                      near_eps=1e-12, check=True):
        """VTEM_IAF's block loop in one launch (vtem.py:165-200): blocks of
        ``block_frames`` frames stepping by block_frames-1, time_count reset
        at each block start, v0 carried.  Returns :class:`DeviceSpikes`; the
        reference's per-block overflow rule (ensemble_encode.py:163-164) is
        checked by the kernel and raised here when ``check``.  time_count is
        left as the reference leaves it after its loop: reset to 0.

        The reference's buffer holds ceil(F / avg_rate) spikes per neuron.
        With ``check`` (and no explicit ``cap``) the scan first runs with
        room for one spike every SMALL_CAP_STRIDE samples and, only if a
        neuron fills that, runs again from the saved state with the full
        buffer; the spikes are the same either way."""
        x, ts, ns, N, F = self._as_input(neural_inputs, layout)
        if N != self.num_neurons:
            raise ValueError("input size should match number of neurons")
        nblocks = max(1, len(range(0, F, block_frames - 1)))
        block_cap = int(np.ceil(block_frames / avg_rate))
        full = max(16, int(np.ceil(F / avg_rate)))
        caps = [full] if cap is not None or not check else [min(full, 64 + -(-F // SMALL_CAP_STRIDE)), full]
        if cap is not None:
            caps = [int(cap)]
        randn = self._draw_randn(nblocks, block_cap, N)
        saved = None
        if len(caps) > 1:
            saved = [self.d_v0.clone(), self.d_time_count.clone()]
            if self.random_thresholds:
                saved.append(self.d_delta_value.clone())
        for i, c in enumerate(caps):
            st, ss, cnt, near, status = self._launch(x, ts, ns, N, F, block_frames, c, 0, randn=randn,
                                                     block_cap=block_cap, near_eps=near_eps,
                                                     block_rate=avg_rate if check else 0.0)
            if not check:
                break
            near_h, code = _read_flags(self._flags)
            if code == VTB_BLOCK_LIMIT or (code == VTB_OVERFLOW and i + 1 == len(caps)):
                self.reset_timer()
                raise ValueError("number of spikes exceeded the limit of buffer")
            if code != VTB_OVERFLOW:
                break
            # a neuron filled the small buffer: rerun from the saved state
            self.d_v0.copy_(saved[0])
            self.d_time_count.copy_(saved[1])
            if self.random_thresholds:
                self.d_delta_value.copy_(saved[2])
        self.reset_timer()
        out = DeviceSpikes(st, ss, cnt, block_frames, self.dt)
        out.near_threshold = near_h if check else near
        return out

    def _draw_randn(self, nblocks, block_cap, N):
        return None


def _read_flags(flags):
    """(near-threshold count, status word) of a launch, one host read."""
    near, word = flags.cpu().tolist()
    code = ((int(word) + (1 << 31)) % (1 << 32)) - (1 << 31)      # the low 32 bits, signed
    return int(near), code


class IAF_encode_rt(IAF_encode):
    """IAF neurons with random thresholds (ensemble_encode.py:175-333).

    After each spike the next threshold is ``randn * sigma + delta``; the
    N(0,1) draws come from ``self.randn_source(shape)`` (default
    ``np.random.normal``, as the reference fills its spike buffer,
    ensemble_encode.py:304-306), so a seeded source reproduces a run.
    """

    random_thresholds = True

    def __init__(self, num_neurons, dt, dtype=np.float64):
        super().__init__(num_neurons, dt, dtype)
        self.randn_source = lambda shape: np.random.normal(size=shape)

    def set_parameters(self):
        """Defaults kappa 1, delta 0.03, bias 0.8, sigma 3e-4 and a first
        threshold drawn from N(delta, sigma) (ensemble_encode.py:199-214)."""
        self.h_kappa = np.zeros(self.num_neurons) + 1.0
        self.h_delta = np.zeros(self.num_neurons) + 0.03
        self.h_bias = np.zeros(self.num_neurons) + 0.8
        self.h_sigma = np.zeros(self.num_neurons) + 0.0003
        self.h_delta_value = np.random.normal(size=self.num_neurons) * self.h_sigma + self.h_delta

    def set_initial_value(self):
        self.h_v0 = np.random.uniform(0, 1, self.num_neurons).astype(np.float64) * self.h_delta_value

    def load_parameters(self, h_kappa=None, h_bias=None, h_delta=None, h_sigma=None, h_delta_value=None,
                        h_time_count=None, h_v0=None):
        """ensemble_encode.py:221-262."""
        if h_kappa is None:
            self.set_parameters()
        else:
            self.h_kappa = np.asarray(h_kappa, np.float64)
            self.h_delta = np.asarray(h_delta, np.float64)
            self.h_bias = np.asarray(h_bias, np.float64)
            self.h_sigma = np.asarray(h_sigma, np.float64)
            self.h_delta_value = np.asarray(h_delta_value, np.float64)
        if h_time_count is None:
            self.set_time_count()
        else:
            self.h_time_count = np.asarray(h_time_count, np.float64).reshape(-1)
        if h_v0 is None:
            self.set_initial_value()
        else:
            self.h_v0 = np.asarray(h_v0, np.float64)
        self.d_delta_value = _dev(self.h_delta_value)
        self.d_kappa = _dev(self.h_kappa)
        self.d_delta = _dev(self.h_delta)
        self.d_bias = _dev(self.h_bias)
        self.d_sigma = _dev(self.h_sigma)
        self.d_v0 = _dev(self.h_v0)
        self.d_time_count = _dev(self.h_time_count)

    def _draw_randn(self, nblocks, block_cap, N):
        r = np.asarray(self.randn_source((nblocks, block_cap, N)), np.float64)
        return _dev(r)


def spikes_per_block(sp: DeviceSpikes, F: int) -> np.ndarray:
    """(blocks, N) spike counts per frame block, from the step indices."""
    bstep = sp.block_frames - 1
    nblocks = max(1, len(range(0, F, bstep)))
    cnt = sp.count
    N, cap = sp.step.shape
    valid = torch.arange(cap, device=cnt.device)[None, :] < cnt[:, None]
    blk = torch.where(valid, sp.step.long() // bstep, torch.full_like(sp.step, nblocks, dtype=torch.long))
    out = torch.zeros((N, nblocks + 1), dtype=torch.int64, device=cnt.device)
    out.scatter_add_(1, blk, torch.ones_like(blk))
    return out[:, :nblocks].t().cpu().numpy()
