"""Video time encoding machines (reference: ``vtem/vtem.py``).

``VTEM_IAF`` keeps the reference's signature and spike-file semantics
(vtem.py:15-206): blocks of ``ONE_TIME_FRAMES`` frames sharing one boundary
frame, time_count reset per block, v0 carried, spikes stored per refresh
interval with block-relative times.  On the B200 the whole clip is filtered
by one RF projection and encoded by one IAF launch that runs the block loop
on the device; the spike store is filled from that result.

Extensions (keyword-only, defaults keep the reference behaviour): ``iaf``
(an ``IAF_encode``/``IAF_encode_rt`` with custom parameters; the reference
always uses the defaults, vtem.py:159-161) and ``return_spikes`` (also
return the device spikes).
"""
from __future__ import annotations

import numpy as np
import torch

from . import ensemble_encode as ee
from . import spike_store as ss
from . import vrf as vrf_mod


def _rf_type(rf):
    if isinstance(rf, vrf_mod.vrf_gabor):
        return "gabor"
    if isinstance(rf, vrf_mod.vrf_cs):
        return "cs"
    if isinstance(rf, vrf_mod.vrf_bank):
        return "bank"
    raise TypeError("Receptive field type not recognized\n.")


def one_time_frames(F):
    """Frames per encode block: min(101, F + 1) (vtem.py:167-169 on a GPU
    whose free memory never limits it)."""
    return int(min(101, F + 1))


def VTEM_IAF(videofile, output_filename, Wt, rf, Wx=2 * np.pi * 4, Wy=2 * np.pi * 4, start_frame=0,
             end_frame=None, dx=1.0 / 16, dy=1.0 / 16, fps=100, domain=None, h5input=True, npinput=False, *,
             iaf=None, return_spikes=False):
    """Encode a video with IAF neurons behind the RF bank ``rf``.

    ``videofile`` is an array (frames, Py, Px) (numpy or torch) when
    ``npinput`` is set, else a ``.npy`` file.  Returns the
    :class:`vtem_storage` (also written to ``output_filename`` when given).
    """
    if npinput:
        videoarray = videofile
    else:
        videoarray = np.load(videofile, mmap_mode="r")
    TotalFrames, Py, Px = videoarray.shape
    if end_frame is None or end_frame > TotalFrames:
        end_frame = TotalFrames
    dt = 1.0 / fps
    kind = _rf_type(rf)
    banks = rf.banks if kind == "bank" else [rf]
    if kind == "bank" and len({_rf_type(b) for b in banks}) != 1:
        store_type = "mixed"
    else:
        store_type = _rf_type(banks[0])
    spikefile = ss.vtem_storage(output_filename, rf.num_neurons, store_type)
    if store_type == "mixed":
        gb0 = next(b for b in banks if _rf_type(b) == "gabor")
        spikefile.data["vrf/KAPPA"] = np.array(float(gb0.KAPPA))
    spikefile.write_video_attributes(Wt, Wx, Wy, rf.Px, rf.Py, float(dx), float(dy))
    for b in banks:
        if _rf_type(b) == "gabor":
            spikefile.write_gabor_parameters(b)
        else:
            spikefile.write_cs_parameters(b)
    if iaf is None:
        iaf = ee.IAF_encode(rf.num_neurons, dt)
        iaf.load_parameters()
    spikefile.write_neuron_parameters(iaf)
    nframes = end_frame - start_frame
    B = one_time_frames(nframes)
    spikefile.write_refresh_interval((B - 1) * dt)
    if isinstance(videoarray, torch.Tensor):
        block = videoarray[start_frame:end_frame]
    else:
        block = torch.as_tensor(np.ascontiguousarray(videoarray[start_frame:end_frame]), dtype=torch.float64)
    L = rf.filter(block, out_layout="neuron")           # (N, frames)
    sp = iaf.encode_blocks(L, block_frames=B, layout="neuron")
    _fill_store(spikefile, sp, nframes)
    spikefile.close()
    if return_spikes:
        return spikefile, sp
    return spikefile


def _fill_store(spikefile, sp, F):
    """Per-refresh-interval spike arrays from one device encode."""
    times, steps, cnt = sp.to_host_lists()
    bstep = sp.block_frames - 1
    nblocks = max(1, len(range(0, F, bstep)))
    N = len(times)
    per = [[None] * N for _ in range(nblocks)]
    for n in range(N):
        blk = steps[n] // bstep
        bounds = np.searchsorted(blk, np.arange(nblocks + 1))
        for b in range(nblocks):
            per[b][n] = times[n][bounds[b]:bounds[b + 1]]
    for b in range(nblocks):
        counts = np.array([len(x) for x in per[b]], np.int32)
        spikefile.write_spike_in_timebin(counts, np.concatenate(per[b]) if N else np.zeros(0))
