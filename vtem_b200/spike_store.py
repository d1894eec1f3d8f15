"""Spike store of the encoder (reference: ``vtem/utils/spike_store.py``).

Same classes and methods as ``vtem_storage`` (:6-156) and
``vtem_storage_read`` (:159-351), including the reference's swap of Wx and
Wy when they are written (:89-90).  The store lives in memory; ``close()``
writes it to ``filename`` as a NumPy ``.npz`` archive when a name is given
(the reference's HDF5 layout needs PyTables, which this stack does not
ship).  ``vtem_storage_read`` accepts such a file or a ``vtem_storage``.
"""
from __future__ import annotations

import numpy as np


class vtem_storage(object):
    def __init__(self, filename, num_neurons, filter_type, title="VTEM_gabor_iaf"):
        self.filename = filename
        self.filter_type = filter_type
        self.title = title
        self.data = {"filter_type": np.array(filter_type)}
        self.vrf = {"alpha": [], "x0": [], "y0": []}
        if filter_type in ("gabor", "mixed"):
            self.vrf["l"] = []
            self.vrf["ab"] = []
        if filter_type == "mixed":
            # extension: Gabor and centre-surround neurons in one store, told
            # apart by vrf/kind (0 Gabor, 1 centre-surround)
            self.vrf["kind"] = []
        self.iaf = {"kappa": [], "delta": [], "bias": [], "sigma": []}
        self.spike_count = []
        self.spikes = []
        self.refresh_interval = 0
        self.closed = False

    def close(self):
        """Finish the store (num_neurons, total_intervals) and save it."""
        if self.closed:
            return
        for k, v in self.vrf.items():
            self.data["vrf/" + k] = np.concatenate(v) if v else np.zeros(0)
        for k, v in self.iaf.items():
            self.data["iaf/" + k] = np.concatenate(v) if v else np.zeros(0)
        self.data["vrf/num_neurons"] = np.array(len(self.data["vrf/alpha"]))
        self.data["spikes/total_intervals"] = np.array(self.refresh_interval)
        for i, (c, s) in enumerate(zip(self.spike_count, self.spikes)):
            self.data["spikes/spike_count%d" % i] = c
            self.data["spikes/spikes%d" % i] = s
        if self.filename:
            np.savez(self.filename, **self.data)
        self.closed = True

    def write_video_attributes(self, Wt, Wx, Wy, Px, Py, dx, dy):
        """Video attributes; Wx and Wy are stored swapped, as the reference
        stores them (spike_store.py:89-90)."""
        self.data["video/Wt"] = np.array(float(Wt))
        self.data["video/Wx"] = np.array(float(Wy))
        self.data["video/Wy"] = np.array(float(Wx))
        self.data["vrf/Px"] = np.array(int(Px))
        self.data["vrf/Py"] = np.array(int(Py))
        self.data["vrf/dx"] = np.array(float(dx))
        self.data["vrf/dy"] = np.array(float(dy))

    def write_gabor_parameters(self, filter):
        if "vrf/KAPPA" not in self.data:
            self.data["vrf/KAPPA"] = np.array(float(filter.KAPPA))
        self.vrf["alpha"].append(np.asarray(filter.h_alpha, np.float64))
        self.vrf["l"].append(np.asarray(filter.h_l, np.float64))
        self.vrf["x0"].append(np.asarray(filter.h_x0, np.float64))
        self.vrf["y0"].append(np.asarray(filter.h_y0, np.float64))
        self.vrf["ab"].append(np.asarray(filter.h_ab, np.int32))
        if "kind" in self.vrf:
            self.vrf["kind"].append(np.zeros(len(filter.h_alpha), np.int32))
        self._gain(filter)

    def _gain(self, filter):
        g = filter.h_gain if filter.h_gain is not None else np.ones(len(filter.h_alpha))
        self.vrf.setdefault("gain", []).append(np.asarray(g, np.float64))

    def write_cs_parameters(self, filter):
        if "vrf/sigma_center" not in self.data:
            self.data["vrf/sigma_center"] = np.array(float(filter.sigma_center))
            self.data["vrf/sigma_surround"] = np.array(float(filter.sigma_surround))
        self.vrf["alpha"].append(np.asarray(filter.h_alpha, np.float64))
        self.vrf["x0"].append(np.asarray(filter.h_x0, np.float64))
        self.vrf["y0"].append(np.asarray(filter.h_y0, np.float64))
        if "kind" in self.vrf:
            n = len(filter.h_alpha)
            self.vrf["l"].append(np.zeros(n))
            self.vrf["ab"].append(np.zeros(n, np.int32))
            self.vrf["kind"].append(np.ones(n, np.int32))
        self._gain(filter)

    def write_neuron_parameters(self, iaf):
        self.iaf["kappa"].append(np.asarray(iaf.h_kappa, np.float64))
        self.iaf["delta"].append(np.asarray(iaf.h_delta, np.float64))
        self.iaf["bias"].append(np.asarray(iaf.h_bias, np.float64))
        self.iaf["sigma"].append(np.asarray(iaf.h_sigma, np.float64))

    def write_refresh_interval(self, time):
        self.data["iaf/refresh_interval"] = np.array(float(time))

    def write_spike_in_timebin(self, spike_count, spikes):
        """One refresh interval: per-neuron counts and the spike times,
        neuron after neuron (spike_store.py:147-156)."""
        self.spike_count.append(np.asarray(spike_count, np.int32))
        self.spikes.append(np.asarray(spikes, np.float64))
        self.refresh_interval += 1


class vtem_storage_read(object):
    def __init__(self, filename):
        if isinstance(filename, vtem_storage):
            filename.close()
            self.d = dict(filename.data)
        else:
            with np.load(filename, allow_pickle=False) as z:
                self.d = {k: z[k] for k in z.files}

    def close(self):
        pass

    def read_num_neurons(self):
        self.num_neurons = int(self.d["vrf/num_neurons"])
        return self.num_neurons

    def read_video_attributes(self):
        """Wt, Wx, Wy, Px, Py, dx, dy (spike_store.py:176-191)."""
        return (float(self.d["video/Wt"]), float(self.d["video/Wx"]), float(self.d["video/Wy"]),
                int(self.d["vrf/Px"]), int(self.d["vrf/Py"]), float(self.d["vrf/dx"]), float(self.d["vrf/dy"]))

    def read_vrf_type(self):
        if "vrf/kind" in self.d:
            self.filter_type = "mixed"
        else:
            self.filter_type = "gabor" if "vrf/ab" in self.d else "cs"

    def read_vrf(self):
        if self.filter_type == "mixed":
            return (self.d["vrf/alpha"], self.d["vrf/l"], self.d["vrf/x0"], self.d["vrf/y0"], self.d["vrf/ab"],
                    float(self.d["vrf/KAPPA"]), float(self.d["vrf/sigma_center"]),
                    float(self.d["vrf/sigma_surround"]), self.d["vrf/kind"])
        if self.filter_type == "gabor":
            return (self.d["vrf/alpha"], self.d["vrf/l"], self.d["vrf/x0"], self.d["vrf/y0"], self.d["vrf/ab"],
                    float(self.d["vrf/KAPPA"]))
        return (self.d["vrf/alpha"], self.d["vrf/x0"], self.d["vrf/y0"], float(self.d["vrf/sigma_center"]),
                float(self.d["vrf/sigma_surround"]))

    def read_gain(self):
        return self.d.get("vrf/gain")

    def read_refresh_interval(self):
        return float(self.d["iaf/refresh_interval"])

    def read_total_intervals(self):
        return int(self.d["spikes/total_intervals"])

    def read_iaf(self):
        return self.d["iaf/kappa"], self.d["iaf/delta"], self.d["iaf/bias"], self.d["iaf/sigma"]

    def select_neurons(self, domain):
        """Neurons centred inside ``domain`` = [x0, x1, y0, y1] (+-0.01),
        with centres shifted to the domain centre (spike_store.py:243-277)."""
        if self.filter_type == "mixed":
            (h_alpha, h_l, h_x0, h_y0, h_ab, self.KAPPA, self.sigma_center, self.sigma_surround,
             h_kind) = self.read_vrf()
        elif self.filter_type == "gabor":
            h_alpha, h_l, h_x0, h_y0, h_ab, self.KAPPA = self.read_vrf()
        else:
            h_alpha, h_x0, h_y0, self.sigma_center, self.sigma_surround = self.read_vrf()
        allind = np.arange(self.num_neurons)
        Sx = domain[1] - domain[0]
        Sy = domain[3] - domain[2]
        shiftx = domain[0] + Sx / 2
        shifty = domain[2] + Sy / 2
        self.choose = allind[(h_x0 > domain[0] - 0.01) & (h_x0 < domain[1] + 0.01) &
                             (h_y0 > domain[2] - 0.01) & (h_y0 < domain[3] + 0.01)]
        self.alpha = h_alpha[self.choose]
        self.x0 = h_x0[self.choose] - shiftx
        self.y0 = h_y0[self.choose] - shifty
        g = self.read_gain()
        self.gain = None if g is None else g[self.choose]
        if self.filter_type in ("gabor", "mixed"):
            self.l = h_l[self.choose]
            self.ab = h_ab[self.choose]
        if self.filter_type == "mixed":
            self.kind = h_kind[self.choose]
        self.decode_neurons = self.choose.size

    def read_select_spikes(self, time_frame):
        """Consecutive spike pairs of the selected neurons inside
        ``time_frame``, plus one spike either side (spike_store.py:279-351).
        Returns tk1, tk2 (relative to time_frame[0]), neuron_ind, and the
        selected kappa, delta, bias plus all sigmas."""
        h_kappa, h_delta, h_bias, h_sigma = self.read_iaf()
        self.kappa = h_kappa[self.choose]
        self.delta = h_delta[self.choose]
        self.bias = h_bias[self.choose]
        R = self.read_refresh_interval()
        total = self.read_total_intervals()
        si = int(np.floor(time_frame[0] / R))
        ei = int(np.floor(time_frame[1] / R))
        intervals = np.arange(max(0, si - 1), min(total, ei + 2))
        D = self.decode_neurons
        # gather per selected neuron, interval by interval (times relative to the window)
        pieces_t = []
        pieces_n = []
        sel = np.full(self.num_neurons, -1, np.int64)
        sel[self.choose] = np.arange(D)
        for i in intervals:
            cnt = self.d["spikes/spike_count%d" % i].astype(np.int64)
            sp = self.d["spikes/spikes%d" % i] + i * R - time_frame[0]
            owner = np.repeat(np.arange(self.num_neurons), cnt)
            keep = sel[owner] >= 0
            pieces_t.append(sp[keep])
            pieces_n.append(sel[owner[keep]])
        if pieces_t:
            t_all = np.concatenate(pieces_t)
            n_all = np.concatenate(pieces_n)
        else:
            t_all = np.zeros(0)
            n_all = np.zeros(0, np.int64)
        order = np.argsort(n_all, kind="stable")
        t_all = t_all[order]
        n_all = n_all[order]
        bounds = np.searchsorted(n_all, np.arange(D + 1))
        T = time_frame[1] - time_frame[0]
        tk1l, tk2l, indl = [], [], []
        count = np.zeros(D, np.int32)
        for j in range(D):
            s = t_all[bounds[j]:bounds[j + 1]]
            a = np.nonzero((s > 0) & (s < T))[0]
            tk = s[max(0, a[0] - 1):min(a[-1] + 2, s.size)] if a.size > 0 else np.zeros(0)
            count[j] = max(0, tk.size - 1)
            if count[j]:
                tk1l.append(tk[:-1])
                tk2l.append(tk[1:])
                indl.append(np.full(count[j], j, np.int32))
        self.count = count
        tk1 = np.concatenate(tk1l) if tk1l else np.zeros(0)
        tk2 = np.concatenate(tk2l) if tk2l else np.zeros(0)
        ind = np.concatenate(indl) if indl else np.zeros(0, np.int32)
        return tk1, tk2, ind, self.kappa, self.delta, self.bias, h_sigma


def device_pairs(spikes, T, t0=0.0):
    """Device-side form of ``read_select_spikes`` for a window that holds the
    whole clip, [t0, T) with t0 = 0 (spike_store.py:279-351): absolute times
    ``t + block * refresh_interval - t0`` (the reference's expression), then
    consecutive pairs of every neuron, grouped by neuron.  ``spikes`` is the
    :class:`~vtem_b200.ensemble_encode.DeviceSpikes` of one encode.  Only valid
    when every spike lies inside (t0, T) (true for a whole-clip window), which
    is checked."""
    import torch
    from ._abi import call, dptr, stream_ptr
    if t0 != 0.0:
        raise ValueError("device_pairs covers the whole-clip window only")
    N, cap = spikes.time.shape
    dev = spikes.time.device
    c1 = (spikes.count.long() - 1).clamp_(min=0)
    incl = torch.cumsum(c1, 0)
    n = int(incl[-1]) if N else 0
    offs = incl - c1
    tk1 = torch.empty(n, dtype=torch.float64, device=dev)
    tk2 = torch.empty(n, dtype=torch.float64, device=dev)
    ind = torch.empty(n, dtype=torch.int32, device=dev)
    outside = torch.zeros(1, dtype=torch.int32, device=dev)
    call("vtb_spike_pairs", dptr(spikes.time), dptr(spikes.step), dptr(spikes.count), N, cap, spikes.block_frames,
         spikes.refresh_interval, float(t0), float(T), dptr(offs), dptr(tk1) if n else None,
         dptr(tk2) if n else None, dptr(ind) if n else None, dptr(outside), stream_ptr())
    if int(outside.item()):
        raise ValueError("spikes outside the window: use read_select_spikes")
    return tk1, tk2, ind
