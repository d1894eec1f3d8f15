"""Benchmark of the vtem decode path on the B200.

Workload ("gpu" configuration, vtem_b200.workloads.gpu_scale): a seeded
Dirichlet-bandlimited video, 64x64 pixels x 10000 samples (1 s at dt=1e-4),
Mx=My=6, Mt=8, encoded by 768 Gabor + 256 centre-surround RFs feeding IAF
neurons (~25k spike intervals).  Encoding and decoder preparation happen
before the timed region.

One step = one decode of the clip: device-resident spike intervals -> the
float64 video (10000, 64, 64) on the device, by the coefficient-space
decoder (same reconstruction as the reference's pseudoinverse decode; its
rel-L2 against the plain n x n path is reported).  value = voxels / s.
e2e = the same decode through the public API from host spike arrays
(host->device copy inside the timed region) with the video read back to
pinned host memory.  The plain float64 n x n path (analytic Gram,
eigendecomposition pseudoinverse, synthesis) is timed once beside it.

L2: the 328 MB output of every step exceeds the 126 MB L2, and a 256 MB
buffer is written between timed steps.

--impl reference: the reference's own kernels compiled for the host
(oracle/_ref) with NumPy for its library calls, on a bounded sample of the
same workload (a decode window of the same spikes), rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "reconstructed voxels/s at >=40 dB SNR (mixed vs FP64 plain)"
SYNTH_KERNEL = "harmonics_kernel<double, 17>"
UNIT = "voxels/s"


def reduce_max(values, device, world):
    """Element-wise maximum over ranks of per-rank timings (the job's time is
    its slowest rank's): an all-reduce MAX on ``device`` (CUDA for NCCL, CPU
    for gloo); a no-op with one rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def weak_value(units_per_rank, world, steps, ms):
    """Whole-job throughput of clip-parallel ranks: every rank processes
    ``units_per_rank`` per step, the job takes the slowest rank's ``ms``."""
    return units_per_rank * world * steps / (ms / 1e3)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- setup

def encode_clip(w, device):
    """Encode the workload's clip on the GPU and prepare the decoder."""
    import torch
    from vtem_b200 import ensemble_encode, spike_store, vrf, vtdm, vtem

    V = w.video(device=device)
    banks = []
    g = w.gabor
    gb = vrf.vrf_gabor((w.Py, w.Px), dx=w.dx, dy=w.dy)
    gb.load_parameters(num_neurons=len(g.h_alpha), h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0,
                       h_ab=g.h_ab, KAPPA=g.KAPPA, h_gain=g.gain)
    banks.append(gb)
    if w.cs is not None:
        c = w.cs
        cb = vrf.vrf_cs((w.Py, w.Px), dx=w.dx, dy=w.dy)
        cb.load_parameters(num_neurons=len(c.h_alpha), h_alpha=c.h_alpha, h_x0=c.h_x0, h_y0=c.h_y0,
                           sigma_center=c.sigma_center, sigma_surround=c.sigma_surround, h_gain=c.gain)
        banks.append(cb)
    bank = vrf.vrf_bank(banks) if len(banks) > 1 else banks[0]
    iaf = ensemble_encode.IAF_encode(w.N, w.dt)
    iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_v0=w.v0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    store, sp = vtem.VTEM_IAF(V, None, w.Wt, bank, w.Wx, w.Wy, dx=w.dx, dy=w.dy, fps=1.0 / w.dt, npinput=True,
                              iaf=iaf, return_spikes=True)
    torch.cuda.synchronize()
    t_enc = time.perf_counter() - t0
    # decoder prep: the decoder-side RF banks on one spatial period (vtdm.py:385-435)
    rfSx, rfSy, rfPx, rfPy = vtdm.period_grid(w.Mx, w.My, w.Wx, w.Wy, w.dx, w.dy)
    dbanks = []
    gd = vrf.vrf_gabor((rfPy, rfPx), dx=rfSx / rfPx, dy=rfSy / rfPy, scale=4)
    gd.load_parameters(num_neurons=len(g.h_alpha), h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0,
                       h_ab=g.h_ab, KAPPA=g.KAPPA, h_gain=g.gain)
    dbanks.append(gd)
    if w.cs is not None:
        c = w.cs
        cd = vrf.vrf_cs((rfPy, rfPx), dx=rfSx / rfPx, dy=rfSy / rfPy, scale=4)
        cd.load_parameters(num_neurons=len(c.h_alpha), h_alpha=c.h_alpha, h_x0=c.h_x0, h_y0=c.h_y0,
                           sigma_center=c.sigma_center, sigma_surround=c.sigma_surround, h_gain=c.gain)
        dbanks.append(cd)
    prep = vtdm.prep_from_banks(dbanks, np.ones(w.N), w.Mx, w.My, w.Wx, w.Wy, w.Px, w.Py, 1.0, 1.0)
    rd = spike_store.vtem_storage_read(store)
    rd.source = store
    rd.num_neurons = w.N
    rd.choose = np.arange(w.N)
    rd.decode_neurons = w.N
    rd.d["iaf/kappa"], rd.d["iaf/delta"], rd.d["iaf/bias"] = w.kappa, w.delta, w.bias
    tk1, tk2, ind, kap, dl, bia, _ = rd.read_select_spikes([0.0, w.T])
    return V, prep, (tk1, tk2, ind), t_enc, sp, rd


def flush_l2(buf):
    buf.add_(1.0)


# ---------------------------------------------------------------- our arm

def time_decoder(dec, inputs, w, u, flush, steps, warmup):
    """Per-step device time of one decode through the public call
    ``decode`` (coefficients + synthesis; the mixed solver queues the
    synthesis before it reads its acceptance), with an L2 flush between
    steps; returns (total ms, synthesis ms per step), the synthesis timed by
    events the decoder records around its launches."""
    import torch
    d_tk1, d_tk2, d_ind, kap, dl, bia = inputs
    for _ in range(warmup):
        dec.decode(d_tk1, d_tk2, d_ind, kap, dl, bia, w.T, w.dt, out=u, assume_sorted=True)
        flush_l2(flush)
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
    try:
        for i in range(steps):
            ev[i][0].record()
            dec.synth_events = (ev[i][1], ev[i][2])
            dec.decode(d_tk1, d_tk2, d_ind, kap, dl, bia, w.T, w.dt, out=u, assume_sorted=True)
            ev[i][3].record()
            flush_l2(flush)
    finally:
        dec.synth_events = None
    torch.cuda.synchronize()
    tot = sum(e[0].elapsed_time(e[3]) for e in ev)
    synth = [e[1].elapsed_time(e[2]) for e in ev]
    return tot, synth


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from vtem_b200 import fast, workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev, timeout=__import__("datetime").timedelta(seconds=600))
    w = workloads.gpu_scale(seed=rank, frames=args.frames)
    V, prep, (tk1, tk2, ind), t_enc, sp, rd = encode_clip(w, dev)
    n = len(tk1)
    Nt = len(np.arange(0, w.T, w.dt))
    voxels = Nt * w.Px * w.Py
    inputs = tuple(torch.as_tensor(x, device=dev) for x in (tk1, tk2, ind, w.kappa, w.delta, w.bias))
    u64 = torch.empty((Nt, w.Py, w.Px), dtype=torch.float64, device=dev)
    umix = torch.empty_like(u64)
    flush = torch.zeros(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    dec64 = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="auto")
    decmix = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=args.sweeps)

    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    mix_ms, mix_synth = time_decoder(decmix, inputs, w, umix, flush, args.steps, args.warmup)
    clk = clocks.stop()
    f64_ms, f64_synth = time_decoder(dec64, inputs, w, u64, flush, args.steps, args.warmup)
    mix_ms, f64_ms = reduce_max([mix_ms, f64_ms], dev, world)
    rel_mix_f64 = float(((umix - u64).norm() / u64.norm()).item())
    resid = decmix.residual_norm(*inputs)
    mix_ratios = list(decmix.last_ratios)
    gram_err = decmix.gram_error()
    # BASELINE configuration 2 as specified: the same mixed decoder with 3 float64 refinement sweeps
    dec3 = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=3)
    u3 = torch.empty_like(u64)
    mix3_ms, _ = time_decoder(dec3, inputs, w, u3, flush, args.steps, args.warmup)
    mix3_ms = reduce_max([mix3_ms], dev, world)[0]
    config2 = {"sweeps": 3, "ms_per_step": mix3_ms / args.steps, "solver": dec3.last_solver,
               "sweep_ratios": list(dec3.last_ratios),
               "rel_l2_vs_coeff_f64": float(((u3 - u64).norm() / u64.norm()).item()),
               "residual_rel": dec3.residual_norm(*inputs), "gram_rel_frobenius": gram_err}
    del u3, dec3
    # the same decoder on cuSOLVER's spotrf/spotrs and the warp-specialised per-frame synthesis, for comparison
    decv = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=args.sweeps,
                          mixed_factor="cusolver", synth="fused")
    uv = torch.empty_like(u64)
    alt_ms, alt_synth = time_decoder(decv, inputs, w, uv, flush, args.steps, args.warmup)
    alt_ms = reduce_max([alt_ms], dev, world)[0]
    alt = {"ms_per_step": alt_ms / args.steps, "synthesis_ms": sum(alt_synth) / len(alt_synth),
           "solver": decv.last_solver, "rel_l2_vs_headline": float(((uv - umix).norm() / umix.norm()).item())}
    del uv, decv

    # --- end to end through the public API with host buffers (mixed decoder)
    h_tk1, h_tk2, h_ind = (torch.as_tensor(x).pin_memory() for x in (tk1, tk2, ind))
    h_u = torch.empty((Nt, w.Py, w.Px), dtype=torch.float64).pin_memory()
    kap, dl, bia = inputs[3:]

    def e2e_step():
        g1 = h_tk1.to(dev, non_blocking=True)
        g2 = h_tk2.to(dev, non_blocking=True)
        gi = h_ind.to(dev, non_blocking=True)
        # synthesis in frame ranges, each range's download overlapping the next range
        decmix.decode_to_host(g1, g2, gi, kap, dl, bia, w.T, w.dt, h_u, chunks=8, assume_sorted=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 5))
    e2e_ms = 0.0
    for _ in range(e2e_steps):
        flush_l2(flush)
        e0.record()
        e2e_step()
        e1.record()
        torch.cuda.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_ms = reduce_max([e2e_ms], dev, world)[0]
    e2e_value = weak_value(voxels, world, e2e_steps, e2e_ms)
    h2d = n * (8 + 8 + 4)
    d2h = voxels * 8

    result = None
    if rank == 0:
        plain = {}
        if not args.no_plain:
            plain = run_plain(w, prep, tk1, tk2, ind, {"mixed": umix, "coeff_f64": u64}, dev, Nt)
        rnn = None if args.no_rnn else run_rnn(w, prep, tk1, tk2, ind, dev, Nt, steps=args.rnn_steps)
        encode = run_encode(w, V, dev)
        snr_mix = plain.get("snr_db", {}).get("mixed")
        headline_mixed = snr_mix is None or snr_mix >= 40.0
        tot_ms = mix_ms if headline_mixed else f64_ms
        synth_ms = mix_synth if headline_mixed else f64_synth
        value = weak_value(voxels, world, args.steps, tot_ms)
        # the synthesis writes the video and reads the K coefficients and the per-pixel weights (P x Kt)
        synth_bytes = voxels * 8 + dec64.K * 16 + 2 * w.Px * w.Py * dec64.Kt * 8
        synth_avg = sum(synth_ms) / len(synth_ms) / 1e3
        peaks = load_peaks()
        achieved = synth_bytes / synth_avg / 1e9
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (split-bf16 tensor-core Gram, f64 refinement)"
            if headline_mixed else "f64",
            "data": "synthetic (seeded Dirichlet-bandlimited video)",
            "config": workload_config(w),
            "config_detail": {"spike_intervals": n, "voxels_per_step": voxels, "K_coeff": dec64.K,
                              "decoder": ("mixed: tensor-core Gram + %d f64 refinement sweeps" % args.sweeps)
                              if headline_mixed else "coefficient-space float64", "clip_per_rank": True,
                              "parallelism": "clip-parallel replicas" if world > 1 else "single GPU"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps * (launches_mixed(decmix) if headline_mixed else launches_per_step(dec64)),
            "roofline": {"bound": "hbm", "kernel": SYNTH_KERNEL + " (rank-%d synthesis; timed with its weights "
                                                                 "kernel)" % dec64.Kt,
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                         "traffic": measured_traffic(voxels, SYNTH_KERNEL), "algorithmic_bytes": synth_bytes,
                         "avg_ms": synth_avg * 1e3},
            "roofline_tensor": gram_gemm_roofline(decmix, peaks),
            "variants_ms_per_step": {"mixed": mix_ms / args.steps, "coeff_f64": f64_ms / args.steps,
                                     "mixed_cusolver_factor_fused_synthesis": alt["ms_per_step"]},
            "variant_cusolver_fused": alt,
            "mixed_vs_coeff_f64_rel_l2": rel_mix_f64, "mixed_residual_rel": resid,
            "stages_ms": {"coefficients": (tot_ms - sum(synth_ms)) / args.steps,
                          "synthesis": sum(synth_ms) / args.steps, "encode_once": t_enc * 1e3},
            "clocks": clk,
            "plain_fp64": plain,
            "rnn": rnn,
            "encode": encode,
            "solver": {"mixed": decmix.last_solver, "f64": dec64.last_solver, "pivots": dec64.last_pivots},
            "near_threshold_events": int(sp.near_threshold),
        }
        result["config2"] = config2
        result["mixed_sweep_ratios"] = mix_ratios
        result["gram_rel_frobenius"] = gram_err
        if not args.no_serve:
            result["serving"] = serve_short(dev, args.serve_requests, args.rate)
        if args.batch_clips > 0:
            # many clips of uneven size decoded as one batch (grouped Grams and solves, CUDA graphs)
            result["batch"] = batch_measure(dev, local, args.batch_clips, 2, args.sweeps, 3, 3, 2,
                                            eig=args.batch_eig)[0]
        if not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(host_clip_from_device(w, prep, rd), windows=2, window=0.1)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def gram_gemm_roofline(dec, peaks, reps=20):
    """The mixed decoder's tensor-core Kronecker Gram (the decode's tensor-
    bound kernel) timed alone with CUDA events on its own operands, at its
    autotuned tile width, against the measured bf16 peak.  Tensor work counts
    the three split-bf16 products (issued from [hi | lo] operand tiles) of the
    symmetric form (the four real sums per pair and upper temporal entry);
    ``complex_form_tflops`` counts the real form of the complex GEMM over all
    Kt^2 entries (twice the products) in the same time.  L2 is flushed before
    each launch (the 54 MB of operands would otherwise stay resident), so the
    RF-bank operand comes from HBM as in a decode."""
    import torch
    from vtem_b200 import autotune, tc
    from vtem_b200._abi import dptr, stream_ptr
    NE, M, K = dec.NE, 2 * dec.npairs, 3 * dec.Kh
    s = stream_ptr()

    def once():
        return autotune.gemm_bf16_tuned(dptr(dec.Lsplit), M, dptr(dec.Rsplit), NE, dec.Kh, dptr(dec.C), dec.ldc, 1, 0,
                                        1.0, 0, dec._stat_ptr(7), s, x3=True)
    bn = once()
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device=dec.C.device)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    torch.cuda.synchronize()
    for e0, e1 in ev:
        flush.fill_(1.0)
        e0.record()
        once()
        e1.record()
    torch.cuda.synchronize()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / reps
    del flush
    flop = 2.0 * M * NE * K
    achieved = flop / (ms / 1e3) / 1e12
    flop_cf = 2.0 * M * dec.Kt * dec.Kt * 3 * tc.padded_k(2 * dec.N)
    return {"bound": "tensor", "kernel": "tc_gemm_kernel<%d, float, x3> (Kronecker Gram, three split-bf16 products)" % bn,
            "achieved": achieved, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
            "frac": achieved / peaks["bf16_tflops"], "peak_source": peaks["source"], "avg_ms": ms,
            "tensor_flop": flop, "shape": [M, NE, K], "operand_bytes": (M + NE) * 2 * dec.Kh * 2,
            "complex_form_tflops": flop_cf / (ms / 1e3) / 1e12, "l2": "flushed before each launch"}



def serve_short(dev, requests=64, rate=200.0, seed=3):
    """A short serving run for the default bench line (BASELINE configuration
    4's request mix): ``requests`` encode+decode jobs sized like the batch
    clips (seed 3), Poisson arrivals at ``rate``/s, 120 GB admission budget,
    2 ms ticks; latency is arrival to result on the host (wall clock)."""
    import torch
    from vtem_b200 import serving, workloads
    clips = workloads.batch_clips(count=requests, seed=seed)
    # a steady-state server: the same request mix once untimed first, so the
    # first use of each size (solver workspaces, graphs, tile widths) is paid
    # before the timed run
    warm = serving.make_requests(clips, rate=rate, seed=seed, device=dev)
    serving.Server(budget_bytes=120 * 10 ** 9, workers=3, device=dev, solvers=2).run(warm)
    del warm
    torch.cuda.synchronize()
    reqs = serving.make_requests(clips, rate=rate, seed=seed, device=dev)
    srv = serving.Server(budget_bytes=120 * 10 ** 9, workers=3, device=dev, solvers=2)
    done = srv.run(reqs)
    st = serving.summary(done, srv.wall_s)
    solvers = {}
    for r in done:
        solvers[r.solver] = solvers.get(r.solver, 0) + 1
    out = {"requests": len(reqs), "rate_per_s": rate, "p50_ms": st["p50_ms"], "p95_ms": st["p95_ms"],
           "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "voxels_per_s": st["voxels_per_s"],
           "completed": st["completed"], "failed": st["failed"], "wall_s": srv.wall_s, "solvers": solvers,
           "max_batch": srv.max_batch}
    del reqs, done, srv
    torch.cuda.empty_cache()
    return out


def launches_mixed(dec):
    # this library's kernels per decode: temporal Gram (1); right-hand side, realify, W_n split, tensor-core
    # Gram, real scatter (5); tile Cholesky (1); initial solve (2 with the inverse: the two product kernels;
    # 1 otherwise); per sweep: unrealify, residual and its reduction (2), realify, solve, norm ratio, axpy;
    # final unrealify (1); synthesis: per-pixel weights and the harmonics product (2).  With
    # mixed_factor="cusolver", cuSOLVER's kernels are not counted.
    solve = 2 if dec.mixed_factor == "inverse" else 1
    return 1 + 5 + 1 + solve + (6 + solve) * dec.mixed_sweeps + 1 + 2


def batch_measure(dev, local, count, seed, sweeps, warmup, steps, plain_count, eig="bucketed"):
    """Decode ``count`` independent clips of uneven size (batch_clips, seed
    ``seed``) as one batch: ``steps`` timed runs of the BatchDecoder after
    ``warmup`` (graph capture) runs, a 256 MB flush before each; the same
    clips decoded one after another by the stand-alone decoders (mixed, and
    float64); the plain float64 decode of the first ``plain_count`` clips for
    the SNR.  ``eig``: how the BatchDecoder eigen-solves the systems that
    both Cholesky factorisations refuse.  Returns (batch result dict, ms per
    step, voxels per step)."""
    import torch
    from vtem_b200 import batch, fast, workloads
    clips = workloads.batch_clips(count=count, seed=seed)
    t0 = time.perf_counter()
    probs = [batch.encode_clip_problem(c, device=dev) for c in clips]
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    voxels = sum(p.voxels for p in probs)
    spikes = [int(p.tk1.numel()) for p in probs]
    bd = batch.BatchDecoder(probs, streams=8, sweeps=sweeps, graph=True, eig=eig)
    flush = torch.zeros(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    for _ in range(warmup):
        bd.run()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ms, phases = 0.0, np.zeros(3)
    for _ in range(steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bd.run(timing=True)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        phases += np.array(bd.phase_ms)
    clk = clocks.stop()
    solvers = bd.solver_counts()

    def sequential(solver):
        decs = [fast.from_prep(p.prep, p.Wt, p.Mt, rcond=p.rcond, solver=solver, mixed_sweeps=sweeps)
                for p in probs]
        for d, p in zip(decs, probs):
            d.decode(p.tk1, p.tk2, p.ind, p.kappa, p.delta, p.bias, p.T, p.dt, assume_sorted=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for d, p in zip(decs, probs):
            d.decode(p.tk1, p.tk2, p.ind, p.kappa, p.delta, p.bias, p.T, p.dt, assume_sorted=True)
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    seq_mixed = sequential("mixed")
    seq_f64 = sequential("auto")
    step_ms = ms / steps
    plain = plain_sample(clips, probs, bd.outs, dev, plain_count)
    res = {"clips": len(probs), "voxels_per_s": voxels * steps / (ms / 1e3), "ms_per_step": step_ms,
           "config": {"workload": "batch: %d clips, side {16,32,48,64}, 0.05-0.5 s, Mt 3..8, M 2..6, 32..1024 RFs"
                                  % len(probs), "voxels_per_step": voxels, "spikes_min": min(spikes),
                      "spikes_max": max(spikes), "groups": len(bd.groups), "solvers": solvers,
                      "cuda_graphs": bd.use_graph, "graph_error": bd.graph_error, "setup_s": t_setup,
                      "eig": eig, "l2": "256 MB flush between steps"},
           "phases_ms": {"grouped_mixed_solve": phases[0] / steps, "f64_fallbacks": phases[1] / steps,
                         "synthesis": phases[2] / steps},
           "sequential_ms": {"mixed": seq_mixed, "f64": seq_f64},
           "batched_speedup": {"vs_sequential_mixed": seq_mixed / step_ms, "vs_sequential_f64": seq_f64 / step_ms},
           "clips_per_s": len(probs) * steps / (ms / 1e3), "clocks": clk,
           "plain_fp64_sample": plain,
           "vs_plain_fp64": (voxels * steps / (ms / 1e3)) / plain["voxels_per_s"] if plain else None}
    del bd, probs, flush
    torch.cuda.empty_cache()
    return res, step_ms, voxels


def run_batch(args, rank, world, local):
    """Many-clip workload: 256 independent clips of uneven size (seed 2).
    One step = decoding every clip of the batch (mixed precision: grouped
    float32 Cholesky, batched triangular solves and float64 refinement,
    replayed as CUDA graphs; float64 fallbacks on worker threads); compared
    with decoding the same clips one after another with the stand-alone
    decoders (mixed, and float64)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    res, step_ms, voxels = batch_measure(dev, local, args.clips, 2 + rank, args.sweeps, args.warmup, args.steps,
                                         args.plain_sample, eig=args.batch_eig)
    out = {"metric": METRIC + " [batch of %d clips]" % res["clips"], "value": res["voxels_per_s"],
           "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64 (split-bf16 tensor-core Gram, f32 Cholesky, f64 refinement)",
           "data": "synthetic (seeded Dirichlet-bandlimited video)"}
    out.update({k: v for k, v in res.items() if k not in ("voxels_per_s", "ms_per_step", "clips")})
    return out


def plain_sample(clips, probs, outs, dev, count):
    """The plain float64 decode of the reference (analytic n x n Gram,
    eigen-pseudoinverse, synthesis) of the first ``count`` clips, one at a
    time: voxels/s, and the SNR of the batched results against it."""
    import torch
    from vtem_b200 import dirichlet, linalg, vrf, vtdm
    tot_s, tot_vox, snrs = 0.0, 0, []
    for w, p, u in list(zip(clips, probs, outs))[:count]:
        rfSx, rfSy, rfPx, rfPy = vtdm.period_grid(w.Mx, w.My, w.Wx, w.Wy, w.dx, w.dy)
        grid = vrf.vrf_gabor((rfPy, rfPx), dx=rfSx / rfPx, dy=rfSy / rfPy, scale=4)
        Ds = p.prep.Ds
        dirich = grid.compute_dirich_space_fft(Ds, w.Mx, w.My, w.Px, w.Py, 1.0, 1.0, w.Wx, w.Wy)
        Dsw = grid.compute_Dsw(Ds, w.Mx, w.My, np.ones(w.N))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cp = dirichlet.dirichlet(w.N, p.tk1, p.tk2, p.ind, w.kappa, w.delta, w.bias, np.ones(w.N), w.Wt, w.Mt)
        cp.compute_q()
        cp.compute_G(Dsw, lower_only=True)
        cp.d_q = linalg.solve_eq_sym(cp.d_G, cp.d_q, rcond=w.rcond)
        cp.freeG()
        up = cp.reconstruct(dirich, [0, w.T], w.dt)
        torch.cuda.synchronize()
        tot_s += time.perf_counter() - t0
        tot_vox += p.voxels
        up = up.reshape(u.shape)
        rel = float((u - up).norm() / up.norm())
        snrs.append(-20 * math.log10(max(rel, 1e-300)))
        del cp, up
        torch.cuda.empty_cache()
    if not tot_vox:
        return None
    return {"clips": min(count, len(probs)), "voxels_per_s": tot_vox / tot_s, "seconds": tot_s,
            "snr_db_min": min(snrs), "snr_db_median": float(np.median(snrs))}


def run_serve(args, rank, world, local):
    """Serving workload: encode+decode requests sized like the batch clips
    (seed 3), float32 video, Poisson arrivals at 200 req/s (seed 3), 120 GB
    device-memory admission budget, 2 ms ticks with batched solves.  The
    warm-up serves a short trace first; the timed run serves the whole trace
    (latencies are wall-clock, arrival to result on the host).  A bounded
    sample of the same requests is then executed one at a time by the plain
    float64 path of the reference, for its service time and the SNR of the
    served results against it."""
    import torch
    from vtem_b200 import serving, workloads
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    clips = workloads.batch_clips(count=args.requests, seed=3 + rank)
    reqs = serving.make_requests(clips, rate=args.rate, seed=3 + rank, device=dev)
    warm = serving.make_requests(workloads.batch_clips(count=max(args.warmup, 8), seed=1000 + rank),
                                 rate=args.rate, seed=7, device=dev)
    serving.Server(device=dev).run(warm)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    srv = serving.Server(budget_bytes=args.budget_gb * 10 ** 9, workers=args.workers, device=dev,
                         solvers=args.solvers)
    done = srv.run(reqs, keep_result=lambda r: r.rid < args.plain_sample)
    clk = clocks.stop()
    st = serving.summary(done, srv.wall_s)
    solvers = {}
    for r in done:
        solvers[r.solver] = solvers.get(r.solver, 0) + 1
    # plain float64 per-request execution on a bounded sample
    sample = [r for r in sorted(done, key=lambda r: r.rid)][:args.plain_sample]
    plain_s, plain_vox, snrs = 0.0, 0, []
    for r in sample:
        u, sec = serving.plain_fp64(r, dev)
        plain_s += sec
        plain_vox += r.voxels
        rel = float((r.result - u).norm() / u.norm())
        snrs.append(-20 * math.log10(max(rel, 1e-300)))
    h2d = sum(r.video.numel() * 4 for r in done)
    d2h = sum(r.voxels * 8 for r in done if r.state == "done")
    return {"metric": "serving: reconstructed voxels/s and p99 latency (ms)", "value": st["voxels_per_s"],
            "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": len(warm), "ms_per_step": srv.wall_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (bf16x3 projection, split-bf16 Gram, f32 Cholesky, f64 refinement)",
            "data": "synthetic (seeded Dirichlet-bandlimited video, float32 input)",
            "config": {"workload": "serve: %d requests, Poisson %.0f/s (seed 3), batch-clip sizes (seed 3), "
                                   "budget %d GB, tick 2 ms, %d encode workers, %d solver threads"
                                   % (len(reqs), args.rate, args.budget_gb, args.workers, args.solvers)},
            "latency_ms": {"p50": st["p50_ms"], "p95": st["p95_ms"], "p99": st["p99_ms"], "mean": st["mean_ms"]},
            "phases_mean_ms": st["phases_mean_ms"],
            "completed": st["completed"], "failed": st["failed"], "solvers": solvers,
            "batched_solve_calls": srv.batched_solves, "max_batch": srv.max_batch,
            "peak_budget_bytes": srv.peak_bytes,
            "e2e": {"value": st["voxels_per_s"], "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "plain_fp64_sample": {"requests": len(sample), "voxels_per_s": plain_vox / max(plain_s, 1e-9),
                                  "ms_per_request": 1e3 * plain_s / max(len(sample), 1),
                                  "snr_db_min": min(snrs) if snrs else None},
            "clocks": clk}


def launches_per_step(dec):
    # temporal_gram 1, kron_gram 1, kron_rhs 1, solve: chol_pivots 1 + 2 per refinement
    # (cuSOLVER's own kernels not counted), synthesis 2
    if dec.last_solver == "chol":
        solve = 1 + 2 * dec.refine
    else:
        solve = 3
    return 1 + 2 + solve + 2


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def measured_traffic(voxels, kernel):
    """DRAM bytes per synthesis launch from the committed ncu summary of the
    same kernel, scaled to this workload's output size (null when no capture
    of that kernel is committed)."""
    p = os.path.join(ROOT, "profiles", "synth_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        if d.get("kernel") != kernel:
            return None
        return d["dram_bytes"] * voxels / d["voxels"]
    except Exception:
        return None


def run_plain(w, prep, tk1, tk2, ind, u_fast_variants, dev, Nt):
    """The plain float64 path of the reference on the whole clip: analytic
    n x n Gram, eigendecomposition pseudoinverse, synthesis."""
    import torch
    from vtem_b200 import dirichlet, linalg

    out = {}
    try:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cp = dirichlet.dirichlet(w.N, tk1, tk2, ind, w.kappa, w.delta, w.bias, np.ones(w.N), w.Wt, w.Mt)
        cp.compute_q()
        cp.compute_G(prep.Dsw, lower_only=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        cp.d_q, kept = linalg.solve_eq_sym(cp.d_G, cp.d_q, rcond=w.rcond, return_kept=True)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        cp.freeG()
        torch.cuda.empty_cache()
        up = cp.reconstruct(prep.dirich, [0, w.T], w.dt)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        rel = {k: float((v - up).norm() / up.norm()) for k, v in u_fast_variants.items()}
        voxels = Nt * w.Px * w.Py
        out = {"value": voxels / (t3 - t0), "unit": UNIT, "seconds": t3 - t0,
               "stages_s": {"q_G": t1 - t0, "pinv_eigh": t2 - t1, "synthesis": t3 - t2},
               "kept": kept, "n": len(tk1), "rel_l2_vs_plain": rel,
               "snr_db": {k: -20 * math.log10(max(r, 1e-300)) for k, r in rel.items()}}
        del up, cp
        torch.cuda.empty_cache()
    except Exception as e:  # report, do not hide
        out = {"error": repr(e)}
    return out


def run_encode(w, V, dev, reps=9):
    """Encoder stages on the clip, device-timed: the RF projection
    L = dx dy V RF^T in float64 and on the tensor cores (split-bf16 operands,
    fp32 accumulation), and the IAF block scan (float64) on the float64
    projection; the rel. error of the tensor-core projection and how many
    spikes its scan changes."""
    import torch
    from vtem_b200 import ensemble_encode, vrf
    g = w.gabor
    banks = []
    gb = vrf.vrf_gabor((w.Py, w.Px), dx=w.dx, dy=w.dy)
    gb.load_parameters(num_neurons=len(g.h_alpha), h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0,
                       h_ab=g.h_ab, KAPPA=g.KAPPA, h_gain=g.gain)
    banks.append(gb)
    if w.cs is not None:
        c = w.cs
        cb = vrf.vrf_cs((w.Py, w.Px), dx=w.dx, dy=w.dy)
        cb.load_parameters(num_neurons=len(c.h_alpha), h_alpha=c.h_alpha, h_x0=c.h_x0, h_y0=c.h_y0,
                           sigma_center=c.sigma_center, sigma_surround=c.sigma_surround, h_gain=c.gain)
        banks.append(cb)
    bank = vrf.vrf_bank(banks) if len(banks) > 1 else banks[0]

    def timed(fn):
        # median of per-call CUDA-event times after a warm-up call (one slow
        # call, e.g. an allocation, does not move the figure)
        out = fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return out, float(np.median(ts))

    L64, t64 = timed(lambda: bank.filter(V, out_layout="neuron", precision="f64"))
    Ltc, ttc = timed(lambda: bank.filter(V, out_layout="neuron", precision="bf16x3"))
    flop = 2.0 * w.F * w.Px * w.Py * w.N

    def encoder():
        iaf = ensemble_encode.IAF_encode(w.N, w.dt)
        iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_v0=w.v0)
        return iaf

    def scan(L):
        return encoder().encode_blocks(L, block_frames=min(101, w.F + 1), layout="neuron")

    # the public call (overflow checks included) and the scan kernel alone, on one
    # encoder whose state carries from call to call as the reference's does
    enc = encoder()
    bf = min(101, w.F + 1)
    _, tscan = timed(lambda: enc.encode_blocks(L64, block_frames=bf, layout="neuron"))
    # the scan kernel alone: one launch with the first-try spike buffer, no host check
    cap0 = 64 + -(-w.F // ensemble_encode.SMALL_CAP_STRIDE)
    _, tkernel = timed(lambda: enc._launch(L64, 1, w.F, w.N, w.F, bf, cap0, 0, block_rate=0.1))
    sp64 = scan(L64)
    sptc = scan(Ltc)
    n64, ntc = int(sp64.count.sum()), int(sptc.count.sum())
    peaks = load_peaks()
    return {"rf_projection": {"f64_ms": t64, "tensor_core_ms": ttc, "algorithmic_gflop": flop / 1e9,
                              "f64_tflops": flop / t64 / 1e9, "tensor_core_tflops": flop / ttc / 1e9,
                              "tensor_core_frac_of_bf16_peak": 3 * flop / ttc / 1e9 / peaks["bf16_tflops"],
                              "tensor_core_rel_err": float((Ltc - L64).norm() / L64.norm())},
            "iaf_scan": {"ms": tscan, "kernel_ms": tkernel,
                         "chain_floor_ms": w.F * 8.0 / (peaks.get("sm_max_mhz", 1965.0) * 1e3),
                         "bytes_read": 8 * w.F * w.N, "gbs": 8.0 * w.F * w.N / tscan / 1e6,
                         "frac_of_hbm": 8.0 * w.F * w.N / tscan / 1e6 / peaks["hbm_gbs"],
                         "spikes": n64, "near_threshold": int(sp64.near_threshold)},
            "spikes_tensor_core_projection": ntc}


def run_encode_only(args, rank, world, local):
    """Encoder stages alone on the GPU configuration's clip (run_encode)."""
    import torch
    from vtem_b200 import workloads
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = workloads.gpu_scale(seed=rank, frames=args.frames)
    V = w.video(device=dev)
    res = run_encode(w, V, dev, reps=max(1, args.steps))
    res["config"] = {"workload": "encode: 64x64 px, %d samples, 768 Gabor + 256 centre-surround RFs" % w.F}
    return res


def run_synth(args, rank, world, local):
    """Synthesis kernels alone at the GPU configuration's decode shape
    (Mx = My = 6, Mt = 8, 64 x 64 px, ``--frames`` frames) on seeded random
    coefficients: vtb_coeff_synth_rank (weights + harmonics, one call),
    vtb_synth_harmonics and vtb_coeff_basis, each timed ``--steps`` times
    with CUDA events after ``--warmup`` calls, a 256 MB add queued before
    each timed call (the host queues ahead of the device; the video, 328 MB,
    exceeds L2); medians."""
    import torch
    from vtem_b200 import _abi
    from vtem_b200.fast import ellipse_storage_index
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    Mx = My = 6
    Mt, Px, Py, Nt = 8, 64, 64, args.frames
    smap = torch.as_tensor(ellipse_storage_index(Mx, My), device=dev)
    Ks, Kt = int(smap.numel()), 2 * Mt + 1
    rng = np.random.default_rng(rank)
    a = torch.as_tensor(rng.standard_normal(Ks * Kt) + 1j * rng.standard_normal(Ks * Kt), dtype=torch.complex128,
                        device=dev)
    H = torch.empty((Px * Py, Kt), dtype=torch.float64, device=dev)
    u = torch.empty((Nt, Py, Px), dtype=torch.float64, device=dev)
    flush = torch.zeros(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    lib, W, dt = _abi.lib(), 2 * np.pi * 20 / Mt, 1e-4

    def rank_call():
        return lib.vtb_coeff_synth_rank(a.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, Px, Py, Px, Py, H.data_ptr(),
                                        Kt, W, 0.0, dt, Nt, u.data_ptr(), 0, _abi.stream_ptr())

    def harm_call():
        return lib.vtb_synth_harmonics(H.data_ptr(), Kt, Px * Py, Mt, W, 0.0, dt, Nt, u.data_ptr(), 0,
                                       _abi.stream_ptr())

    def basis_call():
        return lib.vtb_coeff_basis(a.data_ptr(), smap.data_ptr(), Ks, Mx, My, Mt, Px, Py, Px, Py, H.data_ptr(), Kt,
                                   _abi.stream_ptr())

    out = {}
    for name, fn in (("synth_rank", rank_call), ("harmonics", harm_call), ("basis", basis_call)):
        for _ in range(args.warmup):
            assert fn() == 0
        ts = []
        for _ in range(args.steps):
            flush.add_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            assert fn() == 0
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        med = float(np.median(ts))
        out[name] = {"median_us": med * 1e3, "min_us": min(ts) * 1e3,
                     "video_write_gbs": Nt * Px * Py * 8 / med / 1e6}
    return {"workload": "synth: Mx=My=6, Mt=8, 64x64 px, %d frames, random coefficients" % Nt, "kernels": out}


def run_stitch(args, rank, world, local):
    """Stitched decode of the GPU configuration's clip through the public
    decode_video: spatial tiles of ``--tile`` pixels (20 % overlap, Hann
    blend) and temporal windows of ``--window`` s (20 % overlap, Hann
    cross-fade), every window of every tile decoded (a) one after another by
    the stand-alone coefficient-space decoder and (b) as one batch (grouped
    tensor-core Grams, batched Cholesky, float64 fallbacks).  Host-API
    timing: spike reads, per-tile preparation and the download of the video
    are inside the timed region."""
    import torch
    from vtem_b200 import vtdm, workloads
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = workloads.gpu_scale(seed=rank, frames=args.frames)
    V, prep, _, _, sp, rd = encode_clip(w, dev)
    store = rd.source
    kw = dict(Mt=w.Mt, spatial_stitching=True, spatial_interval=[args.tile, args.tile], stitching=True,
              stitch_interval=args.window, output_format=2)

    def timed(decoder, reps):
        out = None
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = vtdm.decode_video(store, None, None, 0.0, w.T, w.dt, w.Mx, decoder=decoder, **kw)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return out, float(np.median(ts))

    timed("batch", args.warmup)
    ub, tb = timed("batch", args.steps)
    timed("coeff", 1)
    uc, tc = timed("coeff", args.steps)
    voxels = w.F * w.Px * w.Py
    tiles = vtdm.spatial_tiles(w.Px, w.Py, [args.tile, args.tile], [-0.5, 0.5, -0.5, 0.5], w.dx, w.dy)
    plan = vtdm.temporal_plan(0.0, w.T, w.dt, True, args.window)
    Vh = V.cpu().numpy()
    snr = lambda u: float(-20 * np.log10(np.linalg.norm(u - Vh) / np.linalg.norm(Vh)))
    res = {"metric": METRIC + " [stitched decode_video]", "value": voxels / tb, "unit": UNIT, "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": tb * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64 (batched mixed-precision solves)",
           "data": "synthetic (seeded Dirichlet-bandlimited video)",
           "config": {"workload": "stitch: 64x64 px, %d samples, 768 Gabor + 256 centre-surround RFs, "
                                  "%dx%d px tiles, %.3g s windows" % (w.F, args.tile, args.tile, args.window),
                      "tiles": len(tiles), "windows_per_tile": len(plan.windows),
                      "timing": "host wall clock around decode_video (synchronised)"},
           "sequential_coeff": {"s": tc, "voxels_per_s": voxels / tc},
           "batched_speedup": tc / tb,
           "batch_vs_sequential_rel": float(np.linalg.norm(ub - uc) / np.linalg.norm(uc)),
           "snr_db": {"batch": snr(ub), "sequential": snr(uc)}}
    if not args.no_plain:
        up, tp = timed("plain", 1)
        res["sequential_plain"] = {"s": tp, "voxels_per_s": voxels / tp,
                                   "batch_rel": float(np.linalg.norm(ub - up) / np.linalg.norm(up))}
    return res


def run_rnn(w, prep, tk1, tk2, ind, dev, Nt, steps=2000):
    """The RNN decoder (rnn3, step 1/lambda_max, steps+1 updates) on the
    whole clip: on the coefficient system (one cooperative launch) and on the
    reference's n x n spike Gram, same step and updates; device seconds of
    each (coefficients + synthesis) and the rel-L2 between the videos."""
    import torch
    from vtem_b200 import dirichlet, fast, neural_network
    out = {"steps": steps}
    try:
        inputs = tuple(torch.as_tensor(x, device=dev) for x in (tk1, tk2, ind, w.kappa, w.delta, w.bias))
        dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="auto")
        dec.rnn_coefficients(*inputs, steps=10, assume_sorted=True)       # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a, dta = dec.rnn_coefficients(*inputs, steps=steps, assume_sorted=True)
        u = dec.synthesize(a, w.T, w.dt)
        e1.record()
        torch.cuda.synchronize()
        out["coeff_ms"] = e0.elapsed_time(e1)
        out["dt_alpha"] = dta
        out["coeff_voxels_per_s"] = Nt * w.Px * w.Py / (out["coeff_ms"] / 1e3)
        cp = dirichlet.dirichlet(w.N, tk1, tk2, ind, w.kappa, w.delta, w.bias, np.ones(w.N), w.Wt, w.Mt)
        torch.cuda.synchronize()
        e0.record()
        cp.compute_q()
        cp.compute_G(prep.Dsw)
        cp.d_q = neural_network.rnn3(cp.d_G, cp.d_q, dt=dta, alpha=1.0, steps=steps)
        cp.freeG()
        up = cp.reconstruct(prep.dirich, [0, w.T], w.dt)
        e1.record()
        torch.cuda.synchronize()
        out["plain_ms"] = e0.elapsed_time(e1)
        out["plain_voxels_per_s"] = Nt * w.Px * w.Py / (out["plain_ms"] / 1e3)
        out["rel_l2_coeff_vs_plain"] = float((u - up.reshape(u.shape)).norm() / up.norm())
        out["speedup"] = out["plain_ms"] / out["coeff_ms"]
        del cp, up, u
        torch.cuda.empty_cache()
    except Exception as e:  # report, do not hide
        out["error"] = repr(e)
    return out


# ---------------------------------------------------------------- CPU baseline / reference arm

def load_workloads():
    """``vtem_b200/workloads.py`` loaded by path: the seeded workload
    definitions only (NumPy and torch, no kernels), so that the reference arm
    never imports the ``vtem_b200`` package or loads its library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_vtem_workloads", os.path.join(ROOT, "vtem_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


class HostClip(object):
    """A clip encoded and prepared on the host: spike store contents (block
    counts and block-relative times, as vtem_storage keeps them) and the
    decoder preparation (Ds, phi, Dsw)."""

    def __init__(self, w, block_counts, block_spikes, refresh, Ds, dirich, Dsw, seconds):
        self.w, self.block_counts, self.block_spikes, self.refresh = w, block_counts, block_spikes, refresh
        self.Ds, self.dirich, self.Dsw, self.setup_s = Ds, dirich, Dsw, seconds

    def window(self, t0, t1):
        """Spike intervals of [t0, t1), relative to t0 (read_select_spikes)."""
        from oracle import vtem_oracle as O
        return O.read_select_spikes(self.block_counts, self.block_spikes, self.refresh, np.arange(self.w.N),
                                    [t0, t1])


def reference_encode(w):
    """VTEM_IAF + VTDM_prep of the workload's clip with the reference's own
    kernels compiled for the host (oracle/_ref: gabor/cs RFs, the IAF scan,
    fft2Ds, Ds2fft, filter2rec, put_norm) and NumPy for the library calls the
    reference makes (cuBLAS GEMM for the projection and Dsw, cuFFT); the
    stimulus is the seeded video evaluated by NumPy."""
    from oracle import ref_runner as R
    from oracle import vtem_oracle as O
    t0 = time.perf_counter()
    V = O.bandlimited_video(w.coeffs, w.Mx, w.My, w.Mt, w.Wx, w.Wy, w.Wt, w.Px, w.Py, 1.0, 1.0, w.F, w.dt)
    V *= w.scale
    g, c = w.gabor, w.cs
    rf = [R.gabor(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, w.Px, w.Py, 1.0, 1.0, -0.5, -0.5, g.KAPPA)
          * g.gain[:, None, None]]
    if c is not None:
        rf.append(R.cs(c.h_alpha, c.h_x0, c.h_y0, w.Px, w.Py, 1.0, 1.0, -0.5, -0.5, c.sigma_center,
                       c.sigma_surround) * c.gain[:, None, None])
    rf = np.concatenate(rf, 0)
    L = (w.dx * w.dy) * (V.reshape(w.F, -1) @ rf.reshape(w.N, -1).T)       # vrf.py:291 (cuBLAS)
    del V
    B = min(101, w.F + 1)
    v0, tc = w.v0.copy(), np.zeros(w.N)
    counts, spikes = [], []
    for s, e in O.block_schedule(w.F, B):
        sp, cnt = R.iaf_encode(L[s:e], w.dt, w.kappa, w.bias, w.delta, v0, tc)
        tc[:] = 0.0                                                      # reset_timer, vtem.py:197
        counts.append(cnt)
        spikes.append(np.concatenate(sp))
    del L
    # decoder side: RFs at 4x over one spatial period (vtdm.py:385-435)
    rfSx, rfSy, rfPx, rfPy = O.rf_period_grid(w.Mx, w.My, w.Wx, w.Wy, w.dx, w.dy)
    LPx, LPy = rfPx * 4, rfPy * 4
    fdx, fdy = (rfSx / rfPx) / 4, (rfSy / rfPy) / 4
    Sx, Sy = LPx * fdx, LPy * fdy
    fine = [R.gabor(g.h_alpha, g.h_l, g.h_x0, g.h_y0, g.h_ab, LPx, LPy, Sx, Sy, -Sx / 2, -Sy / 2, g.KAPPA)
            * g.gain[:, None, None]]
    if c is not None:
        fine.append(R.cs(c.h_alpha, c.h_x0, c.h_y0, LPx, LPy, Sx, Sy, -Sx / 2, -Sy / 2, c.sigma_center,
                         c.sigma_surround) * c.gain[:, None, None])
    fine = np.concatenate(fine, 0)
    Ds = R.compute_Ds(fine, w.Mx, w.My, fdx * fdy)
    del fine
    Px1 = int(np.round(Sx / w.dx))
    Py1 = int(np.round(Sy / w.dy))
    dirich = R.dirich_space_fft(Ds, w.Mx, w.My, w.Px, w.Py, Px1, Py1)
    Dsw = R.compute_Dsw(Ds, np.ones(w.N))
    return HostClip(w, counts, spikes, (B - 1) * w.dt, Ds, dirich, Dsw, time.perf_counter() - t0)


def window_decode(clip, t0, window, use_ref):
    """One VTDM window of the clip (vtdm.py:630-652) on the host, every frame
    of the window reconstructed: q, the analytic Gram, the pseudoinverse and
    the reconstruction, by the reference's own kernels (q, G, sq,
    reconstruct; NumPy SVD for CULA's gesvd) when ``use_ref``, else by the
    oracle's NumPy restatement (eigh pseudoinverse, factored reconstruction)
    on all host threads.  The spike read is outside the timing.  Returns
    (voxels, seconds, intervals, frames)."""
    from oracle import vtem_oracle as O
    w = clip.w
    t1, t2, ii = clip.window(t0, t0 + window)
    norm = np.ones(w.N)
    tt = np.arange(0, window, w.dt)
    tt = tt[:int(round(window / w.dt))]
    s = time.perf_counter()
    if use_ref:
        from oracle import ref_runner as R
        q = R.compute_q(t1, t2, ii, w.kappa, w.delta, w.bias, norm)
        G = R.compute_G(t1, t2, ii, clip.Dsw, w.Wt, w.Mt)
        cc = R.solve_eq_sym(G, q, w.rcond)
        R.reconstruct(clip.dirich, t1, t2, cc, tt, ii, norm, w.Mt, w.Wt / w.Mt)
    else:
        O.decode_window(t1, t2, ii, w.kappa, w.delta, w.bias, norm, clip.Dsw, clip.dirich, w.Wt, w.Mt,
                        len(tt) * w.dt, w.dt, rcond=w.rcond, threads=os.cpu_count())
    sec = time.perf_counter() - s
    return len(tt) * w.Px * w.Py, sec, len(t1), len(tt)


def sample_desc(window, intervals, frames, w, kind):
    what = ("reference kernels q/G/sq/reconstruct + NumPy SVD (CULA gesvd)" if kind == "reference" else
            "NumPy restatement: q, analytic G, eigh pseudoinverse, factored reconstruction")
    return ("consecutive %.3g s decode windows of the clip's spikes (%d-%d intervals each), all %d frames x "
            "%dx%d px of each window reconstructed; %s" % (window, min(intervals), max(intervals), frames,
                                                          w.Py, w.Px, what))


def cpu_baseline(clip, windows=3, window=0.04, use_ref=False):
    """The oracle port on consecutive windows of the clip (host threads)."""
    vox, sec, ns = 0, 0.0, []
    for i in range(windows):
        v, s, n, f = window_decode(clip, i * window, window, use_ref)
        vox, sec = vox + v, sec + s
        ns.append(n)
    kind = "reference" if use_ref else "port"
    return {"value": vox / sec, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": kind,
            "sample": sample_desc(window, ns, f, clip.w, kind), "seconds": sec}


def host_clip_from_device(w, prep, rd):
    """The GPU-encoded clip's spike store and preparation as a HostClip."""
    return HostClip(w, [np.asarray(c) for c in rd.source.spike_count], [np.asarray(s) for s in rd.source.spikes],
                    float(rd.source.data["iaf/refresh_interval"]), prep.Ds.cpu().numpy(), prep.dirich.cpu().numpy(),
                    prep.Dsw.cpu().numpy(), 0.0)


def run_reference(args, rank, world):
    """The reference arm: the reference's own kernels compiled for the host
    (oracle/_ref), NumPy for its library calls, all host threads.  The clip
    is encoded and prepared by those kernels before the timed steps; each
    step decodes the next window of the clip (its every frame) as VTDM does
    for one window.  Rank 0 only; the package under test is never imported."""
    if rank != 0:
        return None
    from oracle import ref_runner as R
    if not R.available():
        return {"impl": "reference", "unavailable": "oracle/_ref (the reference's kernels built for the host) "
                                                    "is missing: run python oracle/build_ref.py"}
    W = load_workloads()
    w = W.gpu_scale(seed=0, frames=args.frames)
    clip = reference_encode(w)
    nwin = max(1, int(w.T / args.ref_window))
    secs, vox, ns = [], 0, []
    for i in range(args.warmup + args.steps):
        v, s, n, f = window_decode(clip, (i % nwin) * args.ref_window, args.ref_window, True)
        if i >= args.warmup:
            secs.append(s)
            vox += v
            ns.append(n)
    value = vox / sum(secs)
    desc = sample_desc(args.ref_window, ns, f, w, "reference")
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Dirichlet-bandlimited video)", "config": workload_config(w),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                             "sample": desc, "setup_s": clip.setup_s},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def workload_config(w):
    """The ``config`` object both arms print for the GPU configuration."""
    return {"workload": "gpu: %dx%d px, %d samples (%.3g s, dt=1e-4), Mx=My=%d, Mt=%d, 768 Gabor + 256 "
                        "centre-surround RFs, IAF b~U(2,4) delta~N(0.12,0.012), pinv rcond %g"
                        % (w.Px, w.Py, w.F, w.T, w.Mx, w.Mt, w.rcond),
            "l2": "output 328 MB > L2 and a 256 MB flush between steps"}


def run_cpu_full(args):
    """The whole clip decoded on the host by the oracle's NumPy restatement
    (all host threads), as ONE window, the way the GPU decodes it: q and the
    analytic n x n Gram in full, the eigh pseudoinverse in full, and the
    reconstruction of ``--cpu-frames`` frames spread over the clip,
    extrapolated linearly to all frames (reported as such).  The spikes are
    the reference-kernel encode of the clip (``reference_encode``)."""
    from oracle import vtem_oracle as O
    W = load_workloads()
    w = W.gpu_scale(seed=0, frames=args.frames)
    clip = reference_encode(w)
    t1, t2, ii = clip.window(0.0, w.T)
    norm = np.ones(w.N)
    s0 = time.perf_counter()
    q = O.compute_q(t1, t2, ii, w.kappa, w.delta, w.bias, norm)
    G = O.compute_G_threaded(t1, t2, ii, clip.Dsw, w.Wt, w.Mt)
    s1 = time.perf_counter()
    c, kept = O.solve_eq_sym(G, q, w.rcond)
    s2 = time.perf_counter()
    del G
    tt = np.arange(w.F) * w.dt
    pick = np.linspace(0, w.F - 1, args.cpu_frames).astype(np.int64)
    O.reconstruct_factored_threaded(clip.dirich, t1, t2, c, tt[pick], ii, norm, w.Mt, w.Wt / w.Mt)
    s3 = time.perf_counter()
    rec_full = (s3 - s2) * w.F / len(pick)
    total = (s2 - s0) + rec_full
    voxels = w.F * w.Px * w.Py
    return {"metric": METRIC + " [whole clip on the host, one window]", "value": voxels / total, "unit": UNIT,
            "kind": "port", "cores": os.cpu_count() or 1, "intervals": len(t1), "kept": kept,
            "stages_s": {"q_G": s1 - s0, "pinv_eigh": s2 - s1,
                         "reconstruction_extrapolated": rec_full,
                         "reconstruction_measured": {"frames": len(pick), "seconds": s3 - s2}},
            "seconds_total": total, "encode_setup_s": clip.setup_s, "config": workload_config(w)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=10000)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-rnn", action="store_true")
    ap.add_argument("--rnn-steps", type=int, default=2000)
    ap.add_argument("--sweeps", type=int, default=1)
    ap.add_argument("--workload", default="gpu", choices=["gpu", "batch", "serve", "encode", "stitch", "synth", "cpu-full"])
    ap.add_argument("--tile", type=int, default=48)
    ap.add_argument("--window", type=float, default=0.5)
    ap.add_argument("--clips", type=int, default=256)
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--budget-gb", type=int, default=120)
    ap.add_argument("--workers", type=int, default=3)
    ap.add_argument("--solvers", type=int, default=2)
    ap.add_argument("--plain-sample", type=int, default=8)
    ap.add_argument("--no-serve", action="store_true", help="skip the short serving run of the default line")
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--batch-clips", type=int, default=256,
                    help="clips of the batch run in the default line (0: none)")
    ap.add_argument("--batch-eig", default="bucketed", choices=["bucketed", "threads"],
                    help="eigen-solves of the refused batch systems: padded batches or per worker thread")
    ap.add_argument("--ref-window", type=float, default=0.025,
                    help="decode window (s) of one reference-arm step")
    ap.add_argument("--cpu-frames", type=int, default=40,
                    help="frames reconstructed by --workload cpu-full (the rest extrapolated)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    elif args.workload == "batch":
        res = run_batch(args, rank, world, local)
    elif args.workload == "serve":
        res = run_serve(args, rank, world, local)
    elif args.workload == "encode":
        res = run_encode_only(args, rank, world, local)
    elif args.workload == "stitch":
        res = run_stitch(args, rank, world, local)
    elif args.workload == "synth":
        res = run_synth(args, rank, world, local) if rank == 0 else None
    elif args.workload == "cpu-full":
        res = run_cpu_full(args) if rank == 0 else None
    else:
        res = run_ours(args, rank, world, local)
    if rank == 0 and res is not None:
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
