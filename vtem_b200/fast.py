"""Coefficient-space decoder: the reference's pseudoinverse decode without the
spike-by-spike Gram.

``CoeffDecoder.decode`` returns the same video as ``dirichlet.compute_q`` +
``compute_G`` + ``linalg.solve_eq_sym`` + ``dirichlet.reconstruct``
(vtem/dirichlet.py:55-189, vtem/utils/linalg.py:591-631) for one window:
with Phi[k,(s,m)] = norm conj(Ds[n_k,s]) T_k(m), G = Phi Phi^H and the
reconstruction coefficients a = Phi^H G^+ q = M^+ b, M = Phi^H Phi.  M is
K x K (K = ellipse size * (2Mt+1), 1921 for Mx=My=6, Mt=8) whatever the
number of spikes, built from per-neuron Kronecker factors on the device; the
n x n Gram (5 GB at 25k spikes) and its O(n^3) eigendecomposition are never
formed.  See csrc/coeff.cu for the kernels.

Real form: the coefficients of a real video are Hermitian-symmetric, so the
K x K Hermitian system is solved as the equivalent REAL symmetric system
(csrc/realsys.cu; same eigenvalues, a quarter of the arithmetic).

Solver choice: ``"eig"`` applies the reference's truncation rule to the
eigenvalues of M (identical subspace); ``"chol"`` factorises M by float64
Cholesky and is used (under ``"auto"``) only when the pseudoinverse cannot
truncate: the window must have at least K intervals, and the spread of the
squared Cholesky pivots, a lower bound of the condition number that can
underestimate it by orders of magnitude on badly sampled windows, must stay
below 1 / (rcond * CHOL_MARGIN); otherwise the eigen-pseudoinverse runs.
``"mixed"`` builds M on the tensor cores from split-bf16 operands (fp32
accumulation), factorises it by float32 Cholesky (this library's tile
Cholesky, which by default, ``mixed_factor="inverse"``, also forms L^-1 in
the same launch so that every solve is two matrix-vector products;
``"tiles"``: the factor alone and block substitutions; ``"cusolver"``:
cuSOLVER's spotrf), and recovers float64
accuracy with ``mixed_sweeps`` refinement sweeps against the exact float64
residual Phi^H (q - Phi a), applied through the Kronecker factors without
forming M in float64.  A mixed solve is accepted when the factorisation
succeeds, its pivots pass the same test, and the refinement contracts
(estimated remaining error below MIXED_TOL); otherwise the float64 path
decodes the window.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _abi, autotune
from ._abi import VTB_NOT_CONVERGED, VtbError, call, dptr, lib, stream_ptr
from .dirichlet import sort_by_neuron

F64 = torch.float64
C128 = torch.complex128

# Cholesky is trusted only when the pivot spread is this far below 1/rcond
# (a window with pivot spread 1.6e5 had condition number 1.2e10).
CHOL_MARGIN = 1e4
# accepted mixed solves: estimated relative error left after the last sweep
MIXED_TOL = 1e-8


def ellipse_storage_index(Mx, My):
    """Flat Ds storage indices (row My-my, column mx+Mx) of the spatial
    ellipse mx^2 My^2 + my^2 Mx^2 <= Mx^2 My^2 (vrf.py:1331), ascending."""
    idx = []
    Kx = 2 * Mx + 1
    for r in range(2 * My + 1):
        my = My - r
        for c in range(Kx):
            mx = c - Mx
            if mx * mx * My * My + my * my * Mx * Mx <= Mx * Mx * My * My:
                idx.append(r * Kx + c)
    return np.array(idx, np.int32)


def coefficient_count(Mx, My, Mt):
    """K = (ellipse size) * (2 Mt + 1), the size of the coefficient system."""
    return len(ellipse_storage_index(Mx, My)) * (2 * int(Mt) + 1)


class CoeffDecoder(object):
    def __init__(self, Ds, h_norm, Mx, My, Wt, Mt, decPx, decPy, Px1, Py1, rcond=1e-8, solver="auto", refine=0,
                 device="cuda", mixed_sweeps=2, mixed_factor="inverse", synth="harmonics"):
        self.Mx, self.My, self.Mt = int(Mx), int(My), int(Mt)
        self.Wt = float(Wt)
        self.W = self.Wt / self.Mt
        self.decPx, self.decPy, self.Px1, self.Py1 = int(decPx), int(decPy), int(Px1), int(Py1)
        self.rcond = float(rcond)
        self.solver = solver
        self.refine = int(refine)
        Ds = Ds.to(device=device, dtype=C128).contiguous()
        self.Ds = Ds
        self._dsw = None
        self.N = Ds.shape[0]
        self.Kfull = Ds[0].numel()
        self.smap = torch.as_tensor(ellipse_storage_index(self.Mx, self.My), device=device)
        self.Ks = int(self.smap.numel())
        self.Kt = 2 * self.Mt + 1
        self.K = self.Ks * self.Kt
        self.norm = torch.as_tensor(np.asarray(h_norm, np.float64), device=device)
        self.d = torch.empty((self.N, self.Ks), dtype=C128, device=device)
        call("vtb_coeff_pack", dptr(Ds), self.N, self.Kfull, dptr(self.smap), self.Ks, dptr(self.norm),
             dptr(self.d), stream_ptr())
        self.Wn = torch.empty((self.N, self.Kt, self.Kt), dtype=C128, device=device)
        self.gn = torch.empty((self.N, self.Kt), dtype=C128, device=device)
        self.M = torch.empty((self.K, self.K), dtype=C128, device=device)
        self.b = torch.empty((self.K,), dtype=C128, device=device)
        self.a = torch.empty((self.K,), dtype=C128, device=device)
        self.kept = torch.zeros(1, dtype=torch.int32, device=device)
        # real form: Mr (float64), right-hand side, iterate, correction
        self.Mr = torch.empty((self.K, self.K), dtype=F64, device=device)
        self.br = torch.empty((self.K,), dtype=F64, device=device)
        self.xr = torch.empty((self.K,), dtype=F64, device=device)
        self.rr = torch.empty((self.K,), dtype=F64, device=device)
        # status words read once per solve: [flag (int32), min pivot^2, max
        # pivot^2, sweep correction ratios x4, tensor-core error (int32)]
        self.stat = torch.zeros(8, dtype=F64, device=device)
        self.last_ratios = []
        self._work = {}
        self.last_solver = None
        self.last_pivots = (0.0, 0.0)
        self.mixed_sweeps = int(mixed_sweeps)
        if mixed_factor not in ("inverse", "tiles", "cusolver"):
            raise ValueError("mixed_factor must be 'inverse', 'tiles' or 'cusolver'")
        self.mixed_factor = mixed_factor
        if synth not in ("harmonics", "fused"):
            raise ValueError("synth must be 'harmonics' or 'fused'")
        self.synth = synth
        # (start, end) CUDA events that synthesize() records on the current
        # stream around its launches, for timing the synthesis alone
        self.synth_events = None
        self.last_residual = None
        self.last_status = {}
        if solver == "mixed":
            self._init_mixed(device)

    # ------------------------------------------------------------ mixed
    def _init_mixed(self, device):
        iu = np.triu_indices(self.Ks)
        self.ps = torch.as_tensor(iu[0].astype(np.int32), device=device)
        self.ps2 = torch.as_tensor(iu[1].astype(np.int32), device=device)
        self.npairs = int(self.ps.numel())
        from . import tc
        # Gram operands: [hi | lo] over the neurons (Kh = N padded to the
        # GEMM's k-block), rows (pair, re/im) and (upper temporal entry, re/im)
        self.Kh = tc.padded_k(self.N)
        self.NE = self.Kt * (self.Kt + 1)
        self.ldc = (self.NE + 3) // 4 * 4   # 16-byte rows: the GEMM stores C with tensor stores
        self.Lsplit = torch.empty((2 * self.npairs, 2 * self.Kh), dtype=torch.bfloat16, device=device)
        call("vtb_coeff_lhs_sym", dptr(self.d), self.N, self.Ks, dptr(self.ps), dptr(self.ps2), self.npairs,
             dptr(self.Lsplit), stream_ptr())
        self.Rsplit = torch.empty((self.NE, 2 * self.Kh), dtype=torch.bfloat16, device=device)
        self.C = torch.empty((2 * self.npairs, self.ldc), dtype=torch.float32, device=device)
        self.gres = torch.empty((self.N, self.Kt), dtype=C128, device=device)
        self.r = torch.empty((self.K,), dtype=C128, device=device)
        # float32 real system, rows padded to 16 bytes (the tile Cholesky copies 16-byte chunks)
        self.ld32 = (self.K + 3) // 4 * 4
        self.Mr32 = torch.empty((self.K, self.ld32), dtype=torch.float32, device=device)
        # the tile Cholesky's diagonal-tile inverses and flag scratch
        self._cdinv = torch.empty(int(lib().vtb_chol_dinv_floats(self.K)), dtype=torch.float32, device=device)
        self._cwork = torch.empty(int(lib().vtb_chol_work_bytes(self.K)), dtype=torch.uint8, device=device)
        if self.mixed_factor == "inverse":
            self._clinv = torch.empty(int(lib().vtb_chol_inverse_floats(self.K)), dtype=torch.float32, device=device)
            # product-solve scratch: partial sums and tickets (zeroed once; every solve leaves it zeroed)
            self._cy = torch.zeros(int(lib().vtb_chol_solve_inverse_bytes(self.K)), dtype=torch.uint8, device=device)

    def set_norm(self, h_norm):
        """Per-neuron weights norm (vtem/vtdm.py:634-638, 1/(kappa sigma) for
        random-threshold encoders): repacks d = norm * Ds and the operands
        derived from it."""
        dev = self.M.device
        self.norm = torch.as_tensor(np.asarray(h_norm, np.float64), device=dev).contiguous()
        call("vtb_coeff_pack", dptr(self.Ds), self.N, self.Kfull, dptr(self.smap), self.Ks, dptr(self.norm),
             dptr(self.d), stream_ptr())
        self._dsw = None
        if self.solver == "mixed":
            call("vtb_coeff_lhs_sym", dptr(self.d), self.N, self.Ks, dptr(self.ps), dptr(self.ps2), self.npairs,
                 dptr(self.Lsplit), stream_ptr())

    def _workspace(self, mode):
        """Workspace of the real-form solver: mode 0 eigen, 1 float64
        Cholesky, 2 float32 Cholesky."""
        if mode not in self._work:
            nb = np.zeros(1, np.int64)
            call("vtb_sym_workspace", self.K, mode, nb.ctypes.data)
            self._work[mode] = torch.empty(int(nb[0]), dtype=torch.uint8, device=self.M.device)
        return self._work[mode]

    def _stat_ptr(self, i):
        return self.stat.data_ptr() + 8 * i

    def _read_stat(self):
        """(flag, (min, max) squared pivots, sweep ratios, tensor-core error): one synchronising read."""
        h = self.stat.cpu().numpy()
        iv = h.view(np.int32)
        return int(iv[0]), (float(h[1]), float(h[2])), [float(x) for x in h[3:7]], int(iv[14])

    def coefficients(self, tk1, tk2, neuron_ind, kappa, delta, bias, assume_sorted=False):
        """Reconstruction coefficients a[(s, m)] (K complex) of one window.
        ``assume_sorted`` skips the (synchronising) check that the intervals
        are grouped by neuron, for device-resident inputs already sorted."""
        if assume_sorted:
            ind = neuron_ind
        else:
            perm, tk1, tk2, ind = sort_by_neuron(tk1, tk2, neuron_ind)
        n = int(tk1.numel())
        if n == 0:
            raise ValueError("no spikes to decode")
        dev = self.M.device
        kap = torch.as_tensor(np.asarray(kappa, np.float64), device=dev) if not isinstance(kappa, torch.Tensor) else kappa
        dl = torch.as_tensor(np.asarray(delta, np.float64), device=dev) if not isinstance(delta, torch.Tensor) else delta
        bi = torch.as_tensor(np.asarray(bias, np.float64), device=dev) if not isinstance(bias, torch.Tensor) else bias
        s = stream_ptr()
        call("vtb_coeff_temporal_gram", dptr(tk1), dptr(tk2), dptr(ind), n, self.N, dptr(kap), dptr(dl), dptr(bi),
             dptr(self.norm), self.Mt, self.W, dptr(self.Wn), dptr(self.gn), s)
        if self.solver in ("auto", "mixed") and n < self.K:
            # fewer intervals than coefficients: the reference's n x n system is
            # the smaller one (its pseudoinverse, then a = Phi^H c)
            self._solve_spike_space(s, (tk1, tk2, ind, n, kap, dl, bi))
        elif self.solver == "mixed":
            self._solve_mixed(s, (tk1, tk2, ind, n, kap, dl, bi))
        else:
            self._solve(s, n)
        return self.a

    def _solve_spike_space(self, s, spikes):
        tk1, tk2, ind, n, kap, dl, bi = spikes
        dev = self.M.device
        if self._dsw is None:
            self._dsw = torch.empty((self.N, self.N), dtype=torch.float64, device=dev)
            call("vtb_dsw", dptr(self.Ds), self.N, self.Kfull, dptr(self.norm), dptr(self._dsw), self.N, s)
        G = torch.empty((n, n), dtype=torch.float64, device=dev)
        q = torch.empty((n,), dtype=torch.float64, device=dev)
        call("vtb_compute_q", dptr(tk1), dptr(tk2), dptr(ind), n, dptr(kap), dptr(dl), dptr(bi), dptr(self.norm),
             dptr(q), s)
        call("vtb_compute_G", dptr(tk1), dptr(tk2), dptr(ind), n, self.Wt, self.Mt, dptr(self._dsw), self.N, 0.0, 1,
             dptr(G), n, s)
        nb = np.zeros(1, np.int64)
        call("vtb_solve_eq_sym_workspace", n, nb.ctypes.data)
        work = torch.empty(int(nb[0]), dtype=torch.uint8, device=dev)
        c = torch.empty((n,), dtype=torch.float64, device=dev)
        call("vtb_solve_eq_sym", dptr(G), n, dptr(q), dptr(c), n, self.rcond, dptr(work), int(nb[0]),
             dptr(self.kept), s)
        call("vtb_coeff_from_spike_weights", dptr(tk1), dptr(tk2), dptr(ind), n, self.N, dptr(c), self.Mt, self.W,
             dptr(self.d), self.Ks, dptr(self.gn), dptr(self.a), s)
        self.last_solver = "spike-space eig"

    def _solve_mixed(self, s, spikes):
        tk1, tk2, ind, n, kap, dl, bi = spikes
        K, NE = self.K, self.NE
        self.stat.zero_()
        # the right-hand side runs on a side stream beside the Gram, the
        # scatter and the factorisation, which it does not feed
        main = torch.cuda.current_stream(self.M.device)
        side = self._side_stream()
        forked = torch.cuda.Event()
        forked.record(main)
        side.wait_event(forked)
        call("vtb_coeff_rhs", dptr(self.d), self.N, self.Ks, dptr(self.gn), self.Kt, dptr(self.b), side.cuda_stream)
        call("vtb_coeff_realify_vec", dptr(self.b), K, 1, dptr(self.br), side.cuda_stream)
        rhs_done = torch.cuda.Event()
        rhs_done.record(side)
        call("vtb_coeff_wn_sym", dptr(self.Wn), self.N, self.Kt, dptr(self.Rsplit), s)
        autotune.gemm_bf16_tuned(dptr(self.Lsplit), 2 * self.npairs, dptr(self.Rsplit), NE, self.Kh, dptr(self.C),
                                 self.ldc, 1, 0, 1.0, 0, self._stat_ptr(7), s, x3=True)
        ld = self.ld32
        call("vtb_coeff_real_scatter", dptr(self.C), self.ldc, self.Ks, self.Kt, dptr(self.Mr32), ld, 0, s)
        if self.mixed_factor == "inverse":
            # float32 tile Cholesky and L^-1 (one cooperative launch), solves by two products
            call("vtb_chol_factor_inverse", dptr(self.Mr32), ld, K, dptr(self._cdinv), dptr(self._clinv),
                 dptr(self._cwork), self._cwork.numel(), self._stat_ptr(0), self._stat_ptr(1),
                 self.rcond * CHOL_MARGIN, s)
            solve = lambda x: call("vtb_chol_solve_inverse", dptr(self._clinv), K, dptr(x), dptr(self._cy),
                                   self._cy.numel(), s)
        elif self.mixed_factor == "tiles":
            # float32 tile Cholesky (one cooperative launch) and cluster solves
            call("vtb_chol_factor", dptr(self.Mr32), ld, K, dptr(self._cdinv), dptr(self._cwork),
                 self._cwork.numel(), self._stat_ptr(0), self._stat_ptr(1), self.rcond * CHOL_MARGIN, s)
            solve = lambda x: call("vtb_chol_solve", dptr(self.Mr32), ld, dptr(self._cdinv), K, dptr(x), s)
        else:
            work = self._workspace(2)
            call("vtb_sym_factor", dptr(self.Mr32), ld, K, 2, self.rcond * CHOL_MARGIN, dptr(work), work.numel(),
                 self._stat_ptr(0), self._stat_ptr(1), s)
            solve = self._mixed_solver(s, work)
        main.wait_event(rhs_done)
        self.xr.copy_(self.br)
        solve(self.xr)
        for i in range(self.mixed_sweeps):
            call("vtb_coeff_unrealify_vec", dptr(self.xr), K, 1, dptr(self.a), 0, s)
            call("vtb_coeff_residual", dptr(tk1), dptr(tk2), dptr(ind), n, self.N, dptr(kap), dptr(dl), dptr(bi),
                 dptr(self.norm), self.Mt, self.W, dptr(self.d), self.Ks, dptr(self.a), dptr(self.gres),
                 dptr(self.r), s)
            call("vtb_coeff_realify_vec", dptr(self.r), K, 1, dptr(self.rr), s)
            solve(self.rr)
            call("vtb_norm_ratio", dptr(self.rr), dptr(self.xr), K, self._stat_ptr(3 + min(i, 3)), s)
            call("vtb_daxpy1", dptr(self.xr), dptr(self.rr), K, s)
        call("vtb_coeff_unrealify_vec", dptr(self.xr), K, 1, dptr(self.a), 0, s)
        # work that uses the mixed solution is queued before the acceptance
        # read, so the GPU keeps running while the host waits for the status
        spec = getattr(self, "_speculate", None)
        if spec is not None:
            spec()
        flag, piv, ratios, tc_err = self._read_stat()
        self.last_pivots = piv
        self.last_ratios = ratios[:min(self.mixed_sweeps, 4)]
        self.last_status = {"factor_flag": flag, "tensor_core_status": tc_err}
        if tc_err != 0 or flag != 0 or not self._mixed_converged(self.last_ratios):
            # a tensor-core or factorisation wait ran out, the pseudoinverse
            # might truncate, or float32 is not enough: float64 path
            self.solver = "auto"
            try:
                self._solve(s, n)
            finally:
                self.solver = "mixed"
            self.last_solver = "mixed->" + self.last_solver
            return
        self.last_solver = "mixed"
        self._spec_valid = True

    def _side_stream(self):
        """A second stream on the decoder's device for work that overlaps
        the main chain of a decode."""
        st = getattr(self, "_side", None)
        if st is None:
            st = self._side = torch.cuda.Stream(device=self.M.device)
        return st

    def _mixed_solver(self, s, work):
        """The solve with the float32 factor in Mr32: the multi-CTA flag
        hand-off solve (diagonal-block inverses formed here, once per
        factor), or cuSOLVER's spotrs where its CTAs cannot all be resident.
        A wait that runs out sets the factor's flag, which sends the window
        to the float64 path."""
        K = self.K
        if getattr(self, "_flag_work", None) is None:
            dev = self.M.device
            self._dinv = torch.empty(int(lib().vtb_sym_dinv_floats(K)), dtype=torch.float32, device=dev)
            self._flag_work = torch.empty(int(lib().vtb_sym_potrs_flags_bytes(K)), dtype=torch.uint8, device=dev)
            self._flags_ok = (K + 63) // 64 <= torch.cuda.get_device_properties(dev).multi_processor_count
        if not self._flags_ok:
            return lambda x: call("vtb_sym_potrs", dptr(self.Mr32), self.ld32, dptr(x), K, 2, dptr(work), work.numel(),
                                  s)
        call("vtb_sym_dinv", dptr(self.Mr32), self.ld32, K, dptr(self._dinv), s)
        return lambda x: call("vtb_sym_potrs_flags", dptr(self.Mr32), self.ld32, dptr(self._dinv), K, dptr(x),
                              dptr(self._flag_work), self._flag_work.numel(), self._stat_ptr(0), s)

    @staticmethod
    def _mixed_converged(r):
        """Refinement acceptance from the relative sizes of the sweeps'
        corrections: with two or more sweeps the last must shrink and the
        error it leaves (about r_last^2 / r_prev) must be below MIXED_TOL;
        with one sweep its correction alone must be below sqrt(MIXED_TOL)."""
        if not r:
            return True
        if len(r) == 1:
            return r[0] <= MIXED_TOL ** 0.5
        a, b = r[-2], r[-1]
        if b == 0.0:
            return True
        return b < 0.5 * a and b * b / a <= MIXED_TOL

    def residual_norm(self, tk1, tk2, neuron_ind, kappa, delta, bias):
        """||Phi^H (q - Phi a)|| / ||Phi^H q|| of the current coefficients."""
        perm, tk1, tk2, ind = sort_by_neuron(tk1, tk2, neuron_ind)
        dev = self.M.device
        kap, dl, bi = (torch.as_tensor(np.asarray(x, np.float64), device=dev) if not isinstance(x, torch.Tensor)
                       else x for x in (kappa, delta, bias))
        gres = torch.empty((self.N, self.Kt), dtype=C128, device=dev)
        r = torch.empty((self.K,), dtype=C128, device=dev)
        s = stream_ptr()
        call("vtb_coeff_residual", dptr(tk1), dptr(tk2), dptr(ind), int(tk1.numel()), self.N, dptr(kap), dptr(dl),
             dptr(bi), dptr(self.norm), self.Mt, self.W, dptr(self.d), self.Ks, dptr(self.a), dptr(gres), dptr(r), s)
        a0 = self.a.clone()
        self.a.zero_()
        r0 = torch.empty_like(r)
        call("vtb_coeff_residual", dptr(tk1), dptr(tk2), dptr(ind), int(tk1.numel()), self.N, dptr(kap), dptr(dl),
             dptr(bi), dptr(self.norm), self.Mt, self.W, dptr(self.d), self.Ks, dptr(self.a), dptr(gres), dptr(r0), s)
        self.a.copy_(a0)
        return float(r.norm() / r0.norm())

    def gram_error(self):
        """||M_tc - M||_F / ||M||_F of the last mixed solve: the tensor-core
        Gram (split-bf16 operands, fp32 accumulation) scattered into its real
        form again, against the float64 real system built from the same
        temporal Grams.  Overwrites the float64 system buffers (M, Mr)."""
        if self.solver != "mixed":
            raise ValueError("gram_error needs the mixed decoder")
        s = stream_ptr()
        K = self.K
        mtc = torch.empty((K, K), dtype=torch.float32, device=self.M.device)
        call("vtb_coeff_real_scatter", dptr(self.C), self.ldc, self.Ks, self.Kt, dptr(mtc), K, 0, s)
        self._build_real(s)
        return float((mtc.double() - self.Mr).norm() / self.Mr.norm())

    def _build_M(self, s):
        call("vtb_coeff_gram", dptr(self.d), self.N, self.Ks, dptr(self.Wn), dptr(self.gn), self.Kt, dptr(self.M),
             self.K, dptr(self.b), s)

    def _solve(self, s, n=None):
        """Float64 solve in real form: Cholesky (accepted by the pivot test)
        and/or the eigen-pseudoinverse, by solver mode."""
        modes = {"eig": [0], "chol": [1], "auto": [1, 0]}[self.solver]
        if self.solver == "auto" and n is not None and n < self.K:
            modes = [0]          # fewer intervals than unknowns: M is singular
        K = self.K
        self._build_M(s)
        call("vtb_coeff_realify_vec", dptr(self.b), K, 1, dptr(self.br), s)
        for i, mode in enumerate(modes):
            call("vtb_coeff_realify", dptr(self.M), K, K, dptr(self.Mr), K, 1, s)
            work = self._workspace(mode)
            if mode == 1:
                self.stat.zero_()
                call("vtb_sym_factor", dptr(self.Mr), K, K, 1, self.rcond * CHOL_MARGIN, dptr(work), work.numel(),
                     self._stat_ptr(0), self._stat_ptr(1), s)
                self.xr.copy_(self.br)
                call("vtb_sym_potrs", dptr(self.Mr), K, dptr(self.xr), K, 1, dptr(work), work.numel(), s)
                flag, piv, _, _ = self._read_stat()
                self.last_pivots = piv
                if flag == 0:
                    call("vtb_coeff_unrealify_vec", dptr(self.xr), K, 1, dptr(self.a), 0, s)
                    self.kept.fill_(-1)
                    self.last_solver = "chol"
                    return
                if i + 1 < len(modes):
                    continue
                raise VtbError("vtb_sym_factor", VTB_NOT_CONVERGED)
            rng = np.zeros(2, np.float64)
            call("vtb_sym_pinv", dptr(self.Mr), K, dptr(self.br), dptr(self.xr), K, self.rcond, dptr(work),
                 work.numel(), dptr(self.kept), rng.ctypes.data, s)
            call("vtb_coeff_unrealify_vec", dptr(self.xr), K, 1, dptr(self.a), 0, s)
            self.last_pivots = (float(rng[0]), float(rng[1]))
            self.last_solver = "eig"
            return

    def lambda_max(self, iters=40):
        """Largest eigenvalue of the float64 real system Mr (that of the
        spike Gram G = Phi Phi^H as well) by power iteration from a fixed
        start; Mr must be built (``_build_real``)."""
        v = torch.ones(self.K, dtype=F64, device=self.Mr.device)
        lam = torch.zeros((), dtype=F64, device=v.device)
        for _ in range(iters):
            w = torch.mv(self.Mr, v)
            lam = torch.dot(v, w) / torch.dot(v, v)
            v = w / w.norm()
        return float(lam)

    def _build_real(self, s):
        """Float64 M, b and their real forms Mr, br."""
        self._build_M(s)
        call("vtb_coeff_realify_vec", dptr(self.b), self.K, 1, dptr(self.br), s)
        call("vtb_coeff_realify", dptr(self.M), self.K, self.K, dptr(self.Mr), self.K, 1, s)

    def rnn_coefficients(self, tk1, tk2, neuron_ind, kappa, delta, bias, dt_alpha=None, steps=4000,
                         assume_sorted=False):
        """Reconstruction coefficients of the RNN decoder (rnn3,
        vtem/neural_network.py:15-99: steps+1 gradient-flow updates from
        c = 0 with step dt*alpha) run on the coefficient system: the same
        iterates mapped by a = Phi^H c.  ``dt_alpha`` None takes
        1 / lambda_max (power iteration).  Returns (a, dt_alpha)."""
        if assume_sorted:
            ind = neuron_ind
        else:
            perm, tk1, tk2, ind = sort_by_neuron(tk1, tk2, neuron_ind)
        n = int(tk1.numel())
        if n == 0:
            raise ValueError("no spikes to decode")
        dev = self.M.device
        kap, dl, bi = (torch.as_tensor(np.asarray(x, np.float64), device=dev) if not isinstance(x, torch.Tensor)
                       else x for x in (kappa, delta, bias))
        s = stream_ptr()
        call("vtb_coeff_temporal_gram", dptr(tk1), dptr(tk2), dptr(ind), n, self.N, dptr(kap), dptr(dl), dptr(bi),
             dptr(self.norm), self.Mt, self.W, dptr(self.Wn), dptr(self.gn), s)
        self._build_real(s)
        if dt_alpha is None:
            dt_alpha = 1.0 / self.lambda_max()
        bar = torch.zeros(4, dtype=torch.int32, device=dev)
        call("vtb_rnn_coeff", dptr(self.Mr), self.K, dptr(self.br), dptr(self.xr), dptr(self.rr), self.K,
             float(dt_alpha), int(steps), dptr(bar), s)
        call("vtb_coeff_unrealify_vec", dptr(self.xr), self.K, 1, dptr(self.a), 0, s)
        if int(bar[2].item()) != 0:
            raise VtbError("vtb_rnn_coeff", _abi.VTB_TIMEOUT)
        self.last_solver = "rnn"
        return self.a, float(dt_alpha)

    def _harmonic_weights(self, a, s):
        """Per-pixel weights H (P x Kt) of the coefficients a for the
        rank-Kt synthesis (vtb_coeff_basis), or None when the fused kernel
        serves this decoder (synth="fused", or Kt beyond 21)."""
        if self.synth != "harmonics" or self.Kt > 21:
            return None
        P = self.decPx * self.decPy
        if getattr(self, "_H", None) is None or self._H.shape[0] != P:
            self._H = torch.empty((P, self.Kt), dtype=F64, device=self.M.device)
        call("vtb_coeff_basis", dptr(a), dptr(self.smap), self.Ks, self.Mx, self.My, self.Mt, self.decPx, self.decPy,
             self.Px1, self.Py1, dptr(self._H), self.Kt, s)
        return self._H

    def synthesize(self, a, T, dt, t0=0.0, out=None, out_dtype=F64):
        """Video (Nt, decPy, decPx) at t = t0 + arange(0, T, dt)."""
        Nt = len(np.arange(0, T, dt))
        dev = self.M.device
        if out is None:
            out = torch.empty((Nt, self.decPy, self.decPx), dtype=out_dtype, device=dev)
        ev = self.synth_events
        if ev is not None:
            ev[0].record()
        if self.synth == "harmonics" and self.Kt <= 21:
            # weights and harmonics in one call (the second kernel launched programmatically)
            P = self.decPx * self.decPy
            if getattr(self, "_H", None) is None or self._H.shape[0] != P:
                self._H = torch.empty((P, self.Kt), dtype=F64, device=dev)
            call("vtb_coeff_synth_rank", dptr(a), dptr(self.smap), self.Ks, self.Mx, self.My, self.Mt, self.decPx,
                 self.decPy, self.Px1, self.Py1, dptr(self._H), self.Kt, self.W, float(t0), float(dt), Nt, dptr(out),
                 int(out.dtype == torch.float32), stream_ptr())
            if ev is not None:
                ev[1].record()
            return out
        # the fused kernel (2My+1 <= 13) needs no expansion buffer
        A = None if 2 * self.My + 1 <= 13 else torch.empty((Nt, self.Ks), dtype=C128, device=dev)
        call("vtb_coeff_synthesize", dptr(a), dptr(self.smap), self.Ks, self.Mx, self.My, self.Mt, self.W, float(t0),
             float(dt), Nt, self.decPx, self.decPy, self.Px1, self.Py1, dptr(A), dptr(out),
             int(out.dtype == torch.float32), stream_ptr())
        if ev is not None:
            ev[1].record()
        return out

    def decode(self, tk1, tk2, neuron_ind, kappa, delta, bias, T, dt, out=None, out_dtype=F64,
               assume_sorted=False):
        """The window's video (Nt, decPy, decPx) at t = arange(0, T, dt).
        With the mixed solver the synthesis of the mixed solution is queued
        before its acceptance is read and done again only if the window falls
        back to float64."""
        res = {}

        def speculate():
            res["u"] = self.synthesize(self.a, T, dt, out=out, out_dtype=out_dtype)

        self._speculate = speculate
        self._spec_valid = False
        try:
            a = self.coefficients(tk1, tk2, neuron_ind, kappa, delta, bias, assume_sorted=assume_sorted)
        finally:
            self._speculate = None
        if self._spec_valid and "u" in res:
            return res["u"]
        return self.synthesize(a, T, dt, out=out, out_dtype=out_dtype)


    def decode_to_host(self, tk1, tk2, neuron_ind, kappa, delta, bias, T, dt, host_out, chunks=8,
                       assume_sorted=False):
        """Decode into ``host_out`` (pinned host tensor (Nt, decPy, decPx)):
        the synthesis runs in ``chunks`` frame ranges on the current stream
        and each finished range is copied to the host on a copy stream, so
        the download of one range overlaps the synthesis of the next.  The
        current stream waits for the last copy (synchronise it, or an event
        recorded on it, before reading ``host_out``)."""
        a = self.coefficients(tk1, tk2, neuron_ind, kappa, delta, bias, assume_sorted=assume_sorted)
        Nt = int(host_out.shape[0])
        if tuple(host_out.shape) != (Nt, self.decPy, self.decPx) or not host_out.is_pinned():
            raise ValueError("host_out must be a pinned (Nt, decPy, decPx) tensor")
        f32 = host_out.dtype == torch.float32
        dev = self.M.device
        key = (Nt, host_out.dtype)
        if getattr(self, "_e2e_key", None) != key:
            self._e2e_out = torch.empty(host_out.shape, dtype=host_out.dtype, device=dev)
            self._e2e_key = key
            self._copy_stream = torch.cuda.Stream(device=dev)
        out = self._e2e_out
        main = torch.cuda.current_stream(dev)
        cs = self._copy_stream
        bounds = np.linspace(0, Nt, max(1, int(chunks)) + 1).astype(np.int64)
        H = self._harmonic_weights(a, main.cuda_stream)
        A = None if H is not None or 2 * self.My + 1 <= 13 else torch.empty((Nt, self.Ks), dtype=C128, device=dev)
        for f0, f1 in zip(bounds[:-1], bounds[1:]):
            if f1 <= f0:
                continue
            if H is not None:
                call("vtb_synth_harmonics", dptr(H), self.Kt, self.decPx * self.decPy, self.Mt, self.W,
                     float(f0 * dt), float(dt), int(f1 - f0), dptr(out[f0:f1]), int(f32), main.cuda_stream)
            else:
                call("vtb_coeff_synthesize", dptr(a), dptr(self.smap), self.Ks, self.Mx, self.My, self.Mt, self.W,
                     float(f0 * dt), float(dt), int(f1 - f0), self.decPx, self.decPy, self.Px1, self.Py1, dptr(A),
                     dptr(out[f0:f1]), int(f32), main.cuda_stream)
            ev = torch.cuda.Event()
            ev.record(main)
            cs.wait_event(ev)
            with torch.cuda.stream(cs):
                host_out[f0:f1].copy_(out[f0:f1], non_blocking=True)
        done = torch.cuda.Event()
        done.record(cs)
        main.wait_event(done)
        return host_out


def from_prep(prep, Wt, Mt, rcond=1e-8, solver="auto", refine=0, mixed_sweeps=2, mixed_factor="inverse",
              synth="harmonics"):
    """A :class:`CoeffDecoder` on the output of ``vtdm.VTDM_prep``."""
    return CoeffDecoder(prep.Ds, prep.h_norm, prep.Mx, prep.My, Wt, Mt, prep.decPx, prep.decPy, prep.Px1, prep.Py1,
                        rcond=rcond, solver=solver, refine=refine, mixed_sweeps=mixed_sweeps,
                        mixed_factor=mixed_factor, synth=synth)
