"""The float32 tile Cholesky and cluster solves of the mixed decoder, and the
bounded device waits of every kernel that waits on another CTA (GPU).

vtb_chol_factor / vtb_chol_solve (and vtb_chol_factor_inverse /
vtb_chol_solve_inverse, which form L^-1 during the factorisation and solve
by two matrix-vector products) replace cuSOLVER's spotrf / spotrs in the
solve of the coefficient system (vtem/utils/linalg.py:591-631 as called at
vtem/vtdm.py:645-648): checked against float64 NumPy on random symmetric
positive definite matrices of sizes that exercise one tile, ragged tiles and
the GPU configuration's K = 1921.  A wait limit of one poll
(vtb_set_wait_limit) makes the waits between CTAs run out: the calls must
report it and return, later calls must work, and the decoder must fall back
to its float64 path with a correct result."""
import numpy as np
import pytest
import torch

from vtem_b200 import _abi, fast
from vtem_b200._abi import call, dptr, lib, stream_ptr

pytestmark = pytest.mark.gpu


def spd(K, cond, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((K, K)))
    lam = np.geomspace(1.0, 1.0 / cond, K)
    A = (Q * lam) @ Q.T
    return 0.5 * (A + A.T)


def factor(A32, rcond=1e-12):
    K = A32.shape[0]
    dinv = torch.empty(int(lib().vtb_chol_dinv_floats(K)), dtype=torch.float32, device="cuda")
    work = torch.empty(int(lib().vtb_chol_work_bytes(K)), dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    piv = torch.zeros(2, dtype=torch.float64, device="cuda")
    call("vtb_chol_factor", dptr(A32), K, K, dptr(dinv), dptr(work), work.numel(), dptr(status), dptr(piv), rcond,
         stream_ptr())
    torch.cuda.synchronize()
    return dinv, int(status.item()), piv.cpu().numpy()


@pytest.mark.parametrize("K", [40, 64, 130, 257, 1921])
def test_chol_factor_and_solve_match_float64(K):
    A = spd(K, 1e3, K)
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()     # symmetric: layout-free
    dinv, status, piv = factor(A32)
    assert status == 0
    L = np.tril(A32.cpu().numpy().astype(np.float64).T)                           # column-major factor
    Lref = np.linalg.cholesky(A)
    assert np.linalg.norm(L - Lref) / np.linalg.norm(Lref) < 1e-4
    # pivots: squared diagonal of L over the K real rows (padding excluded)
    d2 = np.diag(Lref) ** 2
    assert abs(piv[0] - d2.min()) <= 1e-3 * d2.min() and abs(piv[1] - d2.max()) <= 1e-3 * d2.max()
    # diagonal-tile inverses
    T = (K + 63) // 64
    D = dinv.cpu().numpy().reshape(T, 64, 64)
    for k in range(T):
        r0, r1 = 64 * k, min(K, 64 * k + 64)
        Dk = D[k][: r1 - r0, : r1 - r0]                                           # row-major tile
        ref = np.linalg.inv(Lref[r0:r1, r0:r1])
        assert np.linalg.norm(Dk - ref) / np.linalg.norm(ref) < 1e-3
    # solves: x = A^-1 b to float32 accuracy times the condition number
    rng = np.random.default_rng(1)
    for _ in range(2):                                                            # the same factor twice
        b = rng.standard_normal(K)
        x = torch.as_tensor(b, device="cuda")
        call("vtb_chol_solve", dptr(A32), K, dptr(dinv), K, dptr(x), stream_ptr())
        torch.cuda.synchronize()
        xref = np.linalg.solve(A, b)
        assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-3
    assert lib().vtb_chol_solve_cluster() in (8, 16)


def factor_inverse(A32, rcond=1e-12):
    K = A32.shape[0]
    dinv = torch.empty(int(lib().vtb_chol_dinv_floats(K)), dtype=torch.float32, device="cuda")
    linv = torch.full((int(lib().vtb_chol_inverse_floats(K)),), float("nan"), dtype=torch.float32, device="cuda")
    work = torch.empty(int(lib().vtb_chol_work_bytes(K)), dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    piv = torch.zeros(2, dtype=torch.float64, device="cuda")
    call("vtb_chol_factor_inverse", dptr(A32), K, K, dptr(dinv), dptr(linv), dptr(work), work.numel(), dptr(status),
         dptr(piv), rcond, stream_ptr())
    torch.cuda.synchronize()
    return dinv, linv, int(status.item()), piv.cpu().numpy()


def unpack_inverse(linv, K):
    T = (K + 63) // 64
    X = np.zeros((64 * T, 64 * T))
    t = linv.cpu().numpy().astype(np.float64).reshape(-1, 64, 64)
    for i in range(T):
        for j in range(i + 1):
            X[64 * i:64 * i + 64, 64 * j:64 * j + 64] = t[i * (i + 1) // 2 + j]              # row-major tiles
    return X[:K, :K]


@pytest.mark.parametrize("K", [40, 100, 130, 257, 1921])
def test_chol_factor_inverse_and_product_solve(K):
    """The factor formed with L^-1 equals the plain factor bit for bit (same
    task arithmetic), L^-1 matches float64 NumPy, and the two-product solve
    x = L^-T L^-1 b solves A x = b."""
    A = spd(K, 1e3, K + 1)
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()
    A32b = A32.clone()
    dinv0, status0, piv0 = factor(A32b)
    dinv, linv, status, piv = factor_inverse(A32)
    assert status == 0 and status0 == 0
    assert torch.equal(torch.tril(A32.T), torch.tril(A32b.T))
    assert np.array_equal(piv, piv0)
    assert torch.equal(dinv, dinv0)
    Lref = np.linalg.cholesky(A)
    X = unpack_inverse(linv, K)
    Xref = np.linalg.inv(Lref)
    assert np.isfinite(X).all()
    assert np.linalg.norm(X - Xref) / np.linalg.norm(Xref) < 1e-3
    assert np.abs(np.triu(X, 1)).max() == 0.0                                     # exact zeros above
    work = torch.zeros(int(lib().vtb_chol_solve_inverse_bytes(K)), dtype=torch.uint8, device="cuda")
    rng = np.random.default_rng(2)
    bs = [rng.standard_normal(K), rng.standard_normal(K)]
    outs = []
    for b in bs + [bs[0]]:
        x = torch.as_tensor(b, device="cuda")
        call("vtb_chol_solve_inverse", dptr(linv), K, dptr(x), dptr(work), work.numel(), stream_ptr())
        torch.cuda.synchronize()
        xref = np.linalg.solve(A, b)
        assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-3
        outs.append(x.cpu().numpy())
    assert np.array_equal(outs[0], outs[2])                                       # fixed summation order
    T = (K + 63) // 64
    tickets = work[-8 * T:].view(torch.int32)
    assert int(tickets.abs().sum().item()) == 0                                   # left zeroed


def test_chol_factor_inverse_wait_limit_runs_out():
    K = 1921
    A = spd(K, 1e2, 8)
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()
    with _abi.wait_limit(1):
        _, _, status, _ = factor_inverse(A32.clone())
    assert status == 3
    _, linv, status, _ = factor_inverse(A32)
    assert status == 0
    X = unpack_inverse(linv, K)
    assert np.linalg.norm(X @ np.linalg.cholesky(A) - np.eye(K)) / np.sqrt(K) < 1e-4


def test_chol_flags_bad_pivot_and_spread():
    K = 200
    A = spd(K, 10.0, 3)
    A[150, 150] = -1.0                                                            # not positive definite
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()
    _, status, _ = factor(A32)
    assert status == 1
    A = np.diag(np.geomspace(1.0, 1e-6, K))                                      # pivots = the diagonal
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()
    _, status, piv = factor(A32, rcond=1e-4)
    assert status == 2 and piv[1] / piv[0] * 1e-4 >= 1.0
    _, status, _ = factor(torch.as_tensor(A.astype(np.float32), device="cuda").contiguous(), rcond=1e-7)
    assert status == 0


def test_chol_wait_limit_runs_out_and_recovers():
    K = 1921
    A = spd(K, 1e2, 5)
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()
    with _abi.wait_limit(1):
        _, status, _ = factor(A32.clone())
    assert status == 3                                                           # VTB_TIMEOUT path: flagged
    _, status, _ = factor(A32)
    assert status == 0                                                           # default limit again
    L = np.tril(A32.cpu().numpy().astype(np.float64).T)
    assert np.linalg.norm(L @ L.T - A) / np.linalg.norm(A) < 1e-5


def test_flag_solve_wait_limit_runs_out():
    """The flag hand-off triangular solve (vtb_sym_potrs_flags) reports a
    wait that ran out in its err word and returns."""
    K = 1921
    A = spd(K, 1e2, 6)
    A32 = torch.as_tensor(A.astype(np.float32), device="cuda").contiguous()
    nb = np.zeros(1, np.int64)
    call("vtb_sym_workspace", K, 2, nb.ctypes.data)
    work = torch.empty(int(nb[0]), dtype=torch.uint8, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("vtb_sym_factor", dptr(A32), K, K, 2, 1e-12, dptr(work), work.numel(), dptr(flag), None, stream_ptr())
    dinv = torch.empty(int(lib().vtb_sym_dinv_floats(K)), dtype=torch.float32, device="cuda")
    call("vtb_sym_dinv", dptr(A32), K, K, dptr(dinv), stream_ptr())
    fw = torch.empty(int(lib().vtb_sym_potrs_flags_bytes(K)), dtype=torch.uint8, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = torch.ones(K, dtype=torch.float64, device="cuda")
    with _abi.wait_limit(1):
        call("vtb_sym_potrs_flags", dptr(A32), K, dptr(dinv), K, dptr(x), dptr(fw), fw.numel(), dptr(err),
             stream_ptr())
        torch.cuda.synchronize()
    assert int(err.item()) == 3
    err.zero_()
    x = torch.ones(K, dtype=torch.float64, device="cuda")
    call("vtb_sym_potrs_flags", dptr(A32), K, dptr(dinv), K, dptr(x), dptr(fw), fw.numel(), dptr(err), stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    xref = np.linalg.solve(A, np.ones(K))
    assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-3


def test_rnn_grid_barrier_wait_limit_runs_out():
    K = 1921
    A = spd(K, 1e2, 7)
    Mr = torch.as_tensor(A, device="cuda").contiguous()
    br = torch.ones(K, dtype=torch.float64, device="cuda")
    x = torch.empty(K, dtype=torch.float64, device="cuda")
    xt = torch.empty_like(x)
    bar = torch.zeros(4, dtype=torch.int32, device="cuda")
    with _abi.wait_limit(1):
        call("vtb_rnn_coeff", dptr(Mr), K, dptr(br), dptr(x), dptr(xt), K, 0.5, 50, dptr(bar), stream_ptr())
        torch.cuda.synchronize()
    assert int(bar[2].item()) != 0
    call("vtb_rnn_coeff", dptr(Mr), K, dptr(br), dptr(x), dptr(xt), K, 0.5, 50, dptr(bar), stream_ptr())
    torch.cuda.synchronize()
    assert int(bar[2].item()) == 0


def test_tensor_core_gemm_wait_limit_runs_out():
    """tcgen05 GEMM: a CTA whose mbarrier wait runs out reports VTB_TIMEOUT,
    drains its issued TMA loads and MMAs, frees its tensor memory and
    returns; the next launch is exact again."""
    from vtem_b200 import tc
    M, N, K = 512, 256, 1024
    g = torch.Generator(device="cuda").manual_seed(0)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.empty(M, N, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    with _abi.wait_limit(1):
        call("vtb_tc_gemm_bf16", dptr(A), M, dptr(B), N, K, dptr(C), N, 1, 0, 1.0, 0, dptr(err), stream_ptr())
        torch.cuda.synchronize()
    assert int(err.item()) == _abi.VTB_TIMEOUT
    err.zero_()
    call("vtb_tc_gemm_bf16", dptr(A), M, dptr(B), N, K, dptr(C), N, 1, 0, 1.0, 0, dptr(err), stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.float() @ B.float().T
    assert (C - ref).abs().max().item() <= 1e-3 * ref.abs().max().item()


def _small_window():
    from vtem_b200 import ensemble_encode, spike_store, vrf, vtdm, vtem, workloads
    w = workloads.small()
    V = w.video(device="cuda")
    g = w.gabor
    rf = vrf.vrf_gabor((w.Py, w.Px), dx=w.dx, dy=w.dy)
    rf.load_parameters(num_neurons=w.N, h_alpha=g.h_alpha, h_l=g.h_l, h_x0=g.h_x0, h_y0=g.h_y0, h_ab=g.h_ab,
                       KAPPA=g.KAPPA, h_gain=g.gain)
    iaf = ensemble_encode.IAF_encode(w.N, w.dt)
    iaf.load_parameters(h_kappa=w.kappa, h_bias=w.bias, h_delta=w.delta, h_v0=w.v0)
    store = vtem.VTEM_IAF(V, None, w.Wt, rf, w.Wx, w.Wy, dx=w.dx, dy=w.dy, fps=1.0 / w.dt, npinput=True, iaf=iaf)
    prep = vtdm.VTDM_prep(store, None, None, w.Mx, w.My)
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    return w, prep, rd.read_select_spikes([0.0, w.T])


def test_mixed_decoder_tiles_match_cusolver_and_f64():
    w, prep, (tk1, tk2, ind, kap, dl, bia, sig) = _small_window()
    ref = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="eig").decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    for factor_kind in ("inverse", "tiles", "cusolver"):
        dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=3,
                             mixed_factor=factor_kind)
        u = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
        assert dec.last_solver == "mixed", (factor_kind, dec.last_solver, dec.last_ratios, dec.last_status)
        e = ((u - ref).norm() / ref.norm()).item()
        assert e < 1e-9, (factor_kind, e)


def test_mixed_decoder_falls_back_when_waits_run_out():
    w, prep, (tk1, tk2, ind, kap, dl, bia, sig) = _small_window()
    ref = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="eig").decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=1)
    dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)            # tile-width tuning happens outside the limit
    with _abi.wait_limit(1):
        u = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    assert dec.last_solver.startswith("mixed->"), dec.last_solver
    assert dec.last_status["factor_flag"] == 3 or dec.last_status["tensor_core_status"] == _abi.VTB_TIMEOUT
    assert ((u - ref).norm() / ref.norm()).item() < 1e-8
    u = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)                        # default limit: mixed again
    assert dec.last_solver == "mixed"
    assert ((u - ref).norm() / ref.norm()).item() < 1e-6
