"""Coefficient-space decoder against the reference decode (GPU).

The coefficient-space path must reproduce the pseudoinverse decode of the
spike Gram (the oracle's restatement of solve_eq_sym + reconstruct) to the
same rel-L2 bar as the plain path, and its Gram M = Phi^H Phi must equal the
explicit product of the spike-by-basis matrix."""
import numpy as np
import pytest
import torch

from oracle import vtem_oracle as O
from vtem_b200 import ensemble_encode, fast, spike_store, vrf, vtdm, vtem, workloads

pytestmark = pytest.mark.gpu


def explicit_phi(tk1, tk2, ind, Ds, norm, Mx, My, Mt, W):
    """Phi[k, (s, m)] = norm conj(Ds[n_k, s]) T_k(m), s over the ellipse."""
    smap = fast.ellipse_storage_index(Mx, My)
    D = Ds.reshape(Ds.shape[0], -1)[:, smap]
    m = np.arange(-Mt, Mt + 1)
    T = np.empty((len(tk1), len(m)), np.complex128)
    for j, mm in enumerate(m):
        if mm == 0:
            T[:, j] = tk2 - tk1
        else:
            T[:, j] = (np.exp(1j * mm * W * tk2) - np.exp(1j * mm * W * tk1)) / (1j * mm * W)
    Phi = (norm[ind][:, None, None] * np.conj(D[ind])[:, :, None] * T[:, None, :]).reshape(len(tk1), -1)
    return Phi


def test_coeff_gram_matches_explicit_phi():
    rng = np.random.default_rng(7)
    N, n, Mx, My, Mt = 11, 400, 3, 2, 3
    W = 2 * np.pi * 20 / Mt
    Ds = rng.standard_normal((N, 2 * My + 1, 2 * Mx + 1)) + 1j * rng.standard_normal((N, 2 * My + 1, 2 * Mx + 1))
    # the coefficients of a real RF: Hermitian (Ds[-m] = conj Ds[m]) and zero outside the ellipse
    Ds = 0.5 * (Ds + np.conj(Ds[:, ::-1, ::-1])) * O.ellipse_mask(Mx, My)[None]
    tk1 = rng.uniform(0, 0.3, n)
    tk2 = tk1 + rng.uniform(0.004, 0.03, n)
    ind = np.sort(rng.integers(0, N, n)).astype(np.int32)
    kap, dl, bia = rng.uniform(0.8, 1.2, N), rng.uniform(0.01, 0.05, N), rng.uniform(1, 3, N)
    norm = rng.uniform(0.5, 1.0, N)
    dec = fast.CoeffDecoder(torch.as_tensor(Ds, device="cuda"), norm, Mx, My, 2 * np.pi * 20, Mt, 8, 8, 8, 8,
                            solver="eig")
    # build W_n, g_n, M, b without solving
    perm, t1, t2, ii = fast.sort_by_neuron(tk1, tk2, ind)
    # keep the device copies alive until the kernel has run (the caching
    # allocator would hand a freed temporary's block to the next one)
    kap_d, dl_d, bia_d = (torch.as_tensor(a, device="cuda") for a in (kap, dl, bia))
    from vtem_b200._abi import call, dptr, stream_ptr
    call("vtb_coeff_temporal_gram", dptr(t1), dptr(t2), dptr(ii), n, N, dptr(kap_d), dptr(dl_d), dptr(bia_d),
         dptr(dec.norm), Mt, W, dptr(dec.Wn), dptr(dec.gn), stream_ptr())
    dec._build_M(stream_ptr())
    Phi = explicit_phi(tk1, tk2, ind, Ds, norm, Mx, My, Mt, W)
    Mref = Phi.conj().T @ Phi
    q = O.compute_q(tk1, tk2, ind, kap, dl, bia, norm)
    bref = Phi.conj().T @ q
    M = dec.M.cpu().numpy().T                       # stored column-major
    assert np.abs(M - Mref).max() <= 1e-12 * np.abs(Mref).max()
    assert np.abs(dec.b.cpu().numpy() - bref).max() <= 1e-12 * np.abs(bref).max()
    # the spike Gram of the reference is Re(Phi Phi^H)
    Dsw = (np.conj(Ds.reshape(N, -1)) @ Ds.reshape(N, -1).T).real * np.outer(norm, norm)
    G = O.compute_G(tk1, tk2, ind, Dsw, 2 * np.pi * 20, Mt)
    assert np.abs((Phi @ Phi.conj().T).real - G).max() <= 1e-12 * np.abs(G).max()


@pytest.fixture(scope="module")
def small_encoded():
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
    return w, store, prep


@pytest.mark.parametrize("solver", ["eig", "chol", "auto"])
def test_coeff_decode_matches_oracle_pinv(small_encoded, solver):
    w, store, prep = small_encoded
    u = vtdm.VTDM(store, None, None, 0.0, w.T, w.dt, w.Mx, Mt=w.Mt, rcond=w.rcond, output_format=2, prep=prep,
                  decoder="coeff", coeff_solver=solver)
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    norm = np.ones(w.N)
    uo, c, q, G, kept = O.decode_window(tk1, tk2, ind, kap, dl, bia, norm, prep.Dsw.cpu().numpy(),
                                        prep.dirich.cpu().numpy(), w.Wt, w.Mt, w.T, w.dt, rcond=w.rcond)
    rel = np.linalg.norm(u - uo) / np.linalg.norm(uo)
    assert rel <= 1e-8, rel


def test_coeff_decode_float32_output(small_encoded):
    w, store, prep = small_encoded
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond)
    u64 = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    u32 = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt, out_dtype=torch.float32)
    err = (u32.double() - u64).norm() / u64.norm()
    assert err < 1e-6


def test_mixed_decoder_matches_float64(small_encoded):
    w, store, prep = small_encoded
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    ref = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="eig").decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    dec0 = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=0)
    u0 = dec0.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=3)
    u = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt)
    assert dec.last_solver == "mixed"
    e0 = ((u0 - ref).norm() / ref.norm()).item()
    e = ((u - ref).norm() / ref.norm()).item()
    # tensor-core Gram alone: >= 40 dB; after float64 refinement: float64-level agreement
    assert e0 < 1e-2, e0
    assert e < 1e-9, (e0, e)
    assert dec.residual_norm(tk1, tk2, ind, kap, dl, bia) < 1e-10


def test_real_form_matches_hermitian_system():
    """The real symmetric form (csrc/realsys.cu) of M a = b has the
    eigenvalues of M and the same solution; the tensor-core Gram scattered
    straight into the real form equals the float64 one to its precision."""
    from vtem_b200._abi import call, dptr, stream_ptr
    rng = np.random.default_rng(11)
    # enough neurons and intervals that M is nonsingular (rank <= N * Kt)
    N, n, Mx, My, Mt = 40, 1500, 3, 2, 3
    W = 2 * np.pi * 20 / Mt
    Ds = rng.standard_normal((N, 2 * My + 1, 2 * Mx + 1)) + 1j * rng.standard_normal((N, 2 * My + 1, 2 * Mx + 1))
    Ds = 0.5 * (Ds + np.conj(Ds[:, ::-1, ::-1])) * O.ellipse_mask(Mx, My)[None]
    tk1 = rng.uniform(0, 0.3, n)
    tk2 = tk1 + rng.uniform(0.004, 0.03, n)
    ind = np.sort(rng.integers(0, N, n)).astype(np.int32)
    kap, dl, bia = (torch.as_tensor(x, device="cuda") for x in
                    (rng.uniform(0.8, 1.2, N), rng.uniform(0.01, 0.05, N), rng.uniform(1, 3, N)))
    dec = fast.CoeffDecoder(torch.as_tensor(Ds, device="cuda"), rng.uniform(0.5, 1.0, N), Mx, My, 2 * np.pi * 20,
                            Mt, 8, 8, 8, 8, solver="mixed")
    t1, t2, ii = (torch.as_tensor(x, device="cuda") for x in (tk1, tk2, ind))
    s = stream_ptr()
    K, NE = dec.K, dec.NE
    call("vtb_coeff_temporal_gram", dptr(t1), dptr(t2), dptr(ii), n, N, dptr(kap), dptr(dl), dptr(bia),
         dptr(dec.norm), Mt, W, dptr(dec.Wn), dptr(dec.gn), s)
    dec._build_M(s)
    call("vtb_coeff_realify", dptr(dec.M), K, K, dptr(dec.Mr), K, 1, s)
    call("vtb_coeff_realify_vec", dptr(dec.b), K, 1, dptr(dec.br), s)
    M = dec.M.cpu().numpy().T
    b = dec.b.cpu().numpy()
    Mr = dec.Mr.cpu().numpy()
    br = dec.br.cpu().numpy()
    assert np.abs(Mr - Mr.T).max() <= 1e-13 * np.abs(Mr).max()
    ev_c = np.linalg.eigvalsh(M)
    ev_r = np.linalg.eigvalsh(Mr)
    assert np.abs(ev_c - ev_r).max() <= 1e-11 * ev_c.max()
    a = np.linalg.solve(M, b)
    x = torch.as_tensor(np.linalg.solve(Mr, br), device="cuda")
    call("vtb_coeff_unrealify_vec", dptr(x), K, 1, dptr(dec.a), 0, s)
    assert np.abs(dec.a.cpu().numpy() - a).max() <= 1e-9 * np.abs(a).max()
    # tensor-core Gram -> real form in float32
    call("vtb_coeff_wn_sym", dptr(dec.Wn), N, dec.Kt, dptr(dec.Rsplit), s)
    call("vtb_tc_gemm_bf16x3_bn", dptr(dec.Lsplit), 2 * dec.npairs, dptr(dec.Rsplit), NE, dec.Kh, dptr(dec.C), dec.ldc,
         1, 0, 1.0, 0, dec._stat_ptr(7), 128, s)
    ld = dec.ld32
    call("vtb_coeff_real_scatter", dptr(dec.C), dec.ldc, dec.Ks, dec.Kt, dptr(dec.Mr32), ld, 0, s)
    M32 = dec.Mr32[:, :K].double().cpu().numpy()
    assert np.abs(M32 - Mr).max() <= 2e-5 * np.abs(Mr).max()
    # float32 Cholesky + solve, then a float64 Cholesky solve, against numpy
    work = dec._workspace(2)
    dec.stat.zero_()
    call("vtb_sym_factor", dptr(dec.Mr32), ld, K, 2, 1e-12, dptr(work), work.numel(), dec._stat_ptr(0),
         dec._stat_ptr(1), s)
    x32 = torch.as_tensor(br, device="cuda")
    call("vtb_sym_potrs", dptr(dec.Mr32), ld, dptr(x32), K, 2, dptr(work), work.numel(), s)
    flag, piv, _, tc_err = dec._read_stat()
    assert flag == 0 and tc_err == 0 and piv[0] > 0
    xr = np.linalg.solve(Mr, br)
    assert np.linalg.norm(x32.cpu().numpy() - xr) <= 1e-2 * np.linalg.norm(xr)
    w1 = dec._workspace(1)
    dec.stat.zero_()
    call("vtb_sym_factor", dptr(dec.Mr), K, K, 1, 1e-12, dptr(w1), w1.numel(), dec._stat_ptr(0), dec._stat_ptr(1), s)
    x64 = torch.as_tensor(br, device="cuda")
    call("vtb_sym_potrs", dptr(dec.Mr), K, dptr(x64), K, 1, dptr(w1), w1.numel(), s)
    assert dec._read_stat()[0] == 0
    assert np.linalg.norm(x64.cpu().numpy() - xr) <= 1e-9 * np.linalg.norm(xr)


def test_coefficient_rnn_matches_spike_rnn(small_encoded):
    """The RNN decoder on the coefficient system gives the reconstruction of
    the reference's rnn3 on the n x n spike Gram (same step, same number of
    updates), and the float64 oracle's rnn3 + reconstruction."""
    from vtem_b200 import dirichlet, neural_network
    w, store, prep = small_encoded
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    steps = 300
    dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond)
    a, dta = dec.rnn_coefficients(tk1, tk2, ind, kap, dl, bia, steps=steps)
    u = dec.synthesize(a, w.T, w.dt)
    norm = np.ones(w.N)
    cp = dirichlet.dirichlet(w.N, tk1, tk2, ind, kap, dl, bia, norm, w.Wt, w.Mt)
    cp.compute_q()
    cp.compute_G(prep.Dsw)
    G = cp.d_G
    lam = torch.linalg.eigvalsh(G)[-1].item()
    # the power-iteration estimate of lambda_max (shared by G and M) is a
    # lower bound close to it: a stable step below 2 / lambda_max
    assert 0.5 < 1.0 / (lam * dta) <= 1.0 + 1e-9
    cp.d_q = neural_network.rnn3(G, cp.d_q, dt=dta, alpha=1.0, steps=steps)
    up = cp.reconstruct(prep.dirich, [0, w.T], w.dt)
    rel = ((u - up.reshape(u.shape)).norm() / up.norm()).item()
    assert rel < 1e-9, rel
    # oracle: rnn3 and the reference's reconstruction formula in float64 numpy
    q = O.compute_q(tk1, tk2, ind, kap, dl, bia, norm)
    Go = O.compute_G(tk1, tk2, ind, prep.Dsw.cpu().numpy(), w.Wt, w.Mt)
    co = O.rnn3(Go, q, dta, 1.0, steps)
    t = np.arange(0, w.T, w.dt)
    uo = O.reconstruct_factored(prep.dirich.cpu().numpy(), tk1, tk2, co.ravel(), t, ind, norm, w.Mt, w.Wt / w.Mt)
    rel_o = np.linalg.norm(u.cpu().numpy().ravel() - uo.ravel()) / np.linalg.norm(uo)
    assert rel_o < 1e-8, rel_o


def test_decode_to_host_matches_device_decode(small_encoded):
    """The overlapped end-to-end decode into pinned host memory returns the
    device decode's video (frame ranges synthesised separately)."""
    w, store, prep = small_encoded
    rd = spike_store.vtem_storage_read(store)
    rd.read_vrf_type()
    rd.read_num_neurons()
    rd.select_neurons([-0.5, 0.5, -0.5, 0.5])
    tk1, tk2, ind, kap, dl, bia, sig = rd.read_select_spikes([0.0, w.T])
    dec = fast.from_prep(prep, w.Wt, w.Mt, rcond=w.rcond, solver="mixed", mixed_sweeps=2)
    u = dec.decode(tk1, tk2, ind, kap, dl, bia, w.T, w.dt).cpu()
    h = torch.empty(u.shape, dtype=torch.float64).pin_memory()
    dec.decode_to_host(tk1, tk2, ind, kap, dl, bia, w.T, w.dt, h, chunks=5)
    torch.cuda.synchronize()
    assert ((h - u).norm() / u.norm()).item() < 1e-13


@pytest.mark.parametrize("K", [1, 17, 32, 33, 64, 65, 100, 257, 1000, 1921])
def test_flag_solve_matches_cusolver(K):
    """The multi-CTA flag hand-off solve (vtb_sym_potrs_flags) against
    cuSOLVER's spotrs on the same float32 factor and against a float64 solve,
    for sizes that leave partial 32- and 64-row blocks; twice in a row (the
    flags are reset per call)."""
    from vtem_b200._abi import call, dptr, lib, stream_ptr
    rng = np.random.default_rng(K)
    Q, _ = np.linalg.qr(rng.standard_normal((K, K)))
    A = (Q * rng.uniform(1.0, 100.0, K)) @ Q.T
    A = 0.5 * (A + A.T)
    M = torch.as_tensor(A, dtype=torch.float32, device="cuda").contiguous()
    s = stream_ptr()
    nb = np.zeros(1, np.int64)
    call("vtb_sym_workspace", K, 2, nb.ctypes.data)
    work = torch.empty(int(nb[0]), dtype=torch.uint8, device="cuda")
    stat = torch.zeros(4, dtype=torch.float64, device="cuda")
    call("vtb_sym_factor", dptr(M), K, K, 2, 1e-12, dptr(work), work.numel(), stat.data_ptr(), stat.data_ptr() + 8, s)
    dinv = torch.empty(int(lib().vtb_sym_dinv_floats(K)), dtype=torch.float32, device="cuda")
    fw = torch.empty(int(lib().vtb_sym_potrs_flags_bytes(K)), dtype=torch.uint8, device="cuda")
    call("vtb_sym_dinv", dptr(M), K, K, dptr(dinv), s)
    for _ in range(2):
        b = rng.standard_normal(K)
        x1 = torch.as_tensor(b, device="cuda")
        x2 = torch.as_tensor(b, device="cuda")
        call("vtb_sym_potrs_flags", dptr(M), K, dptr(dinv), K, dptr(x1), dptr(fw), fw.numel(), stat.data_ptr(), s)
        call("vtb_sym_potrs", dptr(M), K, dptr(x2), K, 2, dptr(work), work.numel(), s)
        flag = int(stat[:1].view(torch.int32)[0].item())
        assert flag == 0, flag
        xr = np.linalg.solve(A, b)
        a1, a2 = x1.cpu().numpy(), x2.cpu().numpy()
        assert np.linalg.norm(a1 - a2) <= 1e-4 * np.linalg.norm(xr)
        assert np.linalg.norm(a1 - xr) <= 1e-4 * np.linalg.norm(xr)
