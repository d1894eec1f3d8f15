"""Batched decoding of uneven clips (GPU): every clip of the batch equals its
stand-alone decode, and the whole-clip device pairing equals the reference's
spike reader."""
import numpy as np
import pytest
import torch

from oracle import vtem_oracle as O
from vtem_b200 import batch, ensemble_encode, fast, spike_store, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problems():
    clips = workloads.batch_clips(count=256, seed=2)
    # short clips with few RFs; two (M, Mt) groups of three clips each form
    # batched Cholesky groups, two more clips are groups of one
    small = [c for c in clips if c.F <= 2500 and c.N <= 400]
    keys = {}
    for c in small:
        keys.setdefault((c.Mx, c.Mt), []).append(c)
    groups = sorted(keys.values(), key=len, reverse=True)
    pick = groups[0][:3] + groups[1][:3] + [g[0] for g in groups[2:4]]
    assert len(pick) == 8
    return [batch.encode_clip_problem(c) for c in pick]


@pytest.mark.parametrize("eig", ["threads", "bucketed"])
def test_batch_equals_alone(problems, eig):
    """Every clip of the grouped mixed-precision batch equals its stand-alone
    mixed decode, and both equal the reference's pseudoinverse semantics
    (eigen path), with the refused systems eigen-solved on the worker
    threads or in padded batches; replaying the captured graphs gives the
    same videos."""
    bd = batch.BatchDecoder(problems, streams=4, sweeps=2, graph=True, eig=eig)
    outs = [o.clone() for o in bd.run()]
    torch.cuda.synchronize()
    assert bd.graph_error is None, bd.graph_error
    for p, u, db in zip(problems, outs, bd.decs):
        d = fast.from_prep(p.prep, p.Wt, p.Mt, rcond=p.rcond, solver="mixed", mixed_sweeps=2)
        ua = d.decode(p.tk1, p.tk2, p.ind, p.kappa, p.delta, p.bias, p.T, p.dt)
        rel = ((u - ua).norm() / ua.norm()).item()
        assert rel < 1e-8, (rel, db.last_solver, d.last_solver)
        de = fast.from_prep(p.prep, p.Wt, p.Mt, rcond=p.rcond, solver="eig")
        ue = de.decode(p.tk1, p.tk2, p.ind, p.kappa, p.delta, p.bias, p.T, p.dt)
        assert ((u - ue).norm() / ue.norm()).item() < 1e-8, db.last_solver
    outs2 = bd.run()
    torch.cuda.synchronize()
    for a, b in zip(outs, outs2):
        assert ((a - b).norm() / b.norm()).item() < 1e-12
    bd.close()


def test_batch_eager_equals_graph(problems):
    bg = batch.BatchDecoder(problems, streams=4, sweeps=1, graph=True)
    be = batch.BatchDecoder(problems, streams=4, sweeps=1, graph=False)
    ug = [o.clone() for o in bg.run()]
    ue = be.run()
    torch.cuda.synchronize()
    for a, b in zip(ug, ue):
        assert ((a - b).norm() / b.norm()).item() < 1e-12
    bg.close()
    be.close()


def test_device_pairs_match_reader():
    rng = np.random.default_rng(9)
    N, F = 12, 1234
    L = rng.standard_normal((F, N)) * 0.3
    e = ensemble_encode.IAF_encode(N, 1e-4)
    e.load_parameters(h_kappa=np.ones(N), h_bias=np.full(N, 3.0), h_delta=np.full(N, 0.01),
                      h_v0=rng.uniform(0, 0.01, N))
    sp = e.encode_blocks(L, block_frames=101)
    T = F * 1e-4
    tk1, tk2, ind = spike_store.device_pairs(sp, T)
    times, steps, cnt = sp.to_host_lists()
    bc, bs = [], []
    for b in range(len(range(0, F, 100))):
        c = np.array([np.sum(s // 100 == b) for s in steps], np.int32)
        bc.append(c)
        bs.append(np.concatenate([t[s // 100 == b] for t, s in zip(times, steps)]))
    r1, r2, ri = O.read_select_spikes(bc, bs, 100 * 1e-4, np.arange(N), [0.0, T])
    assert np.array_equal(tk1.cpu().numpy(), r1)
    assert np.array_equal(tk2.cpu().numpy(), r2)
    assert np.array_equal(ind.cpu().numpy(), ri)


def test_pinv_batched_equals_single():
    """Batched eigen-pseudoinverse (rank-deficient and full-rank Hermitian
    systems of one size) equals the single-system mode 0 solve."""
    from vtem_b200._abi import call, dptr, lib, stream_ptr
    rng = np.random.default_rng(11)
    K, B = 72, 5
    Ms, bs = [], []
    for z in range(B):
        r = K if z % 2 else K // 2 + 3 * z          # rank-deficient for even z
        X = rng.standard_normal((K, r)) + 1j * rng.standard_normal((K, r))
        Ms.append(X @ X.conj().T)
        bs.append(rng.standard_normal(K) + 1j * rng.standard_normal(K))
    dev = torch.device("cuda")
    # column-major storage of Hermitian M is its conjugate transpose row-major
    Mb = torch.as_tensor(np.stack([m.T for m in Ms]), device=dev).contiguous()
    bb = torch.as_tensor(np.stack(bs), device=dev)
    ab = torch.empty_like(bb)
    nb = np.zeros(1, np.int64)
    call("vtb_herm_pinv_batched_workspace", K, B, nb.ctypes.data)
    work = torch.empty(int(nb[0]), dtype=torch.uint8, device=dev)
    kept = torch.empty(B, dtype=torch.int32, device=dev)
    infos = torch.empty(B, dtype=torch.int32, device=dev)
    rcond = 1e-8
    call("vtb_herm_pinv_batched", dptr(Mb), dptr(bb), dptr(ab), K, B, rcond, dptr(work), int(nb[0]), dptr(kept),
         dptr(infos), stream_ptr())
    torch.cuda.synchronize()
    assert infos.cpu().tolist() == [0] * B
    for z in range(B):
        M1 = torch.as_tensor(Ms[z].T.copy(), device=dev)
        a1 = torch.empty(K, dtype=torch.complex128, device=dev)
        call("vtb_herm_solve_workspace", K, 0, nb.ctypes.data)
        w1 = torch.empty(int(nb[0]), dtype=torch.uint8, device=dev)
        k1 = torch.zeros(1, dtype=torch.int32, device=dev)
        piv = np.zeros(2)
        st = lib().vtb_herm_solve(dptr(M1), K, dptr(bb[z]), dptr(a1), K, rcond, 0, 0, dptr(w1), w1.numel(),
                                  dptr(k1), piv.ctypes.data, stream_ptr())
        assert st == 0
        torch.cuda.synchronize()
        assert int(kept[z]) == int(k1[0])
        rel = ((ab[z] - a1).norm() / a1.norm()).item()
        assert rel < 1e-10, (z, rel)
        # the truncated solution in numpy's pseudoinverse semantics
        w, V = np.linalg.eigh(Ms[z])
        keep = np.abs(w) > rcond * np.abs(w).max()
        ref = V[:, keep] @ ((V[:, keep].conj().T @ bs[z]) / w[keep])
        assert np.linalg.norm(ab[z].cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-8


def test_pinv_bucketed_equals_single():
    """Eigen-pseudoinverses of systems of different sizes, padded into one
    batched call, equal each system's stand-alone vtb_sym_pinv (same kept
    count, same solution), full-rank and rank-deficient alike."""
    from vtem_b200._abi import call, dptr, stream_ptr

    class Sys(object):
        pass

    rng = np.random.default_rng(5)
    dev = torch.device("cuda")
    systems = []
    # full rank (r > K, well conditioned) and rank-deficient (r < K) systems
    for K, r in ((61, 80), (55, 30), (49, 70), (45, 20), (23, 40)):
        X = rng.standard_normal((K, r))
        A = X @ X.T
        bc = np.zeros(K, np.complex128)
        d = Sys()
        d.K, d.rcond = K, 1e-8
        # pinv_bucketed realifies d.M (complex column-major); give it a real
        # Hermitian-symmetric system through the inverse map of the real form
        d.Mr = torch.empty((K, K), dtype=torch.float64, device=dev)
        d.br = torch.as_tensor(rng.standard_normal(K), device=dev)
        d.xr = torch.empty(K, dtype=torch.float64, device=dev)
        d.a = torch.empty(K, dtype=torch.complex128, device=dev)
        d.kept = torch.zeros(1, dtype=torch.int32, device=dev)
        d.A = A
        systems.append(d)
    # complex M whose real form is A: M = U^H A U for the unitary map of the real form
    for d in systems:
        K, h = d.K, (d.K - 1) // 2
        U = np.zeros((K, K), np.complex128)       # x = U a on Hermitian-symmetric a
        for j in range(h):
            U[j, j] = U[j, K - 1 - j] = 1 / np.sqrt(2)
            U[h + 1 + j, j] = -1j / np.sqrt(2)
            U[h + 1 + j, K - 1 - j] = 1j / np.sqrt(2)
        U[h, h] = 1.0
        M = U.conj().T @ d.A @ U
        d.M = torch.as_tensor(M.T.copy(), device=dev)     # column-major
    batch.pinv_bucketed(systems, stream_ptr())
    torch.cuda.synchronize()
    for d in systems:
        K = d.K
        assert np.abs(d.Mr.cpu().numpy() - d.A).max() <= 1e-12 * np.abs(d.A).max()
        nb = np.zeros(1, np.int64)
        call("vtb_sym_workspace", K, 0, nb.ctypes.data)
        w1 = torch.empty(int(nb[0]), dtype=torch.uint8, device=dev)
        A1 = torch.as_tensor(d.A.copy(), device=dev)
        x1 = torch.empty(K, dtype=torch.float64, device=dev)
        k1 = torch.zeros(1, dtype=torch.int32, device=dev)
        rng2 = np.zeros(2)
        call("vtb_sym_pinv", dptr(A1), K, dptr(d.br), dptr(x1), K, 1e-8, dptr(w1), int(nb[0]), dptr(k1),
             rng2.ctypes.data, stream_ptr())
        torch.cuda.synchronize()
        assert int(d.kept[0]) == int(k1[0])
        rel = ((d.xr - x1).norm() / x1.norm()).item()
        assert rel < 1e-9, (K, rel)
