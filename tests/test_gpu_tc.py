"""Tensor-core (tcgen05) GEMM against float64 references (GPU)."""
import numpy as np
import pytest
import torch

from vtem_b200 import tc

pytestmark = pytest.mark.gpu


def test_bf16_exact_inputs():
    # bf16-representable operands with few terms: fp32 accumulation is exact
    rng = np.random.default_rng(0)
    M, N, K = 200, 130, 192
    A = torch.as_tensor(rng.integers(-8, 9, (M, K)).astype(np.float32) / 8, device="cuda").to(torch.bfloat16)
    B = torch.as_tensor(rng.integers(-8, 9, (N, K)).astype(np.float32) / 8, device="cuda").to(torch.bfloat16)
    out = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    out, err = tc.gemm_bf16(A.contiguous(), B.contiguous(), out)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.double() @ B.double().T
    assert torch.equal(out, ref)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 257, 1000), (1000, 64, 4096)])
def test_split_bf16_accuracy(M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = torch.as_tensor(rng.standard_normal((M, K)), device="cuda")
    B = torch.as_tensor(rng.standard_normal((N, K)), device="cuda")
    C = tc.gemm_split_bf16(A, B, alpha=0.5)
    ref = 0.5 * (A @ B.T)
    rel = ((C - ref).norm() / ref.norm()).item()
    # hi*lo split drops lo*lo: ~2^-16 of the products' scale, plus fp32 accumulation
    assert rel < 5e-5, rel


def test_split_bf16_transposed_output_and_float32():
    rng = np.random.default_rng(3)
    A = torch.as_tensor(rng.standard_normal((257, 300)), device="cuda")
    B = torch.as_tensor(rng.standard_normal((99, 300)), device="cuda")
    C = tc.gemm_split_bf16(A, B, out_layout="col", out_dtype=torch.float32)
    ref = (A @ B.T).T
    assert C.shape == (99, 257)
    rel = ((C.double() - ref).norm() / ref.norm()).item()
    assert rel < 5e-5, rel


def test_rf_filter_split_bf16_matches_f64():
    from vtem_b200 import vrf
    rng = np.random.default_rng(5)
    V = torch.as_tensor(rng.standard_normal((300, 32, 32)), device="cuda")
    gb = vrf.vrf_gabor((32, 32), dx=1 / 32, dy=1 / 32)
    N = 70
    gb.load_parameters(num_neurons=N, h_alpha=rng.uniform(0.05, 0.2, N), h_l=rng.uniform(0, 3, N),
                       h_x0=rng.uniform(-.4, .4, N), h_y0=rng.uniform(-.4, .4, N),
                       h_ab=rng.integers(0, 2, N).astype(np.int32), KAPPA=2.5)
    ref = gb.filter(V, out_layout="neuron")
    got = gb.filter(V, out_layout="neuron", precision="bf16x3")
    rel = ((got - ref).norm() / ref.norm()).item()
    assert rel < 5e-5, rel


@pytest.mark.parametrize("bn", [64, 96, 128, 160, 192, 256, 320])
@pytest.mark.parametrize("N,ldc,alpha", [(289, 289, 1.0), (289, 292, 1.0), (289, 292, 0.5), (306, 308, 1.0)])
def test_every_tile_width_is_exact_on_bf16_inputs(bn, N, ldc, alpha):
    """Each tile width the autotuner may pick computes the same product
    (bf16-exact operands: fp32 accumulation is exact), with partial edge tiles
    in both directions.  Row pitch 289 takes the shared-memory staged stores,
    292 and 308 (16-byte rows) the tensor stores, with the last N mod 4
    columns by plain stores; the padding columns stay untouched."""
    from vtem_b200._abi import call, dptr, stream_ptr
    rng = np.random.default_rng(bn)
    M, K = 300, 256
    A = torch.as_tensor(rng.integers(-8, 9, (M, K)).astype(np.float32) / 8, device="cuda").to(torch.bfloat16)
    B = torch.as_tensor(rng.integers(-8, 9, (N, K)).astype(np.float32) / 8, device="cuda").to(torch.bfloat16)
    out = torch.full((M, ldc), float("nan"), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("vtb_tc_gemm_bf16_bn", dptr(A), M, dptr(B), N, K, dptr(out), ldc, 1, 0, alpha, 0, dptr(err), bn,
         stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(out[:, :N].double(), alpha * (A.double() @ B.double().T))
    assert torch.isnan(out[:, N:]).all()


def test_autotuner_picks_a_candidate_and_caches_it():
    from vtem_b200 import autotune
    rng = np.random.default_rng(1)
    A = torch.as_tensor(rng.standard_normal((513, 200)), device="cuda")
    B = torch.as_tensor(rng.standard_normal((289, 200)), device="cuda")
    C1 = tc.gemm_split_bf16(A, B)
    key = autotune._key(513, 289, tc.padded_k(200), True, x3=True)
    assert autotune._cache[key] in autotune.CANDIDATES
    C2 = tc.gemm_split_bf16(A, B)           # cached choice: same result
    assert torch.equal(C1, C2)


@pytest.mark.parametrize("x3", [False, True])
@pytest.mark.parametrize("bn", [64, 128, 256])
def test_grouped_gemm_equals_single_launches(bn, x3):
    """One grouped launch over problems of uneven sizes gives each problem's
    single-launch result bit for bit (same tiles, same accumulation order),
    in the plain and the three-product mode."""
    from vtem_b200._abi import call, dptr, lib, stream_ptr
    rng = np.random.default_rng(bn + 1)
    shapes = [(300, 289, 384), (97, 49, 128), (513, 121, 192), (128, 225, 64), (40, 81, 256)]
    parts = 2 if x3 else 1
    single = "vtb_tc_gemm_bf16x3_bn" if x3 else "vtb_tc_gemm_bf16_bn"
    As, Bs, Cs, Cref, errs = [], [], [], [], []
    for (M, N, K) in shapes:
        A = torch.as_tensor(rng.standard_normal((M, parts * K)), device="cuda").to(torch.bfloat16).contiguous()
        B = torch.as_tensor(rng.standard_normal((N, parts * K)), device="cuda").to(torch.bfloat16).contiguous()
        As.append(A)
        Bs.append(B)
        Cs.append(torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda"))
        Cref.append(torch.zeros((M, N), dtype=torch.float32, device="cuda"))
        errs.append(torch.zeros(1, dtype=torch.int32, device="cuda"))
        call(single, dptr(A), M, dptr(B), N, K, dptr(Cref[-1]), N, 1, 0, 1.0, 0, dptr(errs[-1]), bn, stream_ptr())
    n = len(shapes)
    u64 = np.uint64
    arr = [np.array([a.data_ptr() for a in As], u64), np.array([s[0] for s in shapes], np.int32),
           np.array([b.data_ptr() for b in Bs], u64), np.array([s[1] for s in shapes], np.int32),
           np.array([s[2] for s in shapes], np.int32), np.array([c.data_ptr() for c in Cs], u64),
           np.array([s[1] for s in shapes], np.int64), np.array([e.data_ptr() for e in errs], u64)]
    host = np.zeros(int(lib().vtb_tc_group_bytes(n)), np.uint8)
    tiles = np.zeros(1, np.int32)
    call("vtb_tc_group_build_x3" if x3 else "vtb_tc_group_build", host.ctypes.data, n, *[a.ctypes.data for a in arr],
         bn, tiles.ctypes.data)
    desc = torch.as_tensor(host).cuda()
    call("vtb_tc_gemm_grouped_x3" if x3 else "vtb_tc_gemm_grouped", dptr(desc), n, int(tiles[0]), bn, stream_ptr())
    torch.cuda.synchronize()
    assert all(int(e.item()) == 0 for e in errs)
    for C, R in zip(Cs, Cref):
        assert torch.equal(C, R)


@pytest.mark.parametrize("bn", [64, 96, 128, 160, 192, 256, 320])
def test_three_product_mode_every_tile_width(bn):
    """vtb_tc_gemm_bf16x3_bn on [hi | lo] operands: the split-bf16 product
    to the same accuracy as the three-part layout, and equal to it up to the
    order of the fp32 sums, for every tile width (partial edge tiles in both
    directions, several k-blocks)."""
    from vtem_b200._abi import call, dptr, stream_ptr
    rng = np.random.default_rng(100 + bn)
    M, N, K = 300, 289, 320
    A = torch.as_tensor(rng.standard_normal((M, K)), device="cuda")
    B = torch.as_tensor(rng.standard_normal((N, K)), device="cuda")
    A2, B2 = tc.split_bf16x2(A), tc.split_bf16x2(B)
    A3, B3 = tc.split_bf16x3(A, 0), tc.split_bf16x3(B, 1)
    Kp = tc.padded_k(K)
    assert A2.shape == (M, 2 * Kp) and A3.shape == (M, 3 * Kp)
    out2 = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    out3 = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("vtb_tc_gemm_bf16x3_bn", dptr(A2), M, dptr(B2), N, Kp, dptr(out2), N, 1, 0, 1.0, 0, dptr(err), bn,
         stream_ptr())
    call("vtb_tc_gemm_bf16_bn", dptr(A3), M, dptr(B3), N, 3 * Kp, dptr(out3), N, 1, 0, 1.0, 0, dptr(err), bn,
         stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A @ B.T
    rel = ((out2.double() - ref).norm() / ref.norm()).item()
    assert rel < 5e-5, rel
    assert (out2 - out3).abs().max().item() <= 1e-5 * ref.abs().max().item()
