"""The allocation-free synthesis entry point (GPU).

vtb_coeff_synthesize_noalloc serves callers that cannot allocate device
memory (a plugin confined to another runtime's memory pool, code that may only
allocate through a framework's allocator): its scratch is a fixed device array
inside the library.  It must give the same video as the allocating
vtb_coeff_synthesize, call after call (the scratch keeps the previous call's
contents), and refuse problems whose per-frame coefficients do not fit.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from vtem_b200 import _abi
from vtem_b200.fast import ellipse_storage_index

pytestmark = pytest.mark.gpu


def _problem(seed, Mx=6, My=6, Mt=8, Nt=5003, P=64):
    rng = np.random.default_rng(seed)
    smap = torch.as_tensor(ellipse_storage_index(Mx, My), device="cuda")
    Ks = int(smap.numel())
    Kt = 2 * Mt + 1
    a = torch.as_tensor(rng.standard_normal(Ks * Kt) + 1j * rng.standard_normal(Ks * Kt), dtype=torch.complex128,
                        device="cuda")
    return dict(a=a, smap=smap, Ks=Ks, Mx=Mx, My=My, Mt=Mt, W=2 * np.pi * 20 / Mt, t0=0.0, dt=1e-4, Nt=Nt, Px=P,
                Py=P, Px1=P, Py1=P)


def _reference(p, dtype):
    lib = _abi.lib()
    u = torch.empty((p["Nt"], p["Py"], p["Px"]), dtype=dtype, device="cuda")
    A = torch.empty((p["Nt"], p["Ks"]), dtype=torch.complex128, device="cuda")
    st = lib.vtb_coeff_synthesize(p["a"].data_ptr(), p["smap"].data_ptr(), p["Ks"], p["Mx"], p["My"], p["Mt"],
                                  p["W"], p["t0"], p["dt"], p["Nt"], p["Px"], p["Py"], p["Px1"], p["Py1"],
                                  A.data_ptr(), u.data_ptr(), int(dtype == torch.float32), _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    return u


def _noalloc(p, dtype):
    lib = _abi.lib()
    u = torch.full((p["Nt"], p["Py"], p["Px"]), float("nan"), dtype=dtype, device="cuda")
    st = lib.vtb_coeff_synthesize_noalloc(p["a"].data_ptr(), p["smap"].data_ptr(), p["Ks"], p["Mx"], p["My"],
                                          p["Mt"], p["W"], p["t0"], p["dt"], p["Nt"], p["Px"], p["Py"], p["Px1"],
                                          p["Py1"], u.data_ptr(), int(dtype == torch.float32), _abi.stream_ptr())
    assert st == 0, _abi.status_string(st)
    return u


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_matches_allocating_entry_point_twice(dtype):
    # 5003 frames x 113 coefficients is larger than the fixed scratch, so the
    # call runs several chunks; two different problems in a row check that
    # nothing of the first call's scratch leaks into the second
    for seed in (1, 2):
        p = _problem(seed)
        ref = _reference(p, dtype)
        got = _noalloc(p, dtype)
        torch.cuda.synchronize()
        assert torch.isfinite(got).all()
        tol = 1e-13 if dtype == torch.float64 else 1e-6
        err = ((got.double() - ref.double()).abs().max() / ref.double().abs().max()).item()
        assert err <= tol, err


def test_noalloc_rejects_oversized_frames():
    lib = _abi.lib()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    # Ks beyond the 4 MiB scratch (262144 complex values per frame): refused
    # before any launch, nothing is read through the dummy pointers
    st = lib.vtb_coeff_synthesize_noalloc(dummy.data_ptr(), dummy.data_ptr(), 262145, 6, 6, 8, 1.0, 0.0, 1e-4, 10,
                                          64, 64, 64, 64, dummy.data_ptr(), 0, _abi.stream_ptr())
    assert st == _abi.VTB_BAD_ARG


def test_noalloc_allocates_no_device_memory():
    """After a first call (which loads the library's module on the device),
    further calls leave both the device's free memory and torch's allocator
    untouched: the scratch is the library's own fixed array."""
    p = _problem(3, Nt=3001)
    u = torch.empty((p["Nt"], p["Py"], p["Px"]), dtype=torch.float64, device="cuda")
    lib = _abi.lib()

    def once():
        st = lib.vtb_coeff_synthesize_noalloc(p["a"].data_ptr(), p["smap"].data_ptr(), p["Ks"], p["Mx"], p["My"],
                                              p["Mt"], p["W"], p["t0"], p["dt"], p["Nt"], p["Px"], p["Py"], p["Px1"],
                                              p["Py1"], u.data_ptr(), 0, _abi.stream_ptr())
        assert st == 0, _abi.status_string(st)

    once()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(4):
        once()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    ref = _reference(p, torch.float64)
    assert ((u - ref).abs().max() / ref.abs().max()).item() <= 1e-13
