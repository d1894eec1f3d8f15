"""The C ABI library loads and exports every symbol include/vtem_b200.h
declares (CPU: no compute call is made)."""
import ctypes
import os
import re

import pytest

from vtem_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "vtem_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vtb_\w+)\s*\(", src)))


def test_library_loads_and_exports_header():
    lib = _abi.lib()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s


def test_every_header_symbol_has_a_binding():
    bound = set(_abi.SIGNATURES) | {"vtb_status_string"}
    missing = [s for s in header_symbols() if s not in bound]
    assert not missing, missing


def test_every_binding_is_declared_in_the_header():
    declared = set(header_symbols())
    undeclared = [s for s in _abi.SIGNATURES if s not in declared]
    assert not undeclared, undeclared


def test_version_and_status_strings():
    lib = _abi.lib()
    assert lib.vtb_version() == 1
    assert _abi.status_string(0) == "ok"
    assert "overflow" in _abi.status_string(_abi.VTB_OVERFLOW)


def test_bad_arguments_rejected_without_gpu():
    # argument validation happens before any CUDA call
    lib = _abi.lib()
    st = lib.vtb_compute_q(None, None, None, -1, None, None, None, None, None, None)
    assert st == _abi.VTB_BAD_ARG
    st = lib.vtb_spike_pairs(None, None, None, 4, 10, 1, 0.01, 0.0, 1.0, None, None, None, None, None, None)
    assert st == _abi.VTB_BAD_ARG
    st = lib.vtb_iaf_encode(None, 0, 0, 4, 10, 0, 1e-4, None, None, None, None, None, None, 0, 0, 0, 0, None,
                            None, None, None, None, 1, None, 0.0, None, 0.0, None)
    assert st == _abi.VTB_BAD_ARG


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_abi, "_lib", None)
    monkeypatch.setattr(_abi, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(RuntimeError, match="not built"):
        _abi.lib()


def header_arities():
    src = open(os.path.join(ROOT, "include", "vtem_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(vtb_\w+)\s*\(([^;{]*?)\)\s*;", src):
        p = params.strip()
        out[name] = 0 if p in ("", "void") else p.count(",") + 1
    return out


def test_bindings_match_header_arity():
    """Every ctypes binding passes as many arguments as the C declaration
    takes (a drift between the two would pass garbage through the ABI)."""
    ar = header_arities()
    bad = {n: (len(a), ar[n]) for n, a in _abi.SIGNATURES.items() if n in ar and len(a) != ar[n]}
    assert not bad, bad


def test_solver_entry_points_reject_bad_sizes_without_gpu():
    lib = _abi.lib()
    assert lib.vtb_sym_dinv(None, 0, 0, None, None) == _abi.VTB_BAD_ARG
    assert lib.vtb_sym_potrs_flags(None, 0, None, 0, None, None, 0, None, None) == _abi.VTB_BAD_ARG
    assert lib.vtb_sym_potrs_flags_bytes(0) == 0


def test_chol_and_wait_limit_entry_points_without_gpu():
    lib = _abi.lib()
    assert lib.vtb_chol_work_bytes(0) == 0 and lib.vtb_chol_dinv_floats(0) == 0
    assert lib.vtb_chol_dinv_floats(1921) == 31 * 4096
    assert lib.vtb_chol_factor(None, 0, 0, None, None, 0, None, None, 1e-8, None) == _abi.VTB_BAD_ARG
    assert lib.vtb_chol_solve(None, 0, None, 0, None, None) == _abi.VTB_BAD_ARG
    assert lib.vtb_chol_inverse_floats(0) == 0 and lib.vtb_chol_inverse_floats(1921) == 31 * 32 // 2 * 4096
    assert lib.vtb_chol_factor_inverse(None, 0, 0, None, None, None, 0, None, None, 1e-8, None) == _abi.VTB_BAD_ARG
    assert lib.vtb_chol_solve_inverse(None, 0, None, None, 0, None) == _abi.VTB_BAD_ARG
    assert lib.vtb_chol_solve_inverse_bytes(1921) == (31 * 32 // 2 * 64 + 31 * 64) * 4 + 2 * 31 * 4
    assert lib.vtb_set_wait_limit(-1, None) == _abi.VTB_BAD_ARG
    with _abi.wait_limit(7):
        import numpy as np
        prev = np.zeros(1, np.int64)
        assert lib.vtb_set_wait_limit(7, prev.ctypes.data) == 0 and prev[0] == 7
    prev = np.zeros(1, np.int64)
    assert lib.vtb_set_wait_limit(0, prev.ctypes.data) == 0 and prev[0] == 0


def test_synth_rank_rejects_unsupported_orders_without_gpu():
    lib = _abi.lib()
    # Mt = 0 and Mt = 11 (23 harmonics, beyond the kernel's 21) are refused before any launch
    assert lib.vtb_coeff_synth_rank(None, None, 29, 3, 3, 0, 8, 8, 8, 8, None, 1, 1.0, 0.0, 1e-3, 4, None, 0,
                                    None) == _abi.VTB_BAD_ARG
    assert lib.vtb_coeff_synth_rank(None, None, 29, 3, 3, 11, 8, 8, 8, 8, None, 23, 1.0, 0.0, 1e-3, 4, 1, 0,
                                    None) == _abi.VTB_BAD_ARG
    # no frames: nothing to do
    assert lib.vtb_coeff_synth_rank(None, None, 29, 3, 3, 4, 8, 8, 8, 8, None, 9, 1.0, 0.0, 1e-3, 0, None, 0,
                                    None) == _abi.VTB_OK
