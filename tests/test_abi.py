"""C ABI surface (CPU only: loads the library, no device compute)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "ssn.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ssn_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from symplectic_projection import _native
    return _native.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name


def test_binding_covers_header():
    from symplectic_projection import _native
    assert set(_native.PROTOTYPES) == set(declared_functions())


def test_version_and_strings(lib):
    assert lib.ssn_version() >= 100
    assert lib.ssn_status_string(0) == b"ok"
    assert b"Newton" in lib.ssn_status_string(3)
    assert b"line search" in lib.ssn_status_string(4)


def test_default_options_match_reference_constants():
    from symplectic_projection import _native
    opt = _native.options()
    assert (opt.max_newton, opt.max_cg, opt.max_backtrack, opt.feas_tol) == (100, 150, 40, 1e-8)


def test_invalid_arguments_rejected_without_device(lib):
    # validation happens on the host before any CUDA call
    assert lib.ssn_solve(None, None, None, None, None, 1, 8, 4, None, 0, None, None) == 1
    assert lib.ssn_solve(16, 16, 16, 16, 16, 1, 8, 3, 16, 1 << 20, None, None) == 1      # odd m
    assert lib.ssn_solve(16, 16, 16, 16, 16, 1, 8, 130, 16, 1 << 20, None, None) == 1    # m > 128
    assert lib.ssn_solve(16, 16, 16, 16, 16, 1, 1, 4, 16, 1 << 20, None, None) == 1      # n < k
    assert lib.ssn_solve(16, 16, 16, 16, 16, 1, 8, 4, 16, 8, None, None) == 7            # workspace too small
    assert lib.ssn_solve(8, 16, 16, 16, 16, 1, 8, 4, 16, 1 << 20, None, None) == 1       # misaligned T


def test_workspace_size_monotone(lib):
    a = lib.ssn_workspace_bytes(64, 4096, 96)
    b = lib.ssn_workspace_bytes(128, 4096, 96)
    assert 0 < a < b
    assert lib.ssn_workspace_bytes(0, 8, 4) == 0
    assert lib.ssn_workspace_bytes(4, 8, 7) == 0


def test_python_api_validates_on_host():
    import torch
    import symplectic_projection as sp
    with pytest.raises(ValueError):
        sp.solve(torch.zeros(2, 8, 4, dtype=torch.float32))
    with pytest.raises(ValueError):
        sp.solve(torch.zeros(2, 7, 4, dtype=torch.float64))
    with pytest.raises(ValueError):
        sp.solve(torch.zeros(2, 2, 4, dtype=torch.float64))   # n < k


def test_ragged_arguments_and_workspace_on_host(lib):
    import ctypes
    ints = lambda *v: (ctypes.c_int * len(v))(*v)
    i64 = lambda *v: (ctypes.c_int64 * len(v))(*v)
    n, m = ints(64, 100, 64), ints(8, 40, 8)
    one = lib.ssn_ragged_workspace_bytes(1, ints(64), ints(8))
    three = lib.ssn_ragged_workspace_bytes(3, n, m)
    assert 0 < one < three
    # two shape groups: at least the uniform workspaces of both plus gathered T, X and omega
    floor = lib.ssn_workspace_bytes(2, 64, 8) + lib.ssn_workspace_bytes(1, 100, 40)
    assert three >= floor + 8 * 2 * (2 * 2 * 64 * 8 + 2 * 100 * 40)
    assert lib.ssn_ragged_workspace_bytes(2, ints(64, 8), ints(8, 20)) == 0          # n < k
    assert lib.ssn_ragged_workspace_bytes(1, ints(64), ints(7)) == 0                 # odd m
    t_off, w_off = i64(0, 1024, 9024), i64(0, 64, 1664)
    args = (16, 16, 16, 16, 16, 3, n, m, t_off, w_off)
    assert lib.ssn_solve_ragged(*args, 16, 8, None, None) == 7                       # workspace too small
    assert lib.ssn_solve_ragged(16, 16, 16, 16, 16, 3, n, m, i64(0, 1025, 9024), w_off, 16, three,
                                None, None) == 1                                     # odd (misaligned) offset
    assert lib.ssn_solve_ragged(None, 16, 16, 16, 16, 3, n, m, t_off, w_off, 16, three, None, None) == 1


def test_adjoint_arguments_on_host(lib):
    a = lib.ssn_adjoint_workspace_bytes(8, 32, 8)
    assert a > 0 and lib.ssn_adjoint_workspace_bytes(8, 32, 7) == 0 and lib.ssn_adjoint_workspace_bytes(0, 32, 8) == 0
    assert lib.ssn_adjoint(16, 16, None, None, 16, 16, None, 8, 32, 8, 16, 8, None, None) == 7   # workspace
    assert lib.ssn_adjoint(None, 16, None, None, 16, 16, None, 8, 32, 8, 16, a, None, None) == 1  # no T
    assert lib.ssn_adjoint(16, 16, 8, None, 16, 16, None, 8, 32, 8, 16, a, None, None) == 1      # misaligned G
    assert lib.ssn_adjoint(16, 16, None, None, 16, 16, None, 8, 2, 8, 16, a, None, None) == 1     # n < k
