"""The C-ABI library builds, loads and exports every symbol include/montmul_b200.h declares.
No compute call is made here (this runs without a GPU)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "montmul_b200.h")).read()
    return sorted(set(re.findall(r"\b(mm_b200_\w+)\s*\(", text)))


def test_header_declares_the_backend_contract():
    syms = declared_symbols()
    for name in ("create", "load", "set_exponent", "run", "mul", "read", "remaining", "destroy",
                 "coefficient_bound", "supported_lengths", "full_k"):
        assert f"mm_b200_{name}" in syms


def test_library_exports_every_declared_symbol():
    from montmul_b200 import backend
    lib = backend.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert name in backend.SIGNATURES, f"{name} has no ctypes signature"


def test_limits_without_device():
    from montmul_b200 import backend
    import ctypes as C
    lib = backend.lib()
    q = (C.c_uint64 * 2)()
    lib.mm_b200_coefficient_bound(q)
    assert (int(q[0]) | int(q[1]) << 64) == ((1 << 31) - 1) * ((1 << 61) - 1)
    n = lib.mm_b200_supported_lengths(None, 0)
    arr = (C.c_size_t * n)()
    lib.mm_b200_supported_lengths(arr, n)
    # Shared-memory lengths 8 .. 16384, then global mode up to 2^24 (the reference's range).
    assert [int(v) for v in arr] == [1 << e for e in range(3, 25)]
    assert lib.mm_b200_batch_bytes(10, 16384, 1) > 10 * 60 * 8192
    # Global mode adds a 24-byte work element per transform position and slot.
    per_slot = lib.mm_b200_batch_bytes(2, 1 << 16, 1) - lib.mm_b200_batch_bytes(1, 1 << 16, 1)
    assert per_slot == (4 + 8 + 48 + 24) * (1 << 15) + 4 + 12
