"""The C-ABI library builds, loads and exports every symbol include/montmul_b200.h declares, and
its default shared/global mode boundary is the reference planner's on a B200 (the planner's
own tests pin the restatement). No compute call is made here (this runs without a GPU)."""
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


# The reference's launch planner (montmul/src/gpu/plan.rs:26-64), restated to pin the mode
# boundary: shared mode when the vector (24 B per complex element) and the carry scratch fit the
# device's opt-in shared memory per block, else global mode.
def _ref_scratch_bytes(threads):
    return 8 * (2 * -(-threads // 32) + 2)


def _ref_plan(n, max_dyn_smem, force_global):
    half = n // 2
    threads = min(max(half // 2, 64), 1024)
    shared_bytes = 24 * n + _ref_scratch_bytes(threads)
    if not force_global and shared_bytes <= max_dyn_smem:
        return ("shared", threads, shared_bytes)
    return ("global", min(max(half, 64), 512), 528 + 24 * min(n, 1 << 11))


def test_reference_planner_restatement_pins():
    """plan.rs:70-100, the reference's own planner tests (RTX 3060 / 5090 limits)."""
    assert _ref_plan(4096, 101_376, False) == ("shared", 1024, 98_832)
    assert [_ref_plan(n, 101_376, False)[1] for n in (1024, 2048, 256)] == [256, 512, 64]
    assert _ref_plan(8192, 101_376, False) == ("global", 512, 49_680)
    assert _ref_plan(4096, 101_376, True)[0] == "global"
    assert _ref_plan(4, 101_376, False) == ("shared", 64, 144)
    assert _ref_plan(4096, 49_152, False)[0] == "global"


def test_default_mode_is_the_reference_planners_on_b200():
    """With a B200's 232,448 B of opt-in shared memory per block the reference's planner puts
    n <= 8192 (L <= 16384) in shared mode and longer lengths in global mode; this backend's
    default mode (visible in its per-slot bytes: global mode adds a 24 B work element per
    position) has the same boundary at every supported length."""
    from montmul_b200 import backend
    lib = backend.lib()
    for m in range(2, 24):
        n = 1 << m
        per_slot = lib.mm_b200_batch_bytes(2, 2 * n, 1) - lib.mm_b200_batch_bytes(1, 2 * n, 1)
        ours = "global" if per_slot == (4 + 8 + 48 + 24) * n + 4 + 12 else "shared"
        assert per_slot in ((4 + 8 + 48) * n + 16, (4 + 8 + 48 + 24) * n + 16)
        assert ours == _ref_plan(n, 232_448, False)[0], f"n = {n}"
