"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/liboracle.so).

The oracle restates the reference `Cpu` backend (montmul/src/cpu.rs, field.rs) and the `Gmp`
backend's REDC (montmul/src/gmp.rs:45-60) in plain C. Only tests, the smoke check and the
bench's CPU-baseline leg import this module; the product never does.

`OracleBackend` implements the same backend protocol as the product's `B200` backend
(create/load/set_exponent/run/mul/read/remaining plus the Limits queries), so both plug into
`montmul_b200.ModBatch` and the parity tests compare raw Montgomery limbs between them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

P1 = (1 << 31) - 1
P2 = (1 << 61) - 1
Q = P1 * P2

PLAIN, FULL_K, WRAP = 0, 1, 2


def build() -> str:
    """Compiles the oracle with its Makefile (gcc, a few seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
        u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
        sz = C.c_size_t
        L.oc_create.restype = C.c_void_p
        L.oc_create.argtypes = [C.c_int, sz, sz, C.c_uint32, sz, u32p, u32p, u32p]
        L.og_create.restype = C.c_void_p
        L.og_create.argtypes = [sz, sz, C.c_uint32, sz, u32p, u32p, u32p]
        L.oc_load.argtypes = [C.c_void_p, sz, u32p]
        L.oc_set_exponent.argtypes = [C.c_void_p, sz, u32p, sz, sz]
        L.oc_run.argtypes = [C.c_void_p, sz, C.c_int]
        L.oc_mul.argtypes = [C.c_void_p, sz, sz, sz]
        L.oc_read.argtypes = [C.c_void_p, sz, u32p]
        L.oc_remaining.restype = sz
        L.oc_remaining.argtypes = [C.c_void_p, sz]
        L.oc_destroy.argtypes = [C.c_void_p]
        L.oc_sylow2_f1.argtypes = [u32p]
        L.oc_sylow2_f2.argtypes = [u64p]
        L.oc_pow_f1.argtypes = [u32p, C.c_uint64, u32p]
        L.oc_pow_f2.argtypes = [u64p, C.c_uint64, u64p]
        L.oc_crt_inv.restype = C.c_uint32
        L.oc_crt.argtypes = [C.c_uint32, C.c_uint64, u64p]
        L.oc_tables.restype = C.c_int
        L.oc_tables.argtypes = [sz] + [u32p] * 4 + [u64p] * 4
        L.oc_upload.argtypes = [u32p, sz, sz, u32p, u64p]
        L.oc_download.argtypes = [u32p, u64p, sz, sz, u64p]
        L.oc_forward.argtypes = [u32p, u64p, sz, sz]
        L.oc_inverse.argtypes = [u32p, u64p, sz, sz]
        L.oc_pointwise.argtypes = [u32p, u64p, u32p, u64p, u32p, u64p, C.c_void_p, sz, sz]
        L.oc_half_factors.restype = C.c_int
        L.oc_half_factors.argtypes = [u32p, sz, u32p, u64p]
        _lib = L
    return _lib


# ---- field checks ----

def sylow2_f1():
    o = np.zeros(2, np.uint32)
    lib().oc_sylow2_f1(o)
    return int(o[0]), int(o[1])


def sylow2_f2():
    o = np.zeros(2, np.uint64)
    lib().oc_sylow2_f2(o)
    return int(o[0]), int(o[1])


def pow_f1(a, e):
    o = np.zeros(2, np.uint32)
    lib().oc_pow_f1(np.array(a, np.uint32), e, o)
    return int(o[0]), int(o[1])


def pow_f2(a, e):
    o = np.zeros(2, np.uint64)
    lib().oc_pow_f2(np.array(a, np.uint64), e, o)
    return int(o[0]), int(o[1])


def crt_inv():
    return int(lib().oc_crt_inv())


def crt(c1, c2):
    o = np.zeros(2, np.uint64)
    lib().oc_crt(c1, c2, o)
    return int(o[0]) | (int(o[1]) << 64)


def tables(n):
    """FieldTables::new(n) of both fields as (F1 arrays [m,2] u32, F2 arrays [m,2] u64)."""
    f1 = [np.zeros((m, 2), np.uint32) for m in (n // 2, n // 2, n, n)]
    f2 = [np.zeros((m, 2), np.uint64) for m in (n // 2, n // 2, n, n)]
    assert lib().oc_tables(n, *f1, *f2) == 0
    return dict(tw1=f1[0], itw1=f1[1], w1=f1[2], iw1=f1[3], tw2=f2[0], itw2=f2[1], w2=f2[2], iw2=f2[3])


# ---- Transform trait (cpu.rs:349-407) ----

def upload(coeffs: np.ndarray, length: int, count: int):
    n = length // 2
    f1 = np.zeros((count * n, 2), np.uint32)
    f2 = np.zeros((count * n, 2), np.uint64)
    lib().oc_upload(np.ascontiguousarray(coeffs, np.uint32), length, count, f1, f2)
    return f1, f2


def download(f1, f2, length: int, count: int):
    out = np.zeros((count * length, 2), np.uint64)
    lib().oc_download(f1, f2, length, count, out)
    return [int(a) | (int(b) << 64) for a, b in out]


def forward(f1, f2, length, count):
    lib().oc_forward(f1, f2, length, count)


def inverse(f1, f2, length, count):
    lib().oc_inverse(f1, f2, length, count)


def pointwise(a, b, scales, length, count):
    o1 = np.zeros_like(a[0])
    o2 = np.zeros_like(a[1])
    sp = None
    if scales is not None:
        s = np.ascontiguousarray(scales, np.uint32)
        sp = s.ctypes.data_as(C.c_void_p)
    lib().oc_pointwise(o1, o2, a[0], a[1], b[0], b[1], sp, length, count)
    return o1, o2


def half_factors(n_limbs: np.ndarray, length: int):
    n = length // 2
    ab1 = np.zeros((n, 2), np.uint32)
    ab2 = np.zeros((n, 2), np.uint64)
    assert lib().oc_half_factors(np.ascontiguousarray(n_limbs, np.uint32), length, ab1, ab2) == 0
    return ab1, ab2


# ---- Backend trait ----

class _State:
    def __init__(self, ptr, k, slots):
        self.ptr, self.k, self.slots = ptr, k, slots

    def __del__(self):
        if self.ptr:
            lib().oc_destroy(self.ptr)
            self.ptr = None


class OracleBackend:
    """`Cpu::default()`, `Cpu::default().with_full_k(true)`, `Cpu::with_wraparound(true)` or `Gmp`."""

    LENGTHS = [1 << e for e in range(3, 25)]

    def __init__(self, mode: int = WRAP, gmp: bool = False, threads: int = 0):
        self.mode, self.gmp, self.threads = mode, gmp, threads

    @classmethod
    def wraparound(cls, threads: int = 0):
        return cls(WRAP, threads=threads)

    @classmethod
    def plain(cls, threads: int = 0):
        return cls(PLAIN, threads=threads)

    @classmethod
    def with_full_k(cls, threads: int = 0):
        return cls(FULL_K, threads=threads)

    @classmethod
    def gmp_backend(cls, threads: int = 0):
        return cls(PLAIN, gmp=True, threads=threads)

    # Limits (transform.rs:11-20)
    def coefficient_bound(self) -> int:
        return (1 << 128) - 1 if self.gmp else Q

    def supported_lengths(self):
        return list(self.LENGTHS)

    def full_k(self) -> bool:
        return (not self.gmp) and self.mode in (FULL_K, WRAP)

    # Backend (transform.rs:61-77)
    def create(self, k, length, base, n, nprime, two_n):
        slots = n.shape[0]
        args = (np.ascontiguousarray(n, np.uint32), np.ascontiguousarray(nprime, np.uint32),
                np.ascontiguousarray(two_n, np.uint32))
        if self.gmp:
            ptr = lib().og_create(k, length, base, slots, *args)
        else:
            ptr = lib().oc_create(self.mode, k, length, base, slots, *args)
        if not ptr:
            raise ValueError("oracle rejected the batch setup")
        return _State(ptr, k, slots)

    def load(self, st, i, limbs):
        lib().oc_load(st.ptr, i, np.ascontiguousarray(limbs, np.uint32))

    def set_exponent(self, st, i, words, nbits):
        w = np.ascontiguousarray(words, np.uint32)
        if w.size == 0:
            w = np.zeros(1, np.uint32)
        lib().oc_set_exponent(st.ptr, i, w, len(words), nbits)

    def run(self, st, bits):
        lib().oc_run(st.ptr, bits, self.threads)

    def mul(self, st, out, a, b):
        lib().oc_mul(st.ptr, out, a, b)

    def read(self, st, i):
        o = np.zeros(st.k, np.uint32)
        lib().oc_read(st.ptr, i, o)
        return o

    def remaining(self, st, i):
        return int(lib().oc_remaining(st.ptr, i))
