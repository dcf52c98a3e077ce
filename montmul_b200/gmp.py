"""GMP through its public C API (libgmp.so.10, called via ctypes).

The reference draws every workload with `rug` over GMP (montmul/src/score.rs:45-61,
tests/common/mod.rs:10-15) and checks results with `pow_mod`. The same GMP calls reproduce its
random streams exactly: `RandState::new()` = gmp_randinit_default, `seed` = gmp_randseed,
`Integer::random_bits` = mpz_urandomb, `random_below` = mpz_urandomm, `next_prime` =
mpz_nextprime. libgmp ships here without its header, so the few prototypes are declared below
from GMP's documented interface.
"""
from __future__ import annotations

import ctypes as C
import ctypes.util

_LIB = None
_F = {}   # "mpz_powm" -> bound __gmpz_powm, etc. (double-underscore names are mangled in classes)


class _Mpz(C.Structure):
    # __mpz_struct: int _mp_alloc; int _mp_size; mp_limb_t *_mp_d
    _fields_ = [("alloc", C.c_int), ("size", C.c_int), ("d", C.c_void_p)]


def _lib():
    global _LIB
    if _LIB is None:
        name = ctypes.util.find_library("gmp") or "libgmp.so.10"
        L = C.CDLL(name)
        P = C.POINTER(_Mpz)
        vp = C.c_void_p
        for fn, args, res in [
            ("__gmpz_init", [P], None),
            ("__gmpz_clear", [P], None),
            ("__gmpz_import", [P, C.c_size_t, C.c_int, C.c_size_t, C.c_int, C.c_size_t, vp], None),
            ("__gmpz_export", [vp, C.POINTER(C.c_size_t), C.c_int, C.c_size_t, C.c_int, C.c_size_t, P], vp),
            ("__gmpz_sizeinbase", [P, C.c_int], C.c_size_t),
            ("__gmpz_powm", [P, P, P, P], None),
            ("__gmpz_gcd", [P, P, P], None),
            ("__gmpz_mul", [P, P, P], None),
            ("__gmpz_mod", [P, P, P], None),
            ("__gmpz_invert", [P, P, P], C.c_int),
            ("__gmpz_nextprime", [P, P], None),
            ("__gmpz_urandomb", [P, vp, C.c_ulong], None),
            ("__gmpz_urandomm", [P, vp, P], None),
            ("__gmp_randinit_default", [vp], None),
            ("__gmp_randseed", [vp, P], None),
            ("__gmp_randclear", [vp], None),
        ]:
            f = getattr(L, fn)
            f.argtypes = args
            f.restype = res
            _F[fn.replace("__gmpz_", "mpz_").replace("__gmp_", "gmp_")] = f
        _LIB = L
    return _LIB


def _f(name):
    if not _F:
        _lib()
    return _F[name]


class Mpz:
    """An owned mpz_t."""

    __slots__ = ("z",)

    def __init__(self, v: int = 0):
        self.z = _Mpz()
        _f("mpz_init")(C.byref(self.z))
        if v:
            self.set(v)

    def set(self, v: int) -> "Mpz":
        if v < 0:
            raise ValueError("negative values are not used with GMP here")
        nb = max(1, (v.bit_length() + 7) // 8)
        buf = v.to_bytes(nb, "little")
        _f("mpz_import")(C.byref(self.z), nb, -1, 1, 0, 0, buf)
        return self

    def get(self) -> int:
        if self.z.size == 0:
            return 0
        nb = (_f("mpz_sizeinbase")(C.byref(self.z), 2) + 7) // 8
        buf = C.create_string_buffer(nb + 8)
        cnt = C.c_size_t(0)
        _f("mpz_export")(buf, C.byref(cnt), -1, 1, 0, 0, C.byref(self.z))
        return int.from_bytes(buf.raw[: cnt.value], "little")

    def __del__(self):
        if _LIB is not None and self.z is not None:
            _F["mpz_clear"](C.byref(self.z))
            self.z = None


def powm(b: int, e: int, m: int) -> int:
    """b^e mod m (rug `pow_mod`)."""
    r, bb, ee, mm = Mpz(), Mpz(b), Mpz(e), Mpz(m)
    _f("mpz_powm")(C.byref(r.z), C.byref(bb.z), C.byref(ee.z), C.byref(mm.z))
    return r.get()


def mulmod(a: int, b: int, m: int) -> int:
    """a * b mod m for nonnegative a, b."""
    r, aa, bb, mm = Mpz(), Mpz(a), Mpz(b), Mpz(m)
    _f("mpz_mul")(C.byref(r.z), C.byref(aa.z), C.byref(bb.z))
    _f("mpz_mod")(C.byref(r.z), C.byref(r.z), C.byref(mm.z))
    return r.get()


def gcd(a: int, b: int) -> int:
    """gcd(a, b) of nonnegative integers (GMP's subquadratic gcd; Python's is quadratic)."""
    r, aa, bb = Mpz(), Mpz(a), Mpz(b)
    _f("mpz_gcd")(C.byref(r.z), C.byref(aa.z), C.byref(bb.z))
    return r.get()


def invert(a: int, m: int) -> int:
    """a^-1 mod m (rug `invert`); raises ValueError when it does not exist."""
    r, aa, mm = Mpz(), Mpz(a % m), Mpz(m)
    if not _f("mpz_invert")(C.byref(r.z), C.byref(aa.z), C.byref(mm.z)):
        raise ValueError("not invertible")
    return r.get()


def next_prime(v: int) -> int:
    r, vv = Mpz(), Mpz(v)
    _f("mpz_nextprime")(C.byref(r.z), C.byref(vv.z))
    return r.get()


class RandState:
    """rug `RandState::new()` (gmp_randinit_default), optionally seeded like `rng.seed(&seed)`."""

    def __init__(self, seed: int | None = None):
        self.st = C.create_string_buffer(64)   # gmp_randstate_t is 32 bytes on LP64
        _f("gmp_randinit_default")(self.st)
        if seed is not None:
            self.seed(seed)

    def seed(self, seed: int) -> None:
        s = Mpz(seed)
        _f("gmp_randseed")(self.st, C.byref(s.z))

    def random_bits(self, bits: int) -> int:
        """`Integer::random_bits(bits, rng)`: uniform in [0, 2^bits)."""
        r = Mpz()
        _f("mpz_urandomb")(C.byref(r.z), self.st, bits)
        return r.get()

    def random_below(self, n: int) -> int:
        """`n.random_below(rng)`: uniform in [0, n)."""
        r, nn = Mpz(), Mpz(n)
        _f("mpz_urandomm")(C.byref(r.z), self.st, C.byref(nn.z))
        return r.get()

    def __del__(self):
        if _LIB is not None and getattr(self, "st", None) is not None:
            _F["gmp_randclear"](self.st)
            self.st = None
