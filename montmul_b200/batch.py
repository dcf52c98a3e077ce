"""Host API above the backend boundary: parameter rules, Montgomery conversion and the Fermat
driver, restating montmul/src/batch.rs (Params 13-31, ModBatch 53-184, fermat 187-198).

Big-integer work stays here, as in the reference: N' = -N^-1 mod R, R mod N and R^-1 mod N per
modulus (computed through GMP, in parallel over moduli like the reference's rayon loop), the
conversion into and out of Montgomery form, and is_one. The backend only sees limb arrays.
A backend is any object with the `Limits` + `Backend` methods of transform.rs:11-77:
coefficient_bound, supported_lengths, full_k, create, load, set_exponent, run, mul, read,
remaining (and optionally load_all / set_exponents for whole-batch uploads).
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import gmp

W = 32  # limb width w (batch.rs:9)


class MontMulError(Exception):
    """A rejected batch or call (the reference's anyhow::Error / panic message)."""


@dataclass(frozen=True)
class Params:
    k: int
    len: int

    @staticmethod
    def for_bits(bits: int, lengths) -> "Params":
        """Smallest k with k w >= b + 4 and the smallest supported L >= 2k (batch.rs:20-25)."""
        k = -(-(bits + 4) // W)
        for length in lengths:
            if length >= 2 * k:
                return Params(k, length)
        raise MontMulError(f"no transform length for {bits} bits")

    def check_exact(self, c: int, bound: int) -> None:
        """The exactness rule c k (2^w - 1)^2 < Q (batch.rs:27-31)."""
        lhs = max(c, 1) * self.k * ((1 << W) - 1) ** 2
        if lhs >= bound:
            raise MontMulError(f"c · k · (2^w − 1)² = {lhs} exceeds the coefficient bound {bound}")


def to_limbs(x: int, k: int) -> np.ndarray:
    """k little-endian 32-bit limbs of x >= 0 (batch.rs:35-40)."""
    if x < 0 or x.bit_length() > 32 * k:
        raise MontMulError(f"value does not fit {k} limbs")
    return np.frombuffer(x.to_bytes(4 * k, "little"), dtype="<u4").astype(np.uint32)


def from_limbs(v) -> int:
    return int.from_bytes(np.ascontiguousarray(v, dtype="<u4").tobytes(), "little")


def exponent_words(e: int):
    """Exponent bits MSB first: bit p is (words[p/32] >> (31 - p%32)) & 1 (batch.rs:140-150)."""
    nbits = e.bit_length()
    nw = -(-nbits // 32)
    if nw == 0:
        return np.zeros(0, np.uint32), 0
    aligned = e << (32 * nw - nbits)
    return np.frombuffer(aligned.to_bytes(4 * nw, "big"), dtype=">u4").astype(np.uint32), nbits


@dataclass
class _Modulus:
    n: int
    r: int      # R mod N
    rinv: int   # R^-1 mod N


def _setup_one(n: int, k: int):
    r = 1 << (32 * k)
    ninv = gmp.invert(n, r)
    nprime = (r - ninv) % r
    rmod = gmp.powm(2, 32 * k, n)
    rinv = gmp.invert(rmod, n)
    return to_limbs(n, k), to_limbs(nprime, k), to_limbs(2 * n, k), _Modulus(n, rmod, rinv)


def _threads() -> int:
    return max(1, min(32, os.cpu_count() or 1))


class ModBatch:
    """A batch of moduli on one backend (batch.rs:53-184)."""

    def __init__(self, backend, moduli, base: int):
        moduli = [int(m) for m in moduli]
        if not moduli:
            raise MontMulError("empty batch")
        if not 1 <= base <= 4:
            raise MontMulError(f"base {base} does not fit the lazy range (c ≤ 4)")
        lengths = list(backend.supported_lengths())
        params = None
        for n in moduli:
            if n <= 1 or n % 2 == 0:
                raise MontMulError("modulus must be odd and > 1")
            p = Params.for_bits(n.bit_length(), lengths)
            if params is None:
                params = p
            elif params.len != p.len:
                raise MontMulError(f"moduli need different transform lengths ({params.len} vs {p.len})")
            else:
                params = Params(max(params.k, p.k), params.len)
        if backend.full_k():
            params = Params(params.len // 2, params.len)
        params.check_exact(base, backend.coefficient_bound())
        k = params.k
        if len(moduli) > 8:
            with ThreadPoolExecutor(_threads()) as ex:
                per = list(ex.map(lambda n: _setup_one(n, k), moduli))
        else:
            per = [_setup_one(n, k) for n in moduli]
        nl = np.stack([p[0] for p in per])
        npl = np.stack([p[1] for p in per])
        tnl = np.stack([p[2] for p in per])
        self.moduli = [p[3] for p in per]
        self.backend = backend
        self.params = params
        self.base = base
        self.state = backend.create(k, params.len, base, nl, npl, tnl)

    def slots(self) -> int:
        return len(self.moduli)

    def modulus(self, i: int) -> int:
        return self.moduli[i].n

    def backend_and_state(self):
        return self.backend, self.state

    def _mont(self, i: int, x: int) -> int:
        m = self.moduli[i]
        x %= m.n
        if x == 1:
            return m.r
        return gmp.mulmod(x, m.r, m.n)

    def load(self, i: int, x: int) -> None:
        """Uploads x (any integer) to slot i in Montgomery form (batch.rs:125-131)."""
        self.backend.load(self.state, i, to_limbs(self._mont(i, int(x)), self.params.k))

    def load_all(self, xs) -> None:
        """`load` on every slot with one upload when the backend supports it."""
        limbs = np.stack([to_limbs(self._mont(i, int(x)), self.params.k) for i, x in enumerate(xs)])
        if hasattr(self.backend, "load_all"):
            self.backend.load_all(self.state, limbs)
        else:
            for i in range(len(xs)):
                self.backend.load(self.state, i, limbs[i])

    def load_raw(self, i: int, xm: int) -> None:
        """Writes a raw Montgomery-form value in [0, 2N) (batch.rs:133-138)."""
        if not 0 <= xm < 2 * self.moduli[i].n:
            raise MontMulError("raw value outside [0, 2N)")
        self.backend.load(self.state, i, to_limbs(xm, self.params.k))

    def set_exponent(self, i: int, e: int) -> None:
        """MSB-first exponent whose bits drive `run` (batch.rs:140-150)."""
        words, nbits = exponent_words(int(e))
        self.backend.set_exponent(self.state, i, words, nbits)

    def set_exponents(self, es) -> None:
        """`set_exponent` on every slot with one upload when the backend supports it."""
        if not hasattr(self.backend, "set_exponents"):
            for i, e in enumerate(es):
                self.set_exponent(i, e)
            return
        ws = [exponent_words(int(e)) for e in es]
        ew = max(1, max(len(w) for w, _ in ws))
        words = np.zeros((len(ws), ew), np.uint32)
        for i, (w, _) in enumerate(ws):
            words[i, : len(w)] = w
        self.backend.set_exponents(self.state, words, np.array([nb for _, nb in ws], np.uint32))

    def run(self, bits: int) -> None:
        """Up to `bits` exponent bits on every active slot (batch.rs:152-155)."""
        self.backend.run(self.state, int(bits))

    def remaining(self, i: int) -> int:
        return self.backend.remaining(self.state, i)

    def mul(self, out: int, a: int, b: int) -> None:
        """a b mod N of slots a, b into slot out; they must share the modulus (batch.rs:162-165)."""
        if not (self.moduli[out].n == self.moduli[a].n == self.moduli[b].n):
            raise MontMulError("mul needs slots that share a modulus")
        self.backend.mul(self.state, out, a, b)

    def read_raw(self, i: int) -> int:
        """Montgomery-form value in [0, 2N) as the backend holds it (batch.rs:168-171)."""
        return from_limbs(self.backend.read(self.state, i))

    def read(self, i: int) -> int:
        """Canonical value in [0, N), out of Montgomery form (batch.rs:173-176)."""
        m = self.moduli[i]
        return gmp.mulmod(self.read_raw(i), m.rinv, m.n)

    def prepare(self, n: int):
        """The host set-up of modulus n for this batch's limb count (N', R mod N, R^-1 mod N, the
        limb rows): what refill computes, done ahead, e.g. while the device runs."""
        n = int(n)
        if n <= 1 or n % 2 == 0:
            raise MontMulError("modulus must be odd and > 1")
        k = self.params.k
        if Params.for_bits(n.bit_length(), self.backend.supported_lengths()).len > self.params.len or \
                n.bit_length() + 4 > 32 * k:
            raise MontMulError("modulus does not fit this batch's length")
        return _setup_one(n, k)

    def refill(self, slots, moduli, xs, exps, setups=None) -> None:
        """Replaces the moduli of `slots` and loads x and an exponent into each, the other slots
        keeping their state on the device (a serving loop's in-place refill; no counterpart in
        the reference). Every new modulus must fit this batch's length and limb count. `setups`
        may carry each modulus's prepare() result, computed earlier."""
        slots = [int(i) for i in slots]
        moduli = [int(n) for n in moduli]
        k = self.params.k
        per = [s if s is not None and s[3].n == n else self.prepare(n)
               for n, s in zip(moduli, setups if setups is not None else [None] * len(moduli))]
        self.backend.set_moduli(self.state, slots, np.stack([p[0] for p in per]), np.stack([p[1] for p in per]))
        for i, p in zip(slots, per):
            self.moduli[i] = p[3]
        x = np.stack([to_limbs(self._mont(i, int(v)), k) for i, v in zip(slots, xs)])
        ws = [exponent_words(int(e)) for e in exps]
        ew = max(1, max(len(w) for w, _ in ws))
        words = np.zeros((len(ws), ew), np.uint32)
        for r, (w, _) in enumerate(ws):
            words[r, : len(w)] = w
        self.backend.write_slots(self.state, slots, x, words, np.array([nb for _, nb in ws], np.uint32))

    def read_raw_slots(self, slots):
        """Raw Montgomery-form values of several slots with one device read."""
        rows = self.backend.read_slots(self.state, [int(i) for i in slots])
        return [from_limbs(r) for r in rows]

    def is_one(self, i: int) -> bool:
        """True if slot i holds 1: raw R mod N or R mod N + N (batch.rs:179-183)."""
        m = self.moduli[i]
        v = self.read_raw(i)
        return v == m.r or v == m.r + m.n


def fermat(backend, moduli, base: int = 3, chunk: int = 1 << 16):
    """Fermat base-`base` PRP test of every modulus: load 1, run N - 1, check for 1 (batch.rs:187-198)."""
    if chunk <= 0:
        raise MontMulError("chunk must be positive")
    b = ModBatch(backend, moduli, base)
    b.load_all([1] * b.slots())
    b.set_exponents([m.n - 1 for m in b.moduli])
    while any(b.remaining(i) > 0 for i in range(b.slots())):
        b.run(chunk)
    return [b.is_one(i) for i in range(b.slots())]
