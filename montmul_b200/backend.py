"""The B200 backend: a ctypes binding of the C ABI in include/montmul_b200.h.

`B200` plays the role of the reference's `Gpu` backend (montmul/src/gpu/mod.rs) behind the
same `Limits` + `Backend` methods, so `ModBatch(B200(), moduli, 3)` drives the CUDA kernels.
There is no CPU fallback: constructing a `B200` without the built library or without a CUDA
device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .batch import MontMulError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmontmul_b200.so")

MM_OK, MM_ERR_ARG, MM_ERR_OOM, MM_ERR_CARRY, MM_ERR_CUDA, MM_ERR_UNSUPPORTED = range(6)

# Every symbol include/montmul_b200.h declares, with (argtypes, restype).
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_sz = C.c_size_t
_vp = C.c_void_p


class Options(C.Structure):
    """mm_b200_options (GpuOptions, gpu/mod.rs:28-45)."""
    _fields_ = [("device", C.c_int), ("force_global", C.c_int), ("wraparound", C.c_int),
                ("max_launch_steps", C.c_int)]


SIGNATURES = {
    "mm_b200_last_error": ([], C.c_char_p),
    "mm_b200_open": ([C.POINTER(Options), C.POINTER(_vp)], C.c_int),
    "mm_b200_close": ([_vp], None),
    "mm_b200_sm_count": ([_vp], C.c_int),
    "mm_b200_free_memory": ([_vp], _sz),
    "mm_b200_max_dyn_smem": ([_vp], C.c_int),
    "mm_b200_device_name": ([_vp], C.c_char_p),
    "mm_b200_coefficient_bound": ([C.POINTER(C.c_uint64)], None),
    "mm_b200_supported_lengths": ([C.POINTER(_sz), _sz], _sz),
    "mm_b200_full_k": ([_vp], C.c_int),
    "mm_b200_batch_bytes": ([_sz, _sz, _sz], _sz),
    "mm_b200_create": ([_vp, _sz, _sz, C.c_uint32, _sz, _u32p, _u32p, _u32p, C.POINTER(_vp)], C.c_int),
    "mm_b200_load": ([_vp, _sz, _u32p], C.c_int),
    "mm_b200_load_all": ([_vp, _u32p], C.c_int),
    "mm_b200_set_exponent": ([_vp, _sz, _u32p, _sz, _sz], C.c_int),
    "mm_b200_set_exponents": ([_vp, _u32p, _sz, _u32p], C.c_int),
    "mm_b200_run": ([_vp, _sz], C.c_int),
    "mm_b200_run_bare": ([_vp, _sz], C.c_int),
    "mm_b200_mul": ([_vp, _sz, _sz, _sz], C.c_int),
    "mm_b200_read": ([_vp, _sz, _u32p], C.c_int),
    "mm_b200_read_all": ([_vp, _u32p], C.c_int),
    "mm_b200_remaining": ([_vp, _sz], _sz),
    "mm_b200_slots": ([_vp], _sz),
    "mm_b200_destroy": ([_vp], None),
    "mm_b200_run_async": ([_vp, _sz], C.c_int),
    "mm_b200_sync": ([_vp], C.c_int),
    "mm_b200_push": ([_vp], C.c_int),
    "mm_b200_stream": ([_vp], _vp),
    "mm_b200_launches": ([_vp], C.c_uint64),
    "mm_b200_mul_noalloc": ([_vp, _sz, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "mm_b200_wait_check": ([_vp, C.c_uint64], C.c_int),
    "mm_b200_run_items_async": ([_vp, _sz, _vp, _vp], C.c_int),
    "mm_b200_blocks_per_sm": ([_vp], C.c_int),
    "mm_b200_busy": ([_vp], C.c_int),
    "mm_b200_bfly_peak": ([C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "mm_b200_set_schedule": ([_vp, _vp], C.c_int),
    "mm_b200_get_schedule": ([_vp, _vp], C.c_int),
    "mm_b200_set_moduli": ([_vp, _sz, _vp, _vp, _vp], C.c_int),
    "mm_b200_write_slots": ([_vp, _sz, _vp, _vp, _vp, _sz, _vp], C.c_int),
    "mm_b200_read_slots": ([_vp, _sz, _vp, _vp], C.c_int),
    "mm_b200_plan_create": ([_vp, _sz, _sz, C.POINTER(_vp)], C.c_int),
    "mm_b200_plan_run_async": ([_vp, _sz], C.c_int),
    "mm_b200_plan_sync": ([_vp], C.c_int),
    "mm_b200_plan_run_each_async": ([_vp, _vp], C.c_int),
    "mm_b200_plan_run_each": ([_vp, _vp], C.c_int),
    "mm_b200_plan_run_items": ([_vp, _sz, _vp, _vp, _vp], C.c_int),
    "mm_b200_plan_blocks": ([_vp], C.c_int),
    "mm_b200_plan_wide_blocks": ([_vp], C.c_int),
    "mm_b200_plan_batch_wide": ([_vp, _sz], C.c_int),
    "mm_b200_plan_run": ([_vp, _sz], C.c_int),
    "mm_b200_plan_stream": ([_vp], _vp),
    "mm_b200_plan_launches": ([_vp], C.c_uint64),
    "mm_b200_plan_graph_launches": ([_vp], C.c_uint64),
    "mm_b200_plan_destroy": ([_vp], None),
    "mm_b200_t_upload": ([_vp, _vp, _sz, _sz, C.POINTER(_vp)], C.c_int),
    "mm_b200_t_download_raw": ([_vp, _vp, _vp], C.c_int),
    "mm_b200_t_forward": ([_vp, _sz, _sz], C.c_int),
    "mm_b200_t_inverse": ([_vp, _sz, _sz], C.c_int),
    "mm_b200_t_pointwise": ([_vp, _vp, _vp, _vp, _sz, _sz], C.c_int),
    "mm_b200_t_load_forward": ([_vp, _vp, _sz, _sz, _sz, C.POINTER(_vp)], C.c_int),
    "mm_b200_t_count": ([_vp], _sz),
    "mm_b200_t_len": ([_vp], _sz),
    "mm_b200_t_free": ([_vp], None),
}

P1, P2 = (1 << 31) - 1, (1 << 61) - 1
_CRT_INV = pow(P2 % P1, -1, P1)


def crt(c1: int, c2: int) -> int:
    """The coefficient in [0, M31 M61) with residues c1 mod M31 and c2 mod M61 (field.rs:284-294)."""
    return c2 + P2 * (((c1 - c2) * _CRT_INV) % P1)


class TBuf:
    """Transform-domain data of `count` vectors of one length (the Transform trait's Buf)."""

    def __init__(self, ptr, length, count, owner):
        self.ptr, self.len, self.count, self.owner = ptr, length, count, owner

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().mm_b200_t_free(self.ptr)
            self.ptr = None


class Schedule(C.Structure):
    """mm_b200_schedule: global mode, steps per launch, measured ns per slot-step."""
    _fields_ = [("global_", C.c_int), ("launch_steps", C.c_int), ("step_ns", C.c_double), ("threads", C.c_int)]


def _ptr(a):
    return a.ctypes.data_as(_vp) if a is not None else None

_lib = None


def lib():
    """Loads the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MontMulError(f"{LIB_PATH} is missing: build it with `python -m montmul_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def bfly_peak(device: int = 0, iters: int = 1 << 14):
    """(butterfly pairs per second, kernel ms) of the integer roofline probe."""
    r, ms = C.c_double(), C.c_double()
    _check(lib().mm_b200_bfly_peak(device, iters, C.byref(r), C.byref(ms)))
    return r.value, ms.value


def _check(rc: int) -> None:
    if rc != MM_OK:
        msg = lib().mm_b200_last_error().decode()
        raise MontMulError(msg)


class _Batch:
    def __init__(self, ptr, k, slots):
        self.ptr, self.k, self.slots = ptr, k, slots

    def __del__(self):
        if self.ptr:
            lib().mm_b200_destroy(self.ptr)
            self.ptr = None


class B200:
    """`Gpu`-equivalent backend on one B200 (wraparound path, k = L/2)."""

    def __init__(self, device: int = 0, max_launch_steps: int = 0, force_global: bool = False, tuned: bool = True,
                 wraparound: bool = True):
        """tuned: every new batch takes its length's row of the autotuner's schedule table
        (montmul_b200.tune), unless max_launch_steps or force_global fix the schedule.
        wraparound: GpuOptions::wraparound (gpu/mod.rs:36-44): k = L/2 and the half-length cyclic
        REDC (bit-identical to Cpu::with_wraparound); off, k = k0 and the plain REDC
        (bit-identical to Cpu::default)."""
        self.device = device
        self.wraparound = bool(wraparound)
        opts = Options(device, int(force_global), int(wraparound), max_launch_steps)
        self._tuned = tuned and not max_launch_steps and not force_global
        self._table = None
        ptr = _vp()
        _check(lib().mm_b200_open(C.byref(opts), C.byref(ptr)))
        self._dev = ptr
        n = lib().mm_b200_supported_lengths(None, 0)
        arr = (_sz * n)()
        lib().mm_b200_supported_lengths(arr, n)
        self._lengths = [int(v) for v in arr]

    def __del__(self):
        if getattr(self, "_dev", None):
            lib().mm_b200_close(self._dev)
            self._dev = None

    # Limits (transform.rs:11-20)
    def coefficient_bound(self) -> int:
        q = (C.c_uint64 * 2)()
        lib().mm_b200_coefficient_bound(q)
        return int(q[0]) | (int(q[1]) << 64)

    def supported_lengths(self):
        return list(self._lengths)

    def full_k(self) -> bool:
        return bool(lib().mm_b200_full_k(self._dev))

    # device facts (gpu/mod.rs:83-99)
    def sm_count(self) -> int:
        return int(lib().mm_b200_sm_count(self._dev))

    def free_memory(self) -> int:
        return int(lib().mm_b200_free_memory(self._dev))

    def device_name(self) -> str:
        return lib().mm_b200_device_name(self._dev).decode()

    # Backend (transform.rs:61-77)
    def create(self, k, length, base, n, nprime, two_n):
        slots = n.shape[0]
        ptr = _vp()
        _check(lib().mm_b200_create(self._dev, k, length, base, slots, np.ascontiguousarray(n, np.uint32),
                                    np.ascontiguousarray(nprime, np.uint32),
                                    np.ascontiguousarray(two_n, np.uint32), C.byref(ptr)))
        st = _Batch(ptr, k, slots)
        st.owner = self   # keep the device open while the batch lives
        if self._tuned:
            from . import tune
            if self._table is None:
                self._table = tune.load_table()
            sc = tune.schedule_for(self.device_name(), length, self._table, self.wraparound)
            if sc:
                self.set_schedule(st, sc["global"], sc["launch_steps"], sc["step_ns"], sc.get("block_threads", 0))
        return st

    def load(self, st, i, limbs):
        _check(lib().mm_b200_load(st.ptr, i, np.ascontiguousarray(limbs, np.uint32)))

    def load_all(self, st, limbs):
        _check(lib().mm_b200_load_all(st.ptr, np.ascontiguousarray(limbs, np.uint32)))

    def set_exponent(self, st, i, words, nbits):
        w = np.ascontiguousarray(words, np.uint32)
        if w.size == 0:
            w = np.zeros(1, np.uint32)
        _check(lib().mm_b200_set_exponent(st.ptr, i, w, len(words), nbits))

    def set_exponents(self, st, words, nbits):
        words = np.ascontiguousarray(words, np.uint32)
        _check(lib().mm_b200_set_exponents(st.ptr, words, words.shape[1], np.ascontiguousarray(nbits, np.uint32)))

    def run(self, st, bits):
        _check(lib().mm_b200_run(st.ptr, bits))

    def run_bare(self, st, bits):
        """Gpu::run_bare: steps that stop after the squaring, x unchanged (gpu/mod.rs:109-111)."""
        _check(lib().mm_b200_run_bare(st.ptr, bits))

    def run_async(self, st, bits):
        _check(lib().mm_b200_run_async(st.ptr, bits))

    def push(self, st):
        _check(lib().mm_b200_push(st.ptr))

    def sync(self, st):
        _check(lib().mm_b200_sync(st.ptr))

    def stream(self, st) -> int:
        return int(lib().mm_b200_stream(st.ptr) or 0)

    def launches(self, st) -> int:
        return int(lib().mm_b200_launches(st.ptr))

    def mul(self, st, out, a, b):
        _check(lib().mm_b200_mul(st.ptr, out, a, b))

    def run_items_async(self, st, slots, steps) -> None:
        """One launch over a list: slot slots[i] runs up to steps[i] steps (each slot once);
        returns at once, sync() waits and checks errors."""
        s = np.ascontiguousarray(slots, np.uintp)
        t = np.ascontiguousarray(steps, np.uint32)
        assert s.size == t.size
        _check(lib().mm_b200_run_items_async(st.ptr, s.size, _ptr(s), _ptr(t)))

    def busy(self, st) -> bool:
        """True while work enqueued on the batch's stream is still running."""
        return bool(lib().mm_b200_busy(st.ptr))

    def blocks_per_sm(self, st) -> int:
        """Blocks of the batch's step kernel one SM holds at once."""
        return int(lib().mm_b200_blocks_per_sm(st.ptr))

    def wait_check(self, st, limit_ns: int) -> None:
        """Runs a bulk-copy wait that is bound to run out after limit_ns on the batch's stream;
        raises MontMulError with the time-out message, as run does after a late copy."""
        _check(lib().mm_b200_wait_check(st.ptr, int(limit_ns)))

    def read(self, st, i):
        o = np.zeros(st.k, np.uint32)
        _check(lib().mm_b200_read(st.ptr, i, o))
        return o

    def read_all(self, st):
        o = np.zeros((st.slots, st.k), np.uint32)
        _check(lib().mm_b200_read_all(st.ptr, o))
        return o

    def remaining(self, st, i):
        return int(lib().mm_b200_remaining(st.ptr, i))

    # The Transform trait (transform.rs:22-46; the Gpu impl, gpu/mod.rs:286-319).
    def upload(self, coeffs, length: int, count: int) -> TBuf:
        c = np.ascontiguousarray(coeffs, np.uint32).reshape(-1)
        assert c.size == length * count
        ptr = _vp()
        _check(lib().mm_b200_t_upload(self._dev, _ptr(c), length, count, C.byref(ptr)))
        return TBuf(ptr, length, count, self)

    def download_raw(self, buf: TBuf):
        """(f1, f2): count x L/2 x (re, im) field values in the reference's element order."""
        n = buf.len // 2
        f1 = np.zeros((buf.count * n, 2), np.uint32)
        f2 = np.zeros((buf.count * n, 2), np.uint64)
        _check(lib().mm_b200_t_download_raw(buf.ptr, _ptr(f1), _ptr(f2)))
        return f1, f2

    def download(self, buf: TBuf):
        """Exact coefficients in [0, Q) (CRT of the two fields), count x L, row-major."""
        f1, f2 = self.download_raw(buf)
        n = buf.len // 2
        out = [0] * (buf.count * buf.len)
        for v in range(buf.count):
            for j in range(n):
                e = v * n + j
                out[v * buf.len + j] = crt(int(f1[e, 0]), int(f2[e, 0]))
                out[v * buf.len + j + n] = crt(int(f1[e, 1]), int(f2[e, 1]))
        return out

    def upload_scales(self, scales):
        return np.ascontiguousarray(scales, np.uint32)

    def forward(self, buf: TBuf, length: int, count: int) -> None:
        _check(lib().mm_b200_t_forward(buf.ptr, length, count))

    def inverse(self, buf: TBuf, length: int, count: int) -> None:
        _check(lib().mm_b200_t_inverse(buf.ptr, length, count))

    def pointwise(self, out: TBuf, a: TBuf, b: TBuf, scales, length: int, count: int) -> None:
        sc = None if scales is None else np.ascontiguousarray(scales, np.uint32)
        _check(lib().mm_b200_t_pointwise(out.ptr, a.ptr, b.ptr, _ptr(sc), length, count))

    def load_forward(self, limbs, k: int, length: int, count: int) -> TBuf:
        """k limbs per vector, zero-padded to the length, forward-transformed (gpu/mod.rs load_forward)."""
        li = np.ascontiguousarray(limbs, np.uint32).reshape(-1)
        assert li.size == k * count
        ptr = _vp()
        _check(lib().mm_b200_t_load_forward(self._dev, _ptr(li), k, length, count, C.byref(ptr)))
        return TBuf(ptr, length, count, self)

    # Schedules and in-place refill (no counterpart in the reference's Backend trait).
    def set_schedule(self, st, global_mode, launch_steps: int = 0, step_ns: float = 0.0, threads: int = 0):
        """global_mode: 0 (or False) shared memory, 1 (or True) global mode, 2 cluster mode
        (L = 32768 and 65536: one thread-block cluster per slot, the vector in the cluster's
        shared memory). threads: threads per block of the shared-memory step (0: the default); in
        cluster mode, threads per SM (0 or 512: one block of 8,192 elements per SM; 1024 at
        L = 32768: two blocks of 4,096 elements per SM)."""
        sc = Schedule(int(global_mode), int(launch_steps), float(step_ns), int(threads))
        _check(lib().mm_b200_set_schedule(st.ptr, C.byref(sc)))

    def get_schedule(self, st):
        sc = Schedule()
        _check(lib().mm_b200_get_schedule(st.ptr, C.byref(sc)))
        return {"global": bool(sc.global_), "mode": ("shared", "global", "cluster")[sc.global_],
                "launch_steps": sc.launch_steps, "step_ns": sc.step_ns, "threads": sc.threads}

    def set_moduli(self, st, slots, n, nprime):
        ids = np.ascontiguousarray(slots, np.uintp)
        n = np.ascontiguousarray(n, np.uint32)
        nprime = np.ascontiguousarray(nprime, np.uint32)
        assert n.shape == nprime.shape == (len(ids), st.k)
        _check(lib().mm_b200_set_moduli(st.ptr, len(ids), _ptr(ids), _ptr(n), _ptr(nprime)))

    def write_slots(self, st, slots, x=None, words=None, nbits=None):
        ids = np.ascontiguousarray(slots, np.uintp)
        xa = None if x is None else np.ascontiguousarray(x, np.uint32)
        wa = None if words is None else np.ascontiguousarray(words, np.uint32)
        nb = None if nbits is None else np.ascontiguousarray(nbits, np.uint32)
        if xa is not None:
            assert xa.shape == (len(ids), st.k)
        ew = 0 if wa is None else wa.shape[1]
        _check(lib().mm_b200_write_slots(st.ptr, len(ids), _ptr(ids), _ptr(xa), _ptr(wa), ew, _ptr(nb)))

    def read_slots(self, st, slots):
        ids = np.ascontiguousarray(slots, np.uintp)
        o = np.zeros((len(ids), st.k), np.uint32)
        _check(lib().mm_b200_read_slots(st.ptr, len(ids), _ptr(ids), _ptr(o)))
        return o


class Plan:
    """A mixed-length persistent launch over every slot of several batches on one device
    (mm_b200_plan_*): `run(bits)` advances every slot like ModBatch.run on each batch, in
    launches of `quantum` steps replayed from a CUDA graph. The batches must outlive the plan."""

    def __init__(self, batches, quantum: int = 1 << 16):
        states = [b.backend_and_state()[1] if hasattr(b, "backend_and_state") else b for b in batches]
        arr = (_vp * len(states))(*[s.ptr for s in states])
        ptr = _vp()
        _check(lib().mm_b200_plan_create(arr, len(states), int(quantum), C.byref(ptr)))
        self._p = ptr
        self._keep = list(batches)

    def run(self, bits: int) -> None:
        _check(lib().mm_b200_plan_run(self._p, int(bits)))

    def run_async(self, bits: int) -> None:
        _check(lib().mm_b200_plan_run_async(self._p, int(bits)))

    def run_items(self, batch, slot, steps) -> None:
        """One launch over an explicit list: item i runs up to steps[i] steps of slot slot[i]
        of batch batch[i] (each slot at most once), taken in list order."""
        b = np.ascontiguousarray(batch, np.uint32)
        s = np.ascontiguousarray(slot, np.uint32)
        t = np.ascontiguousarray(steps, np.uint32)
        assert b.size == s.size == t.size and (t.size == 0 or t.min() >= 1)
        _check(lib().mm_b200_plan_run_items(self._p, b.size, _ptr(b), _ptr(s), _ptr(t)))

    def blocks(self) -> int:
        """Workers of the plan's launch that take items other than wide ones (items that run
        at once; two per block)."""
        return int(lib().mm_b200_plan_blocks(self._p))

    def wide_blocks(self) -> int:
        """Blocks of the plan's launch; each takes wide items (L = 16384 in shared mode) one
        at a time, before its two workers take the other items."""
        return int(lib().mm_b200_plan_wide_blocks(self._p))

    def batch_wide(self, i: int) -> bool:
        """Whether the slots of batch i run as wide items."""
        return bool(lib().mm_b200_plan_batch_wide(self._p, i))

    def run_each(self, steps) -> None:
        """One launch in which the slots of batch i run up to steps[i] steps."""
        s = np.ascontiguousarray(steps, np.uintp)
        assert s.size == len(self._keep)
        _check(lib().mm_b200_plan_run_each(self._p, _ptr(s)))

    def sync(self) -> None:
        _check(lib().mm_b200_plan_sync(self._p))

    def stream(self) -> int:
        return int(lib().mm_b200_plan_stream(self._p) or 0)

    def launches(self) -> int:
        return int(lib().mm_b200_plan_launches(self._p))

    def graph_launches(self) -> int:
        return int(lib().mm_b200_plan_graph_launches(self._p))

    def close(self) -> None:
        if getattr(self, "_p", None):
            lib().mm_b200_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        self.close()
