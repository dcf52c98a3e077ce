"""mm_b200_mul_noalloc: the product entry point for callers that cannot allocate device memory
when they multiply (a service whose device memory belongs to its own pool allocator, or a loop
that cannot take cudaFree's device synchronization).

The test owns its device buffers (allocated here, as such a caller would have them already),
calls the entry point twice in a row with different operands, and requires each result to equal,
limb for limb, what the allocating entry point mm_b200_mul writes for the same operands and what
the oracle (the reference Cpu backend with the wraparound path) computes for the same product.
It runs last in the suite, and also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import common
from montmul_b200 import ModBatch, to_limbs
from montmul_b200.gmp import RandState

pytestmark = pytest.mark.gpu


def _device_limbs(torch, limbs):
    return torch.from_numpy(np.ascontiguousarray(limbs, np.uint32).view(np.int32)).cuda()


@pytest.mark.parametrize("bits", [1000, 87_914, 200_000])
def test_mul_noalloc_matches_mul(bits, oracle):
    torch = pytest.importorskip("torch")
    from montmul_b200 import B200
    from montmul_b200.backend import lib

    rng = RandState(bits)
    n = common.rand_odd(rng, bits)
    batch = ModBatch(B200(), [n, n, n, n], 3)
    k = batch.params.k
    vals = [rng.random_below(n) for _ in range(3)]
    for i, v in enumerate(vals):
        batch.load(i, v)
    be, st = batch.backend_and_state()
    ref = ModBatch(oracle.OracleBackend.wraparound(), [n, n, n, n], 3)
    for i, v in enumerate(vals):
        ref.load(i, v)

    out = torch.zeros(k, dtype=torch.int32, device="cuda")
    err = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    for a, b in [(0, 1), (2, 0)]:   # two calls in a row, different operands
        # The allocating entry point's result for the same operands, via slot 3.
        batch.mul(3, a, b)
        want = to_limbs(batch.read_raw(3), k)
        da = _device_limbs(torch, to_limbs(batch.read_raw(a), k))
        db = _device_limbs(torch, to_limbs(batch.read_raw(b), k))
        torch.cuda.synchronize()
        rc = lib().mm_b200_mul_noalloc(st.ptr, 3, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()),
                                       C.c_void_p(out.data_ptr()), C.c_void_p(err.data_ptr()), None)
        assert rc == 0, lib().mm_b200_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32)
        assert int(err.item()) == 0
        assert np.array_equal(got, want), f"bits {bits} operands ({a}, {b})"
        ref.mul(3, a, b)
        assert np.array_equal(got, to_limbs(ref.read_raw(3), k)), f"bits {bits} operands ({a}, {b}): oracle"
        assert batch.read(3) == vals[a] * vals[b] % n
