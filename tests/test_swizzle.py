"""The shared-memory swizzle, read from the header itself (swz_c in montmul_b200/csrc/mm_common.h,
built for the host with g++): it permutes every aligned run of 16 elements, is linear over XOR
(the pass loops form swz(b + k q) as swz(b) ^ swz(k q)), and every warp access of the
shared-memory kernels' passes and carries takes the minimum number of shared-memory wavefronts.

Wavefront model: a warp's 16-byte accesses are served in phases of 8 lanes and its 8-byte
accesses in phases of 16 lanes; a phase costs the largest number of distinct 4-byte words that
fall into one of the 32 banks (at least 1)."""
import os
import shutil
import subprocess
import tempfile

import pytest

from montmul_b200 import tune

CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "montmul_b200", "csrc")
SPAN = 1 << 13   # the shared-memory lengths: n <= 8192


@pytest.fixture(scope="module")
def swz():
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not found")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "swz.cpp"), os.path.join(d, "swz")
        with open(src, "w") as f:
            f.write('#include "mm_common.h"\n#include <cstdio>\n'
                    "int main() { for (int e = 0; e < %d; ++e) std::printf(\"%%d\\n\", mm::swz_c(e)); }\n" % SPAN)
        subprocess.run([gxx, "-std=c++17", "-I", CSRC, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [int(v) for v in out]


def test_permutes_each_run_of_16(swz):
    for b in range(0, SPAN, 16):
        assert sorted(swz[b:b + 16]) == list(range(b, b + 16))


def test_linear_over_xor(swz):
    assert swz[0] == 0
    for i in range(13):
        for a in range(SPAN):
            assert swz[a ^ (1 << i)] == swz[a] ^ swz[1 << i]


def wavefronts(lane_elems, size, swz):
    """Wavefronts of one warp access: lane_elems are the elements of the active lanes."""
    per = {16: 8, 8: 16}[size]
    cost = ideal = 0
    for p in range(0, 32, per):
        phase = [e for e in lane_elems[p:p + per] if e is not None]
        if not phase:
            continue
        banks = {}
        for e in phase:
            a = size * swz[e]
            for w in range(a // 4, (a + size) // 4):
                banks.setdefault(w % 32, set()).add(w)
        cost += max(len(s) for s in banks.values())
        ideal += 1
    return cost, ideal


def accesses(m, nt):
    """Every (lane elements) warp access of one slot's step at n = 2^m with nt threads: the radix
    passes of the length-n and length-n/2 transforms (group g of a pass with span q = 2^lq holds
    elements ((g >> lq) << (lq + log2 R)) + (g mod q) + k q), and the carries (thread t holds E
    consecutive coefficients from t E; the packing reads or writes element (t E + e) / 2)."""
    n = 1 << m
    for mm in (m, m - 1):
        if mm < 1:
            continue
        lq = mm
        for r in tune.radix_schedule(mm):
            lr = r.bit_length() - 1
            lq -= lr
            q, groups = 1 << lq, (1 << mm) // r
            for w in range(0, min(groups, nt), 32):
                for k in range(r):
                    yield [((g >> lq) << (lq + lr)) + (g & (q - 1)) + k * q if g < groups else None
                           for g in range(w, w + 32)]
    for count in (2 * n, n):
        e_per = max(2, count // nt)
        active = count // e_per
        for w in range(0, min(active, nt), 32):
            for e in range(e_per):
                yield [((t * e_per) % n) + e if t < active else None for t in range(w, w + 32)]
    e_per = max(2, n // nt)
    active = n // e_per
    for w in range(0, min(active, nt), 32):
        for e in range(0, e_per, 2):
            yield [(t * e_per + e) >> 1 if t < active else None for t in range(w, w + 32)]


# (log2 n, threads per slot) of every shared-memory step shape: the uniform kernels' default and
# alternative shapes, the mixed launch's 256-thread workers and its 512-thread wide items.
SHAPES = [(6, 32), (7, 32), (8, 32), (9, 64), (10, 128), (11, 256), (12, 512), (13, 512),
          (11, 256), (12, 256), (13, 1024), (7, 256), (8, 256), (9, 256), (10, 256)]


@pytest.mark.parametrize("m,nt", SHAPES)
def test_every_access_takes_the_minimum_wavefronts(swz, m, nt):
    for lanes in accesses(m, nt):
        for size in (16, 8):
            cost, ideal = wavefronts(lanes, size, swz)
            assert cost == ideal, (m, nt, size, lanes)
