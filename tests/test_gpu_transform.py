"""The Transform trait on the B200 against the oracle's (the reference Cpu's, cpu.rs:349-407),
through the C ABI: raw field values after forward bit for bit, exact coefficients after the
round trip, pointwise scales above M31, load_forward, exactness and batching. Restates
montmul/tests/gpu.rs:26-90 and the transform cases of tests/common/mod.rs:24-91."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from montmul_b200 import B200
    return B200()


def _coeffs(seed, length, count, half=True):
    """Random 32-bit coefficients; with `half`, only the low half of each vector (a product of
    two such vectors then fits the length)."""
    c = np.random.default_rng(seed).integers(0, 1 << 32, size=(count, length), dtype=np.uint64).astype(np.uint32)
    if half:
        c[:, length // 2:] = 0
    return c.reshape(-1)


def _value(cs):
    """sum c_q 2^(32 q), by halves (linear-time additions stay cheap at 2^16 coefficients)."""
    vals = [int(v) for v in cs]
    width = 32
    while len(vals) > 1:
        if len(vals) % 2:
            vals.append(0)
        vals = [vals[i] + (vals[i + 1] << width) for i in range(0, len(vals), 2)]
        width *= 2
    return vals[0] if vals else 0


@pytest.mark.parametrize("e", range(3, 21))
def test_transform_matches_oracle_bit_for_bit(gpu, oracle, e):
    """tests/gpu.rs:26-42: forward then download_raw, inverse then download, L = 2^3 .. 2^20."""
    length, count = 1 << e, 3
    coeffs = _coeffs(e, length, count)
    gx = gpu.upload(coeffs, length, count)
    cx = oracle.upload(coeffs, length, count)
    gpu.forward(gx, length, count)
    oracle.forward(*cx, length, count)
    g1, g2 = gpu.download_raw(gx)
    assert np.array_equal(g1, cx[0]) and np.array_equal(g2, cx[1]), f"forward, len {length}"
    gpu.inverse(gx, length, count)
    oracle.inverse(*cx, length, count)
    want = oracle.download(*cx, length, count)
    assert gpu.download(gx) == want, f"round trip, len {length}"
    # the round trip restores the input coefficients exactly
    assert want == [int(v) for v in coeffs]


def test_pointwise_scales_above_m31_match_oracle(gpu, oracle):
    """tests/gpu.rs:57-71"""
    length, count = 64, 4
    scales = [0x7FFFFFFF, 0x80000004, 0xFFFFFFFE, 0xFFFFFFFF]
    coeffs = _coeffs(2, length, count, half=False)
    gx = gpu.upload(coeffs, length, count)
    cx = oracle.upload(coeffs, length, count)
    gpu.forward(gx, length, count)
    oracle.forward(*cx, length, count)
    go = gpu.upload(np.zeros(length * count, np.uint32), length, count)
    gpu.pointwise(go, gx, gx, gpu.upload_scales(scales), length, count)
    co = oracle.pointwise(cx, cx, scales, length, count)
    g1, g2 = gpu.download_raw(go)
    assert np.array_equal(g1, co[0]) and np.array_equal(g2, co[1])


@pytest.mark.parametrize("e", [3, 8, 13, 16])
def test_load_forward_matches_upload_forward(gpu, oracle, e):
    """tests/gpu.rs:74-90"""
    length, count = 1 << e, 5
    k = length // 2 - 1
    limbs = _coeffs(e + 100, k * count, 1, half=False)
    padded = np.zeros(length * count, np.uint32)
    for v in range(count):
        padded[v * length:v * length + k] = limbs[v * k:(v + 1) * k]
    cx = oracle.upload(padded, length, count)
    oracle.forward(*cx, length, count)
    g1, g2 = gpu.download_raw(gpu.load_forward(limbs, k, length, count))
    assert np.array_equal(g1, cx[0]) and np.array_equal(g2, cx[1]), f"len {length}"


@pytest.mark.parametrize("length", [1 << e for e in range(3, 19)])
def test_exactness_bound(gpu, length):
    """tests/common/mod.rs:24-53 up to L = 2^18: (2^(32k) - 1)^2 * 4 through forward, pointwise
    with scale 4 and inverse, every coefficient exact."""
    k, c = length // 2, 4
    coeffs = np.zeros(length, np.uint32)
    coeffs[:k] = 0xFFFFFFFF
    x = gpu.upload(coeffs, length, 1)
    gpu.forward(x, length, 1)
    y = gpu.upload(coeffs, length, 1)
    gpu.forward(y, length, 1)
    out = gpu.upload(np.zeros(length, np.uint32), length, 1)
    gpu.pointwise(out, x, y, gpu.upload_scales([c]), length, 1)
    gpu.inverse(out, length, 1)
    got = gpu.download(out)
    sq = (1 << 32) - 1
    for q in range(length):
        cnt = q + 1 if q < k else (2 * k - 1 - q if q < 2 * k - 1 else 0)
        assert got[q] == c * sq * sq * cnt, f"len {length} coeff {q}"


def test_transform_batched(gpu):
    """tests/common/mod.rs:55-91 up to L = 2^16: three vectors with scales [1, 3, 4], then none;
    every product equals the big-integer product."""
    for length in [1 << e for e in range(3, 17)]:
        count = 3
        coeffs = [_coeffs(length + i, length, count) for i in range(2)]
        for scales in ([1, 3, 4], None):
            x = gpu.upload(coeffs[0], length, count)
            gpu.forward(x, length, count)
            y = gpu.upload(coeffs[1], length, count)
            gpu.forward(y, length, count)
            out = gpu.upload(np.zeros(length * count, np.uint32), length, count)
            gpu.pointwise(out, x, y, None if scales is None else gpu.upload_scales(scales), length, count)
            gpu.inverse(out, length, count)
            got = gpu.download(out)
            for v in range(count):
                val = _value(got[v * length:(v + 1) * length])
                a = int.from_bytes(coeffs[0][v * length:(v + 1) * length].tobytes(), "little")
                b = int.from_bytes(coeffs[1][v * length:(v + 1) * length].tobytes(), "little")
                assert val == a * b * (scales[v] if scales else 1), f"len {length} vector {v}"
