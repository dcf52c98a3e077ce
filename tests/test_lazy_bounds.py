"""The lazy GF(M61) arithmetic of the kernels never overflows 64 bits and keeps every value
stored between passes below 2^61 + 2^34 (interval model in lazy_bounds_model.py). CPU only."""
import lazy_bounds_model as m


def test_butterfly_bounds():
    m.check_butterflies()


def test_pointwise_bounds():
    m.check_pointwise()


def test_model_rejects_a_short_offset():
    """The model itself catches an offset smaller than the subtrahend's bound."""
    import pytest
    with pytest.raises(AssertionError):
        m.sub(m.V(0), m.V(m.ONE), 1)
