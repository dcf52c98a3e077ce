"""montmul_b200 — a B200-native backend for MontMul's batched Montgomery step.

x <- x^2 c R^-1 mod N (and a b R^-1 mod N) over many independent odd moduli, computed with the
reference's exact integer method (an M31 x M61 right-angle NTT over GF(p^2), Montgomery REDC
with the wraparound correction, CRT and carry) in CUDA kernels for sm_100a.

    from montmul_b200 import B200, ModBatch, fermat
    b = ModBatch(B200(), moduli, 3)
"""
from .batch import ModBatch, MontMulError, Params, fermat, from_limbs, to_limbs, exponent_words  # noqa: F401


def __getattr__(name):
    # The CUDA backend loads its shared library on first use, so the host-only parts of the
    # package import without a GPU.
    if name == "B200":
        from .backend import B200
        return B200
    raise AttributeError(name)
