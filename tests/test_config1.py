"""The CPU-sized Fermat batch: 64 random odd 4,096-bit moduli (GMP seed 2026) with 4 of them
replaced by next_prime primes, base 3, every slot loaded with 1 and run through its whole
exponent N - 1 (4,096 bit-steps at L = 512, k = 256), as `fermat` does (batch.rs:187-198).

Every slot's value is checked against GMP's pow_mod and every verdict against (that value == 1):
on the oracle (the reference Cpu backend with the wraparound path), and on the B200 backend,
whose raw Montgomery limbs must equal the oracle's slot for slot."""
import pytest

from montmul_b200.score import fermat_checked, fermat_workload


@pytest.fixture(scope="module")
def workload():
    return fermat_workload(slots=64, bits=4096, primes=4, seed=2026)


def test_workload_shape(workload):
    moduli, primes = workload
    assert len(moduli) == 64 and len(primes) == 4 and len(set(primes)) == 4
    assert all(n.bit_length() == 4096 and n & 1 for n in moduli)


@pytest.fixture(scope="module")
def oracle_run(workload, oracle):
    moduli, _ = workload
    return fermat_checked(oracle.OracleBackend.wraparound(), moduli, 3)


def test_oracle_fermat_every_slot(workload, oracle_run):
    _, primes = workload
    verdicts, raws, _ = oracle_run
    assert [i for i, v in enumerate(verdicts) if v] == primes
    assert len(raws) == 64


@pytest.mark.gpu
def test_b200_fermat_equals_oracle(workload, oracle_run):
    from montmul_b200 import B200
    moduli, primes = workload
    verdicts, raws, _ = fermat_checked(B200(), moduli, 3)
    assert [i for i, v in enumerate(verdicts) if v] == primes
    assert raws == oracle_run[1]
