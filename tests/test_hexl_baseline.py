"""The timed CPU baseline (oracle/hexl_ifma.c, the reference's HEXL-style
AVX-512 IFMA52 path) returns exactly the scalar restatement's canonical values;
skipped on hosts without avx512ifma."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(not O.hexl_available(), reason="host without avx512ifma")


@pytest.mark.parametrize("log_n", [4, 5, 8, 11, 16])
def test_hexl_matches_scalar(log_n):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, 3)
    t = O.DcrtTable(log_n, moduli)
    hx = O.HexlDcrt(t)
    x = np.concatenate([O.uniform_rns(0x4E, 10 * p, moduli, n).ravel() for p in range(2)])
    x[:3] = [0, moduli[0] - 1, 1]
    assert np.array_equal(hx.forward(x), t.forward(x))
    assert np.array_equal(hx.inverse(x), t.inverse(x))
    plain = O.uniform_rns(0x4F, 0, moduli, n)
    assert np.array_equal(hx.polymul_roundtrip(x.copy(), plain, hx.prepare(plain), threads=2),
                          t.polymul_roundtrip(x, plain))


def test_hexl_rejects_large_moduli():
    t = O.DcrtTable(10, O.ntt_primes(1 << 54, 2048, 1))
    with pytest.raises(ValueError):
        O.HexlDcrt(t)
