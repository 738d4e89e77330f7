"""The FP64 schedule's twiddle tables store only wq = w / q (a correctly rounded
double); the kernels recover w as rint(wq * q) with one FMA against the
1.5 * 2^52 rounding constant.  That is exact when |wq * q - w| < 1/2; the
kernel comment states the sharper bound |wq * q - w| <= q * 2^-53 < 1/8 for
q < 2^50.  These checks run the same arithmetic exactly (Fraction) on the host
over every twiddle the table builder produces for primes just below 2^50 and on
the extreme values w = 1 and w = q - 1, so the bound is pinned without a GPU.
"""
import random
from fractions import Fraction

import pytest

import primus_b200.ntt as NT

MAGIC = 6755399441055744  # 1.5 * 2^52: doubles in [2^52, 2^53) are the integers


def recover(wq: float, q: int) -> int:
    """fma(wq, q, 1.5 * 2^52) - 1.5 * 2^52: the exact product plus the constant,
    rounded once to the nearest double (an integer in this range)."""
    exact = Fraction(wq) * q + MAGIC
    lo = exact.numerator // exact.denominator
    frac = exact - lo
    r = lo + (1 if frac > Fraction(1, 2) or (frac == Fraction(1, 2) and lo % 2) else 0)
    return r - MAGIC


def check(w: int, q: int):
    wq = w / q  # IEEE division of two exactly represented integers: correctly rounded
    assert 0.0 < wq < 1.0
    assert abs(Fraction(wq) * q - w) <= Fraction(q, 2**53) < Fraction(1, 8)
    assert recover(wq, q) == w


@pytest.mark.parametrize("log_n", [10, 16])
def test_table_twiddles_recover_exactly(log_n):
    for q in NT.ntt_primes(1 << 50, 1 << 17, 2):
        t = NT.host_tables(log_n, q)
        ws = set(int(v) for v in t["root_powers"][1:]) | set(int(v) for v in t["inv_root_powers"][:-1])
        ws.discard(0)
        for w in sorted(ws):
            check(w, q)


def test_extreme_and_random_values():
    rng = random.Random(20250)
    qs = NT.ntt_primes(1 << 50, 1 << 17, 3) + NT.ntt_primes(1 << 40, 1 << 17, 1) + [12289, 3]
    for q in qs:
        for w in {1, 2, q - 1, q - 2, q // 2, q // 2 + 1} - {0}:
            if 0 < w < q:
                check(w, q)
        for _ in range(2000 if q > 1000 else 0):
            check(rng.randrange(1, q), q)
