"""Seeded random configurations for the FP64 schedule: ring degrees 2^1..2^16,
1-4 limbs, primes of 14 to 50 bits (q = 1 mod 2N), inputs uniform in the ranges
each transform accepts with extreme rows mixed in.  The FP64 schedule must equal
the integer schedule (itself pinned to the oracle) on the canonical forward, the
inverse and the fused round trip; small cases are also checked against the
oracle directly."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _configs(count=40, seed=0xF9):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        log_n = int(rng.integers(1, 17))
        L = int(rng.integers(1, 5))
        bits = int(rng.integers(max(14, log_n + 3), 51))
        try:
            moduli = O.ntt_primes(1 << bits, 2 << log_n, L)
        except ValueError:
            continue
        out.append((log_n, moduli, int(rng.integers(0, 1 << 30))))
    return out


@pytest.mark.parametrize("log_n,moduli,seed", _configs())
def test_fp64_matches_integer_schedule(gpu, log_n, moduli, seed):
    P = gpu
    n, L = 1 << log_n, len(moduli)
    polys = max(1, min(8, (1 << 18) // (n * L)))
    rng = np.random.default_rng(seed)
    q = np.array(moduli, np.uint64)[None, :, None]
    fwd_in = (rng.integers(0, 1 << 62, (polys, L, n), dtype=np.uint64) % (4 * q))
    inv_in = (rng.integers(0, 1 << 62, (polys, L, n), dtype=np.uint64) % (2 * q))
    rt_in = fwd_in % q
    fwd_in[0, :, : n // 2] = (4 * q - 1)[0]  # extremes in the first poly
    inv_in[0, :, : n // 2] = (2 * q - 1)[0]
    plain = (rng.integers(0, 1 << 62, (L, n), dtype=np.uint64) % q[0])
    t = P.DcrtTable(log_n, moduli)
    assert t.fp64
    dp, dq = P.DeviceBuffer.from_numpy(plain), P.DeviceBuffer(plain.size)
    t.shoup_prepare(dp, dq, 1)
    res = {}
    for fp in (True, False):
        t.set_fp64(fp)
        d = P.DeviceBuffer.from_numpy(fwd_in)
        t.forward(d, polys)
        f = d.numpy(fwd_in.shape)
        d = P.DeviceBuffer.from_numpy(inv_in)
        t.inverse(d, polys)
        i = d.numpy(inv_in.shape)
        d = P.DeviceBuffer.from_numpy(rt_in)
        t.polymul_ntt_plain(d, dp, dq, polys)
        res[fp] = (f, i, d.numpy(rt_in.shape))
    for k, name in enumerate(("forward", "inverse", "round trip")):
        assert np.array_equal(res[True][k], res[False][k]), name
    if n * L * polys <= 1 << 14:
        ref = O.DcrtTable(log_n, moduli)
        assert np.array_equal(res[True][0].ravel(), ref.forward(fwd_in.ravel().copy()))
        assert np.array_equal(res[True][2].ravel(), ref.polymul_roundtrip(rt_in.ravel().copy(), plain.ravel()))
