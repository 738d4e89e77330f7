"""The headline workload's shape (N = 2^16, L = 24 primes just below 2^50) at full
size, beyond what the oracle checks in seconds: the FP64 schedule and the
integer-only schedule (each pinned to the oracle at smaller sizes) must give the
same residues for the fused round trip, the forward and the inverse, and the
forward followed by the inverse must return the input."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def test_fp64_equals_integer_schedule_at_full_size(gpu):
    P = gpu
    log_n, L, polys = 16, 24, 64  # 0.8 GB of residues: beyond L2
    n = 1 << log_n
    t = P.DcrtTable(log_n, O.ntt_primes(1 << 50, 2 * n, L))
    assert t.fp64
    src = P.DeviceBuffer(polys * L * n)
    t.fill_uniform(src, polys, seed=0xF00D)
    plain, plain_q = P.DeviceBuffer(L * n), P.DeviceBuffer(L * n)
    t.fill_uniform(plain, 1, seed=0xF00E)
    t.shoup_prepare(plain, plain_q, 1)
    x = src.numpy()
    results = {}
    for fp in (True, False):
        t.set_fp64(fp)
        d = P.DeviceBuffer.from_numpy(x)
        t.polymul_ntt_plain(d, plain, plain_q, polys)
        rt = d.numpy()
        d = P.DeviceBuffer.from_numpy(x)
        t.forward(d, polys)
        fwd = d.numpy()
        t.inverse(d, polys)
        assert np.array_equal(d.numpy(), x), f"inverse(forward(x)) != x, fp64={fp}"
        results[fp] = (rt, fwd)
    assert np.array_equal(results[True][0], results[False][0]), "round trip differs between schedules"
    assert np.array_equal(results[True][1], results[False][1]), "forward differs between schedules"
    t.set_fp64(True)
