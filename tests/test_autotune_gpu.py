"""Kernel shapes and the autotuner: every alternative shape of a ring degree
returns exactly the default shape's values (and the oracle's) for the canonical
forward, the inverse and the fused round trip; pg_ntt_autotune picks a valid
shape per mode and the table keeps computing the same values afterwards."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 15, 16])
def test_every_shape_matches_default_and_oracle(gpu, log_n):
    P = gpu
    n, L, polys = 1 << log_n, 3, 3
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    t = P.DcrtTable(log_n, moduli)
    ref = O.DcrtTable(log_n, moduli)
    x = np.concatenate([O.uniform_rns(0xA7 + log_n, 10 * p, moduli, n).ravel() for p in range(polys)])
    plain = O.uniform_rns(0xB7, 0, moduli, n)
    exp_fwd = ref.forward(x.copy())
    exp_inv = ref.inverse(x.copy())
    exp_rt = ref.polymul_roundtrip(x.copy(), plain)
    dplain = P.DeviceBuffer.from_numpy(plain)
    dq = P.DeviceBuffer(plain.size)
    t.shoup_prepare(dplain, dq, 1)
    for v in range(P.variant_count(log_n)):
        for mode in range(3):
            t.set_variant(mode, v)
        d = P.DeviceBuffer.from_numpy(x)
        t.forward(d, polys)
        assert np.array_equal(d.numpy(), exp_fwd), f"forward, shape {v}"
        d = P.DeviceBuffer.from_numpy(x)
        t.inverse(d, polys)
        assert np.array_equal(d.numpy(), exp_inv), f"inverse, shape {v}"
        d = P.DeviceBuffer.from_numpy(x)
        t.polymul_ntt_plain(d, dplain, dq, polys)
        assert np.array_equal(d.numpy(), exp_rt), f"round trip, shape {v}"
        # the lazy forward keeps the default shape whatever the setting
        d = P.DeviceBuffer.from_numpy(x)
        t.forward(d, polys, lazy=True)
        assert np.array_equal(d.numpy(), ref.forward(x.copy(), lazy=True)), f"lazy forward, shape {v}"


@pytest.mark.parametrize("log_n", [11, 15])
def test_autotune_picks_valid_shapes(gpu, log_n):
    P = gpu
    n, L = 1 << log_n, 4
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    t = P.DcrtTable(log_n, moduli)
    res = t.autotune(16)
    for mode in ("forward", "inverse", "round_trip"):
        assert 0 <= res[mode]["variant"] < P.variant_count(log_n)
        assert res[mode]["us"] > 0
    assert res["rows"] == 16 * L
    x = np.concatenate([O.uniform_rns(0xC1, 10 * p, moduli, n).ravel() for p in range(2)])
    d = P.DeviceBuffer.from_numpy(x)
    t.forward(d, 2)
    t.inverse(d, 2)
    assert np.array_equal(d.numpy(), x)


def test_bad_variant_rejected(gpu):
    P = gpu
    t = P.DcrtTable(12, O.ntt_primes(1 << 50, 1 << 13, 1))
    with pytest.raises(P.PrimusGpuError):
        t.set_variant(0, P.variant_count(12))
    with pytest.raises(P.PrimusGpuError):
        t.set_variant(3, 0)
