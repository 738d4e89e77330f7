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


def _fp_variants(P, log_n):
    return [v for v in range(1, P.variant_count(log_n)) if P.variant_name(log_n, v).startswith("fp64")]


@pytest.mark.parametrize("log_n,bits", [(10, 50), (10, 20), (12, 50), (13, 45), (16, 50), (16, 24)])
def test_fp64_shapes_at_the_bounds(gpu, log_n, bits):
    """The FP64 schedule's bounds are tight for q just below 2^50: forward inputs up to
    4q - 1 (the reference's accepted range), inverse inputs up to 2q - 1, all-(q-1)
    rows and plaintexts, zeros; small moduli too.  Every FP64 shape equals the oracle."""
    P = gpu
    n, L = 1 << log_n, 3
    moduli = O.ntt_primes(1 << bits, 2 * n, L)
    t = P.DcrtTable(log_n, moduli)
    ref = O.DcrtTable(log_n, moduli)
    q = np.array(moduli, np.uint64)[:, None]
    rng = np.random.default_rng(log_n * 100 + bits)
    rows_fwd = [np.broadcast_to(4 * q - 1, (L, n)), np.zeros((L, n), np.uint64), np.broadcast_to(q - 1, (L, n)),
                (rng.integers(0, 1 << 62, (L, n), dtype=np.uint64) % (4 * q))]
    rows_inv = [np.broadcast_to(2 * q - 1, (L, n)), np.broadcast_to(q - 1, (L, n)),
                (rng.integers(0, 1 << 62, (L, n), dtype=np.uint64) % (2 * q)), np.zeros((L, n), np.uint64)]
    xf = np.concatenate([r.astype(np.uint64).ravel() for r in rows_fwd])
    xi = np.concatenate([r.astype(np.uint64).ravel() for r in rows_inv])
    xc = xf % np.tile(np.repeat(np.array(moduli, np.uint64), n), len(rows_fwd))
    plain = np.broadcast_to(q - 1, (L, n)).astype(np.uint64).ravel().copy()
    polys = len(rows_fwd)
    exp_fwd = ref.forward(xf.copy())
    exp_inv = ref.inverse(xi.copy())
    exp_rt = ref.polymul_roundtrip(xc.copy(), plain)
    dplain = P.DeviceBuffer.from_numpy(plain)
    dq = P.DeviceBuffer(plain.size)
    t.shoup_prepare(dplain, dq, 1)
    fps = _fp_variants(P, log_n)
    assert fps, "no FP64 shape for this degree"
    for v in [0] + fps:  # variant 0: the default dispatch, FP64 for these moduli
        for mode in range(3):
            t.set_variant(mode, v)
        d = P.DeviceBuffer.from_numpy(xf)
        t.forward(d, polys)
        assert np.array_equal(d.numpy(), exp_fwd), f"forward, {P.variant_name(log_n, v)}"
        d = P.DeviceBuffer.from_numpy(xi)
        t.inverse(d, polys)
        assert np.array_equal(d.numpy(), exp_inv), f"inverse, {P.variant_name(log_n, v)}"
        d = P.DeviceBuffer.from_numpy(xc)
        t.polymul_ntt_plain(d, dplain, dq, polys)
        assert np.array_equal(d.numpy(), exp_rt), f"round trip, {P.variant_name(log_n, v)}"


def test_fp64_shapes_skip_wide_moduli(gpu):
    """A modulus at or above 2^50 keeps the integer schedules whatever shape is set."""
    P = gpu
    log_n, n = 12, 1 << 12
    moduli = O.ntt_primes(1 << 50, 2 * n, 1) + O.ntt_primes(1 << 55, 2 * n, 1)
    t = P.DcrtTable(log_n, moduli)
    ref = O.DcrtTable(log_n, moduli)
    x = O.uniform_rns(0xD1, 0, moduli, n).ravel()
    for v in _fp_variants(P, log_n):
        for mode in range(3):
            t.set_variant(mode, v)
        d = P.DeviceBuffer.from_numpy(x)
        t.forward(d, 1)
        assert np.array_equal(d.numpy(), ref.forward(x.copy()))
        t.inverse(d, 1)
        assert np.array_equal(d.numpy(), x)


def test_fp64_switch_keeps_values(gpu):
    """pg_ntt_set_fp64: integer-only and FP64 schedules give the same residues; the
    switch is refused for a modulus at or above 2^50."""
    P = gpu
    log_n, n, L, polys = 14, 1 << 14, 3, 2
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    t = P.DcrtTable(log_n, moduli)
    assert t.fp64
    ref = O.DcrtTable(log_n, moduli)
    x = np.concatenate([O.uniform_rns(0xE1, 10 * p, moduli, n).ravel() for p in range(polys)])
    plain = O.uniform_rns(0xE2, 0, moduli, n)
    dplain = P.DeviceBuffer.from_numpy(plain)
    dq = P.DeviceBuffer(plain.size)
    t.shoup_prepare(dplain, dq, 1)
    for fp in (False, True, False):
        t.set_fp64(fp)
        assert t.fp64 == fp
        d = P.DeviceBuffer.from_numpy(x)
        t.forward(d, polys)
        assert np.array_equal(d.numpy(), ref.forward(x.copy()))
        t.inverse(d, polys)
        assert np.array_equal(d.numpy(), x)
        d = P.DeviceBuffer.from_numpy(x)
        t.polymul_ntt_plain(d, dplain, dq, polys)
        assert np.array_equal(d.numpy(), ref.polymul_roundtrip(x.copy(), plain))
    wide = P.DcrtTable(12, O.ntt_primes(1 << 55, 2 << 12, 1))
    assert not wide.fp64
    with pytest.raises(P.PrimusGpuError):
        wide.set_fp64(True)


def test_calibration_ceilings(gpu):
    """pg_calibrate: the built-in ceilings are positive and in a sane range for a B200."""
    c = gpu.calibrate()
    assert 1000 < c["hbm_copy_gbs"] < 20000
    assert 50 < c["int_butterflies_gps"] < 10000
    assert 50 < c["fp64_butterflies_gps"] < 10000
