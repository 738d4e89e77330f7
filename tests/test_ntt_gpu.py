"""GPU parity of the NTT family against the oracle (bit-exact, lazy values too).

Covers every supported ring degree (2^1 .. 2^16: single-CTA and cluster
kernels), single and multi-prime tables, ragged batch counts, the reference's
input ranges ([0,4q) forward, [0,2q) inverse), host-slice drop-in calls,
monomial transforms, the fused fwd -> x plain -> inv launch and the golden
fixtures.  Full-size batches are checked through round-trip identities.
"""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def primes_for(log_n, count, bits=50):
    return O.ntt_primes(1 << bits, 2 << log_n, count)


def lazy_inputs(moduli, n, polys, seed, top):
    """[polys][L][n] values uniform below top*q_l (top = 4 for forward, 2 for inverse)."""
    L = len(moduli)
    out = np.empty((polys, L, n), np.uint64)
    for p in range(polys):
        for l, q in enumerate(moduli):
            out[p, l] = O.uniform(seed, p * L + l, top * q, n)
    return out


@pytest.mark.parametrize("log_n", list(range(1, 17)))
@pytest.mark.parametrize("L", [1, 3])
def test_forward_inverse_bit_exact(gpu, log_n, L):
    n = 1 << log_n
    moduli = primes_for(log_n, L)
    polys = 1 if log_n >= 15 else (3 if log_n >= 12 else 5)
    ref = O.DcrtTable(log_n, moduli)
    tab = gpu.DcrtTable(log_n, moduli)
    for lazy in (True, False):
        x = lazy_inputs(moduli, n, polys, 100 + log_n, 4)
        buf = gpu.DeviceBuffer.from_numpy(x)
        tab.forward(buf, polys, lazy=lazy)
        got = buf.numpy(x.shape)
        exp = ref.forward(x, lazy=lazy)
        assert np.array_equal(got, exp.reshape(x.shape)), f"forward lazy={lazy}"
        y = lazy_inputs(moduli, n, polys, 200 + log_n, 2)
        buf = gpu.DeviceBuffer.from_numpy(y)
        tab.inverse(buf, polys, lazy=lazy)
        got = buf.numpy(y.shape)
        exp = ref.inverse(y, lazy=lazy)
        assert np.array_equal(got, exp.reshape(y.shape)), f"inverse lazy={lazy}"


@pytest.mark.parametrize("log_n", [1, 4, 9, 10, 12, 13, 14, 16])
def test_ragged_batches(gpu, log_n):
    # batch counts that do not fill the last CTA of the multi-row kernels
    n = 1 << log_n
    moduli = primes_for(log_n, 2)
    ref = O.DcrtTable(log_n, moduli)
    tab = gpu.DcrtTable(log_n, moduli)
    for polys in ([0, 1, 7, 33, 65] if log_n < 12 else [0, 1, 2]):
        x = lazy_inputs(moduli, n, max(polys, 1), 7, 4)[:polys].copy()
        buf = gpu.DeviceBuffer(max(x.size, 1))
        if polys:
            buf.upload(x)
        tab.forward(buf, polys)
        if polys:
            assert np.array_equal(buf.numpy()[: x.size].reshape(x.shape), ref.forward(x).reshape(x.shape))


@pytest.mark.parametrize("log_n", [1, 5, 10, 11, 13, 14, 15, 16])
def test_fused_polymul_round_trip(gpu, log_n):
    n = 1 << log_n
    L = 3
    moduli = primes_for(log_n, L)
    polys = 2
    ref = O.DcrtTable(log_n, moduli)
    tab = gpu.DcrtTable(log_n, moduli)
    x = lazy_inputs(moduli, n, polys, 31, 1)
    plain = lazy_inputs(moduli, n, 1, 32, 1)[0]
    exp = ref.polymul_roundtrip(x, plain)
    buf = gpu.DeviceBuffer.from_numpy(x)
    pbuf = gpu.DeviceBuffer.from_numpy(plain)
    qbuf = gpu.DeviceBuffer(plain.size)
    tab.shoup_prepare(pbuf, qbuf, 1)
    tab.polymul_ntt_plain(buf, pbuf, qbuf, polys)
    assert np.array_equal(buf.numpy(x.shape), exp.reshape(x.shape))
    # and it is the product of the three reference calls
    b2 = gpu.DeviceBuffer.from_numpy(x)
    tab.forward(b2, polys)
    tab.mul(b2, pbuf, polys, rhs_polys=1)
    tab.inverse(b2, polys)
    assert np.array_equal(b2.numpy(x.shape), exp.reshape(x.shape))


def test_polymul_equals_schoolbook(gpu):
    # config-1 shape: N = 1024, q = largest prime < 2^50 with q = 1 mod 2048, 64 pairs
    q = O.ntt_primes(1 << 50, 2048, 1)[0]
    tab = gpu.NttTable(10, q)
    a = np.stack([O.uniform(0x5EED0000, 2 * i, q, 1024) for i in range(64)])
    b = np.stack([O.uniform(0x5EED0000, 2 * i + 1, q, 1024) for i in range(64)])
    da, db = gpu.DeviceBuffer.from_numpy(a), gpu.DeviceBuffer.from_numpy(b)
    tab.forward(da, 64)
    tab.forward(db, 64)
    tab.mul(da, db, 64)
    tab.inverse(da, 64)
    got = da.numpy(a.shape)
    for i in range(0, 64, 9):
        assert np.array_equal(got[i], O.naive_negacyclic(a[i], b[i], q))


def test_golden_fixtures(gpu):
    import json
    arrays = np.load(os.path.join(GOLD, "ntt_golden.npz"))
    kats = json.load(open(os.path.join(GOLD, "kats.json")))
    for case in kats["ntt_cases"]:
        label, log_n, q = case["label"], case["log_n"], case["q"]
        tab = gpu.NttTable(log_n, q)
        a = arrays[f"{label}/a"].copy()
        tab.transform_slice(a)
        assert np.array_equal(a, arrays[f"{label}/ntt_a"]), label
        tab.inverse_transform_slice(a)
        assert np.array_equal(a, arrays[f"{label}/a"]), label


def test_host_slice_dropin_lazy(gpu):
    q = O.ntt_primes(1 << 50, 1 << 12, 1)[0]
    tab = gpu.NttTable(11, q)
    ref = O.NttTable(11, q)
    a = O.uniform(5, 5, 4 * q, 2048)
    x = a.copy()
    tab.lazy_transform_slice(x)
    assert np.array_equal(x, ref.forward(a, lazy=True))
    y = x % np.uint64(2 * q)
    z = y.copy()
    tab.lazy_inverse_transform_slice(z)
    assert np.array_equal(z, ref.inverse(y, lazy=True))
    with pytest.raises(ValueError):
        tab.transform_slice(np.zeros(1000, np.uint64))


def test_host_slices_pipelined(gpu):
    # 12 polys of 24 limbs at N = 2^16 (12.6 MB each): 64 MB chunks of 5, 5 and 2
    # polys on the three pipeline streams, in pinned and in pageable host memory
    import ctypes as C
    from primus_b200 import _native as nat
    log_n, L, polys = 16, 24, 12
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    tab = gpu.DcrtTable(log_n, moduli)
    d = gpu.DeviceBuffer(polys * L * n)
    tab.fill_uniform(d, polys, seed=0x9A)
    x = d.numpy()
    plain = gpu.DeviceBuffer(L * n)
    tab.fill_uniform(plain, 1, seed=0x9B)
    plain_q = gpu.DeviceBuffer(L * n)
    tab.shoup_prepare(plain, plain_q, 1)
    want_fwd = gpu.DeviceBuffer.from_numpy(x)
    tab.forward(want_fwd, polys)
    want_rt = gpu.DeviceBuffer.from_numpy(x)
    tab.polymul_ntt_plain(want_rt, plain, plain_q, polys)
    gpu.synchronize()
    # pageable
    y = x.copy()
    tab.transform_slice(y)
    assert np.array_equal(y, want_fwd.numpy())
    tab.inverse_transform_slice(y)
    assert np.array_equal(y, x)
    # pinned, fused round trip on the caller's stream
    hp = C.c_void_p()
    nat.call("pg_host_alloc", C.byref(hp), x.nbytes)
    try:
        host = np.ctypeslib.as_array((C.c_uint64 * x.size).from_address(hp.value))
        host[:] = x
        st = gpu.Stream()
        nat.call("pg_dcrt_polymul_ntt_plain_host", tab.h, hp.value, plain.ptr, plain_q.ptr, polys, st.h)
        assert np.array_equal(host, want_rt.numpy())
    finally:
        nat.call("pg_host_free", hp.value)


@pytest.mark.parametrize("log_n", [1, 6, 11, 16])
def test_monomials(gpu, log_n):
    n = 1 << log_n
    moduli = primes_for(log_n, 2)
    tab = gpu.DcrtTable(log_n, moduli)
    refs = [O.NttTable(log_n, q) for q in moduli]
    out = np.zeros(2 * n, np.uint64)
    # degrees at and above N wrap mod 2N with X^N = -1 (primitive.rs:319 masks the exponent)
    for coeff, deg in [(5, min(7, n - 1)), (1, n - 1), (0, 1), (123456789, 0), (moduli[0] - 1, 1), (5, n + 3),
                       (moduli[0] - 1, 2 * n - 1), (1, 3 * n + 5)]:
        tab.transform_monomial(coeff, deg, out)
        exp = np.concatenate([r.monomial(coeff, deg) for r in refs])
        assert np.array_equal(out, exp), (coeff, deg)
    for deg in (0, 1, n - 1, n, 2 * n - 1, 5 * n + 1):
        tab.transform_coeff_one_monomial(deg, out)
        assert np.array_equal(out, np.concatenate([r.coeff_one_monomial(deg) for r in refs]))
        tab.transform_coeff_minus_one_monomial(deg, out)
        assert np.array_equal(out, np.concatenate([r.coeff_minus_one_monomial(deg) for r in refs]))


def test_extreme_moduli(gpu):
    # 60-bit HEXL prime (4q < 2^64 still holds) and a tiny prime
    for log_n, q in [(11, 1152921504606830593), (3, 17), (12, 536813569)]:
        n = 1 << log_n
        ref = O.NttTable(log_n, q)
        tab = gpu.NttTable(log_n, q)
        a = O.uniform(9, 1, 4 * q, n)
        buf = gpu.DeviceBuffer.from_numpy(a)
        tab.forward(buf, 1, lazy=True)
        assert np.array_equal(buf.numpy(), ref.forward(a, lazy=True))


def _threads():
    return max(1, len(os.sched_getaffinity(0)))


def test_full_size_batched_round_trip(gpu):
    # the batched workload's shape: N = 2^16, L = 24 primes q = 1 mod 2^17, 128 polys;
    # fwd -> inv is the identity on every row, repeated so that an ordering race
    # between the cluster CTAs' shared-memory exchange would show up; the forward
    # outputs of all 128 polys equal the oracle bit for bit
    log_n, L, polys = 16, 24, 128
    moduli = O.ntt_primes(1 << 50, 1 << 17, L)
    tab = gpu.DcrtTable(log_n, moduli)
    buf = gpu.DeviceBuffer(polys * L * (1 << log_n))
    tab.fill_uniform(buf, polys, seed=0x5EED0001)
    orig = buf.numpy()
    ref = O.DcrtTable(log_n, moduli)
    for rep in range(3):
        tab.forward(buf, polys)
        if rep == 0:
            fwd = buf.numpy()
            exp = ref.forward(orig.copy(), threads=_threads())
            bad = np.nonzero((fwd != exp).reshape(polys * L, -1).any(axis=1))[0]
            assert bad.size == 0, f"forward rows {bad[:8].tolist()} differ from the oracle"
        tab.inverse(buf, polys)
        got = buf.numpy()
        bad = np.nonzero((got != orig).reshape(polys * L, -1).any(axis=1))[0]
        assert bad.size == 0, f"rep {rep}: rows {bad[:8].tolist()} differ"
    # device generator equals the oracle generator
    assert np.array_equal(orig[: 1 << log_n], O.uniform(0x5EED0001, 0, moduli[0], 1 << log_n))


def test_full_size_fused_round_trip_repeatable(gpu):
    # fused fwd -> x plain -> inv at full size (the batched workload: N = 2^16,
    # L = 24, 128 polys): every poly equals the oracle and the whole batch is
    # identical across repeated launches (no exchange races)
    log_n, L, polys = 16, 24, 128
    moduli = O.ntt_primes(1 << 50, 1 << 17, L)
    tab = gpu.DcrtTable(log_n, moduli)
    src = gpu.DeviceBuffer(polys * L * (1 << log_n))
    tab.fill_uniform(src, polys, seed=0x5EED0002)
    x = src.numpy()
    plain = O.uniform_rns(0x5EED0003, 0, moduli, 1 << log_n)
    pb, qb = gpu.DeviceBuffer.from_numpy(plain), gpu.DeviceBuffer(plain.size)
    tab.shoup_prepare(pb, qb, 1)
    first = None
    for rep in range(3):
        buf = gpu.DeviceBuffer.from_numpy(x)
        tab.polymul_ntt_plain(buf, pb, qb, polys)
        got = buf.numpy()
        if first is None:
            first = got
            exp = O.DcrtTable(log_n, moduli).polymul_roundtrip(x.copy(), plain, threads=_threads())
            bad = np.nonzero((got != exp).reshape(polys * L, -1).any(axis=1))[0]
            assert bad.size == 0, f"rows {bad[:8].tolist()} (poly = row // {L}) differ from the oracle"
        else:
            assert np.array_equal(got, first), f"rep {rep} differs"


def test_ntt_tables_views(gpu):
    """DcrtTable::ntt_tables / iter: per-prime views over the DCRT table's device arrays
    (pg_ntt_table_view) transform like single-prime tables of the same primes."""
    log_n, L = 12, 3
    n = 1 << log_n
    moduli = primes_for(log_n, L)
    tab = gpu.DcrtTable(log_n, moduli)
    views = tab.ntt_tables()
    assert [v.moduli for v in views] == [[q] for q in moduli]
    assert [v.moduli for v in tab.iter()] == [[q] for q in moduli]
    x = lazy_inputs(moduli, n, 2, 77, 4)
    for l, (v, q) in enumerate(zip(views, moduli)):
        ref = O.NttTable(log_n, q)
        rows = np.ascontiguousarray(x[:, l, :])
        d = gpu.DeviceBuffer.from_numpy(rows)
        v.forward(d, 2)
        assert np.array_equal(d.numpy(rows.shape), np.stack([ref.forward(r.copy()) for r in rows]))
        slice_ = rows[0] % np.uint64(q)
        v.transform_slice(slice_)
        assert np.array_equal(slice_, ref.forward((rows[0] % np.uint64(q)).copy()))
    from primus_b200 import _native as nat
    import ctypes as C
    h = C.c_void_p()
    assert nat.lib().pg_ntt_table_view(tab.h, L, 1, C.byref(h)) == nat.PG_ERR_INVALID_ARGUMENT
    assert nat.lib().pg_ntt_table_view(tab.h, 1, L, C.byref(h)) == nat.PG_ERR_INVALID_ARGUMENT
    del views
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.forward(d, 2)  # the parent keeps working after its views are gone
    assert np.array_equal(d.numpy(x.shape), O.DcrtTable(log_n, moduli).forward(x).reshape(x.shape))
