"""GPU parity of the element-wise DCRT ops (primus_poly) against the oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def setup(gpu, log_n=10, L=3, polys=4, seed=1):
    moduli = O.ntt_primes(1 << 50, 2 << log_n, L)
    n = 1 << log_n
    tab = gpu.DcrtTable(log_n, moduli)
    mk = lambda s: np.stack([O.uniform_rns(seed * 100 + s, p * L, moduli, n) for p in range(polys)])
    return tab, moduli, n, mk


def per_limb(fn, x, *rest, moduli):
    out = x.copy()
    for p in range(x.shape[0]):
        for l, q in enumerate(moduli):
            out[p, l] = fn(x[p, l], *[r[p, l] if r.ndim == 3 else r[l] for r in rest], q)
    return out


@pytest.mark.parametrize("broadcast", [False, True])
def test_mul_add_sub_neg(gpu, broadcast):
    tab, moduli, n, mk = setup(gpu)
    x, y, z = mk(1), mk(2), mk(3)
    if broadcast:
        y, z = y[:1].copy(), z[:1].copy()
    rp = 1 if broadcast else 4
    yb = np.broadcast_to(y, x.shape).copy()
    zb = np.broadcast_to(z, x.shape).copy()
    for name, ref in [("mul", lambda: per_limb(O.mul, x, yb, moduli=moduli)),
                      ("add", lambda: per_limb(O.add, x, yb, moduli=moduli)),
                      ("sub", lambda: per_limb(O.sub, x, yb, moduli=moduli))]:
        d = gpu.DeviceBuffer.from_numpy(x)
        getattr(tab, name)(d, gpu.DeviceBuffer.from_numpy(y), 4, rhs_polys=rp)
        assert np.array_equal(d.numpy(x.shape), ref()), name
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.add_mul(d, gpu.DeviceBuffer.from_numpy(y), gpu.DeviceBuffer.from_numpy(z), 4, rhs_polys=rp)
    exp = x.copy()
    for p in range(4):
        for l, q in enumerate(moduli):
            exp[p, l] = O.add_mul(x[p, l], yb[p, l], zb[p, l], q)
    assert np.array_equal(d.numpy(x.shape), exp)
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.neg(d, 4)
    exp = per_limb(O.neg, x, moduli=moduli)
    assert np.array_equal(d.numpy(x.shape), exp)


def test_neg_of_zero_is_zero(gpu):
    tab, moduli, n, mk = setup(gpu, polys=1)
    d = gpu.DeviceBuffer.from_numpy(np.zeros((1, 3, n), np.uint64))
    tab.neg(d, 1)
    assert not d.numpy().any()


def test_scalar_ops(gpu):
    tab, moduli, n, mk = setup(gpu)
    x, y = mk(4), mk(5)
    sc = [int(O.uniform(9, l, q, 1)[0]) for l, q in enumerate(moduli)]
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.mul_scalar(d, sc, 4)
    exp = x.copy()
    for p in range(4):
        for l, q in enumerate(moduli):
            exp[p, l] = O.mul_scalar(x[p, l], sc[l], q)
    assert np.array_equal(d.numpy(x.shape), exp)
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.add_mul_scalar(d, gpu.DeviceBuffer.from_numpy(y), sc, 4)
    for p in range(4):
        for l, q in enumerate(moduli):
            exp[p, l] = O.add_mul_scalar(x[p, l], y[p, l], sc[l], q)
    assert np.array_equal(d.numpy(x.shape), exp)
    with pytest.raises(gpu.PrimusGpuError):
        tab.mul_scalar(d, [moduli[0], 1, 1], 4)  # scalar must be below its modulus


def test_shoup_prepare_and_prepared_mul(gpu):
    tab, moduli, n, mk = setup(gpu)
    x, w = mk(6), mk(7)[:1].copy()
    dw, dq = gpu.DeviceBuffer.from_numpy(w), gpu.DeviceBuffer(w.size)
    tab.shoup_prepare(dw, dq, 1)
    wq = dq.numpy(w.shape)
    for l, q in enumerate(moduli):
        exp = np.array([O.lib().orc_shoup_quotient(int(v), q) for v in w[0, l]], np.uint64)
        assert np.array_equal(wq[0, l], exp)
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.mul_prepared(d, dw, dq, 4, rhs_polys=1)
    exp = per_limb(O.mul, x, np.broadcast_to(w, x.shape).copy(), moduli=moduli)
    assert np.array_equal(d.numpy(x.shape), exp)


def test_butterfly_mul_factor(gpu):
    tab, moduli, n, mk = setup(gpu, polys=2)
    a, s, w = mk(8), mk(9), mk(10)[:1].copy()
    dw, dq = gpu.DeviceBuffer.from_numpy(w), gpu.DeviceBuffer(w.size)
    tab.shoup_prepare(dw, dq, 1)
    da, ds, db = gpu.DeviceBuffer.from_numpy(a), gpu.DeviceBuffer.from_numpy(s), gpu.DeviceBuffer(a.size)
    tab.butterfly_mul_factor(da, ds, dw, dq, db, 2)
    for p in range(2):
        for l, q in enumerate(moduli):
            ea, eb = O.butterfly_mul_factor(a[p, l], s[p, l], w[0, l], q)
            assert np.array_equal(da.numpy(a.shape)[p, l], ea)
            assert np.array_equal(db.numpy(a.shape)[p, l], eb)


@pytest.mark.parametrize("bits", [15, 31, 45, 55, 60, 62])
def test_products_across_modulus_widths(gpu, bits):
    """The multiply paths hold for every modulus width the table accepts, with
    operands at the extremes (0, 1, q-1) mixed into uniform residues."""
    log_n, L, polys = 10, 2, 2
    n = 1 << log_n
    moduli = O.ntt_primes(1 << bits, 2 << log_n, L)
    tab = gpu.DcrtTable(log_n, moduli)
    rng = np.random.default_rng(bits)

    def operand(s):
        v = np.stack([O.uniform_rns(1000 * bits + s, p * L, moduli, n) for p in range(polys)])
        for l, q in enumerate(moduli):
            pick = rng.integers(0, 4, size=(polys, n))
            v[:, l] = np.where(pick == 0, np.uint64(q - 1), np.where(pick == 1, np.uint64(0), v[:, l]))
        return v

    x, y, z = operand(1), operand(2), operand(3)
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.mul(d, gpu.DeviceBuffer.from_numpy(y), polys)
    assert np.array_equal(d.numpy(x.shape), per_limb(O.mul, x, y, moduli=moduli))
    d = gpu.DeviceBuffer.from_numpy(x)
    tab.add_mul(d, gpu.DeviceBuffer.from_numpy(y), gpu.DeviceBuffer.from_numpy(z), polys)
    exp = x.copy()
    for p in range(polys):
        for l, q in enumerate(moduli):
            exp[p, l] = O.add_mul(x[p, l], y[p, l], z[p, l], q)
    assert np.array_equal(d.numpy(x.shape), exp)
    for sc in ([q - 1 for q in moduli], [1, 0], [int(O.uniform(bits, l, q, 1)[0]) for l, q in enumerate(moduli)]):
        d = gpu.DeviceBuffer.from_numpy(x)
        tab.mul_scalar(d, sc, polys)
        exp = x.copy()
        for p in range(polys):
            for l, q in enumerate(moduli):
                exp[p, l] = O.mul_scalar(x[p, l], sc[l], q)
        assert np.array_equal(d.numpy(x.shape), exp)
        d = gpu.DeviceBuffer.from_numpy(x)
        tab.add_mul_scalar(d, gpu.DeviceBuffer.from_numpy(y), sc, polys)
        for p in range(polys):
            for l, q in enumerate(moduli):
                exp[p, l] = O.add_mul_scalar(x[p, l], y[p, l], sc[l], q)
        assert np.array_equal(d.numpy(x.shape), exp)
