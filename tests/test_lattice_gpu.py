"""GPU parity of RNS compose/decompose, fast base conversion, gadget
decomposition, GLev MAC, external product and key switch against the oracle
(bit-exact), plus the reference's decryption properties (ext_prod.rs, ksk.rs)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def big_to_int(row):
    return sum(int(v) << (64 * i) for i, v in enumerate(row))


@pytest.mark.parametrize("L", [1, 2, 3, 8, 16, 24])
def test_compose_decompose(gpu, L):
    moduli = O.ntt_primes(1 << 50, 1 << 12, L)
    base, ref = gpu.RnsBase(moduli), O.RnsBase(moduli)
    assert base.W == ref.W
    n = 1000
    res = O.uniform_rns(11, 0, moduli, n)
    res[:, 0] = 0
    res[:, 1] = [q - 1 for q in moduli]
    dres = gpu.DeviceBuffer.from_numpy(res)
    dval = gpu.DeviceBuffer(n * base.W)
    base.compose(dres, dval, n)
    vals = dval.numpy((n, base.W))
    assert np.array_equal(vals, ref.compose_multiple(res))
    back = gpu.DeviceBuffer(L * n)
    base.decompose(dval, back, n)
    assert np.array_equal(back.numpy((L, n)), res)


def test_rns_kats_on_device(gpu):
    for moduli, residues, value in [([3, 5, 7], [2, 3, 2], 23), ([256, 257], [2, 3], 65538)]:
        base = gpu.RnsBase(moduli)
        d = gpu.DeviceBuffer.from_numpy(np.array(residues, np.uint64).reshape(len(moduli), 1))
        v = gpu.DeviceBuffer(base.W)
        base.compose(d, v, 1)
        assert big_to_int(v.numpy()) == value


def test_not_coprime_error(gpu):
    with pytest.raises(gpu.RnsError) as e:
        gpu.RnsBase([6, 9])
    assert "co-prime" in str(e.value)


def test_wrapping_decompose_small(gpu):
    moduli = [1099511592961, 1099511590913]
    base = gpu.RnsBase(moduli)
    ref = O.RnsBase(moduli)
    for t in (2, 257, 12289):
        small = np.arange(t, dtype=np.uint64) if t < 5000 else O.uniform(3, 3, t, 5000)
        d = gpu.DeviceBuffer.from_numpy(small)
        out = gpu.DeviceBuffer(2 * small.size)
        base.wrapping_decompose_small(d, out, small.size, t)
        assert np.array_equal(out.numpy((2, small.size)), ref.wrapping_decompose_small(small, t))


def test_add_wrapping_decompose_small_scaled(gpu):
    """RNSBase::add_wrapping_decompose_small_values_scaled (base.rs:238-283) equals the
    lift followed by the per-limb scaled add (the oracle's two steps), for t = 2 (no
    centering) and odd / even t, with factors at 0, 1 and q - 1 among them."""
    moduli = O.ntt_primes(1 << 50, 1 << 12, 3)
    base = gpu.RnsBase(moduli)
    ref = O.RnsBase(moduli)
    n = 3000
    for t, factor in ((2, [5, 0, moduli[2] - 1]), (257, [1, moduli[1] - 1, 12345]), (4096, [7, 8, 9])):
        small = O.uniform(11, t, t, n)
        dest = O.uniform_rns(12, t, moduli, n)
        lifted = ref.wrapping_decompose_small(small, t)
        exp = dest.copy()
        for l, q in enumerate(moduli):
            exp[l] = O.add_mul_scalar(dest[l], lifted[l], factor[l], q)
        dd = gpu.DeviceBuffer.from_numpy(dest)
        base.add_wrapping_decompose_small_scaled(gpu.DeviceBuffer.from_numpy(small), dd, n, t, factor)
        assert np.array_equal(dd.numpy(dest.shape), exp), t
    with pytest.raises(gpu.PrimusGpuError):
        base.add_wrapping_decompose_small_scaled(gpu.DeviceBuffer.from_numpy(small), dd, n, 4096,
                                                 [moduli[0], 1, 1])  # factor not below its modulus


@pytest.mark.parametrize("li,lo", [(2, 2), (4, 3), (16, 4), (24, 2)])
def test_fast_convert(gpu, li, lo):
    qs = O.ntt_primes(1 << 50, 1 << 13, li)
    ps = O.ntt_primes(1 << 48, 1 << 13, lo)
    conv = gpu.BaseConverter(gpu.RnsBase(qs), gpu.RnsBase(ps))
    ref = O.BaseConverter(O.RnsBase(qs), O.RnsBase(ps))
    n = 777
    x = O.uniform_rns(5, 0, qs, n)
    dx, dy = gpu.DeviceBuffer.from_numpy(x), gpu.DeviceBuffer(lo * n)
    conv.fast_convert_array(dx, dy, n)
    assert np.array_equal(dy.numpy((lo, n)), ref.fast_convert_array(x))


def test_fast_convert_t_gamma(gpu):
    # the BFV decryption shape of primus_rns/tests/rns.rs: q -> {t, gamma}
    qs = [1125899906826241, 1125899906629633]
    for gamma in (2199023190017, 2305843009213554689):
        conv = gpu.BaseConverter(gpu.RnsBase(qs), gpu.RnsBase([12289, gamma]))
        ref = O.BaseConverter(O.RnsBase(qs), O.RnsBase([12289, gamma]))
        x = O.uniform_rns(8, 0, qs, 512)
        dx, dy = gpu.DeviceBuffer.from_numpy(x), gpu.DeviceBuffer(2 * 512)
        conv.fast_convert_array(dx, dy, 512)
        assert np.array_equal(dy.numpy((2, 512)), ref.fast_convert_array(x))


@pytest.mark.parametrize("moduli_bits,L,lb,rl", [(50, 1, 7, None), (54, 1, 7, None), (50, 2, 30, None),
                                                 (50, 2, 20, None), (50, 3, 1, None), (50, 4, 17, 5),
                                                 (50, 16, 30, None), (50, 24, 25, None), (50, 2, 25, 4)])
def test_gadget_digits(gpu, moduli_bits, L, lb, rl):
    moduli = O.ntt_primes(1 << moduli_bits, 1 << 12, L)
    base, rbase = gpu.RnsBase(moduli), O.RnsBase(moduli)
    g, rg = gpu.GadgetBasis(base, lb, rl), O.GadgetBasis(rbase, lb, rl)
    assert (g.d, g.drop_bits) == (rg.d, rg.drop_bits)
    assert np.array_equal(g.scalar_residues, rg.scalar_residues)
    n = 600
    res = O.uniform_rns(21, 0, moduli, n)
    vals = rbase.compose_multiple(res)
    # edge values: 0, Q - 1, the largest and smallest representable
    Q = 1
    for q in moduli:
        Q *= q
    for i, v in enumerate([0, Q - 1, Q // 2, Q // 2 + 1]):
        vals[i] = [(v >> (64 * w)) & ((1 << 64) - 1) for w in range(rbase.W)]
    dv = gpu.DeviceBuffer.from_numpy(vals)
    dd = gpu.DeviceBuffer(g.d * n)
    g.decompose(dv, dd, n)
    exp = rg.decompose_all(vals)
    assert np.array_equal(dd.numpy((g.d, n)), exp)
    dl = gpu.DeviceBuffer(g.d * L * n)
    g.decompose_lift(dv, dl, n)
    lifted = dl.numpy((g.d, L, n))
    for j in range(g.d):
        assert np.array_equal(lifted[j], rbase.wrapping_decompose_small(exp[j], 1 << lb))


def lattice_setup(log_n, moduli, lb, rl=None):
    table = O.DcrtTable(log_n, moduli)
    rbase = O.RnsBase(moduli)
    rg = O.GadgetBasis(rbase, lb, rl)
    return O.Lattice(table, rbase, rg)


@pytest.mark.parametrize("log_n,L,k,lb,batch", [(9, 2, 1, 30, 3), (9, 2, 2, 20, 2), (11, 1, 1, 7, 5),
                                                (10, 3, 1, 25, 2), (12, 2, 1, 30, 1)])
def test_external_product_bit_exact(gpu, log_n, L, k, lb, batch):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    lat = lattice_setup(log_n, moduli, lb)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    d = g.d
    ggsw = np.concatenate([O.uniform_rns(77, 100 * i, moduli, n).ravel() for i in range((k + 1) * d * (k + 1))])
    glwe = np.concatenate([O.uniform_rns(55, 1000 * b + 10 * i, moduli, n).ravel()
                           for b in range(batch) for i in range(k + 1)])
    exp = lat.external_product(k, glwe, ggsw, batch=batch)
    din, dk = gpu.DeviceBuffer.from_numpy(glwe), gpu.DeviceBuffer.from_numpy(ggsw)
    dout = gpu.DeviceBuffer(glwe.size)
    gpu.external_product(table, g, k, din, dk, dout, batch)
    assert np.array_equal(dout.numpy(), exp)
    # caller-provided workspace gives the same result
    ws = gpu.DeviceBuffer(gpu.ext_product_workspace_size(table, g, k, batch) // 8 + 1)
    dout2 = gpu.DeviceBuffer(glwe.size)
    gpu.external_product(table, g, k, din, dk, dout2, batch, workspace=ws)
    assert np.array_equal(dout2.numpy(), exp)
    # the library's scratch pool, trimmed to nothing, is refilled on the next call
    from primus_b200 import _native as nat
    nat.call("pg_scratch_trim", 0)
    dout3 = gpu.DeviceBuffer(glwe.size)
    gpu.external_product(table, g, k, din, dk, dout3, batch)
    assert np.array_equal(dout3.numpy(), exp)


def test_external_product_decrypts(gpu):
    # primus_fhe_core/tests/ext_prod.rs on the device: Dec(ct (x) GGSW(X^deg)) = m X^deg
    moduli = [1125899906826241, 1125899906629633]
    k, log_n, t, gamma = 2, 9, 12289, 2199023190017
    lat = lattice_setup(log_n, moduli, 30)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), 30)
    sk = np.concatenate([lat.ternary(3, 10 + i) for i in range(k)])
    sk_ntt = lat.table.forward(sk)
    for deg in (0, 100, 511):
        msg_small = O.uniform(40 + deg, 1, t, 512)
        ct = lat.encrypt(k, sk_ntt, lat.base.wrapping_decompose_small(msg_small, t), lat.delta(t), 9 + deg)
        ggsw = lat.ggsw_monomial(k, sk_ntt, [1, 1], deg, 600 + deg)
        din, dk = gpu.DeviceBuffer.from_numpy(lat.table.inverse(ct)), gpu.DeviceBuffer.from_numpy(ggsw)
        dout = gpu.DeviceBuffer(ct.size)
        gpu.external_product(table, g, k, din, dk, dout, 1)
        m = lat.decrypt(k, sk_ntt, dout.numpy(), t, gamma)
        exp = np.roll(msg_small.astype(np.int64), deg)
        exp[:deg] = (t - exp[:deg]) % t
        assert np.array_equal(m, exp.astype(np.uint64))


@pytest.mark.parametrize("k", [1, 3])
def test_glev_mac(gpu, k):
    moduli = O.ntt_primes(1 << 50, 1 << 10, 2)
    log_n, n = 9, 512
    lat = lattice_setup(log_n, moduli, 20)
    table = gpu.DcrtTable(log_n, moduli)
    base = gpu.RnsBase(moduli)
    g = gpu.GadgetBasis(base, 20)
    glev = np.concatenate([O.uniform_rns(1, 50 * i, moduli, n).ravel() for i in range(g.d * (k + 1))])
    acc = np.concatenate([O.uniform_rns(2, 7 * i, moduli, n).ravel() for i in range(k + 1)])
    poly = O.uniform_rns(3, 0, moduli, n).ravel()
    exp = lat.glev_mac_crt_poly(k, acc, glev, poly)
    dacc = gpu.DeviceBuffer.from_numpy(acc)
    gpu.glev_mac_crt_poly(table, g, k, dacc, gpu.DeviceBuffer.from_numpy(glev), gpu.DeviceBuffer.from_numpy(poly))
    assert np.array_equal(dacc.numpy(), exp)
    # BigUint form of the same poly
    big = lat.base.compose_multiple(poly.reshape(2, n))
    dacc2 = gpu.DeviceBuffer.from_numpy(acc)
    gpu.glev_mac_big_uint_poly(table, g, k, dacc2, gpu.DeviceBuffer.from_numpy(glev), gpu.DeviceBuffer.from_numpy(big))
    assert np.array_equal(dacc2.numpy(), exp)


@pytest.mark.parametrize("k_in,k_out,L,batch", [(3, 3, 2, 2), (1, 2, 3, 3), (2, 1, 4, 1)])
def test_key_switch_bit_exact(gpu, k_in, k_out, L, batch):
    log_n, n = 9, 512
    moduli = O.ntt_primes(1 << 50, 1 << 10, L)
    lat = lattice_setup(log_n, moduli, 20)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), 20)
    key = np.concatenate([O.uniform_rns(4, 9 * i, moduli, n).ravel() for i in range(k_in * g.d * (k_out + 1))])
    cin = np.concatenate([O.uniform_rns(5, 100 * b + i, moduli, n).ravel()
                          for b in range(batch) for i in range(k_in + 1)])
    per_in, per_out = (k_in + 1) * L * n, (k_out + 1) * L * n
    exp = np.concatenate([lat.key_switch(k_in, k_out, key, cin[b * per_in:(b + 1) * per_in]) for b in range(batch)])
    dout = gpu.DeviceBuffer(batch * per_out)
    gpu.key_switch(table, g, k_in, k_out, gpu.DeviceBuffer.from_numpy(key), gpu.DeviceBuffer.from_numpy(cin), dout,
                   batch)
    assert np.array_equal(dout.numpy(), exp)


def test_key_switch_decrypts(gpu):
    # primus_fhe_core/tests/ksk.rs on the device
    moduli = [1125899906826241, 1125899906629633]
    k, log_n, t, gamma = 3, 9, 12289, 2305843009213554689
    lat = lattice_setup(log_n, moduli, 20)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), 20)
    sk1 = np.concatenate([lat.ternary(31, 10 + i) for i in range(k)])
    sk2 = np.concatenate([lat.ternary(32, 10 + i) for i in range(k)])
    sk1n, sk2n = lat.table.forward(sk1), lat.table.forward(sk2)
    key = lat.ksk(k, k, sk1, sk2n, 77)
    msg_small = O.uniform(41, 1, t, 512)
    ct = lat.encrypt(k, sk1n, lat.base.wrapping_decompose_small(msg_small, t), lat.delta(t), 42)
    dout = gpu.DeviceBuffer(ct.size)
    gpu.key_switch(table, g, k, k, gpu.DeviceBuffer.from_numpy(key),
                   gpu.DeviceBuffer.from_numpy(lat.table.inverse(ct)), dout, 1)
    assert np.array_equal(lat.decrypt(k, sk2n, dout.numpy(), t, gamma), msg_small)


def test_mismatched_base_rejected(gpu):
    moduli = O.ntt_primes(1 << 50, 1 << 10, 2)
    table = gpu.DcrtTable(9, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli[:1] + [O.ntt_primes(1 << 49, 1 << 10, 1)[0]]), 20)
    d = gpu.DeviceBuffer(4 * 512)
    with pytest.raises(gpu.PrimusGpuError):
        gpu.external_product(table, g, 1, d, d, d, 1)
