"""Secret-key GLWE encryption on the device (pg_glwe_encrypt): bit-exact
against the oracle's restatement with the same samplers
(DcrtGlweSecretKey::encrypt_inplace, primus_fhe_core/src/secret_key/glwe.rs:386-424),
and a device-only encrypt -> decrypt round trip returns the messages."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _lat(log_n, moduli):
    tab = O.DcrtTable(log_n, moduli)
    base = O.RnsBase(moduli)
    return O.Lattice(tab, base, O.GadgetBasis(base, 20))


@pytest.mark.parametrize("log_n,L,k,batch,with_msg", [(10, 2, 1, 3, True), (11, 1, 2, 2, True), (12, 4, 1, 2, False),
                                                       (15, 3, 1, 1, True)])
def test_encrypt_matches_oracle(gpu, log_n, L, k, batch, with_msg):
    n = 1 << log_n
    t = 16
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli)
    sk = np.concatenate([lat.ternary(3, 10 + i) for i in range(k)])
    sk_ntt = lat.table.forward(sk.copy())
    msgs = [lat.base.wrapping_decompose_small(O.uniform(40 + j, 1, t, n), t) for j in range(batch)]
    delta = lat.delta(t)
    exp = np.concatenate([lat.encrypt_cdt(k, sk_ntt, msgs[j] if with_msg else None, delta, 0xE1, 500, j)
                          for j in range(batch)])
    table = gpu.DcrtTable(log_n, moduli)
    enc = gpu.GlweEncryptor(table, 3.2)
    ct = gpu.DeviceBuffer(exp.size)
    dmsg = gpu.DeviceBuffer.from_numpy(np.concatenate([m.ravel() for m in msgs])) if with_msg else None
    enc.encrypt(k, gpu.DeviceBuffer.from_numpy(sk_ntt), dmsg, delta if with_msg else None, 0xE1, 500, ct, batch)
    assert np.array_equal(ct.numpy(), exp)


def test_device_encrypt_decrypt_round_trip(gpu):
    log_n, L, k, t, gamma, batch = 11, 2, 1, 12289, 2199023190017, 4
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli)
    sk_ntt = lat.table.forward(lat.ternary(7, 1).copy())
    msg = np.stack([O.uniform(90 + j, 2, t, n) for j in range(batch)])
    lifted = np.concatenate([lat.base.wrapping_decompose_small(m, t).ravel() for m in msg])
    table = gpu.DcrtTable(log_n, moduli)
    enc = gpu.GlweEncryptor(table)
    dec = gpu.BfvDecryptor(table, t, gamma)
    dsk = gpu.DeviceBuffer.from_numpy(sk_ntt)
    ct = gpu.DeviceBuffer(batch * (k + 1) * L * n)
    enc.encrypt(k, dsk, gpu.DeviceBuffer.from_numpy(lifted), lat.delta(t), 0x77, 0, ct, batch)
    out = gpu.DeviceBuffer(batch * n)
    dec.decrypt(k, dsk, ct, out, batch)
    assert np.array_equal(out.numpy().reshape(batch, n), msg)


def test_wire_format_round_trip(gpu):
    # primus_lattice/src/macros/mod.rs:39-97: containers travel as little-endian u64 bytes
    from primus_b200 import _native as nat
    import ctypes as C
    x = O.uniform(3, 4, (1 << 50) - 27, 4096)
    d = gpu.DeviceBuffer.from_bytes(x.astype("<u8").tobytes())
    assert np.array_equal(d.numpy(), x)
    assert d.to_bytes() == x.astype("<u8").tobytes()
    bad = (C.c_uint8 * 15)()
    assert nat.lib().pg_from_bytes(d.ptr, d.count, bad, 15) == nat.PG_ERR_INVALID_ARGUMENT
    assert nat.lib().pg_to_bytes(d.ptr, d.count, bad, 15) == nat.PG_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("log_n,L,k,batch,with_msg", [(10, 2, 1, 3, True), (11, 1, 2, 2, False), (12, 3, 2, 2, True)])
def test_pk_encrypt_matches_oracle(gpu, log_n, L, k, batch, with_msg):
    """DcrtGlwePublicKey::new / encrypt (primus_fhe_core/src/public_key/glwe.rs:33-126)."""
    n = 1 << log_n
    t = 16
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli)
    sk = np.concatenate([lat.ternary(5, 10 + i) for i in range(k)])
    sk_ntt = lat.table.forward(sk.copy())
    pk = lat.encrypt_cdt(k, sk_ntt, None, [0] * L, 0xF1, 0, 0)
    msgs = [lat.base.wrapping_decompose_small(O.uniform(60 + j, 1, t, n), t) for j in range(batch)]
    delta = lat.delta(t)
    exp = np.concatenate([lat.pk_encrypt_cdt(k, pk, msgs[j] if with_msg else None, delta if with_msg else None,
                                             0xF2, 700, j) for j in range(batch)])
    table = gpu.DcrtTable(log_n, moduli)
    enc = gpu.GlweEncryptor(table, 3.2)
    dpk = gpu.DeviceBuffer(pk.size)
    enc.public_key(k, gpu.DeviceBuffer.from_numpy(sk_ntt), 0xF1, 0, dpk)
    assert np.array_equal(dpk.numpy(), pk)
    ct = gpu.DeviceBuffer(exp.size)
    dmsg = gpu.DeviceBuffer.from_numpy(np.concatenate([m.ravel() for m in msgs])) if with_msg else None
    enc.pk_encrypt(k, dpk, dmsg, delta if with_msg else None, 0xF2, 700, ct, batch)
    assert np.array_equal(ct.numpy(), exp)


@pytest.mark.parametrize("log_n,L,k,lb,degree", [(9, 2, 1, 30, 0), (9, 2, 2, 30, 301), (11, 1, 1, 7, 2047)])
def test_ggsw_pk_monomial_matches_oracle_and_decrypts(gpu, log_n, L, k, lb, degree):
    """DcrtGlwePublicKey::encrypt_monomial_ggsw (public_key/glwe.rs:214-263): bit-exact,
    and its external product with a ciphertext decrypts to m X^degree (tests/ext_prod.rs:58-113)."""
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    tab = O.DcrtTable(log_n, moduli)
    base = O.RnsBase(moduli)
    lat = O.Lattice(tab, base, O.GadgetBasis(base, lb))
    sk = np.concatenate([lat.ternary(6, 10 + i) for i in range(k)])
    sk_ntt = lat.table.forward(sk.copy())
    pk = lat.encrypt_cdt(k, sk_ntt, None, [0] * L, 0xF3, 0, 0)
    coeff = [1] * L
    exp = lat.ggsw_pk_encrypt_monomial(k, pk, coeff, degree, 0xF4, 900)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    enc = gpu.GlweEncryptor(table, 3.2)
    dpk = gpu.DeviceBuffer.from_numpy(pk)
    ggsw = gpu.DeviceBuffer(exp.size)
    enc.ggsw_pk_encrypt_monomial(g, k, dpk, coeff, degree, 0xF4, 900, ggsw)
    assert np.array_equal(ggsw.numpy(), exp)
    if L == 2:
        t, gamma = 12289, 2199023190017
        msg_small = O.uniform(77, 1, t, n)
        ct = lat.encrypt(k, sk_ntt, base.wrapping_decompose_small(msg_small, t), lat.delta(t), 13)
        out = gpu.DeviceBuffer(ct.size)
        gpu.external_product(table, g, k, gpu.DeviceBuffer.from_numpy(lat.table.inverse(ct.copy())), ggsw, out, 1)
        want = np.roll(msg_small.astype(np.int64), degree)
        want[:degree] = (t - want[:degree]) % t
        assert np.array_equal(lat.decrypt(k, sk_ntt, out.numpy(), t, gamma), want.astype(np.uint64))
    with pytest.raises(gpu.PrimusGpuError):
        enc.ggsw_pk_encrypt_monomial(g, k, dpk, coeff, n, 0xF4, 900, ggsw)  # degree must be below N
