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
