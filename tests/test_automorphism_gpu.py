"""GLWE automorphism X -> X^degree in the NTT domain (pg_glwe_automorphism):
bit-exact against the oracle's DcrtGlweAutoKey::automorphism_inplace
(primus_fhe_core/src/automorphism/glwe/dcrt.rs:269-331) and, with a real
automorphism key, decryption to m(X^degree)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _lat(log_n, moduli, lb):
    tab = O.DcrtTable(log_n, moduli)
    base = O.RnsBase(moduli)
    return O.Lattice(tab, base, O.GadgetBasis(base, lb))


@pytest.mark.parametrize("log_n,L,k,lb,degree,batch", [(10, 2, 1, 20, 3, 3), (11, 1, 1, 7, 2047 * 2 + 1, 2),
                                                        (12, 3, 2, 30, 5, 2), (15, 4, 1, 25, 17, 1),
                                                        (9, 2, 1, 30, 1, 2)])
def test_automorphism_bit_exact(gpu, log_n, L, k, lb, degree, batch):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli, lb)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    key = np.concatenate([O.uniform_rns(0xA1, 50 * r, moduli, n).ravel() for r in range(k * g.d * (k + 1))])
    ct = np.concatenate([O.uniform_rns(0xA2, 10 * b + i, moduli, n).ravel() for b in range(batch)
                         for i in range(k + 1)])
    per = (k + 1) * L * n
    exp = np.concatenate([lat.automorphism(k, degree, key, ct[b * per:(b + 1) * per]) for b in range(batch)])
    out = gpu.DeviceBuffer(ct.size)
    gpu.glwe_automorphism(table, g, k, degree, gpu.DeviceBuffer.from_numpy(key), gpu.DeviceBuffer.from_numpy(ct),
                          out, batch)
    assert np.array_equal(out.numpy(), exp)


def test_automorphism_decrypts(gpu):
    log_n, k, t, gamma = 11, 1, 16, 257
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, 2)
    lat = _lat(log_n, moduli, 20)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), 20)
    sk = lat.ternary(3, 10)
    sk_ntt = lat.table.forward(sk.copy())
    for degree in (3, 2 * n - 1):
        perm = O.ntt_auto_perm(log_n, degree)
        s_auto = lat.table.inverse(np.concatenate([sk_ntt.reshape(2, n)[l][perm] for l in range(2)]))
        key = lat.ksk(k, k, s_auto, sk_ntt, 77 + degree)
        msg = O.uniform(41, degree, t, n)
        ct = lat.encrypt(k, sk_ntt, lat.base.wrapping_decompose_small(msg, t), lat.delta(t), 9)
        out = gpu.DeviceBuffer(ct.size)
        gpu.glwe_automorphism(table, g, k, degree, gpu.DeviceBuffer.from_numpy(key), gpu.DeviceBuffer.from_numpy(ct),
                              out, 1)
        m = lat.decrypt(k, sk_ntt, out.numpy(), t, gamma)
        exp = np.zeros(n, np.int64)
        for i in range(n):
            j = (i * degree) % (2 * n)
            if j < n:
                exp[j] = (exp[j] + int(msg[i])) % t
            else:
                exp[j - n] = (exp[j - n] - int(msg[i])) % t
        assert np.array_equal(m, exp.astype(np.uint64)), degree


def test_automorphism_rejects(gpu):
    from primus_b200 import _native as nat
    moduli = O.ntt_primes(1 << 50, 2048, 1)
    table = gpu.DcrtTable(10, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), 20)
    d = gpu.DeviceBuffer(2 * 1024 * 4)
    e = gpu.DeviceBuffer(2 * 1024)
    assert nat.lib().pg_glwe_automorphism(table.h, g.h, 1, 4, d.ptr, e.ptr, d.ptr, 1, None, 0, None) \
        == nat.PG_ERR_INVALID_ARGUMENT  # even degree
    assert nat.lib().pg_glwe_automorphism(table.h, g.h, 1, 3, d.ptr, e.ptr, e.ptr, 1, None, 0, None) \
        == nat.PG_ERR_INVALID_ARGUMENT  # in place
