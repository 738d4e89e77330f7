"""Field trace and coefficient expansion (sums of NTT-domain automorphisms).

CPU: the oracle's trace / reverse trace / expansion decrypt as the
reference's own tests require (primus_fhe_core/tests/trace.rs:121-211,
:214-285 and tests/expand.rs:139-253): Tr(m) = N m_0, Tr(N^-1 m) = m_0, the
reverse trace gives m_0, and expansion output j holds m_j at coefficient 0.
GPU: pg_glwe_trace / pg_glwe_expand_coefficients are bit-exact against the
oracle (random keys and ciphertexts) and decrypt the same way.
"""
import numpy as np
import pytest

import oracle as O

T_PLAIN, GAMMA = 12289, 2199023190017  # plaintext and correction moduli of the reference tests


def _lat(log_n, moduli, lb):
    tab = O.DcrtTable(log_n, moduli)
    base = O.RnsBase(moduli)
    return O.Lattice(tab, base, O.GadgetBasis(base, lb))


def _auto_key(lat, k, sk_ntt, degree, seed):
    """GLev of sigma_degree(s_i) under s (DcrtGlweAutoKey::new)."""
    log_n = lat.n.bit_length() - 1
    perm = O.ntt_auto_perm(log_n, degree)
    comps = sk_ntt.reshape(k, lat.L, lat.n)
    s_auto = np.concatenate([lat.table.inverse(np.ascontiguousarray(comps[i][:, perm]).ravel()) for i in range(k)])
    return lat.ksk(k, k, s_auto, sk_ntt, seed)


def _setup(log_n=9, L=2, k=2, lb=20, seed=5):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli, lb)
    sk = np.concatenate([lat.ternary(seed, 10 + i) for i in range(k)])
    sk_ntt = np.concatenate([lat.table.forward(sk[i * L * n:(i + 1) * L * n].copy()) for i in range(k)])
    return lat, moduli, n, sk_ntt


def _keys(lat, k, sk_ntt, degrees, seed):
    return np.concatenate([_auto_key(lat, k, sk_ntt, d, seed + i) for i, d in enumerate(degrees)])


def _encrypt(lat, k, sk_ntt, msg, seed):
    return lat.encrypt(k, sk_ntt, lat.base.wrapping_decompose_small(msg, T_PLAIN), lat.delta(T_PLAIN), seed)


def _fwd_degrees(n):
    return [n // (1 << r) + 1 for r in range(n.bit_length() - 1)]


def _rev_degrees(n):
    return [(2 << r) + 1 for r in range(n.bit_length() - 1)]


def test_oracle_trace_decrypts():
    k = 2
    lat, moduli, n, sk_ntt = _setup(k=k)
    msg = O.uniform(0x7A, 1, T_PLAIN, n)
    ct = _encrypt(lat, k, sk_ntt, msg, 3)
    keys = _keys(lat, k, sk_ntt, _fwd_degrees(n), 100)
    m = lat.decrypt(k, sk_ntt, lat.trace(k, keys, ct), T_PLAIN, GAMMA)
    assert int(m[0]) == int(msg[0]) * n % T_PLAIN and not m[1:].any()
    # scaled by N^-1 mod q_l first, the trace returns m_0 itself (trace.rs:196-210)
    scaled = ct.copy().reshape(k + 1, len(moduli), n)
    for l, q in enumerate(moduli):
        scaled[:, l] = O.mul_scalar(scaled[:, l].ravel(), O.lib().orc_invmod(n, q), q).reshape(k + 1, n)
    m = lat.decrypt(k, sk_ntt, lat.trace(k, keys, scaled.ravel()), T_PLAIN, GAMMA)
    assert int(m[0]) == int(msg[0]) and not m[1:].any()


def test_oracle_rev_trace_decrypts():
    k = 2
    lat, moduli, n, sk_ntt = _setup(k=k)
    msg = O.uniform(0x7B, 1, T_PLAIN, n)
    ct = _encrypt(lat, k, sk_ntt, msg, 4)
    keys = _keys(lat, k, sk_ntt, _rev_degrees(n), 200)
    m = lat.decrypt(k, sk_ntt, lat.trace(k, keys, ct, reverse=True), T_PLAIN, GAMMA)
    assert int(m[0]) == int(msg[0]) and not m[1:].any()


def test_oracle_expand_decrypts():
    k = 2
    lat, moduli, n, sk_ntt = _setup(k=k)
    keys = _keys(lat, k, sk_ntt, _fwd_degrees(n), 300)
    msg = O.uniform(0x7C, 1, T_PLAIN, n)
    per = (k + 1) * lat.L * n
    out = lat.expand(k, keys, n, _encrypt(lat, k, sk_ntt, msg, 5))
    for j in range(n):
        m = lat.decrypt(k, sk_ntt, out[j * per:(j + 1) * per], T_PLAIN, GAMMA)
        assert int(m[0]) == int(msg[j]) and not m[1:].any(), j
    # partial expansion: a message with coefficients 256.. zero (expand.rs:235-252)
    msg[256:] = 0
    out = lat.expand(k, keys, 256, _encrypt(lat, k, sk_ntt, msg, 6))
    for j in range(256):
        m = lat.decrypt(k, sk_ntt, out[j * per:(j + 1) * per], T_PLAIN, GAMMA)
        assert int(m[0]) == int(msg[j]) and not m[1:].any(), j


# ------------------------------------------------------------------ GPU
def _gpu_args(gpu, log_n, moduli, lb):
    table = gpu.DcrtTable(log_n, moduli)
    return table, gpu.GadgetBasis(gpu.RnsBase(moduli), lb)


@pytest.mark.gpu
@pytest.mark.parametrize("log_n,L,k,lb,batch,reverse", [(10, 2, 1, 20, 3, False), (10, 2, 1, 20, 2, True),
                                                        (9, 3, 2, 30, 2, False), (11, 1, 1, 7, 1, True)])
def test_trace_bit_exact(gpu, log_n, L, k, lb, batch, reverse):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli, lb)
    table, g = _gpu_args(gpu, log_n, moduli, lb)
    keys = np.concatenate([O.uniform_rns(0xB1, 50 * r, moduli, n).ravel()
                           for r in range(log_n * k * g.d * (k + 1))])
    per = (k + 1) * L * n
    ct = np.concatenate([O.uniform_rns(0xB2, 10 * b + i, moduli, n).ravel() for b in range(batch)
                         for i in range(k + 1)])
    exp = np.concatenate([lat.trace(k, keys, ct[b * per:(b + 1) * per], reverse) for b in range(batch)])
    dk = gpu.DeviceBuffer.from_numpy(keys)
    out = gpu.DeviceBuffer(ct.size)
    gpu.glwe_trace(table, g, k, dk, gpu.DeviceBuffer.from_numpy(ct), out, batch, reverse=reverse)
    assert np.array_equal(out.numpy(), exp)
    inplace = gpu.DeviceBuffer.from_numpy(ct)  # the same buffer as input and output
    gpu.glwe_trace(table, g, k, dk, inplace, inplace, batch, reverse=reverse)
    assert np.array_equal(inplace.numpy(), exp)


@pytest.mark.gpu
@pytest.mark.parametrize("log_n,L,k,lb,count", [(9, 2, 1, 20, 512), (10, 2, 1, 25, 1024), (10, 1, 2, 10, 64),
                                                (9, 2, 1, 20, 1)])
def test_expand_bit_exact(gpu, log_n, L, k, lb, count):
    """count = 1024 runs its last level as two automorphism calls of 256 ciphertexts each."""
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L)
    lat = _lat(log_n, moduli, lb)
    table, g = _gpu_args(gpu, log_n, moduli, lb)
    levels = max(1, count.bit_length() - 1)
    keys = np.concatenate([O.uniform_rns(0xC1, 50 * r, moduli, n).ravel() for r in range(levels * k * g.d * (k + 1))])
    ct = np.concatenate([O.uniform_rns(0xC2, i, moduli, n).ravel() for i in range(k + 1)])
    exp = lat.expand(k, keys, count, ct)
    out = gpu.DeviceBuffer(exp.size)
    gpu.glwe_expand_coefficients(table, g, k, gpu.DeviceBuffer.from_numpy(keys), count,
                                 gpu.DeviceBuffer.from_numpy(ct), out)
    assert np.array_equal(out.numpy(), exp)


@pytest.mark.gpu
def test_expand_and_trace_decrypt_on_device(gpu):
    k = 1
    lat, moduli, n, sk_ntt = _setup(k=k, seed=9)
    table, g = _gpu_args(gpu, 9, moduli, 20)
    keys = _keys(lat, k, sk_ntt, _fwd_degrees(n), 400)
    msg = O.uniform(0x7D, 1, T_PLAIN, n)
    ct = _encrypt(lat, k, sk_ntt, msg, 7)
    per = (k + 1) * lat.L * n
    out = gpu.DeviceBuffer(n * per)
    gpu.glwe_expand_coefficients(table, g, k, gpu.DeviceBuffer.from_numpy(keys), n, gpu.DeviceBuffer.from_numpy(ct),
                                 out)
    res = out.numpy()
    for j in range(0, n, 37):
        m = lat.decrypt(k, sk_ntt, res[j * per:(j + 1) * per], T_PLAIN, GAMMA)
        assert int(m[0]) == int(msg[j]) and not m[1:].any(), j
    tr = gpu.DeviceBuffer(per)
    gpu.glwe_trace(table, g, k, gpu.DeviceBuffer.from_numpy(keys), gpu.DeviceBuffer.from_numpy(ct), tr, 1)
    m = lat.decrypt(k, sk_ntt, tr.numpy(), T_PLAIN, GAMMA)
    assert int(m[0]) == int(msg[0]) * n % T_PLAIN and not m[1:].any()


@pytest.mark.gpu
def test_trace_expand_reject(gpu):
    from primus_b200 import _native as nat
    moduli = O.ntt_primes(1 << 50, 2048, 1)
    table, g = _gpu_args(gpu, 10, moduli, 20)
    d = gpu.DeviceBuffer(2 * 1024 * 8)
    assert nat.lib().pg_glwe_expand_coefficients(table.h, g.h, 1, d.ptr, 3, d.ptr, d.ptr, None, 0, None) \
        == nat.PG_ERR_INVALID_ARGUMENT  # count not a power of two
    assert nat.lib().pg_glwe_expand_coefficients(table.h, g.h, 1, d.ptr, 2048, d.ptr, d.ptr, None, 0, None) \
        == nat.PG_ERR_INVALID_ARGUMENT  # count above N
    assert nat.lib().pg_glwe_trace(table.h, g.h, 1, d.ptr, 0, d.ptr, d.ptr + 8, 1, None, 0, None) \
        == nat.PG_ERR_INVALID_ARGUMENT  # partial overlap
