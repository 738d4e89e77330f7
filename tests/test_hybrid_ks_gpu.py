"""Hybrid RNS key switch with special primes (pg_key_switch_hybrid): bit-exact
against the oracle's restatement of the same definition, and decryption after
a key switch with a key built by GLWE encryption.  The reference has no such
key switch, so these pins are the definition's own (parity unpinned against
the reference)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


# (log_n, L, K, alpha, k_in, k_out, batch): the served shape (N=2^15, L=16, K=4,
# 4-limb groups) in batches of 2 and 1, a ragged last group, a single group, and larger k
# (N = 2^13 .. 2^16 and batches of at most 8 run the fused form: conversions inside
# the transforms' loads and stores; smaller N and larger batches the separate kernels;
# at N = 2^15 fused launches of at most 32 rows run 8 elements per thread)
SHAPES = [(15, 16, 4, 4, 1, 1, 2), (15, 16, 4, 4, 1, 1, 1), (10, 7, 2, 3, 1, 1, 3), (11, 4, 1, 4, 1, 1, 2),
          (10, 6, 3, 2, 2, 2, 2), (12, 5, 2, 1, 1, 3, 1), (13, 6, 2, 3, 2, 1, 2), (14, 7, 3, 2, 1, 2, 3),
          (16, 5, 1, 4, 1, 1, 1), (13, 4, 2, 2, 1, 1, 9)]


@pytest.mark.parametrize("log_n,L,K,alpha,k_in,k_out,batch", SHAPES)
def test_hybrid_key_switch_bit_exact(gpu, log_n, L, K, alpha, k_in, k_out, batch):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L + K)
    ref = O.HybridKeySwitch(log_n, moduli, L, K, alpha)
    table = gpu.DcrtTable(log_n, moduli)
    hks = gpu.HybridKeySwitch(table, L, K, alpha)
    assert hks.dnum == ref.dnum
    rows = k_in * hks.dnum * (k_out + 1)
    key = np.concatenate([O.uniform_rns(0x4B, 50 * r, moduli, n).ravel() for r in range(rows)])
    c_in = np.concatenate([O.uniform_rns(0x1C, 40 * b + 20 * i, moduli[:L], n).ravel()
                           for b in range(batch) for i in range(k_in + 1)])
    c_in[:3] = [0, moduli[0] - 1, moduli[0] // 2]
    per_in, per_out = (k_in + 1) * L * n, (k_out + 1) * L * n
    exp = np.concatenate([ref.key_switch(k_in, k_out, key, c_in[b * per_in:(b + 1) * per_in])
                          for b in range(batch)])
    dk, di = gpu.DeviceBuffer.from_numpy(key), gpu.DeviceBuffer.from_numpy(c_in)
    do = gpu.DeviceBuffer(batch * per_out)
    hks.key_switch(k_in, k_out, dk, di, do, batch)
    assert np.array_equal(do.numpy(), exp)
    # caller workspace gives the same result
    ws = gpu.DeviceBuffer(hks.workspace_size(k_in, k_out, batch) // 8 + 1)
    do2 = gpu.DeviceBuffer(batch * per_out)
    hks.key_switch(k_in, k_out, dk, di, do2, batch, workspace=ws)
    assert np.array_equal(do2.numpy(), exp)
    # the integer-only schedule (FP64 off: NTTs and base conversions on the integer pipe)
    table.set_fp64(False)
    do3 = gpu.DeviceBuffer(batch * per_out)
    hks.key_switch(k_in, k_out, dk, di, do3, batch)
    assert np.array_equal(do3.numpy(), exp)


def test_hybrid_key_switch_wide_moduli(gpu):
    """Moduli between 2^50 and 2^59 run every step on the integer pipe."""
    log_n, L, K, alpha, k_in, k_out, batch = 10, 5, 2, 2, 1, 1, 2
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 58, 2 * n, L + K)
    ref = O.HybridKeySwitch(log_n, moduli, L, K, alpha)
    table = gpu.DcrtTable(log_n, moduli)
    assert not table.fp64
    hks = gpu.HybridKeySwitch(table, L, K, alpha)
    rows = k_in * hks.dnum * (k_out + 1)
    key = np.concatenate([O.uniform_rns(0x4C, 50 * r, moduli, n).ravel() for r in range(rows)])
    c_in = np.concatenate([O.uniform_rns(0x1D, 40 * b + 20 * i, moduli[:L], n).ravel()
                           for b in range(batch) for i in range(k_in + 1)])
    per_in, per_out = (k_in + 1) * L * n, (k_out + 1) * L * n
    exp = np.concatenate([ref.key_switch(k_in, k_out, key, c_in[b * per_in:(b + 1) * per_in])
                          for b in range(batch)])
    do = gpu.DeviceBuffer(batch * per_out)
    hks.key_switch(k_in, k_out, gpu.DeviceBuffer.from_numpy(key), gpu.DeviceBuffer.from_numpy(c_in), do, batch)
    assert np.array_equal(do.numpy(), exp)


def test_hybrid_key_switch_decrypts(gpu):
    log_n, L, K, alpha, k = 11, 8, 2, 4, 1
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L + K)
    ref = O.HybridKeySwitch(log_n, moduli, L, K, alpha)
    Q = moduli[:L]
    tq, bq = O.DcrtTable(log_n, Q), O.RnsBase(Q)
    latq = O.Lattice(tq, bq, O.GadgetBasis(bq, 30))
    tqp, bqp = O.DcrtTable(log_n, moduli), O.RnsBase(moduli)
    latqp = O.Lattice(tqp, bqp, O.GadgetBasis(bqp, 30))
    s_in, s_out = latqp.ternary(1, 1), latqp.ternary(2, 2)
    s_out_ntt = tqp.forward(s_out.copy())
    key = np.concatenate([latqp.encrypt(k, s_out_ntt, s_in, ref.factor(g), 1000 + g) for g in range(ref.dnum)])
    t, gamma = 16, 257
    msg = O.uniform(5, 5, t, n)
    ct = latq.encrypt(k, tq.forward(s_in[:L * n].copy()), bq.wrapping_decompose_small(msg, t), latq.delta(t), 77)
    table = gpu.DcrtTable(log_n, moduli)
    hks = gpu.HybridKeySwitch(table, L, K, alpha)
    do = gpu.DeviceBuffer(ct.size)
    hks.key_switch(k, k, gpu.DeviceBuffer.from_numpy(key), gpu.DeviceBuffer.from_numpy(tq.inverse(ct.copy())), do, 1)
    m = latq.decrypt(k, tq.forward(s_out[:L * n].copy()), do.numpy(), t, gamma)
    assert np.array_equal(m, msg)


def test_hybrid_rejects_bad_parameters(gpu):
    from primus_b200 import _native as nat
    import ctypes as C
    moduli = O.ntt_primes(1 << 50, 2048, 6)
    table = gpu.DcrtTable(10, moduli)
    h = C.c_void_p()
    for L, K, alpha in [(5, 2, 1), (4, 2, 5), (4, 2, 0), (0, 6, 1), (4, 2, 9)]:
        st = nat.lib().pg_hybrid_ks_create(table.h, L, K, alpha, C.byref(h))
        assert st == nat.PG_ERR_INVALID_ARGUMENT
