"""The one-kernel external product (k = 1, one prime, single-word gadget values,
N = 2^10..2^12, batches of 64 ciphertexts or more): decomposition, forward NTT of every digit row, MAC and, for the
coefficient-form entry point, the inverse NTT of both outputs, all inside one
CTA per ciphertext.  Every output is compared bit for bit with the oracle's
CrtGlwe::mul_dcrt_ggsw_inplace (primus_lattice/src/glwe/crt.rs:202-229) and,
for pg_ext_product_coeff, with the oracle's inverse_transform_slice of it."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _setup(log_n, q, lb):
    table = O.DcrtTable(log_n, [q])
    rbase = O.RnsBase([q])
    return O.Lattice(table, rbase, O.GadgetBasis(rbase, lb))


# (log_n, modulus bound, log_basis, batch): the blind-rotation shape (2^11, q < 2^54,
# 7-bit digits), 16-bit digits, wide digits kept as 64-bit words, a modulus above
# 2^58 (lazy Harvey forward schedule), and base 2 (many digits, many folds)
# (the fused kernel runs for batches of 64 and more; the batch of 5 takes the pipeline;
# bases up to 256 below 2^58 take the first forward stage from a table: the largest
# table at N = 2^12, and a modulus just below 2^58)
SHAPES = [(11, 1 << 54, 7, 100), (10, 1 << 54, 7, 5), (10, 1 << 54, 7, 64), (12, 1 << 50, 10, 65),
          (11, 1 << 50, 16, 64), (11, 1 << 54, 20, 70), (11, 1 << 61, 16, 64), (10, 1 << 40, 1, 64),
          (12, 1 << 50, 8, 64), (11, 1 << 58, 6, 64)]


@pytest.mark.parametrize("log_n,bound,lb,batch", SHAPES)
def test_fused_external_product_bit_exact(gpu, log_n, bound, lb, batch):
    n, k = 1 << log_n, 1
    q = O.ntt_primes(bound, 2 * n, 1)[0]
    lat = _setup(log_n, q, lb)
    table = gpu.DcrtTable(log_n, [q])
    g = gpu.GadgetBasis(gpu.RnsBase([q]), lb)
    d = g.d
    ggsw = np.concatenate([O.uniform_rns(91, 7 * i, [q], n).ravel() for i in range(2 * d * 2)])
    glwe = np.concatenate([O.uniform_rns(92, 3 * b + i, [q], n).ravel() for b in range(batch) for i in range(2)])
    # edge values: 0, q-1 and the split neighbourhood in the first ciphertext
    glwe[:4] = [0, q - 1, q // 2, q // 2 + 1]
    exp = lat.external_product(k, glwe, ggsw, batch=batch)
    din, dk = gpu.DeviceBuffer.from_numpy(glwe), gpu.DeviceBuffer.from_numpy(ggsw)
    dout = gpu.DeviceBuffer(glwe.size)
    gpu.external_product(table, g, k, din, dk, dout, batch)
    assert np.array_equal(dout.numpy(), exp)
    # coefficient form: the oracle's inverse transform of every output poly
    exp_coeff = lat.table.inverse(exp.copy())
    dcoef = gpu.DeviceBuffer(glwe.size)
    gpu.external_product_coeff(table, g, k, din, dk, dcoef, batch)
    assert np.array_equal(dcoef.numpy(), exp_coeff)


def test_coeff_form_pipeline_shape(gpu):
    # two primes: the pipeline (compose -> digits -> NTT -> MAC) plus an inverse launch
    log_n, k, lb, batch = 10, 1, 25, 3
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, 2)
    table_o = O.DcrtTable(log_n, moduli)
    rbase = O.RnsBase(moduli)
    lat = O.Lattice(table_o, rbase, O.GadgetBasis(rbase, lb))
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    ggsw = np.concatenate([O.uniform_rns(5, 100 * i, moduli, n).ravel() for i in range(2 * g.d * 2)])
    glwe = np.concatenate([O.uniform_rns(6, 10 * b + i, moduli, n).ravel() for b in range(batch) for i in range(2)])
    exp = table_o.inverse(lat.external_product(k, glwe, ggsw, batch=batch))
    dout = gpu.DeviceBuffer(glwe.size)
    gpu.external_product_coeff(table, g, k, gpu.DeviceBuffer.from_numpy(glwe), gpu.DeviceBuffer.from_numpy(ggsw),
                               dout, batch)
    assert np.array_equal(dout.numpy(), exp)


def test_fused_blind_rotation_steps_decrypt(gpu):
    # three accumulator steps ct <- ct (x) GGSW(X^deg) in coefficient form with a
    # real encryption (primus_fhe_core/tests/ext_prod.rs): Dec gives m X^(sum deg)
    log_n, lb, t = 11, 7, 16
    n, k = 1 << log_n, 1
    q = O.ntt_primes(1 << 54, 2 * n, 1)[0]
    lat = _setup(log_n, q, lb)
    table = gpu.DcrtTable(log_n, [q])
    g = gpu.GadgetBasis(gpu.RnsBase([q]), lb)
    sk = lat.ternary(3, 10)
    sk_ntt = lat.table.forward(sk)
    msg = O.uniform(41, 1, t, n)
    ct = lat.encrypt(k, sk_ntt, lat.base.wrapping_decompose_small(msg, t), lat.delta(t), 9)
    # 64 copies of the ciphertext so that the one-kernel form runs
    cur = gpu.DeviceBuffer.from_numpy(np.tile(lat.table.inverse(ct), 64))
    nxt = gpu.DeviceBuffer(64 * ct.size)
    total = 0
    for step, deg in enumerate((5, 300, 1000)):
        dk = gpu.DeviceBuffer.from_numpy(lat.ggsw_monomial(k, sk_ntt, [1], deg, 700 + step))
        gpu.external_product_coeff(table, g, k, cur, dk, nxt, 64)
        cur, nxt = nxt, cur
        total += deg
    res = cur.numpy().reshape(64, -1)
    assert (res == res[0]).all()
    m = lat.decrypt(k, sk_ntt, lat.table.forward(res[0].copy()), t, 257)  # small gamma: one 54-bit prime
    exp = np.roll(msg.astype(np.int64), total)
    exp[:total] = (t - exp[:total]) % t
    assert np.array_equal(m, exp.astype(np.uint64))
