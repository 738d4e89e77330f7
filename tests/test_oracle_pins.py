"""Pins the CPU oracle to the reference before parity tests rely on it.

The reference (a Rust workspace) is not compiled or run alongside these tests, so the oracle is pinned by
(a) the golden fixtures in tests/golden/ -- pure-Python big-integer values of
the definitions the reference encodes -- and (b) ports of the reference's own
known-answer and property tests, with fixed seeds:

* primus_ntt/tests/root.rs:9-25            INTT(NTT(a)) == a, N=1024, q=132120577
* primus_ntt/tests/hexl.rs:18-130          the three HEXL primes (canonical == definition)
* primus_rns/tests/rns.rs:14-34            compose/decompose KATs
* primus_decompose/tests/non_pow_of_2.rs   signed decomposition recomposes
* primus_decompose/tests/big_uint.rs       BigUint decomposition recomposes
* primus_modulus/src/barrett/ops.rs:533    dot product == naive fold
* primus_fhe_core/tests/ext_prod.rs:14-115 Dec(ct (x) GGSW(X^d)) == m X^d
* primus_fhe_core/tests/ksk.rs:12-98       Dec_s2(KS(Enc_s1(m))) == m
"""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def golden():
    arrays = np.load(os.path.join(GOLD, "ntt_golden.npz"))
    with open(os.path.join(GOLD, "kats.json")) as f:
        kats = json.load(f)
    return arrays, kats


def test_ntt_matches_golden_definition(golden):
    arrays, kats = golden
    for case in kats["ntt_cases"]:
        label, log_n, q = case["label"], case["log_n"], case["q"]
        t = O.NttTable(log_n, q)
        assert t.export()["root"] == case["psi"], label
        a = arrays[f"{label}/a"]
        assert np.array_equal(t.forward(a), arrays[f"{label}/ntt_a"]), label
        assert np.array_equal(t.inverse(arrays[f"{label}/ntt_a"]), a), label
        if f"{label}/a_times_b" in arrays:
            b = arrays[f"{label}/b"]
            assert np.array_equal(O.naive_negacyclic(a, b, q), arrays[f"{label}/a_times_b"]), label
            prod = t.inverse(O.mul(t.forward(a), t.forward(b), q))
            assert np.array_equal(prod, arrays[f"{label}/a_times_b"]), label


def test_prime_search_matches_golden(golden):
    _, kats = golden
    pr = kats["primes"]
    assert O.ntt_primes(1 << 50, 2048, 1)[0] == pr["polymul_2^50_mod_2048"]
    assert O.ntt_primes(1 << 54, 4096, 1)[0] == pr["extprod_2^54_mod_4096"]
    assert O.ntt_primes(1 << 50, 1 << 17, 24) == pr["rns24_2^50_mod_2^17"]


def test_root_rs_roundtrip():
    # primus_ntt/tests/root.rs: M = 132120577, N = 1024
    q = 132120577
    t = O.NttTable(10, q)
    a = O.uniform(7, 0, q, 1024)
    assert np.array_equal(t.inverse(t.forward(a)), a)


@pytest.mark.parametrize("q", [536813569, 562949953392641, 1152921504606830593])
def test_hexl_primes_lazy_ranges(q):
    # primus_ntt/tests/hexl.rs uses these primes at N = 2048; the lazy outputs
    # stay in [0, 4q) and reduce to the canonical transform
    t = O.NttTable(11, q)
    a = O.uniform(11, 3, q, 2048)
    lazy = t.forward(a, lazy=True)
    assert int(lazy.max()) < 4 * q
    canon = t.forward(a)
    assert np.array_equal(lazy % np.uint64(q), canon)
    back = t.inverse(canon, lazy=True)
    assert np.array_equal(back, a)


def test_monomials_match_transform():
    q = O.ntt_primes(1 << 50, 2048, 1)[0]
    t = O.NttTable(10, q)
    for coeff, deg in [(5, 7), (1, 1023), (q - 1, 3), (123456789, 0), (0, 9)]:
        poly = np.zeros(1024, np.uint64)
        poly[deg] = coeff
        assert np.array_equal(t.monomial(coeff, deg), t.forward(poly))
    for deg in (0, 1, 511):
        poly = np.zeros(1024, np.uint64)
        poly[deg] = 1
        assert np.array_equal(t.coeff_one_monomial(deg), t.forward(poly))
        poly[deg] = q - 1
        assert np.array_equal(t.coeff_minus_one_monomial(deg), t.forward(poly))


def test_rns_kats(golden):
    _, kats = golden
    for case in kats["rns"]:
        base = O.RnsBase(case["moduli"])
        v = base.compose(case["residues"])
        value = sum(int(x) << (64 * i) for i, x in enumerate(v))
        assert value == case["value"]
        assert [int(x) for x in base.decompose(v)] == case["residues"]


def test_rns_wrapping_decompose_kat():
    # primus_rns/tests/rns.rs:36-68 (test_rns3): small signed values lift to q_i - (t - r)
    moduli = [1099511592961, 1099511590913]
    base = O.RnsBase(moduli)
    t = 257
    small = np.arange(t, dtype=np.uint64)
    res = base.wrapping_decompose_small(small, t)
    for r in range(t):
        for i, m in enumerate(moduli):
            assert int(res[i, r]) == (r if r < (t + 1) // 2 else m - (t - r))


def test_non_pow_of_2_decompose():
    # primus_decompose/tests/non_pow_of_2.rs:14-80
    modulus, lb, length, value = 0b111000110, 3, 2, 0b11111101
    b = O.ApproxBasis(modulus, lb, length)
    digits = b.decompose(value)
    result = sum(int(s) * int(d) for s, d in zip(b.scalars, digits)) % modulus
    diff = min((result - value) % modulus, (value - result) % modulus)
    assert diff <= (1 << (b.drop_bits - 1) if b.drop_bits else 0)


@pytest.mark.parametrize("seed", range(4))
def test_approx_signed_decompose(seed):
    # primus_decompose/tests/non_pow_of_2.rs:108-150 with a seeded modulus
    rng = np.random.default_rng(seed)
    modulus = int(rng.integers(512, 1 << 30))
    b = O.ApproxBasis(modulus, 4)
    bound = (1 << (b.drop_bits - 1)) if b.drop_bits else 0
    for value in rng.integers(0, modulus, 200):
        digits = b.decompose(int(value))
        result = sum(int(s) * int(d) for s, d in zip(b.scalars, digits)) % modulus
        diff = min((result - int(value)) % modulus, (int(value) - result) % modulus)
        assert diff <= bound


@pytest.mark.parametrize("moduli,lb", [([134215681, 134176769], 7),
                                       ([1125899906826241, 1125899906629633], 30),
                                       ([1125899906826241, 1125899906629633, 1125899906617345], 20)])
def test_big_uint_decompose_recomposes(moduli, lb):
    # primus_decompose/tests/big_uint.rs: sum of signed digits * gadget ~ value
    base = O.RnsBase(moduli)
    g = O.GadgetBasis(base, lb)
    Q = 1
    for m in moduli:
        Q *= m
    bits = Q.bit_length()
    rng = np.random.default_rng(lb)
    count = 300
    vals = [int(rng.integers(0, 1 << 62)) * int(rng.integers(0, 1 << 62)) * int(rng.integers(0, 1 << 40)) % Q
            for _ in range(count)]
    vals[0], vals[1], vals[2] = 0, Q - 1, Q // 2
    W = base.W
    arr = np.array([[(v >> (64 * i)) & ((1 << 64) - 1) for i in range(W)] for v in vals], dtype=np.uint64)
    digits = g.decompose_all(arr)
    B = 1 << lb
    for x, v in enumerate(vals):
        s = 0
        for j in range(g.d):
            d = int(digits[j, x])
            sd = d if d < B // 2 else d - B
            s += sd << (g.drop_bits + j * lb)
        diff = (s - v) % Q
        diff = min(diff, Q - diff)
        assert diff <= (1 << g.drop_bits), (x, diff)
    assert bits - g.d * lb == g.drop_bits


def test_barrett_dot_product_matches_naive():
    q = 0x3FFFFFFB
    rng = np.random.default_rng(5)
    for n in [0, 1, 7, 15, 16, 17, 31, 32, 33, 127, 128, 129, 1000]:
        a = rng.integers(0, q, n, dtype=np.uint64)
        b = rng.integers(0, q, n, dtype=np.uint64)
        got = O.lib().orc_barrett_dot_product(O.p64(a), O.p64(b), n, q) if n else 0
        exp = 0
        for x, y in zip(a, b):
            exp = (exp + int(x) * int(y)) % q
        assert got == exp


def test_barrett_reduce_matches_mod():
    rng = np.random.default_rng(9)
    for q in [3, 97, 132120577, (1 << 50) - 27, (1 << 61) - 1]:
        ratio = np.zeros(2, np.uint64)
        O.lib().orc_barrett_ratio(q, O.p64(ratio))
        assert int(ratio[0]) + (int(ratio[1]) << 64) == (1 << 128) // q
        for _ in range(200):
            a, b, c = (int(x) for x in rng.integers(0, q, 3, dtype=np.uint64))
            assert O.lib().orc_barrett_reduce_mul_add(a, b, c, q, O.p64(ratio)) == (a * b + c) % q


def _bfv_setup(k, n_log, moduli, lb):
    table = O.DcrtTable(n_log, moduli)
    base = O.RnsBase(moduli)
    basis = O.GadgetBasis(base, lb)
    return table, base, basis, O.Lattice(table, base, basis)


@pytest.mark.parametrize("k", [1, 2])
def test_external_product_decrypts(k):
    # primus_fhe_core/tests/ext_prod.rs (dimension reduced from 8 for speed)
    moduli = [1125899906826241, 1125899906629633]
    table, base, basis, lat = _bfv_setup(k, 9, moduli, 30)
    t, gamma = 12289, 2199023190017
    sk = np.concatenate([lat.ternary(21, 10 + i) for i in range(k)])
    sk_ntt = table.forward(sk)
    delta = lat.delta(t)
    for trial in range(3):
        degree = [0, 37, 511][trial]
        msg_small = O.uniform(100 + trial, 1, t, 512)
        msg = base.wrapping_decompose_small(msg_small, t)
        ct = lat.encrypt(k, sk_ntt, msg, delta, 500 + trial)
        ggsw = lat.ggsw_monomial(k, sk_ntt, [1, 1], degree, 900 + trial)
        out = lat.external_product(k, table.inverse(ct), ggsw)
        exp = np.roll(msg_small.astype(np.int64), degree)
        exp[:degree] = (t - exp[:degree]) % t
        assert np.array_equal(lat.decrypt(k, sk_ntt, out, t, gamma), exp.astype(np.uint64))


@pytest.mark.parametrize("k", [1, 2])
def test_public_key_ggsw_external_product_decrypts(k):
    # primus_fhe_core/tests/ext_prod.rs:58-113: the GGSW of X^degree is encrypted
    # under the public key (DcrtGlwePublicKey::encrypt_monomial_ggsw), and a
    # public-key GLWE encryption decrypts to its message
    moduli = [1125899906826241, 1125899906629633]
    table, base, basis, lat = _bfv_setup(k, 9, moduli, 30)
    t, gamma = 12289, 2199023190017
    sk = np.concatenate([lat.ternary(31, 10 + i) for i in range(k)])
    sk_ntt = table.forward(sk)
    pk = lat.encrypt_cdt(k, sk_ntt, None, [0, 0], 0x9C, 0, 0)
    delta = lat.delta(t)
    for trial, degree in enumerate([0, 101, 511]):
        msg_small = O.uniform(200 + trial, 1, t, 512)
        msg = base.wrapping_decompose_small(msg_small, t)
        ct = lat.pk_encrypt_cdt(k, pk, msg, delta, 0x9D, 0, trial)
        assert np.array_equal(lat.decrypt(k, sk_ntt, ct, t, gamma), msg_small)
        ggsw = lat.ggsw_pk_encrypt_monomial(k, pk, [1, 1], degree, 0x9E, (1 << 20) + 100 * trial)
        out = lat.external_product(k, table.inverse(ct), ggsw)
        exp = np.roll(msg_small.astype(np.int64), degree)
        exp[:degree] = (t - exp[:degree]) % t
        assert np.array_equal(lat.decrypt(k, sk_ntt, out, t, gamma), exp.astype(np.uint64))


def test_key_switch_decrypts():
    # primus_fhe_core/tests/ksk.rs: dimension 3, N = 512, log_basis 20
    moduli = [1125899906826241, 1125899906629633]
    k = 3
    table, base, basis, lat = _bfv_setup(k, 9, moduli, 20)
    t, gamma = 12289, 2305843009213554689
    sk1 = np.concatenate([lat.ternary(31, 10 + i) for i in range(k)])
    sk2 = np.concatenate([lat.ternary(32, 10 + i) for i in range(k)])
    sk1_ntt, sk2_ntt = table.forward(sk1), table.forward(sk2)
    key = lat.ksk(k, k, sk1, sk2_ntt, 77)
    msg_small = O.uniform(41, 1, t, 512)
    msg = base.wrapping_decompose_small(msg_small, t)
    ct = lat.encrypt(k, sk1_ntt, msg, lat.delta(t), 42)
    assert np.array_equal(lat.decrypt(k, sk1_ntt, ct, t, gamma), msg_small)
    out = lat.key_switch(k, k, key, table.inverse(ct))
    assert np.array_equal(lat.decrypt(k, sk2_ntt, out, t, gamma), msg_small)


def test_fast_convert_matches_crt():
    # fast_convert_array (converter.rs:147-175) = (x + alpha Q) mod p_j, alpha in [0, L)
    qs = O.ntt_primes(1 << 50, 1 << 13, 4)
    ps = O.ntt_primes(1 << 49, 1 << 13, 3)
    ib, ob = O.RnsBase(qs), O.RnsBase(ps)
    conv = O.BaseConverter(ib, ob)
    n = 64
    x = O.uniform_rns(3, 0, qs, n)
    y = conv.fast_convert_array(x)
    Q = 1
    for q in qs:
        Q *= q
    for c in range(n):
        v = ib.compose(x[:, c])
        val = sum(int(w) << (64 * i) for i, w in enumerate(v))
        ok = False
        for alpha in range(len(qs)):
            if all(int(y[j, c]) == (val + alpha * Q) % p for j, p in enumerate(ps)):
                ok = True
        assert ok


def test_automorphism_decrypts_to_permuted_message():
    # DcrtGlweAutoKey (primus_fhe_core/src/automorphism/glwe/dcrt.rs): decrypting the
    # automorphism of an encryption of m gives m(X^degree) mod X^N + 1
    log_n, k, t, gamma = 9, 1, 16, 257
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, 2)
    tab = O.DcrtTable(log_n, moduli)
    base = O.RnsBase(moduli)
    lat = O.Lattice(tab, base, O.GadgetBasis(base, 20))
    sk = lat.ternary(3, 10)
    sk_ntt = tab.forward(sk.copy())
    for degree in (3, 2 * n - 1, 257):
        perm = O.ntt_auto_perm(log_n, degree)
        s_auto = tab.inverse(np.concatenate([sk_ntt.reshape(2, n)[l][perm] for l in range(2)]))
        key = lat.ksk(k, k, s_auto, sk_ntt, 5 + degree)
        msg = O.uniform(41, degree, t, n)
        ct = lat.encrypt(k, sk_ntt, base.wrapping_decompose_small(msg, t), lat.delta(t), 9)
        m = lat.decrypt(k, sk_ntt, lat.automorphism(k, degree, key, ct), t, gamma)
        exp = np.zeros(n, np.int64)
        for i in range(n):
            j = (i * degree) % (2 * n)
            if j < n:
                exp[j] = (exp[j] + int(msg[i])) % t
            else:
                exp[j - n] = (exp[j - n] - int(msg[i])) % t
        assert np.array_equal(m, exp.astype(np.uint64)), degree
