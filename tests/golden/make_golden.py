"""Generate the golden fixtures in tests/golden/ with pure-Python big integers.

Independent of both the C oracle and the CUDA library: every value here is
computed from the mathematical definitions the reference encodes, so the
fixtures pin the oracle (and through it the GPU path) to the reference.

* minimal primitive 2N-th root of unity (try_minimal_primitive_root,
  primus_ntt/src/root.rs:89-111): the smallest odd power of any primitive root;
* forward NTT output order (transform_monomial, primus_ntt/src/ntt/primitive.rs:321-328):
  out[i] = sum_j a_j psi^((2 rev(i) + 1) j) mod q;
* negacyclic product (Polynomial::naive_mul_inplace, primus_poly/src/poly/mul.rs:111-142);
* CRT composition (RNSBase::compose, primus_rns/src/base.rs:369-394) as the
  unique x in [0, Q) with x = r_i mod q_i;
* the reference's own known-answer tests, transcribed as data.

Inputs come from the counter-based generator the library uses (restated here):
uniform(seed, stream, index, q).

    python tests/golden/make_golden.py      # rewrites tests/golden/*.npz / *.json
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
M64 = (1 << 64) - 1


def mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def hash64(seed, stream, index, attempt):
    h = mix64((seed * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) & M64)
    h = mix64(h ^ ((stream * 0xD1B54A32D192ED03) & M64))
    h = mix64(h ^ ((index * 0xA0761D6478BD642F) & M64) ^ ((attempt * 0xE7037ED1A0B428DB) & M64))
    return h


def uniform(seed, stream, index, q):
    if q <= 1:
        return 0
    bits = (q - 1).bit_length()
    for attempt in range(64):
        v = hash64(seed, stream, index, attempt) >> (64 - bits)
        if v < q:
            return v
    return 0


def is_prime(n):
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 325, 9375, 28178, 450775, 9780504, 1795265022):
        a %= n
        if a == 0:
            continue
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def prev_prime_congruent(bound, m):
    v = ((bound - 2) // m) * m + 1
    while v >= 2:
        if is_prime(v):
            return v
        v -= m
    return 0


def minimal_root(two_n, q):
    assert (q - 1) % two_n == 0
    for r in range(2, q):
        w = pow(r, (q - 1) // two_n, q)
        if pow(w, two_n // 2, q) == q - 1:
            break
    return min(pow(w, k, q) for k in range(1, 2 * two_n, 2))


def rev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def ntt_def(a, psi, q, log_n):
    n = len(a)
    out = []
    for i in range(n):
        e = 2 * rev(i, log_n) + 1
        step = pow(psi, e, q)
        acc, p = 0, 1
        for aj in a:
            acc = (acc + aj * p) % q
            p = p * step % q
        out.append(acc)
    return out


def negacyclic(a, b, q):
    n = len(a)
    c = [0] * n
    for i in range(n):
        for j in range(n):
            k = i + j
            if k < n:
                c[k] = (c[k] + a[i] * b[j]) % q
            else:
                c[k - n] = (c[k - n] - a[i] * b[j]) % q
    return c


def main():
    cases = []
    # (label, log_n, q): the reference's own test primes plus the workload primes
    specs = [
        ("root_rs_q132120577", 10, 132120577),                   # primus_ntt/tests/root.rs:6-7
        ("hexl_shift32_q536813569", 11, 536813569),              # primus_ntt/tests/hexl.rs (32-bit shift)
        ("hexl_shift52_q562949953392641", 11, 562949953392641),  # (52-bit shift)
        ("hexl_shift64_q1152921504606830593", 11, 1152921504606830593),  # (64-bit shift)
        ("polymul_n1024_q50", 10, prev_prime_congruent(1 << 50, 2048)),
        ("extprod_n2048_q54", 11, prev_prime_congruent(1 << 54, 4096)),
        ("small_n16_q97", 4, 97),
        ("small_n2_q5", 1, 5),
    ]
    arrays = {}
    for label, log_n, q in specs:
        n = 1 << log_n
        psi = minimal_root(2 * n, q)
        a = [uniform(0x601D, 1, i, q) for i in range(n)]
        b = [uniform(0x601D, 2, i, q) for i in range(n)]
        arrays[f"{label}/a"] = np.array(a, dtype=np.uint64)
        arrays[f"{label}/b"] = np.array(b, dtype=np.uint64)
        arrays[f"{label}/ntt_a"] = np.array(ntt_def(a, psi, q, log_n), dtype=np.uint64)
        if n <= 1024:
            arrays[f"{label}/a_times_b"] = np.array(negacyclic(a, b, q), dtype=np.uint64)
        cases.append({"label": label, "log_n": log_n, "q": q, "psi": psi})
    # primes the workloads search for (descending below the bound, q = 1 mod 2N)
    primes = {
        "polymul_2^50_mod_2048": prev_prime_congruent(1 << 50, 2048),
        "extprod_2^54_mod_4096": prev_prime_congruent(1 << 54, 4096),
    }
    ps, b = [], 1 << 50
    for _ in range(24):
        b = prev_prime_congruent(b, 1 << 17)
        ps.append(b)
    primes["rns24_2^50_mod_2^17"] = ps
    # CRT composition checks (value in [0, Q))
    crt = []
    for moduli, residues in [([3, 5, 7], [2, 3, 2]), ([256, 257], [2, 3]),
                             ([1099511592961, 1099511590913], [12345, 678910]),
                             ([1125899906826241, 1125899906629633], [1, 1125899906629632])]:
        Q = 1
        for m in moduli:
            Q *= m
        x = 0
        for m, r in zip(moduli, residues):
            Mi = Q // m
            x = (x + r * Mi * pow(Mi, -1, m)) % Q
        crt.append({"moduli": moduli, "residues": residues, "value": x})
    kats = {
        # primus_rns/tests/rns.rs:14-34: compose then decompose round-trips
        "rns": crt,
        # primus_decompose/tests/non_pow_of_2.rs:14-80: modulus 0b111_000_110,
        # log_basis 3, reverse length 2, value 0b11_111_101 recomposes within
        # the init-carry bound
        "non_pow_of_2": {"modulus": 0b111000110, "log_basis": 3, "length": 2, "value": 0b11111101},
        "ntt_cases": cases,
        "primes": primes,
    }
    np.savez_compressed(os.path.join(HERE, "ntt_golden.npz"), **arrays)
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f, indent=1)
    print("wrote", len(arrays), "arrays")


if __name__ == "__main__":
    main()
