"""ctypes bindings for the CPU oracle (oracle/primus_oracle.c).

TEST INFRASTRUCTURE ONLY.  This package is the parity oracle: tests/, the smoke
check in __graft_entry__.py and bench.py's CPU-baseline / reference arm import
it.  The product package (primus_b200) never imports it.

The oracle restates the reference's Rust functions in C (each C function
cites the crate file:line it follows).  The reference itself is a Rust
workspace that is not compiled or run next to this package, so the restatement
is pinned by the reference's own known-answer and property tests
(tests/test_oracle_pins.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "primus_oracle.c")
SRCS = [SRC, os.path.join(HERE, "hexl_ifma.c")]
HDR = os.path.join(HERE, "primus_oracle.h")

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u8p = C.POINTER(C.c_uint8)


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (OpenMP for the multi-threaded CPU baseline)."""
    newest = max(os.path.getmtime(f) for f in SRCS + [HDR])
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        # hexl_ifma.c marks its AVX-512 functions with target attributes; the rest is x86-64-v3
        cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-fopenmp", "-o", LIB_PATH, *SRCS, "-lm"]
        subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        sig = {
            "orc_hash64": (C.c_uint64, [C.c_uint64] * 4),
            "orc_uniform_at": (C.c_uint64, [C.c_uint64] * 4),
            "orc_fill_uniform": (None, [C.c_uint64, C.c_uint64, C.c_uint64, C.c_size_t, u64p]),
            "orc_fill_uniform_rns": (None, [C.c_uint64, C.c_uint64, u64p, C.c_uint32, C.c_size_t, u64p]),
            "orc_mulmod": (C.c_uint64, [C.c_uint64] * 3),
            "orc_powmod": (C.c_uint64, [C.c_uint64] * 3),
            "orc_invmod": (C.c_uint64, [C.c_uint64] * 2),
            "orc_is_prime": (C.c_int, [C.c_uint64]),
            "orc_prev_prime_congruent": (C.c_uint64, [C.c_uint64, C.c_uint64]),
            "orc_ntt_primes": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint32, u64p]),
            "orc_shoup_quotient": (C.c_uint64, [C.c_uint64, C.c_uint64]),
            "orc_shoup_lazy_mul": (C.c_uint64, [C.c_uint64] * 4),
            "orc_shoup_mul": (C.c_uint64, [C.c_uint64] * 4),
            "orc_barrett_ratio": (None, [C.c_uint64, u64p]),
            "orc_barrett_reduce_mul": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64, u64p]),
            "orc_barrett_reduce_mul_add": (C.c_uint64, [C.c_uint64] * 4 + [u64p]),
            "orc_barrett_dot_product": (C.c_uint64, [u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_minimal_primitive_root": (C.c_int, [C.c_uint32, C.c_uint64, u64p]),
            "orc_ntt_table_new": (C.c_void_p, [C.c_uint32, C.c_uint64]),
            "orc_ntt_table_delete": (None, [C.c_void_p]),
            "orc_ntt_table_export": (None, [C.c_void_p] + [u64p] * 10),
            "orc_ntt_lazy_forward": (None, [C.c_void_p, u64p]),
            "orc_ntt_forward": (None, [C.c_void_p, u64p]),
            "orc_ntt_lazy_inverse": (None, [C.c_void_p, u64p]),
            "orc_ntt_inverse": (None, [C.c_void_p, u64p]),
            "orc_ntt_monomial": (None, [C.c_void_p, C.c_uint64, C.c_size_t, u64p]),
            "orc_ntt_coeff_one_monomial": (None, [C.c_void_p, C.c_size_t, u64p]),
            "orc_ntt_coeff_minus_one_monomial": (None, [C.c_void_p, C.c_size_t, u64p]),
            "orc_ntt_forward_rows": (None, [C.c_void_p, u64p, C.c_size_t, C.c_int, C.c_int]),
            "orc_ntt_inverse_rows": (None, [C.c_void_p, u64p, C.c_size_t, C.c_int, C.c_int]),
            "orc_ntt_by_definition": (None, [C.c_void_p, u64p, u64p]),
            "orc_dcrt_forward": (None, [C.c_void_p, C.c_uint32, u64p, C.c_size_t, C.c_int, C.c_int]),
            "orc_dcrt_inverse": (None, [C.c_void_p, C.c_uint32, u64p, C.c_size_t, C.c_int, C.c_int]),
            "orc_dcrt_polymul_roundtrip": (None, [C.c_void_p, C.c_uint32, u64p, u64p, C.c_size_t, C.c_int]),
            "orc_mul_assign": (None, [u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_add_mul_assign": (None, [u64p, u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_mul_scalar_assign": (None, [u64p, C.c_uint64, C.c_size_t, C.c_uint64]),
            "orc_add_mul_scalar_assign": (None, [u64p, u64p, C.c_uint64, C.c_size_t, C.c_uint64]),
            "orc_mul_factor_assign": (None, [u64p, C.c_uint64, C.c_uint64, C.c_size_t, C.c_uint64]),
            "orc_add_assign": (None, [u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_sub_assign": (None, [u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_neg_assign": (None, [u64p, C.c_size_t, C.c_uint64]),
            "orc_butterfly_mul_factor": (None, [u64p, u64p, u64p, u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_naive_negacyclic_mul": (None, [u64p, u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_rns_base_new": (C.c_void_p, [u64p, C.c_uint32]),
            "orc_rns_base_delete": (None, [C.c_void_p]),
            "orc_rns_base_width": (C.c_uint32, [C.c_void_p]),
            "orc_rns_base_export": (None, [C.c_void_p, u64p, u64p, u64p]),
            "orc_rns_compose": (None, [C.c_void_p, u64p, u64p]),
            "orc_rns_compose_multiple": (None, [C.c_void_p, u64p, u64p, C.c_size_t]),
            "orc_rns_decompose": (None, [C.c_void_p, u64p, u64p]),
            "orc_rns_decompose_multiple": (None, [C.c_void_p, u64p, u64p, C.c_size_t]),
            "orc_rns_wrapping_decompose_small": (None, [C.c_void_p, u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_base_converter_new": (C.c_void_p, [C.c_void_p, C.c_void_p]),
            "orc_base_converter_delete": (None, [C.c_void_p]),
            "orc_fast_convert_array": (None, [C.c_void_p, u64p, u64p, C.c_size_t]),
            "orc_gadget_basis_new": (C.c_void_p, [C.c_void_p, C.c_uint32, C.c_int32]),
            "orc_gadget_basis_delete": (None, [C.c_void_p]),
            "orc_gadget_basis_info": (None, [C.c_void_p, u32p, u32p, u64p]),
            "orc_gadget_init_carry": (None, [C.c_void_p, u64p, u8p, C.c_size_t]),
            "orc_gadget_unsigned_digit": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u8p, C.c_size_t]),
            "orc_gadget_decompose_all": (None, [C.c_void_p, u64p, u64p, C.c_size_t]),
            "orc_approx_basis_new": (C.c_void_p, [C.c_int, C.c_uint64, C.c_uint32, C.c_int32]),
            "orc_approx_basis_delete": (None, [C.c_void_p]),
            "orc_approx_basis_info": (None, [C.c_void_p, u32p, u32p, u32p, u64p]),
            "orc_approx_decompose": (None, [C.c_void_p, C.c_uint64, u64p]),
            "orc_glev_mac_crt_poly": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p]),
            "orc_glev_mac_big_uint_poly": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p]),
            "orc_external_product": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p]),
            "orc_external_product_batch": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p, C.c_size_t, C.c_int]),
            "orc_key_switch": (None, [C.c_void_p, C.c_uint32, C.c_uint32, u64p, u64p, u64p]),
            "orc_sample_ternary": (None, [C.c_uint64, C.c_uint64, u64p, C.c_uint32, C.c_size_t, u64p]),
            "orc_sample_gaussian": (None, [C.c_uint64, C.c_uint64, C.c_double, u64p, C.c_uint32, C.c_size_t, u64p]),
            "orc_glwe_encrypt": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p, C.c_uint64, C.c_double, u64p]),
            "orc_ggsw_encrypt_monomial": (None, [C.c_void_p, C.c_uint32, u64p, u64p, C.c_size_t, C.c_uint64,
                                                 C.c_double, u64p]),
            "orc_ksk_generate": (None, [C.c_void_p, C.c_uint32, C.c_uint32, u64p, u64p, C.c_uint64, C.c_double, u64p]),
            "orc_glwe_decrypt": (None, [C.c_void_p, C.c_uint32, u64p, u64p, C.c_uint64, C.c_uint64, u64p]),
            "orc_bfv_delta": (None, [C.c_void_p, C.c_uint64, u64p]),
            "orc_ntt_auto_perm": (None, [C.c_uint32, C.c_uint64, u32p]),
            "orc_glwe_automorphism": (None, [C.c_void_p, C.c_uint32, C.c_uint64, u64p, u64p, u64p]),
            "orc_glwe_trace": (None, [C.c_void_p, C.c_uint32, u64p, C.c_int, u64p, u64p]),
            "orc_glwe_pk_encrypt_cdt": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p, C.c_double, C.c_uint64,
                                                C.c_uint64, C.c_uint64, u64p]),
            "orc_ggsw_pk_encrypt_monomial": (None, [C.c_void_p, C.c_uint32, u64p, u64p, C.c_size_t, C.c_double,
                                                     C.c_uint64, C.c_uint64, u64p]),
            "orc_glwe_expand": (None, [C.c_void_p, C.c_uint32, u64p, C.c_size_t, u64p, u64p]),
            "orc_cdt_table": (C.c_uint32, [C.c_double, u64p, C.c_uint32]),
            "orc_cdt_sample": (C.c_int64, [u64p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64]),
            "orc_glwe_encrypt_cdt": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p, C.c_double, C.c_uint64,
                                            C.c_uint64, C.c_uint64, u64p]),
            "orc_hexl_available": (C.c_int, []),
            "orc_hexl_table_new": (C.c_void_p, [C.c_void_p]),
            "orc_hexl_table_delete": (None, [C.c_void_p]),
            "orc_hexl_forward": (None, [C.c_void_p, u64p]),
            "orc_hexl_inverse": (None, [C.c_void_p, u64p]),
            "orc_hexl_precon52": (None, [u64p, u64p, C.c_size_t, C.c_uint64]),
            "orc_hexl_polymul_roundtrip": (None, [C.c_void_p, C.c_uint32, u64p, u64p, u64p, C.c_size_t, C.c_int]),
            "orc_hybrid_ks_new": (C.c_void_p, [C.c_uint32, u64p, C.c_uint32, C.c_uint32, C.c_uint32]),
            "orc_hybrid_ks_delete": (None, [C.c_void_p]),
            "orc_hybrid_ks_dnum": (C.c_uint32, [C.c_void_p]),
            "orc_hybrid_ks_factor": (None, [C.c_void_p, C.c_uint32, u64p]),
            "orc_hybrid_key_switch": (None, [C.c_void_p, C.c_uint32, C.c_uint32, u64p, u64p, u64p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def p64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(u64p)


def u64(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.uint64))


# ---------------------------------------------------------------- inputs

def uniform(seed: int, stream: int, q: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    lib().orc_fill_uniform(seed, stream, q, n, p64(out))
    return out


def uniform_rns(seed: int, stream0: int, moduli, n: int) -> np.ndarray:
    m = u64(moduli)
    out = np.empty((len(m), n), dtype=np.uint64)
    lib().orc_fill_uniform_rns(seed, stream0, p64(m), len(m), n, p64(out))
    return out


def ntt_primes(bound: int, m: int, count: int):
    out = np.zeros(count, dtype=np.uint64)
    rc = lib().orc_ntt_primes(bound, m, count, p64(out))
    if rc != 0:
        raise ValueError("not enough primes")
    return [int(x) for x in out]


# ---------------------------------------------------------------- NTT

class NttTable:
    """Restatement of UintNttTable (primus_ntt/src/ntt/primitive.rs)."""

    def __init__(self, log_n: int, q: int):
        self.log_n, self.q, self.n = log_n, q, 1 << log_n
        self.h = lib().orc_ntt_table_new(log_n, q)
        if not self.h:
            raise ValueError(f"no NTT table for log_n={log_n} q={q}")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_ntt_table_delete(self.h)
            self.h = None

    def export(self):
        n = self.n
        vals = [np.zeros(1, np.uint64) for _ in range(4)]
        arrs = [np.zeros(n, np.uint64) for _ in range(4)] + [np.zeros(2 * n, np.uint64) for _ in range(2)]
        lib().orc_ntt_table_export(self.h, *[p64(v) for v in vals], *[p64(a) for a in arrs])
        keys = ["root", "inv_root", "inv_n", "inv_n_q"]
        d = {k: int(v[0]) for k, v in zip(keys, vals)}
        for k, a in zip(["root_powers", "root_powers_q", "inv_root_powers", "inv_root_powers_q",
                         "ordinal", "ordinal_q"], arrs):
            d[k] = a
        return d

    def _rows(self, fn, a, *extra):
        a = u64(a).copy()
        rows = a.size // self.n
        getattr(lib(), fn)(self.h, p64(a), rows, *extra)
        return a

    def forward(self, a, lazy=False, threads=1):
        return self._rows("orc_ntt_forward_rows", a, int(lazy), threads)

    def inverse(self, a, lazy=False, threads=1):
        return self._rows("orc_ntt_inverse_rows", a, int(lazy), threads)

    def by_definition(self, a):
        a = u64(a)
        out = np.zeros(self.n, np.uint64)
        lib().orc_ntt_by_definition(self.h, p64(a), p64(out))
        return out

    def monomial(self, coeff, degree):
        out = np.zeros(self.n, np.uint64)
        lib().orc_ntt_monomial(self.h, coeff, degree, p64(out))
        return out

    def coeff_one_monomial(self, degree):
        out = np.zeros(self.n, np.uint64)
        lib().orc_ntt_coeff_one_monomial(self.h, degree, p64(out))
        return out

    def coeff_minus_one_monomial(self, degree):
        out = np.zeros(self.n, np.uint64)
        lib().orc_ntt_coeff_minus_one_monomial(self.h, degree, p64(out))
        return out


class DcrtTable:
    """Restatement of UintCrtNttTable (primus_ntt/src/dcrt/primitive.rs)."""

    def __init__(self, log_n: int, moduli):
        self.moduli = [int(q) for q in moduli]
        self.L, self.n, self.log_n = len(self.moduli), 1 << log_n, log_n
        self.tables = [NttTable(log_n, q) for q in self.moduli]
        self._arr = (C.c_void_p * self.L)(*[t.h for t in self.tables])

    def forward(self, a, lazy=False, threads=1):
        a = u64(a).copy()
        polys = a.size // (self.L * self.n)
        lib().orc_dcrt_forward(self._arr, self.L, p64(a), polys, int(lazy), threads)
        return a

    def inverse(self, a, lazy=False, threads=1):
        a = u64(a).copy()
        polys = a.size // (self.L * self.n)
        lib().orc_dcrt_inverse(self._arr, self.L, p64(a), polys, int(lazy), threads)
        return a

    def polymul_roundtrip(self, a, plain, threads=1):
        a = u64(a).copy()
        polys = a.size // (self.L * self.n)
        lib().orc_dcrt_polymul_roundtrip(self._arr, self.L, p64(a), p64(u64(plain)), polys, threads)
        return a


# ---------------------------------------------------------------- pointwise

def _pw(fn, q, *arrays, scalars=()):
    arrs = [u64(x).copy() for x in arrays]
    n = arrs[0].size
    getattr(lib(), fn)(*[p64(a) for a in arrs[:1]], *[p64(a) for a in arrs[1:]], *scalars, n, q)
    return arrs


def mul(x, y, q):
    return _pw("orc_mul_assign", q, x, y)[0]


def add_mul(acc, b, c, q):
    return _pw("orc_add_mul_assign", q, acc, b, c)[0]


def add(x, y, q):
    return _pw("orc_add_assign", q, x, y)[0]


def sub(x, y, q):
    return _pw("orc_sub_assign", q, x, y)[0]


def neg(x, q):
    return _pw("orc_neg_assign", q, x)[0]


def mul_scalar(x, s, q):
    x = u64(x).copy()
    lib().orc_mul_scalar_assign(p64(x), s, x.size, q)
    return x


def add_mul_scalar(x, y, s, q):
    x = u64(x).copy()
    lib().orc_add_mul_scalar_assign(p64(x), p64(u64(y)), s, x.size, q)
    return x


def mul_factor(x, w, q):
    x = u64(x).copy()
    lib().orc_mul_factor_assign(p64(x), w, lib().orc_shoup_quotient(w, q), x.size, q)
    return x


def butterfly_mul_factor(a, s, w, q):
    a = u64(a).copy()
    s, w = u64(s), u64(w)
    wq = np.array([lib().orc_shoup_quotient(int(v), q) for v in w], dtype=np.uint64)
    b = np.zeros_like(a)
    lib().orc_butterfly_mul_factor(p64(a), p64(s), p64(w), p64(wq), p64(b), a.size, q)
    return a, b


def naive_negacyclic(a, b, q):
    a, b = u64(a), u64(b)
    c = np.zeros_like(a)
    lib().orc_naive_negacyclic_mul(p64(a), p64(b), p64(c), a.size, q)
    return c


# ---------------------------------------------------------------- RNS

class RnsBase:
    """Restatement of RNSBase (primus_rns/src/base.rs)."""

    def __init__(self, moduli):
        self.moduli = u64(moduli)
        self.L = len(self.moduli)
        self.h = lib().orc_rns_base_new(p64(self.moduli), self.L)
        if not self.h:
            raise ValueError("moduli are not co-prime")
        self.W = lib().orc_rns_base_width(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_rns_base_delete(self.h)
            self.h = None

    def export(self):
        prod = np.zeros(self.W, np.uint64)
        punct = np.zeros((self.L, self.W), np.uint64)
        inv = np.zeros(self.L, np.uint64)
        lib().orc_rns_base_export(self.h, p64(prod), p64(punct), p64(inv))
        return prod, punct, inv

    def compose(self, residues):
        out = np.zeros(self.W, np.uint64)
        lib().orc_rns_compose(self.h, p64(u64(residues)), p64(out))
        return out

    def compose_multiple(self, multi):
        multi = u64(multi)
        count = multi.size // self.L
        out = np.zeros((count, self.W), np.uint64)
        lib().orc_rns_compose_multiple(self.h, p64(multi), p64(out), count)
        return out

    def decompose(self, value):
        out = np.zeros(self.L, np.uint64)
        lib().orc_rns_decompose(self.h, p64(u64(value)), p64(out))
        return out

    def decompose_multiple(self, values):
        values = u64(values)
        count = values.size // self.W
        out = np.zeros((self.L, count), np.uint64)
        lib().orc_rns_decompose_multiple(self.h, p64(values), p64(out), count)
        return out

    def wrapping_decompose_small(self, small, small_modulus):
        small = u64(small)
        out = np.zeros((self.L, small.size), np.uint64)
        lib().orc_rns_wrapping_decompose_small(self.h, p64(small), p64(out), small.size, small_modulus)
        return out


class BaseConverter:
    """Restatement of BaseConverter (primus_rns/src/converter.rs)."""

    def __init__(self, ibase: RnsBase, obase: RnsBase):
        self.ibase, self.obase = ibase, obase
        self.h = lib().orc_base_converter_new(ibase.h, obase.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_base_converter_delete(self.h)
            self.h = None

    def fast_convert_array(self, x):
        x = u64(x)
        n = x.size // self.ibase.L
        out = np.zeros((self.obase.L, n), np.uint64)
        lib().orc_fast_convert_array(self.h, p64(x), p64(out), n)
        return out


class GadgetBasis:
    """Restatement of BigUintApproxSignedBasis (primus_decompose/src/big_integer)."""

    def __init__(self, base: RnsBase, log_basis: int, reverse_length: int | None = None):
        self.base = base
        self.h = lib().orc_gadget_basis_new(base.h, log_basis, -1 if reverse_length is None else reverse_length)
        if not self.h:
            raise ValueError("bad gadget basis")
        d, drop = C.c_uint32(), C.c_uint32()
        lib().orc_gadget_basis_info(self.h, C.byref(d), C.byref(drop), None)
        self.d, self.drop_bits, self.log_basis = d.value, drop.value, log_basis
        self.scalar_residues = np.zeros((self.d, base.L), np.uint64)
        lib().orc_gadget_basis_info(self.h, None, None, p64(self.scalar_residues))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_gadget_basis_delete(self.h)
            self.h = None

    def decompose_all(self, values):
        values = u64(values)
        count = values.size // self.base.W
        out = np.zeros((self.d, count), np.uint64)
        lib().orc_gadget_decompose_all(self.h, p64(values), p64(out), count)
        return out


class ApproxBasis:
    """Restatement of ApproxSignedBasis (primus_decompose/src/primitive)."""

    def __init__(self, modulus: int | None, log_basis: int, reverse_length: int | None = None):
        self.h = lib().orc_approx_basis_new(0 if modulus is None else 1, modulus or 0, log_basis,
                                            -1 if reverse_length is None else reverse_length)
        if not self.h:
            raise ValueError("bad basis")
        d, drop, vb = C.c_uint32(), C.c_uint32(), C.c_uint32()
        lib().orc_approx_basis_info(self.h, C.byref(d), C.byref(drop), C.byref(vb), None)
        self.d, self.drop_bits, self.value_bits = d.value, drop.value, vb.value
        self.scalars = np.zeros(self.d, np.uint64)
        lib().orc_approx_basis_info(self.h, None, None, None, p64(self.scalars))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_approx_basis_delete(self.h)
            self.h = None

    def decompose(self, value: int):
        out = np.zeros(self.d, np.uint64)
        lib().orc_approx_decompose(self.h, value, p64(out))
        return out


class LatticeCtx(C.Structure):
    _fields_ = [("tables", C.c_void_p), ("L", C.c_uint32), ("n", C.c_size_t),
                ("base", C.c_void_p), ("basis", C.c_void_p)]


class Lattice:
    """GLev MAC / external product / key switch / GLWE enc-dec over one DCRT table."""

    def __init__(self, table: DcrtTable, base: RnsBase, basis: GadgetBasis):
        self.table, self.base, self.basis = table, base, basis
        self.L, self.n, self.d = table.L, table.n, basis.d
        self.ctx = LatticeCtx(C.cast(table._arr, C.c_void_p), table.L, table.n, base.h, basis.h)
        self.pctx = C.byref(self.ctx)

    def external_product(self, k, glwe_in, ggsw, batch=1, threads=1):
        glwe_in = u64(glwe_in)
        out = np.zeros_like(glwe_in)
        lib().orc_external_product_batch(self.pctx, k, p64(glwe_in), p64(u64(ggsw)), p64(out), batch, threads)
        return out

    def glev_mac_crt_poly(self, k, acc, glev, crt_poly):
        acc = u64(acc).copy()
        lib().orc_glev_mac_crt_poly(self.pctx, k, p64(acc), p64(u64(glev)), p64(u64(crt_poly)))
        return acc

    def key_switch(self, k_in, k_out, key, c_in):
        out = np.zeros((k_out + 1) * self.L * self.n, np.uint64)
        lib().orc_key_switch(self.pctx, k_in, k_out, p64(u64(key)), p64(u64(c_in)), p64(out))
        return out

    def automorphism(self, k, degree, key, ct_in):
        """DcrtGlweAutoKey::automorphism_inplace: NTT-domain GLWE in and out."""
        out = np.zeros((k + 1) * self.L * self.n, np.uint64)
        lib().orc_glwe_automorphism(self.pctx, k, degree, p64(u64(key)), p64(u64(ct_in)), p64(out))
        return out

    def trace(self, k, keys, ct_in, reverse=False):
        """DcrtGlweTraceKey / DcrtGlweRevTraceKey::trace_inplace (keys in the order applied)."""
        out = np.zeros((k + 1) * self.L * self.n, np.uint64)
        lib().orc_glwe_trace(self.pctx, k, p64(u64(keys)), int(reverse), p64(u64(ct_in)), p64(out))
        return out

    def expand(self, k, keys, count, ct_in):
        """DcrtGlweExpandCoeffKey::expand_partial_coefficients_inplace: [count][k+1][L][N]."""
        out = np.zeros(count * (k + 1) * self.L * self.n, np.uint64)
        lib().orc_glwe_expand(self.pctx, k, p64(u64(keys)), count, p64(u64(ct_in)), p64(out))
        return out

    def encrypt_cdt(self, k, sk_ntt, msg, scale, seed, stream0, index, sigma=3.2):
        """GLWE encryption with the CDT Gaussian sampler (ciphertext `index` of a batch)."""
        ct = np.zeros((k + 1) * self.L * self.n, np.uint64)
        mp = p64(u64(msg)) if msg is not None else None
        lib().orc_glwe_encrypt_cdt(self.pctx, k, p64(u64(sk_ntt)), mp, p64(u64(scale)), sigma, seed, stream0, index,
                                   p64(ct))
        return ct

    def pk_encrypt_cdt(self, k, pk, msg, scale, seed, stream0, index, sigma=3.2):
        """DcrtGlwePublicKey::encrypt of ciphertext `index` with the counter-based samplers."""
        ct = np.zeros((k + 1) * self.L * self.n, np.uint64)
        mp = p64(u64(msg)) if msg is not None else None
        sp = p64(u64(scale)) if scale is not None else None
        lib().orc_glwe_pk_encrypt_cdt(self.pctx, k, p64(u64(pk)), mp, sp, sigma, seed, stream0, index, p64(ct))
        return ct

    def ggsw_pk_encrypt_monomial(self, k, pk, coeff_res, degree, seed, stream0, sigma=3.2):
        """DcrtGlwePublicKey::encrypt_monomial_ggsw: [k+1][d][k+1][L][N]."""
        out = np.zeros((k + 1) * self.d * (k + 1) * self.L * self.n, np.uint64)
        lib().orc_ggsw_pk_encrypt_monomial(self.pctx, k, p64(u64(pk)), p64(u64(coeff_res)), degree, sigma, seed,
                                           stream0, p64(out))
        return out

    def ternary(self, seed, stream):
        out = np.zeros(self.L * self.n, np.uint64)
        lib().orc_sample_ternary(seed, stream, p64(u64(self.table.moduli)), self.L, self.n, p64(out))
        return out

    def encrypt(self, k, sk_ntt, msg, delta_res, seed, sigma=3.2):
        ct = np.zeros((k + 1) * self.L * self.n, np.uint64)
        lib().orc_glwe_encrypt(self.pctx, k, p64(u64(sk_ntt)), p64(u64(msg)), p64(u64(delta_res)), seed, sigma,
                               p64(ct))
        return ct

    def ggsw_monomial(self, k, sk_ntt, coeff_res, degree, seed, sigma=3.2):
        g = np.zeros((k + 1) * self.d * (k + 1) * self.L * self.n, np.uint64)
        lib().orc_ggsw_encrypt_monomial(self.pctx, k, p64(u64(sk_ntt)), p64(u64(coeff_res)), degree, seed, sigma,
                                        p64(g))
        return g

    def ksk(self, k_in, k_out, sk_in_coeff, sk_out_ntt, seed, sigma=3.2):
        key = np.zeros(k_in * self.d * (k_out + 1) * self.L * self.n, np.uint64)
        lib().orc_ksk_generate(self.pctx, k_in, k_out, p64(u64(sk_in_coeff)), p64(u64(sk_out_ntt)), seed, sigma,
                               p64(key))
        return key

    def decrypt(self, k, sk_ntt, ct, t, gamma):
        out = np.zeros(self.n, np.uint64)
        lib().orc_glwe_decrypt(self.pctx, k, p64(u64(sk_ntt)), p64(u64(ct)), t, gamma, p64(out))
        return out

    def delta(self, t):
        out = np.zeros(self.L, np.uint64)
        lib().orc_bfv_delta(self.base.h, t, p64(out))
        return out


class HybridKeySwitch:
    """Hybrid RNS key switch with K special primes and digit groups of alpha
    limbs (a definition of this build; the reference has no such key switch).
    moduli = Q (L primes) followed by P (K primes)."""

    def __init__(self, log_n: int, moduli, L: int, K: int, alpha: int):
        self.moduli = [int(q) for q in moduli]
        assert len(self.moduli) == L + K
        self.log_n, self.n, self.L, self.K, self.alpha = log_n, 1 << log_n, L, K, alpha
        self.h = lib().orc_hybrid_ks_new(log_n, p64(u64(self.moduli)), L, K, alpha)
        if not self.h:
            raise ValueError("hybrid key switch parameters rejected")
        self.dnum = int(lib().orc_hybrid_ks_dnum(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_hybrid_ks_delete(self.h)
            self.h = None

    def factor(self, g: int) -> np.ndarray:
        out = np.zeros(self.L + self.K, np.uint64)
        lib().orc_hybrid_ks_factor(self.h, g, p64(out))
        return out

    def key_switch(self, k_in: int, k_out: int, key, c_in) -> np.ndarray:
        out = np.zeros((k_out + 1) * self.L * self.n, np.uint64)
        lib().orc_hybrid_key_switch(self.h, k_in, k_out, p64(u64(key)), p64(u64(c_in)), p64(out))
        return out


def hexl_available() -> bool:
    """True when this host runs the AVX-512 IFMA52 transforms (the reference's HEXL path)."""
    return bool(lib().orc_hexl_available())


class HexlDcrt:
    """HEXL-style AVX-512 IFMA52 transforms over a DcrtTable's primes (q < 2^50):
    the reference's fastest CPU path, used as the timed CPU baseline."""

    def __init__(self, table: "DcrtTable"):
        self.table, self.L, self.n = table, table.L, table.n
        self.h = []
        for i in range(table.L):
            h = lib().orc_hexl_table_new(table._arr[i])
            if not h:
                raise ValueError("HEXL path needs q < 2^50 and n >= 16")
            self.h.append(h)
        self._harr = (C.c_void_p * table.L)(*self.h)

    def __del__(self):
        for h in getattr(self, "h", []):
            lib().orc_hexl_table_delete(h)
        self.h = []

    def forward(self, a):
        a = u64(a).copy()
        for r in range(a.size // self.n):
            lib().orc_hexl_forward(self.h[r % self.L], p64(a[r * self.n:]))
        return a

    def inverse(self, a):
        a = u64(a).copy()
        for r in range(a.size // self.n):
            lib().orc_hexl_inverse(self.h[r % self.L], p64(a[r * self.n:]))
        return a

    def prepare(self, plain):
        plain = np.ascontiguousarray(u64(plain).ravel())
        pp = np.zeros_like(plain)
        for l in range(self.L):
            lib().orc_hexl_precon52(p64(plain[l * self.n:]), p64(pp[l * self.n:]), self.n, self.table.moduli[l])
        return pp

    def polymul_roundtrip(self, a, plain, plain_p, threads=1):
        """In place on a: forward, x plain (NTT domain, quotients from prepare), inverse."""
        plain = np.ascontiguousarray(u64(plain).ravel())
        plain_p = np.ascontiguousarray(u64(plain_p).ravel())
        lib().orc_hexl_polymul_roundtrip(self._harr, self.L, p64(a), p64(plain), p64(plain_p),
                                         a.size // (self.L * self.n), threads)
        return a


def ntt_auto_perm(log_n: int, degree: int) -> np.ndarray:
    """generate_ntt_permutation: out[d] = in[perm[d]] in bit-reversed NTT storage."""
    perm = np.zeros(1 << log_n, np.uint32)
    lib().orc_ntt_auto_perm(log_n, degree, perm.ctypes.data_as(u32p))
    return perm
