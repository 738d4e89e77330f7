"""Python mirror of primus_rns / primus_decompose / primus_lattice operations
over the C ABI (device buffers in, device buffers out).

    RnsBase        RNSBase              primus_rns/src/base.rs
    BaseConverter  BaseConverter        primus_rns/src/converter.rs
    GadgetBasis    BigUintApproxSignedBasis  primus_decompose/src/big_integer/basis.rs
    external_product  CrtGlwe::mul_dcrt_ggsw_inplace   primus_lattice/src/glwe/crt.rs:202
    glev_mac_*        DcrtGlwe::add_dcrt_glev_mul_*     primus_lattice/src/glwe/dcrt.rs:170,249
    key_switch        CrtGlweKeySwitchingKey::key_swithching_inplace  primus_fhe_core/src/key_switch.rs:79
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import DeviceBuffer, PrimusGpuError, call, ptr


def _sh(stream):
    return None if stream is None else stream.h


class RnsError(PrimusGpuError):
    pass


class RnsBase:
    def __init__(self, moduli):
        self.moduli = [int(q) for q in moduli]
        m = np.asarray(self.moduli, dtype=np.uint64)
        h = C.c_void_p()
        st = nat.lib().pg_rns_base_create(ptr(m), len(self.moduli), C.byref(h))
        if st != nat.PG_OK:
            raise RnsError(st, "pg_rns_base_create", nat.lib().pg_last_error().decode())
        self.h = h.value
        L, W = C.c_uint32(), C.c_uint32()
        call("pg_rns_base_info", self.h, C.byref(L), C.byref(W), None)
        self.L, self.W = L.value, W.value
        prod = np.zeros(self.W, np.uint64)
        call("pg_rns_base_info", self.h, None, None, ptr(prod))
        self.product = sum(int(v) << (64 * i) for i, v in enumerate(prod))

    def moduli_count(self):
        return self.L

    def big_uint_value_len(self):
        return self.W

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_rns_base_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compose(self, residues: DeviceBuffer, values: DeviceBuffer, count: int, stream=None):
        call("pg_rns_compose", self.h, residues.ptr, values.ptr, count, _sh(stream))

    def decompose(self, values: DeviceBuffer, residues: DeviceBuffer, count: int, stream=None):
        call("pg_rns_decompose", self.h, values.ptr, residues.ptr, count, _sh(stream))

    def wrapping_decompose_small(self, small: DeviceBuffer, residues: DeviceBuffer, count: int, small_modulus: int,
                                 stream=None):
        call("pg_rns_wrapping_decompose_small", self.h, small.ptr, residues.ptr, count, small_modulus, _sh(stream))

    def add_wrapping_decompose_small_scaled(self, small: DeviceBuffer, dest: DeviceBuffer, count: int,
                                            small_modulus: int, factor, stream=None):
        """RNSBase::add_wrapping_decompose_small_values_scaled: dest += factor * lift(small)."""
        f = np.ascontiguousarray(np.asarray(factor, dtype=np.uint64))
        call("pg_rns_add_wrapping_decompose_small_scaled", self.h, small.ptr, dest.ptr, count, small_modulus, ptr(f),
             _sh(stream))


class BaseConverter:
    def __init__(self, ibase: RnsBase, obase: RnsBase):
        self.ibase, self.obase = ibase, obase
        h = C.c_void_p()
        call("pg_base_converter_create", ibase.h, obase.h, C.byref(h))
        self.h = h.value

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_base_converter_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def fast_convert_array(self, x: DeviceBuffer, out: DeviceBuffer, n: int, stream=None):
        call("pg_fast_convert_array", self.h, x.ptr, out.ptr, n, _sh(stream))


class GadgetBasis:
    def __init__(self, base: RnsBase, log_basis: int, reverse_length: int | None = None):
        self.base = base
        h = C.c_void_p()
        call("pg_gadget_basis_create", base.h, log_basis, -1 if reverse_length is None else reverse_length,
             C.byref(h))
        self.h = h.value
        d, drop = C.c_uint32(), C.c_uint32()
        call("pg_gadget_basis_info", self.h, C.byref(d), C.byref(drop), None)
        self.d, self.drop_bits, self.log_basis = d.value, drop.value, log_basis
        self.scalar_residues = np.zeros((self.d, base.L), np.uint64)
        call("pg_gadget_basis_info", self.h, None, None, ptr(self.scalar_residues))

    def decompose_length(self):
        return self.d

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_gadget_basis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def decompose(self, values: DeviceBuffer, digits: DeviceBuffer, count: int, stream=None):
        call("pg_gadget_decompose", self.h, values.ptr, digits.ptr, count, _sh(stream))

    def decompose_lift(self, values: DeviceBuffer, residues: DeviceBuffer, count: int, stream=None):
        call("pg_gadget_decompose_lift", self.h, values.ptr, residues.ptr, count, _sh(stream))


def external_product(table, basis: GadgetBasis, k: int, glwe_in: DeviceBuffer, ggsw: DeviceBuffer,
                     glwe_out: DeviceBuffer, batch: int, workspace: DeviceBuffer | None = None, stream=None):
    ws = workspace.ptr if workspace is not None else None
    wsb = workspace.count * 8 if workspace is not None else 0
    call("pg_ext_product", table.h, basis.h, k, glwe_in.ptr, ggsw.ptr, glwe_out.ptr, batch, ws, wsb, _sh(stream))


def external_product_coeff(table, basis: GadgetBasis, k: int, glwe_in: DeviceBuffer, ggsw: DeviceBuffer,
                           glwe_out: DeviceBuffer, batch: int, workspace: DeviceBuffer | None = None, stream=None):
    """external_product followed by the inverse NTT of every output poly: the
    GLWE comes back in coefficient form (one kernel for k = 1, one prime,
    N = 2^10..2^12)."""
    ws = workspace.ptr if workspace is not None else None
    wsb = workspace.count * 8 if workspace is not None else 0
    call("pg_ext_product_coeff", table.h, basis.h, k, glwe_in.ptr, ggsw.ptr, glwe_out.ptr, batch, ws, wsb,
         _sh(stream))


def ext_product_workspace_size(table, basis: GadgetBasis, k: int, batch: int) -> int:
    return int(nat.lib().pg_ext_product_workspace_size(table.h, basis.h, k, batch))


def key_switch_workspace_size(table, basis: GadgetBasis, k_in: int, k_out: int, batch: int) -> int:
    return int(nat.lib().pg_key_switch_workspace_size(table.h, basis.h, k_in, k_out, batch))


def glwe_automorphism(table, basis: GadgetBasis, k: int, degree: int, key: DeviceBuffer, c_in: DeviceBuffer,
                      c_out: DeviceBuffer, batch: int, workspace: DeviceBuffer | None = None, stream=None):
    """DcrtGlweAutoKey::automorphism_inplace on device buffers (NTT domain)."""
    ws = workspace.ptr if workspace is not None else None
    wsb = workspace.count * 8 if workspace is not None else 0
    call("pg_glwe_automorphism", table.h, basis.h, k, degree, key.ptr, c_in.ptr, c_out.ptr, batch, ws, wsb,
         _sh(stream))


def glwe_trace(table, basis: GadgetBasis, k: int, keys: DeviceBuffer, c_in: DeviceBuffer, c_out: DeviceBuffer,
               batch: int, reverse: bool = False, workspace: DeviceBuffer | None = None, stream=None):
    """DcrtGlweTraceKey::trace_inplace (reverse=False; keys of degrees N+1, N/2+1, .., 3)
    or DcrtGlweRevTraceKey::trace_inplace (reverse=True; degrees 3, 5, .., N+1),
    keys concatenated in the order applied."""
    ws = workspace.ptr if workspace is not None else None
    wsb = workspace.count * 8 if workspace is not None else 0
    call("pg_glwe_trace", table.h, basis.h, k, keys.ptr, int(bool(reverse)), c_in.ptr, c_out.ptr, batch, ws, wsb,
         _sh(stream))


def glwe_expand_coefficients(table, basis: GadgetBasis, k: int, keys: DeviceBuffer, count: int, c_in: DeviceBuffer,
                             out: DeviceBuffer, workspace: DeviceBuffer | None = None, stream=None):
    """DcrtGlweExpandCoeffKey::expand_partial_coefficients_inplace: out[count][k+1][L][N]."""
    ws = workspace.ptr if workspace is not None else None
    wsb = workspace.count * 8 if workspace is not None else 0
    call("pg_glwe_expand_coefficients", table.h, basis.h, k, keys.ptr, count, c_in.ptr, out.ptr, ws, wsb,
         _sh(stream))


def glev_mac_crt_poly(table, basis: GadgetBasis, k: int, acc: DeviceBuffer, glev: DeviceBuffer,
                      crt_poly: DeviceBuffer, stream=None):
    call("pg_glev_mac_crt_poly", table.h, basis.h, k, acc.ptr, glev.ptr, crt_poly.ptr, None, 0, _sh(stream))


def glev_mac_big_uint_poly(table, basis: GadgetBasis, k: int, acc: DeviceBuffer, glev: DeviceBuffer,
                           big_poly: DeviceBuffer, stream=None):
    call("pg_glev_mac_big_uint_poly", table.h, basis.h, k, acc.ptr, glev.ptr, big_poly.ptr, None, 0, _sh(stream))


def key_switch(table, basis: GadgetBasis, k_in: int, k_out: int, key: DeviceBuffer, c_in: DeviceBuffer,
               c_out: DeviceBuffer, batch: int, workspace: DeviceBuffer | None = None, stream=None):
    ws = workspace.ptr if workspace is not None else None
    wsb = workspace.count * 8 if workspace is not None else 0
    call("pg_key_switch", table.h, basis.h, k_in, k_out, key.ptr, c_in.ptr, c_out.ptr, batch, ws, wsb, _sh(stream))


class HybridKeySwitch:
    """Hybrid RNS key switch over a table of L + K primes (Q then P) with digit
    groups of `alpha` Q limbs (pg_hybrid_ks_*).  No reference counterpart."""

    def __init__(self, table, L: int, K: int, alpha: int):
        h = C.c_void_p()
        call("pg_hybrid_ks_create", table.h, L, K, alpha, C.byref(h))
        self.h = h.value
        self.table, self.L, self.K, self.alpha = table, L, K, alpha
        self.dnum = int(nat.lib().pg_hybrid_ks_dnum(self.h))

    def workspace_size(self, k_in: int, k_out: int, batch: int) -> int:
        return int(nat.lib().pg_hybrid_ks_workspace_size(self.h, k_in, k_out, batch))

    def key_switch(self, k_in: int, k_out: int, key: DeviceBuffer, c_in: DeviceBuffer, c_out: DeviceBuffer,
                   batch: int, workspace: DeviceBuffer | None = None, stream=None):
        ws = workspace.ptr if workspace is not None else None
        wsb = workspace.count * 8 if workspace is not None else 0
        call("pg_key_switch_hybrid", self.h, k_in, k_out, key.ptr, c_in.ptr, c_out.ptr, batch, ws, wsb,
             _sh(stream))

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_hybrid_ks_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BfvDecryptor:
    """BFV decryption through fast base conversion on the device
    (DcrtGlweSecretKey::decrypt_inplace); pg_bfv_decryptor_* / pg_bfv_decrypt."""

    def __init__(self, table, plain_modulus: int, gamma: int):
        h = C.c_void_p()
        call("pg_bfv_decryptor_create", table.h, plain_modulus, gamma, C.byref(h))
        self.h = h.value
        self.table, self.t, self.gamma = table, plain_modulus, gamma

    def decrypt(self, k: int, sk_ntt: DeviceBuffer, ct: DeviceBuffer, msg: DeviceBuffer, batch: int,
                workspace: DeviceBuffer | None = None, stream=None):
        ws = workspace.ptr if workspace is not None else None
        wsb = workspace.count * 8 if workspace is not None else 0
        call("pg_bfv_decrypt", self.h, k, sk_ntt.ptr, ct.ptr, msg.ptr, batch, ws, wsb, _sh(stream))

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_bfv_decryptor_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GlweEncryptor:
    """Secret-key GLWE encryption on the device with reproducible samplers
    (pg_glwe_encryptor_* / pg_glwe_encrypt)."""

    def __init__(self, table, sigma: float = 3.2):
        h = C.c_void_p()
        call("pg_glwe_encryptor_create", table.h, float(sigma), C.byref(h))
        self.h = h.value
        self.table, self.sigma = table, sigma

    def encrypt(self, k: int, sk_ntt: DeviceBuffer, msg: DeviceBuffer | None, scale, seed: int, stream0: int,
                ct: DeviceBuffer, batch: int, stream=None):
        sc = np.ascontiguousarray(np.asarray(scale if scale is not None else [0] * self.table.L, dtype=np.uint64))
        call("pg_glwe_encrypt", self.h, k, sk_ntt.ptr, msg.ptr if msg is not None else None, ptr(sc), seed, stream0,
             ct.ptr, batch, _sh(stream))

    def public_key(self, k: int, sk_ntt: DeviceBuffer, seed: int, stream0: int, pk: DeviceBuffer, stream=None):
        """DcrtGlwePublicKey::new: a secret-key encryption of zero, [k+1][L][N]."""
        self.encrypt(k, sk_ntt, None, None, seed, stream0, pk, 1, stream=stream)

    def pk_encrypt(self, k: int, pk: DeviceBuffer, msg: DeviceBuffer | None, scale, seed: int, stream0: int,
                   ct: DeviceBuffer, batch: int, stream=None):
        """DcrtGlwePublicKey::encrypt of `batch` ciphertexts."""
        sc = np.ascontiguousarray(np.asarray(scale if scale is not None else [0] * self.table.L, dtype=np.uint64))
        call("pg_glwe_pk_encrypt", self.h, k, pk.ptr, msg.ptr if msg is not None else None, ptr(sc), seed, stream0,
             ct.ptr, batch, _sh(stream))

    def ggsw_pk_encrypt_monomial(self, basis: GadgetBasis, k: int, pk: DeviceBuffer, coeff_residues, degree: int,
                                 seed: int, stream0: int, ggsw: DeviceBuffer, stream=None):
        """DcrtGlwePublicKey::encrypt_monomial_ggsw_inplace: [k+1][d][k+1][L][N]."""
        cr = np.ascontiguousarray(np.asarray(coeff_residues, dtype=np.uint64))
        call("pg_ggsw_pk_encrypt_monomial", self.h, basis.h, k, pk.ptr, ptr(cr), degree, seed, stream0, ggsw.ptr,
             _sh(stream))

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_glwe_encryptor_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
