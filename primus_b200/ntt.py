"""Python mirror of primus_ntt's `NttTable` / `DcrtTable` traits over the C ABI.

Method names, argument meaning and error behaviour follow the Rust traits
(primus_ntt/src/ntt/mod.rs:20-117, primus_ntt/src/dcrt/mod.rs:17-129):

* ``*_slice`` methods transform a host slice (a uint64 numpy array) in place,
  exactly like the reference's `&mut [u64]` calls;
* ``forward`` / ``inverse`` run on device buffers (``DeviceBuffer``) on a
  stream and are the form the batched workloads use;
* construction errors raise ``NttError`` (NoPrimitiveRoot / DegreeTooLarge /
  ...), the counterpart of ``NttError`` (primus_ntt/src/error.rs:7-35).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import DeviceBuffer, PrimusGpuError, call, ptr


class NttError(PrimusGpuError):
    pass


def _sh(stream):
    return None if stream is None else stream.h


def ntt_primes(bound: int, m: int, count: int) -> list[int]:
    """`count` descending primes below `bound`, each congruent to 1 mod m."""
    out = np.zeros(count, dtype=np.uint64)
    call("pg_ntt_primes", bound, m, count, ptr(out))
    return [int(v) for v in out]


def prev_prime_congruent(bound: int, m: int) -> int:
    return int(nat.lib().pg_prev_prime_congruent(bound, m))


def minimal_primitive_root(log_degree: int, q: int) -> int:
    r = C.c_uint64()
    call("pg_minimal_primitive_root", log_degree, q, C.byref(r))
    return r.value


def host_tables(log_n: int, q: int) -> dict:
    """The product's table construction run on the host only (no device)."""
    n = 1 << log_n
    vals = [C.c_uint64() for _ in range(3)]
    arrs = [np.zeros(n, np.uint64) for _ in range(4)]
    st = nat.lib().pg_ntt_host_tables(log_n, q, *[C.byref(v) for v in vals], *[ptr(a) for a in arrs])
    if st != nat.PG_OK:
        raise NttError(st, "pg_ntt_host_tables", nat.lib().pg_last_error().decode())
    d = {"root": vals[0].value, "inv_root": vals[1].value, "inv_n": vals[2].value}
    for k, a in zip(["root_powers", "root_powers_q", "inv_root_powers", "inv_root_powers_q"], arrs):
        d[k] = a
    return d


class NttTuning(C.Structure):
    _fields_ = [("variant", C.c_int32 * 3), ("us", C.c_float * 3), ("default_us", C.c_float * 3),
                ("rows", C.c_uint64)]


def variant_count(log_n: int) -> int:
    """Kernel shapes available for degree 2^log_n (0 is the default)."""
    return int(nat.lib().pg_ntt_variant_count(log_n))


def variant_name(log_n: int, variant: int) -> str:
    r = nat.lib().pg_ntt_variant_name(log_n, variant)
    return r.decode() if r else ""


class Calibration(C.Structure):
    _fields_ = [("hbm_copy_gbs", C.c_double), ("int_butterflies_gps", C.c_double),
                ("fp64_butterflies_gps", C.c_double)]


def calibrate() -> dict:
    """Built-in ceilings on the current device (pg_calibrate): streaming-copy GB/s and the
    register-only forward-butterfly rate (G/s) on the integer and the FP64 schedule."""
    c = Calibration()
    call("pg_calibrate", C.byref(c))
    return {"hbm_copy_gbs": c.hbm_copy_gbs, "int_butterflies_gps": c.int_butterflies_gps,
            "fp64_butterflies_gps": c.fp64_butterflies_gps}


class DcrtTable:
    """Device-resident NTT tables for L primes of degree N = 2^log_n
    (UintCrtNttTable, primus_ntt/src/dcrt/primitive.rs)."""

    def __init__(self, log_n: int, moduli):
        self.moduli = [int(q) for q in moduli]
        m = np.asarray(self.moduli, dtype=np.uint64)
        h = C.c_void_p()
        st = nat.lib().pg_ntt_table_create(log_n, ptr(m), len(self.moduli), C.byref(h))
        if st != nat.PG_OK:
            raise NttError(st, "pg_ntt_table_create", nat.lib().pg_last_error().decode())
        self.h = h.value
        self.log_n = log_n
        self.n = 1 << log_n
        self.L = len(self.moduli)

    @classmethod
    def new(cls, log_n: int, moduli):
        return cls(log_n, moduli)

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_ntt_table_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- trait accessors
    def ntt_tables(self) -> list:
        """DcrtTable::ntt_tables: one single-prime table per limb, sharing this table's
        device arrays (pg_ntt_table_view); they must not outlive this table."""
        out = []
        for l in range(len(self.moduli)):
            h = C.c_void_p()
            call("pg_ntt_table_view", self.h, l, 1, C.byref(h))
            out.append(_TableView(h.value, self, self.log_n, [self.moduli[l]]))
        return out

    def iter(self):
        """DcrtTable::iter: the per-prime tables in limb order."""
        return iter(self.ntt_tables())

    def poly_length(self) -> int:
        return self.n

    def moduli_count(self) -> int:
        return self.L

    def crt_poly_length(self) -> int:
        return self.n * self.L

    def export(self, limb: int = 0) -> dict:
        n = self.n
        vals = [C.c_uint64() for _ in range(3)]
        arrs = [np.zeros(n, np.uint64) for _ in range(4)]
        call("pg_ntt_table_export", self.h, limb, *[C.byref(v) for v in vals], *[ptr(a) for a in arrs])
        d = {"root": vals[0].value, "inv_root": vals[1].value, "inv_n": vals[2].value}
        for k, a in zip(["root_powers", "root_powers_q", "inv_root_powers", "inv_root_powers_q"], arrs):
            d[k] = a
        return d

    # ---- host-slice transforms (in place), reference call semantics
    def _host(self, fn: str, a: np.ndarray, lazy: bool):
        if not (isinstance(a, np.ndarray) and a.dtype == np.uint64 and a.flags.c_contiguous):
            raise TypeError("expected a C-contiguous uint64 numpy array")
        per = self.n * self.L
        if a.size % per:
            raise ValueError(f"slice length {a.size} is not a multiple of crt_poly_length {per}")
        call(fn, self.h, ptr(a), a.size // per, int(bool(lazy)))

    def lazy_transform_slice(self, a: np.ndarray):
        self._host("pg_ntt_forward_host", a, True)

    def transform_slice(self, a: np.ndarray):
        self._host("pg_ntt_forward_host", a, False)

    def lazy_inverse_transform_slice(self, a: np.ndarray):
        self._host("pg_ntt_inverse_host", a, True)

    def inverse_transform_slice(self, a: np.ndarray):
        self._host("pg_ntt_inverse_host", a, False)

    def transform_inplace(self, poly: np.ndarray) -> np.ndarray:
        self.transform_slice(poly)
        return poly

    def inverse_transform_inplace(self, values: np.ndarray) -> np.ndarray:
        self.inverse_transform_slice(values)
        return values

    def _mono(self, fn: str, values: np.ndarray, *args):
        buf = DeviceBuffer(self.n * self.L)
        call(fn, self.h, *args, buf.ptr, None)
        values[...] = buf.numpy().reshape(values.shape)

    def transform_monomial(self, coeff: int, degree: int, values: np.ndarray):
        self._mono("pg_ntt_monomial", values, coeff, degree)

    def transform_coeff_one_monomial(self, degree: int, values: np.ndarray):
        self._mono("pg_ntt_coeff_one_monomial", values, degree)

    def transform_coeff_minus_one_monomial(self, degree: int, values: np.ndarray):
        self._mono("pg_ntt_coeff_minus_one_monomial", values, degree)

    # ---- device forms
    def forward(self, buf: DeviceBuffer, polys: int, lazy: bool = False, stream=None):
        call("pg_ntt_forward", self.h, buf.ptr, polys, int(bool(lazy)), _sh(stream))

    def inverse(self, buf: DeviceBuffer, polys: int, lazy: bool = False, stream=None):
        call("pg_ntt_inverse", self.h, buf.ptr, polys, int(bool(lazy)), _sh(stream))

    def polymul_ntt_plain(self, buf: DeviceBuffer, plain: DeviceBuffer, plain_q: DeviceBuffer, polys: int,
                          stream=None):
        """fwd -> x plain (NTT domain, Shoup-prepared) -> inv, one launch."""
        call("pg_dcrt_polymul_ntt_plain", self.h, buf.ptr, plain.ptr, plain_q.ptr, polys, _sh(stream))

    def fill_uniform(self, buf: DeviceBuffer, polys: int, seed: int, stream0: int = 0, stream=None):
        call("pg_fill_uniform", self.h, buf.ptr, polys, seed, stream0, _sh(stream))

    # ---- kernel shapes (autotuner)
    def autotune(self, polys: int) -> dict:
        """Time every kernel shape of this degree on `polys` seeded polys and keep
        the fastest per mode in the table (pg_ntt_autotune)."""
        r = NttTuning()
        call("pg_ntt_autotune", self.h, polys, C.byref(r))
        names = ["forward", "inverse", "round_trip"]
        return {n: {"variant": r.variant[i], "name": variant_name(self.log_n, r.variant[i]), "us": r.us[i],
                    "default_us": r.default_us[i]}
                for i, n in enumerate(names)} | {"rows": r.rows}

    def set_variant(self, mode: int, variant: int):
        """Force kernel shape `variant` for mode 0 (canonical forward), 1 (inverse) or 2 (round trip)."""
        call("pg_ntt_set_variant", self.h, mode, variant)

    def set_fp64(self, enable: bool):
        """Switch the FP64 butterfly schedule on or off (pg_ntt_set_fp64); off keeps every
        transform on the integer pipe.  Same results either way."""
        call("pg_ntt_set_fp64", self.h, int(bool(enable)))

    @property
    def fp64(self) -> bool:
        return bool(nat.lib().pg_ntt_fp64_enabled(self.h))

    # ---- pointwise (device)
    def mul(self, x, y, polys, rhs_polys=None, stream=None):
        call("pg_dcrt_mul", self.h, x.ptr, y.ptr, polys, polys if rhs_polys is None else rhs_polys, _sh(stream))

    def add_mul(self, x, y, z, polys, rhs_polys=None, stream=None):
        call("pg_dcrt_add_mul", self.h, x.ptr, y.ptr, z.ptr, polys, polys if rhs_polys is None else rhs_polys,
             _sh(stream))

    def add(self, x, y, polys, rhs_polys=None, stream=None):
        call("pg_dcrt_add", self.h, x.ptr, y.ptr, polys, polys if rhs_polys is None else rhs_polys, _sh(stream))

    def sub(self, x, y, polys, rhs_polys=None, stream=None):
        call("pg_dcrt_sub", self.h, x.ptr, y.ptr, polys, polys if rhs_polys is None else rhs_polys, _sh(stream))

    def neg(self, x, polys, stream=None):
        call("pg_dcrt_neg", self.h, x.ptr, polys, _sh(stream))

    def mul_scalar(self, x, scalars, polys, stream=None):
        s = np.asarray(scalars, dtype=np.uint64)
        call("pg_dcrt_mul_scalar", self.h, x.ptr, ptr(s), polys, _sh(stream))

    def add_mul_scalar(self, x, y, scalars, polys, stream=None):
        s = np.asarray(scalars, dtype=np.uint64)
        call("pg_dcrt_add_mul_scalar", self.h, x.ptr, y.ptr, ptr(s), polys, _sh(stream))

    def shoup_prepare(self, values, quotients, polys, stream=None):
        call("pg_dcrt_shoup_prepare", self.h, values.ptr, quotients.ptr, polys, _sh(stream))

    def mul_prepared(self, x, w, wq, polys, rhs_polys=None, stream=None):
        call("pg_dcrt_mul_prepared", self.h, x.ptr, w.ptr, wq.ptr, polys, polys if rhs_polys is None else rhs_polys,
             _sh(stream))

    def butterfly_mul_factor(self, a, s, w, wq, b, polys, stream=None):
        call("pg_dcrt_butterfly_mul_factor", self.h, a.ptr, s.ptr, w.ptr, wq.ptr, b.ptr, polys, _sh(stream))


class _TableView(DcrtTable):
    """A table over some limbs of another table (pg_ntt_table_view): the same
    methods, the parent's device arrays; keeps its parent alive."""

    def __init__(self, h, parent, log_n, moduli):
        self.h, self.parent, self.log_n, self.moduli = h, parent, log_n, list(moduli)
        self.n = 1 << log_n
        self.L = len(self.moduli)


class NttTable(DcrtTable):
    """Single-prime table (UintNttTable, primus_ntt/src/ntt/primitive.rs)."""

    def __init__(self, log_n: int, modulus: int):
        super().__init__(log_n, [modulus])
        self.modulus = int(modulus)

    @classmethod
    def new(cls, log_n: int, modulus: int):
        return cls(log_n, modulus)


class PolymulJob(C.Structure):
    _fields_ = [("d_a", C.c_void_p), ("d_b", C.c_void_p), ("log_n", C.c_uint32), ("moduli_count", C.c_uint32)]


class PolymulBatch:
    """Uneven batches of products a <- a*b over several ring degrees in one
    (graph-captured) submission; one table per degree (pg_polymul_batch_*)."""

    def __init__(self, tables):
        self.tables = list(tables)
        arr = (C.c_void_p * len(self.tables))(*[t.h for t in self.tables])
        h = C.c_void_p()
        call("pg_polymul_batch_create", arr, len(self.tables), C.byref(h))
        self.h = h.value

    @staticmethod
    def prepare(jobs):
        """The C job array for `jobs` ((a, b, log_n, moduli_count) tuples), built once:
        a caller that resubmits the same job set passes it to run() and skips the
        per-call Python conversion (what a C or Rust caller holds anyway)."""
        return (PolymulJob * len(jobs))(*[PolymulJob(a.ptr, b.ptr, ln, L) for a, b, ln, L in jobs])

    def run(self, jobs, use_graph=True, stream=None):
        """jobs: iterable of (a: DeviceBuffer, b: DeviceBuffer, log_n, moduli_count), or
        the array prepare() returned."""
        arr = jobs if isinstance(jobs, C.Array) else self.prepare(jobs)
        call("pg_polymul_batch_run", self.h, arr, len(arr), int(bool(use_graph)), _sh(stream))

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_polymul_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
