"""CPU checks of the product library: it loads, exports every symbol that
include/primus_gpu.h declares, and its host-side setup (prime search, minimal
root, twiddle tables, error reporting) equals the oracle's.  No device calls."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import primus_b200 as P
from primus_b200 import _native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
            syms |= set(re.findall(r"\b(pg_\w+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) > 40
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (pg_\w+)", out))
    missing = syms - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for s in syms:
        assert hasattr(nat.lib(), s)


def test_rust_bindings_declare_every_symbol():
    """rust/primus_gpu/src/ffi.rs (the drop-in crate's bindings) declares exactly
    the entry points of the header, with the same parameter counts."""
    text = open(os.path.join(ROOT, "include", "primus_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    want = {m.group(1): (0 if m.group(2).strip() in ("", "void") else m.group(2).count(",") + 1)
            for m in re.finditer(r"\b(pg_\w+)\s*\(([^)]*)\)\s*;", text)}
    rs = open(os.path.join(ROOT, "rust", "primus_gpu", "src", "ffi.rs")).read()
    got = {m.group(1): (0 if not m.group(2).strip() else m.group(2).count(",") + 1)
           for m in re.finditer(r"pub fn (pg_\w+)\(([^)]*)\)", rs)}
    assert got == want


def test_status_strings():
    assert nat.lib().pg_status_string(0) == b"ok"
    assert nat.lib().pg_status_string(2) == b"no primitive root"
    assert nat.lib().pg_version().startswith(b"primus_b200")


@pytest.mark.parametrize("bound,m,count", [(1 << 50, 2048, 1), (1 << 54, 4096, 1), (1 << 50, 1 << 17, 24),
                                           (1 << 50, 1 << 11, 8), (1 << 40, 1 << 5, 5)])
def test_prime_search_equals_oracle(bound, m, count):
    assert P.ntt_primes(bound, m, count) == O.ntt_primes(bound, m, count)


@pytest.mark.parametrize("log_n,q", [(1, 5), (4, 97), (10, 132120577), (11, 536813569), (11, 562949953392641),
                                     (11, 1152921504606830593), (12, 1125899906826241), (16, 1125899906826241)])
def test_host_tables_equal_oracle(log_n, q):
    if (q - 1) % (2 << log_n):
        q = O.ntt_primes(1 << 50, 2 << log_n, 1)[0]
    mine = P.host_tables(log_n, q)
    ref = O.NttTable(log_n, q).export()
    for k in ["root", "inv_root", "inv_n"]:
        assert mine[k] == ref[k], k
    for k in ["root_powers", "root_powers_q", "inv_root_powers", "inv_root_powers_q"]:
        assert np.array_equal(mine[k], ref[k]), k


def test_construction_errors_mirror_ntt_error():
    with pytest.raises(P.NttError) as e:
        P.host_tables(10, 1000003)  # q - 1 not divisible by 2N: NoPrimitiveRoot
    assert e.value.status == nat.PG_ERR_NO_PRIMITIVE_ROOT
    assert "no primitive root" in str(e.value).lower()


def test_degree_too_large():
    # q = 17: 2N = 16 divides q - 1 for N = 8 (ok); N = 16 needs 32 | 16 (no root)
    P.host_tables(3, 17)
    with pytest.raises(P.NttError) as e:
        P.host_tables(4, 17)
    assert e.value.status == nat.PG_ERR_NO_PRIMITIVE_ROOT


def test_host_generator_equals_oracle():
    out = np.zeros(1000, np.uint64)
    nat.call("pg_fill_uniform_host", 0x5EED, 7, 1125899906826241, 1000, nat.ptr(out))
    assert np.array_equal(out, O.uniform(0x5EED, 7, 1125899906826241, 1000))
    nat.call("pg_fill_uniform_host", 1, 2, 12289, 1000, nat.ptr(out))
    assert np.array_equal(out, O.uniform(1, 2, 12289, 1000))


def test_minimal_root_equals_oracle():
    for log_deg, q in [(11, 1125899906826241), (17, 1125899906826241), (12, 18014398509404161)]:
        r = C.c_uint64()
        st = O.lib().orc_minimal_primitive_root(log_deg, q, C.cast(C.pointer(r), O.u64p))
        if st == 0:
            assert P.minimal_primitive_root(log_deg, q) == r.value
