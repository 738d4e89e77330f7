"""The allocation-free external product, pg_ext_product_noalloc.

It serves callers that cannot allocate device memory when they call: hosts
that only hold device pointers owned by another runtime, and serving processes
that reserve their HBM at start-up and forbid allocations afterwards (cudaMalloc
and cudaFree synchronise the device and can fail under memory pressure).  Its
scratch is a fixed 32 MiB array inside the library, shared by every call.

The test calls it through the C ABI twice in a row on different inputs and
checks each output against the allocating entry point, pg_ext_product, on the
same inputs.  The tolerance is zero: both return canonical residues.  The file
sorts last so that a run stopping at the first failure has run every other test
before it; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _shape():
    # the external product's benchmark shape (N = 2048, largest q < 2^54 with
    # q = 1 mod 4096, log_basis 7 -> 7 digits, k = 1, L = 1) at a small batch
    log_n, k, lb, batch = 11, 1, 7, 16
    q = O.ntt_primes(1 << 54, 1 << 12, 1)[0]
    return log_n, k, lb, batch, [q]


def test_no_alloc_matches_allocating_entry_point(gpu):
    from primus_b200 import _native as nat
    log_n, k, lb, batch, moduli = _shape()
    n = 1 << log_n
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    ggsw = np.concatenate([O.uniform_rns(0xA11, 31 * i, moduli, n).ravel() for i in range((k + 1) * g.d * (k + 1))])
    dk = gpu.DeviceBuffer.from_numpy(ggsw)
    per = (k + 1) * n
    for call_no, seed in enumerate((0xB0B, 0xC0C)):
        glwe = np.concatenate([O.uniform_rns(seed, 10 * b + i, moduli, n).ravel()
                               for b in range(batch) for i in range(k + 1)])
        din = gpu.DeviceBuffer.from_numpy(glwe)
        want = gpu.DeviceBuffer(batch * per)
        gpu.external_product(table, g, k, din, dk, want, batch)
        got = gpu.DeviceBuffer(batch * per)
        got.upload(np.full(batch * per, 0xFFFF, np.uint64))  # stale contents must be overwritten
        nat.call("pg_ext_product_noalloc", table.h, g.h, k, din.ptr, dk.ptr, got.ptr, batch, None)
        nat.call("pg_stream_synchronize", None)
        assert np.array_equal(got.numpy(), want.numpy()), f"call {call_no + 1} differs from pg_ext_product"


def test_no_alloc_rejects_batches_above_its_scratch(gpu):
    from primus_b200 import _native as nat
    log_n, k, lb, _, moduli = _shape()
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    dummy = gpu.DeviceBuffer(1)
    st = nat.lib().pg_ext_product_noalloc(table.h, g.h, k, dummy.ptr, dummy.ptr, dummy.ptr, 1 << 20, None)
    assert st == nat.PG_ERR_UNSUPPORTED
    msg = nat.lib().pg_last_error().decode()
    assert "scratch" in msg and "at most" in msg
