"""The allocation-free external product, pg_ext_product_noalloc.

It serves callers that cannot allocate device memory when they call: hosts
that only hold device pointers owned by another runtime, and serving processes
that reserve their HBM at start-up and forbid allocations afterwards (cudaMalloc
and cudaFree synchronise the device and can fail under memory pressure).
Shapes the fused external-product kernel takes need no scratch; every other
shape keeps its scratch in a fixed 32 MiB array inside the library, shared by
every call.

Each test calls it through the C ABI twice in a row on different inputs and
checks every output against the oracle (CrtGlwe::mul_dcrt_ggsw_inplace,
primus_lattice/src/glwe/crt.rs:202-229) and against the allocating entry point,
pg_ext_product, on the same inputs.  The tolerance is zero: both return
canonical residues.  The file sorts last so that a run stopping at the first
failure has run every other test before it; it also passes alone in a fresh
process.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

# the fixed scratch array inside the library
SCRATCH_BYTES = 32 << 20


def _lattice(log_n, moduli, lb):
    rbase = O.RnsBase(moduli)
    return O.Lattice(O.DcrtTable(log_n, moduli), rbase, O.GadgetBasis(rbase, lb))


def _run_twice(gpu, log_n, moduli, lb, k, batch):
    from primus_b200 import _native as nat
    n = 1 << log_n
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    lat = _lattice(log_n, moduli, lb)
    ggsw = np.concatenate([O.uniform_rns(0xA11, 31 * i, moduli, n).ravel() for i in range((k + 1) * g.d * (k + 1))])
    dk = gpu.DeviceBuffer.from_numpy(ggsw)
    per = (k + 1) * len(moduli) * n
    for call_no, seed in enumerate((0xB0B, 0xC0C)):
        glwe = np.concatenate([O.uniform_rns(seed, 10 * b + i, moduli, n).ravel()
                               for b in range(batch) for i in range(k + 1)])
        exp = lat.external_product(k, glwe, ggsw, batch=batch, threads=8)
        din = gpu.DeviceBuffer.from_numpy(glwe)
        want = gpu.DeviceBuffer(batch * per)
        gpu.external_product(table, g, k, din, dk, want, batch)
        got = gpu.DeviceBuffer(batch * per)
        got.upload(np.full(batch * per, 0xFFFF, np.uint64))  # stale contents must be overwritten
        nat.call("pg_ext_product_noalloc", table.h, g.h, k, din.ptr, dk.ptr, got.ptr, batch, None)
        nat.call("pg_stream_synchronize", None)
        out = got.numpy()
        assert np.array_equal(out, exp), f"call {call_no + 1} differs from the oracle"
        assert np.array_equal(out, want.numpy()), f"call {call_no + 1} differs from pg_ext_product"


def test_no_alloc_pipeline_shape_matches_oracle(gpu):
    # the external product's benchmark shape (N = 2048, largest q < 2^54 with
    # q = 1 mod 4096, log_basis 7 -> 7 digits, k = 1) at a batch below the fused
    # kernel's minimum: the pipeline, with its scratch in the fixed array
    q = O.ntt_primes(1 << 54, 1 << 12, 1)[0]
    _run_twice(gpu, 11, [q], 7, 1, 16)


def test_no_alloc_two_primes_k2_matches_oracle(gpu):
    # two primes and k = 2: always the pipeline (compose over two limbs)
    moduli = O.ntt_primes(1 << 50, 1 << 11, 2)
    _run_twice(gpu, 10, moduli, 20, 2, 5)


def test_no_alloc_fused_shape_beyond_the_array(gpu):
    # the benchmark shape at 256 ciphertexts: the pipeline would need 64 MiB of
    # scratch (twice the array); the fused kernel needs none
    q = O.ntt_primes(1 << 54, 1 << 12, 1)[0]
    _run_twice(gpu, 11, [q], 7, 1, 256)


def test_no_alloc_rejects_batches_above_its_scratch(gpu):
    from primus_b200 import _native as nat
    log_n, k, lb = 10, 2, 20
    moduli = O.ntt_primes(1 << 50, 1 << 11, 2)
    table = gpu.DcrtTable(log_n, moduli)
    g = gpu.GadgetBasis(gpu.RnsBase(moduli), lb)
    lib = nat.lib()
    # scratch per call: one ws_bytes of (batch * (k + 1)) polys
    per = lib.pg_ext_product_workspace_size(table.h, g.h, k, 1)
    max_batch = (SCRATCH_BYTES - 256) // (per - 256)
    assert lib.pg_ext_product_workspace_size(table.h, g.h, k, max_batch) <= SCRATCH_BYTES
    assert lib.pg_ext_product_workspace_size(table.h, g.h, k, max_batch + 1) > SCRATCH_BYTES
    # NULL buffers: the size check comes first, so a regression of it shows as a
    # host-side PG_ERR_INVALID_ARGUMENT, never as a launch
    for batch in (max_batch + 1, 1 << 20, 1 << 62, (1 << 64) - 1):
        st = lib.pg_ext_product_noalloc(table.h, g.h, k, None, None, None, batch, None)
        assert st == nat.PG_ERR_UNSUPPORTED, batch
        msg = lib.pg_last_error().decode()
        assert "scratch" in msg and f"at most {max_batch} " in msg, msg
    # sizes that do not fit size_t saturate instead of wrapping to a small size
    assert lib.pg_ext_product_workspace_size(table.h, g.h, k, 1 << 62) == (1 << 64) - 1
    assert lib.pg_key_switch_workspace_size(table.h, g.h, k, k, 1 << 62) == (1 << 64) - 1
