"""Uneven batches (ragged ring degrees and limb counts in one submission,
descriptor-driven launches, CUDA-graph replay) against the oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def make_jobs(seed, count, log_ns, max_L, rng):
    jobs = []
    for j in range(count):
        ln = int(rng.choice(log_ns))
        L = int(rng.integers(1, max_L + 1))
        jobs.append((ln, L))
    return jobs


def run_case(gpu, log_ns, max_L, count, seed, graph_reps=3, bound=1 << 50):
    rng = np.random.default_rng(seed)
    primes = {ln: O.ntt_primes(bound, 2 << ln, max_L) for ln in log_ns}
    tables = {ln: gpu.DcrtTable(ln, primes[ln]) for ln in log_ns}
    refs = {ln: O.DcrtTable(ln, primes[ln]) for ln in log_ns}
    batch = gpu.PolymulBatch(list(tables.values()))
    shape = make_jobs(seed, count, log_ns, max_L, rng)
    for rep in range(graph_reps):
        host, bufs = [], []
        for j, (ln, L) in enumerate(shape):
            n = 1 << ln
            a = O.uniform_rns(seed * 1000 + rep, 64 * j, primes[ln][:L], n)
            b = O.uniform_rns(seed * 1000 + rep, 64 * j + 32, primes[ln][:L], n)
            host.append((a, b))
            bufs.append((gpu.DeviceBuffer.from_numpy(a), gpu.DeviceBuffer.from_numpy(b), ln, L))
        batch.run(bufs, use_graph=True)
        gpu.synchronize()
        for (a, b), (da, db, ln, L) in zip(host, bufs):
            sub = O.DcrtTable(ln, primes[ln][:L])
            exp = sub.inverse(_mul(sub, a, b, primes[ln][:L])).reshape(a.shape)
            assert np.array_equal(da.numpy(a.shape), exp), (rep, ln, L)
            assert np.array_equal(db.numpy(b.shape), sub.forward(b).reshape(b.shape)), (rep, ln, L)


def _mul(sub, a, b, moduli):
    fa, fb = sub.forward(a).reshape(a.shape), sub.forward(b).reshape(b.shape)
    return np.stack([O.mul(fa[l], fb[l], q) for l, q in enumerate(moduli)])


def test_uneven_small(gpu):
    run_case(gpu, [4, 7, 10, 11], 5, 24, seed=1)


def test_uneven_cluster_sizes(gpu):
    run_case(gpu, [10, 13, 14, 15, 16], 4, 12, seed=2, graph_reps=2)


def test_uneven_tiny_degrees(gpu):
    # N <= 2^12 with moduli below 2^50: one launch per degree (the pair form), several rows per CTA
    run_case(gpu, [1, 2, 3, 5, 6, 8, 9, 12], 3, 24, seed=3, graph_reps=2)


def test_uneven_wide_moduli(gpu):
    # moduli above 2^50 (no FP64 schedule): the forward and the fused inverse launches
    run_case(gpu, [3, 10, 12, 14], 3, 12, seed=4, graph_reps=2, bound=1 << 62)


def test_single_job_plain_form(gpu):
    # one job per call without a graph: the per-call drop-in form
    ln, L = 12, 3
    primes = O.ntt_primes(1 << 50, 2 << ln, L)
    t = gpu.DcrtTable(ln, primes)
    batch = gpu.PolymulBatch([t])
    a = O.uniform_rns(9, 0, primes, 1 << ln)
    b = O.uniform_rns(9, 7, primes, 1 << ln)
    da, db = gpu.DeviceBuffer.from_numpy(a), gpu.DeviceBuffer.from_numpy(b)
    batch.run([(da, db, ln, L)], use_graph=False)
    gpu.synchronize()
    sub = O.DcrtTable(ln, primes)
    assert np.array_equal(da.numpy(a.shape), sub.inverse(_mul(sub, a, b, primes)).reshape(a.shape))
    for row in range(L):
        assert np.array_equal(da.numpy(a.shape)[row], O.naive_negacyclic(a[row], b[row], primes[row]))


def test_rejects_bad_jobs(gpu):
    primes = O.ntt_primes(1 << 50, 2 << 10, 2)
    batch = gpu.PolymulBatch([gpu.DcrtTable(10, primes)])
    d = gpu.DeviceBuffer(4096)
    with pytest.raises(gpu.PrimusGpuError):
        batch.run([(d, d, 11, 1)])   # no table for N = 2^11
    with pytest.raises(gpu.PrimusGpuError):
        batch.run([(d, d, 10, 3)])   # more limbs than the table
    with pytest.raises(gpu.PrimusGpuError):
        batch.run([(d, d, 10, 1)])   # a and b are the same row (both are transformed in place)

    class View:  # a device pointer into d
        def __init__(self, off):
            self.ptr = d.ptr + 8 * off
    with pytest.raises(gpu.PrimusGpuError):
        batch.run([(View(0), View(1000), 10, 2)])  # b starts inside a's two rows
