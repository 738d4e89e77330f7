"""Parity at the workloads' own shapes.

* The uneven batch: the benchmark's 512 products (N uniform in 2^10..2^16, L
  uniform in 1..32, 32-prime tables per degree, primes below 2^50 with
  q = 1 mod 2N) in one graph-replayed submission; every job's a <- a * b and
  b <- NTT(b) equal the oracle (UintCrtNttTable transforms and the pointwise
  product, primus_ntt/src/dcrt/primitive.rs:117-123, primus_poly/src/dcrt/mul.rs:27-60).
* The served mixed stream at the served shapes: RNS products N = 2^12..2^16
  with L = 4..24, the N = 2048 external product (q < 2^54, B = 2^7, k = 1) and
  the hybrid key switch (N = 2^15, L = 16, K = 4, 4-limb groups) submitted as
  one stream; every served result equals the same request run alone through the
  plain API, and equals the oracle (every product and external product, and
  three key switches).
"""
import hashlib
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _threads():
    return max(1, len(os.sched_getaffinity(0)))


def _oracle_polymul(sub, a, b, moduli):
    t = _threads()
    fa = sub.forward(a.copy(), threads=t).reshape(a.shape)
    fb = sub.forward(b.copy(), threads=t).reshape(b.shape)
    prod = np.stack([O.mul(fa[l], fb[l], q) for l, q in enumerate(moduli)])
    return sub.inverse(prod, threads=t).reshape(a.shape), fb


def test_uneven_batch_512_jobs(gpu):
    # the benchmark's job set (same generator and seed as bench.py's uneven batch)
    rng = np.random.default_rng(0x5EED0002)
    log_ns = list(range(10, 17))
    shape = [(int(rng.choice(log_ns)), int(rng.integers(1, 33))) for _ in range(512)]
    assert {ln for ln, _ in shape} == set(log_ns) and max(L for _, L in shape) == 32
    primes = {ln: O.ntt_primes(1 << 50, 2 << ln, 32) for ln in log_ns}
    tables = {ln: gpu.DcrtTable(ln, primes[ln]) for ln in log_ns}
    batch = gpu.PolymulBatch(list(tables.values()))

    def inputs(j):  # regenerated on demand: the whole set is 2.5 GB
        ln, L = shape[j]
        return (O.uniform_rns(0x5EED0003, 64 * j, primes[ln][:L], 1 << ln),
                O.uniform_rns(0x5EED0004, 64 * j, primes[ln][:L], 1 << ln))

    bufs = []
    for j, (ln, L) in enumerate(shape):
        a, b = inputs(j)
        bufs.append((gpu.DeviceBuffer.from_numpy(a), gpu.DeviceBuffer.from_numpy(b), ln, L))
    jobs = batch.prepare(bufs)
    batch.run(jobs, use_graph=True)
    gpu.synchronize()
    digest = []
    refs = {}
    for j, (da, db, ln, L) in enumerate(bufs):
        a, b = inputs(j)
        if (ln, L) not in refs:
            refs[(ln, L)] = O.DcrtTable(ln, primes[ln][:L])
        exp_a, exp_b = _oracle_polymul(refs[(ln, L)], a, b, primes[ln][:L])
        got = da.numpy(a.shape)
        assert np.array_equal(got, exp_a), (j, ln, L)
        assert np.array_equal(db.numpy(b.shape), exp_b), (j, ln, L)
        digest.append(hashlib.sha256(got.tobytes()).digest())
    # the captured graph replayed on the same inputs, uploaded again
    for j, (da, db, _, _) in enumerate(bufs):
        a, b = inputs(j)
        da.upload(a)
        db.upload(b)
    batch.run(jobs, use_graph=True)
    gpu.synchronize()
    for j, (da, _, _, _) in enumerate(bufs):
        assert hashlib.sha256(da.numpy().tobytes()).digest() == digest[j], j


def test_served_mix_at_served_shapes(gpu):
    P = gpu
    # RNS products: tables of 24 primes for N = 2^12 .. 2^16
    pm_lns = list(range(12, 17))
    pm_primes = {ln: O.ntt_primes(1 << 50, 2 << ln, 24) for ln in pm_lns}
    pm_tables = {ln: P.DcrtTable(ln, pm_primes[ln]) for ln in pm_lns}
    # external product: N = 2048, q = largest prime < 2^54 with q = 1 mod 4096, B = 2^7, k = 1
    xq = O.ntt_primes(1 << 54, 1 << 12, 1)[0]
    xt, xg = P.DcrtTable(11, [xq]), P.GadgetBasis(P.RnsBase([xq]), 7)
    xkey = np.concatenate([O.uniform_rns(0x5E, 11 * i, [xq], 2048).ravel() for i in range(2 * xg.d * 2)])
    dxkey = P.DeviceBuffer.from_numpy(xkey)
    xrb = O.RnsBase([xq])
    xlat = O.Lattice(O.DcrtTable(11, [xq]), xrb, O.GadgetBasis(xrb, 7))
    # hybrid key switch: N = 2^15, L = 16 + K = 4 special primes, 4-limb digit groups, k = 1
    ks_moduli = O.ntt_primes(1 << 50, 1 << 16, 20)
    kt = P.DcrtTable(15, ks_moduli)
    hks = P.HybridKeySwitch(kt, 16, 4, 4)
    kref = O.HybridKeySwitch(15, ks_moduli, 16, 4, 4)
    kkey = np.concatenate([O.uniform_rns(0x6E, 50 * r, ks_moduli, 1 << 15).ravel() for r in range(hks.dnum * 2)])
    dkkey = P.DeviceBuffer.from_numpy(kkey)

    srv = P.Server(memory_budget_bytes=4 << 30, slots=4, max_batch=64, polymul_tables=list(pm_tables.values()))
    xid = srv.register_key(2, xt, xg, 1, 1, dxkey)
    kid = srv.register_hybrid_key(hks, 1, 1, dkkey)
    rng = np.random.default_rng(0x5EED0005)
    kinds = rng.choice(3, size=60, p=[0.5, 0.3, 0.2])
    kinds[:3] = [0, 1, 2]  # at least one of each kind
    items, served, tickets = [], [], []
    for i, kd in enumerate(kinds):
        if kd == 0:
            ln, L = int(rng.choice(pm_lns)), int(rng.integers(4, 25))
            if i == 0:
                ln, L = 16, 24  # the largest product of the stream
            a = O.uniform_rns(0x70 + i, 0, pm_primes[ln][:L], 1 << ln)
            b = O.uniform_rns(0x170 + i, 0, pm_primes[ln][:L], 1 << ln)
            da, db = P.DeviceBuffer.from_numpy(a), P.DeviceBuffer.from_numpy(b)
            items.append(("pm", ln, L, a, b))
            served.append((da, db))
            tickets.append(srv.submit(P.polymul_request(da, db, ln, L)))
        elif kd == 1:
            x = O.uniform_rns(0x270 + i, 0, [xq], 2 * 2048)
            di, do = P.DeviceBuffer.from_numpy(x), P.DeviceBuffer(x.size)
            items.append(("xp", x))
            served.append((di, do))
            tickets.append(srv.submit(P.ext_product_request(xid, di, do)))
        else:
            x = np.concatenate([O.uniform_rns(0x370 + i, 20 * c, ks_moduli[:16], 1 << 15).ravel() for c in range(2)])
            di, do = P.DeviceBuffer.from_numpy(x), P.DeviceBuffer(x.size)
            items.append(("ks", x))
            served.append((di, do))
            tickets.append(srv.submit(P.key_switch_request(kid, di, do)))
    for t in tickets:
        srv.wait(t, timeout_us=60_000_000)
    stats = srv.stats()
    assert stats["completed"] == len(items) and stats["rejected"] == 0
    ks_checked = 0
    for it, bufs in zip(items, served):
        if it[0] == "pm":
            _, ln, L, a, b = it
            got = bufs[0].numpy(a.shape)
            # alone: the plain per-call API on the same inputs
            sub = P.DcrtTable(ln, pm_primes[ln][:L])
            da, db = P.DeviceBuffer.from_numpy(a), P.DeviceBuffer.from_numpy(b)
            P.PolymulBatch([sub]).run([(da, db, ln, L)], use_graph=False)
            P.synchronize()
            assert np.array_equal(got, da.numpy(a.shape)), (ln, L)
            exp, _ = _oracle_polymul(O.DcrtTable(ln, pm_primes[ln][:L]), a, b, pm_primes[ln][:L])
            assert np.array_equal(got, exp), (ln, L)
        elif it[0] == "xp":
            got = bufs[1].numpy()
            alone = P.DeviceBuffer(it[1].size)
            P.external_product(xt, xg, 1, P.DeviceBuffer.from_numpy(it[1]), dxkey, alone, 1)
            assert np.array_equal(got, alone.numpy())
            assert np.array_equal(got, xlat.external_product(1, it[1], xkey).ravel())
        else:
            got = bufs[1].numpy()
            alone = P.DeviceBuffer(it[1].size)
            hks.key_switch(1, 1, dkkey, P.DeviceBuffer.from_numpy(it[1]), alone, 1)
            assert np.array_equal(got, alone.numpy())
            if ks_checked < 3:
                assert np.array_equal(got, np.asarray(kref.key_switch(1, 1, kkey, it[1])).ravel())
                ks_checked += 1
    assert ks_checked >= 1
    srv.close()
