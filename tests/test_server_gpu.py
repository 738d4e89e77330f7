"""The continuous-batching server: every result is the same alone and in the
mix (bit-exact against the plain per-call API and the oracle), admission by
memory budget, refusal of malformed requests, bounded waits, load replay."""
import threading

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(gpu):
    P = gpu
    e = {}
    # polymul tables for three ring degrees, 4 primes each
    e["pm"] = {ln: P.DcrtTable(ln, O.ntt_primes(1 << 50, 2 << ln, 4)) for ln in (10, 12, 14)}
    # external product key: N = 2048, q < 2^54, log_basis 7, k = 1
    q = O.ntt_primes(1 << 54, 1 << 12, 1)[0]
    e["xt"] = P.DcrtTable(11, [q])
    e["xg"] = P.GadgetBasis(P.RnsBase([q]), 7)
    e["xk_host"] = np.concatenate([O.uniform_rns(7, 11 * i, [q], 2048).ravel() for i in range(2 * e["xg"].d * 2)])
    e["xk"] = P.DeviceBuffer.from_numpy(e["xk_host"])
    # key switch key: N = 1024, L = 2, log_basis 20, k_in = k_out = 1
    ks_moduli = O.ntt_primes(1 << 50, 1 << 11, 2)
    e["kt"] = P.DcrtTable(10, ks_moduli)
    e["kg"] = P.GadgetBasis(P.RnsBase(ks_moduli), 20)
    e["kk_host"] = np.concatenate([O.uniform_rns(8, 13 * i, ks_moduli, 1024).ravel() for i in range(e["kg"].d * 2)])
    e["kk"] = P.DeviceBuffer.from_numpy(e["kk_host"])
    return e


def make_server(P, env, budget=256 << 20, slots=3, max_batch=64, max_queue=0):
    srv = P.Server(memory_budget_bytes=budget, slots=slots, max_batch=max_batch, max_queue=max_queue,
                   polymul_tables=list(env["pm"].values()))
    xid = srv.register_key(2, env["xt"], env["xg"], 1, 1, env["xk"])
    kid = srv.register_key(3, env["kt"], env["kg"], 1, 1, env["kk"])
    return srv, xid, kid


def test_mixed_stream_equals_alone(gpu, env):
    P = gpu
    srv, xid, kid = make_server(P, env)
    rng = np.random.default_rng(3)
    items = []
    for i in range(90):
        kind = rng.choice(["pm", "xp", "ks"])
        if kind == "pm":
            ln = int(rng.choice([10, 12, 14]))
            L = int(rng.integers(1, 5))
            t = env["pm"][ln]
            a = O.uniform_rns(100 + i, 0, t.moduli[:L], 1 << ln)
            b = O.uniform_rns(200 + i, 0, t.moduli[:L], 1 << ln)
            items.append(("pm", ln, L, a, b))
        elif kind == "xp":
            x = O.uniform_rns(300 + i, 0, env["xt"].moduli, 2 * 2048)
            items.append(("xp", x))
        else:
            x = O.uniform_rns(400 + i, 0, env["kt"].moduli, 2 * 1024)
            items.append(("ks", x))
    served, tickets = [], []
    for it in items:
        if it[0] == "pm":
            da, db = P.DeviceBuffer.from_numpy(it[3]), P.DeviceBuffer.from_numpy(it[4])
            req = P.polymul_request(da, db, it[1], it[2])
            served.append((da, db))
        elif it[0] == "xp":
            di, do = P.DeviceBuffer.from_numpy(it[1]), P.DeviceBuffer(it[1].size)
            req = P.ext_product_request(xid, di, do)
            served.append((di, do))
        else:
            di, do = P.DeviceBuffer.from_numpy(it[1]), P.DeviceBuffer(it[1].size)
            req = P.key_switch_request(kid, di, do)
            served.append((di, do))
        tickets.append(srv.submit(req))
    for t in tickets:
        srv.wait(t, timeout_us=30_000_000)
    stats = srv.stats()
    assert stats["completed"] == len(items) and stats["rejected"] == 0
    assert stats["batches"] < len(items)  # requests were batched
    # each result equals the same request run alone through the plain API
    for it, bufs in zip(items, served):
        if it[0] == "pm":
            _, ln, L, a, b = it
            sub = P.DcrtTable(ln, env["pm"][ln].moduli[:L])
            batch = P.PolymulBatch([sub])
            da, db = P.DeviceBuffer.from_numpy(a), P.DeviceBuffer.from_numpy(b)
            batch.run([(da, db, ln, L)], use_graph=False)
            P.synchronize()
            assert np.array_equal(bufs[0].numpy(), da.numpy())
            for r in range(L):
                if ln == 10 and r == 0:
                    assert np.array_equal(bufs[0].numpy().reshape(L, -1)[r],
                                          O.naive_negacyclic(a[r], b[r], env["pm"][ln].moduli[r]))
        elif it[0] == "xp":
            alone = P.DeviceBuffer(it[1].size)
            P.external_product(env["xt"], env["xg"], 1, P.DeviceBuffer.from_numpy(it[1]), env["xk"], alone, 1)
            assert np.array_equal(bufs[1].numpy(), alone.numpy())
        else:
            alone = P.DeviceBuffer(it[1].size)
            P.key_switch(env["kt"], env["kg"], 1, 1, env["kk"], P.DeviceBuffer.from_numpy(it[1]), alone, 1)
            assert np.array_equal(bufs[1].numpy(), alone.numpy())
    srv.close()


def test_concurrent_submitters(gpu, env):
    P = gpu
    srv, xid, _ = make_server(P, env)
    x = O.uniform_rns(9, 0, env["xt"].moduli, 2 * 2048)
    want = P.DeviceBuffer(x.size)
    P.external_product(env["xt"], env["xg"], 1, P.DeviceBuffer.from_numpy(x), env["xk"], want, 1)
    want = want.numpy()
    outs, errors = [], []

    def client(n):
        try:
            mine = []
            for _ in range(n):
                di, do = P.DeviceBuffer.from_numpy(x), P.DeviceBuffer(x.size)
                mine.append((srv.submit(P.ext_product_request(xid, di, do)), di, do))
            for t, di, do in mine:
                srv.wait(t, timeout_us=30_000_000)
                outs.append(do.numpy())
        except Exception as ex:  # pragma: no cover - reported below
            errors.append(ex)

    th = [threading.Thread(target=client, args=(25,)) for _ in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
    assert len(outs) == 100 and all(np.array_equal(o, want) for o in outs)
    srv.close()


def test_admission_by_memory_budget(gpu, env):
    P = gpu
    # one slot of 64 KiB cannot hold a single external product's scratch
    srv, xid, kid = make_server(P, env, budget=64 << 10, slots=1)
    d = P.DeviceBuffer(4 * 2048)
    st, _ = srv.try_submit(P.ext_product_request(xid, d, d))
    from primus_b200 import _native as nat
    assert st == nat.PG_ERR_REJECTED
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_malformed_requests_refused(gpu, env):
    P = gpu
    from primus_b200 import _native as nat
    srv, xid, kid = make_server(P, env)
    d = P.DeviceBuffer(8192)
    bad = [P.ext_product_request(99, d, d),                      # unknown key
           P.key_switch_request(xid, d, d),                      # key of another kind
           P.polymul_request(d, d, 11, 1),                       # no table for N = 2^11
           P.polymul_request(d, d, 10, 5),                       # more limbs than the table
           P.polymul_request(d, d, 10, 1)]                       # a and b the same row
    for r in bad:
        st, _ = srv.try_submit(r)
        assert st == nat.PG_ERR_INVALID_ARGUMENT
    r = P.Request(7, 0, None, None, 0, 0, None, None)           # unknown kind
    assert srv.try_submit(r)[0] == nat.PG_ERR_INVALID_ARGUMENT
    with pytest.raises(P.PrimusGpuError):
        srv.wait(123456)                                         # unknown ticket
    srv.close()


def test_queue_limit_rejects(gpu, env):
    P = gpu
    from primus_b200 import _native as nat
    # a one-entry queue behind one slot: a burst is partly refused, never lost
    srv, xid, _ = make_server(P, env, slots=1, max_batch=1, max_queue=1)
    x = P.DeviceBuffer(4 * 2048)
    outs = [P.DeviceBuffer(4 * 2048) for _ in range(200)]
    sts = [srv.try_submit(P.ext_product_request(xid, x, o)) for o in outs]
    accepted = [t for s, t in sts if s == nat.PG_OK]
    rejected = [s for s, _ in sts if s != nat.PG_OK]
    assert all(s == nat.PG_ERR_REJECTED for s in rejected)
    for t in accepted:
        srv.wait(t, timeout_us=30_000_000)
    st = srv.stats()
    assert st["completed"] == len(accepted) and st["rejected"] == len(rejected)
    assert len(rejected) > 0
    srv.close()


def test_replay_reports_latencies(gpu, env):
    P = gpu
    srv, xid, _ = make_server(P, env)
    x = O.uniform_rns(5, 0, env["xt"].moduli, 2 * 2048)
    di = P.DeviceBuffer.from_numpy(x)
    outs = [P.DeviceBuffer(x.size) for _ in range(64)]
    reqs = [P.ext_product_request(xid, di, o) for o in outs]
    arrivals = np.arange(64, dtype=np.float64) * 20.0
    lat = srv.replay(reqs, arrivals)
    assert (lat > 0).all()
    want = P.DeviceBuffer(x.size)
    P.external_product(env["xt"], env["xg"], 1, di, env["xk"], want, 1)
    assert all(np.array_equal(o.numpy(), want.numpy()) for o in outs)
    srv.close()


def test_hybrid_key_requests(gpu, env):
    # hybrid key switch keys in the server: every result equals the plain call
    P = gpu
    log_n, L, K, alpha = 10, 4, 2, 2
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 50, 2 * n, L + K)
    table = P.DcrtTable(log_n, moduli)
    hks = P.HybridKeySwitch(table, L, K, alpha)
    key = np.concatenate([O.uniform_rns(21, 9 * r, moduli, n).ravel() for r in range(hks.dnum * 2)])
    dk = P.DeviceBuffer.from_numpy(key)
    srv, xid, _ = make_server(P, env)
    hid = srv.register_hybrid_key(hks, 1, 1, dk)
    ins = [O.uniform_rns(30 + i, 0, moduli[:L], 2 * n) for i in range(24)]
    bufs = [(P.DeviceBuffer.from_numpy(x), P.DeviceBuffer(2 * L * n)) for x in ins]
    tickets = [srv.submit(P.key_switch_request(hid, di, do)) for di, do in bufs]
    for t in tickets:
        srv.wait(t, timeout_us=30_000_000)
    for (di, do) in bufs:
        alone = P.DeviceBuffer(2 * L * n)
        hks.key_switch(1, 1, dk, di, alone, 1)
        assert np.array_equal(do.numpy(), alone.numpy())
    srv.close()
