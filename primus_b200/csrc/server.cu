// Continuous-batching request server for mixed polynomial products, external
// products and key switches.
//
// Clients submit single requests on device buffers they keep resident in HBM
// (keys, ciphertexts); the server keeps twiddle tables and keys resident too.
// A worker thread forms batches from whatever is pending whenever one of its
// slots is free: a slot is a stream plus a fixed share of the scratch memory
// budget, so admission is by memory -- a batch takes as many pending requests
// of one kind and shape as fit in its slot's scratch.  Requests that arrive
// while other batches are on the GPU wait for the next free slot, and batches
// on different slots overlap on the device.  Completion is an event recorded
// after each batch's last launch and polled by a completion thread (no
// device-side waiting), which frees the slot, timestamps each request and wakes
// the worker and any waiting clients.  The idle worker spins briefly before it
// sleeps, so a request arriving right after a batch is not delayed by a wake-up.
//
// Batches reuse the library's batched paths: pg_polymul_batch (descriptor
// driven NTT launches), and for external products / key switches a gather of
// the requests' inputs into contiguous scratch, the batched pg_ext_product /
// pg_key_switch pipeline, and a scatter of the outputs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "internal.hpp"

using namespace pg;

namespace {

double now_us() {
    using namespace std::chrono;
    return duration<double, std::micro>(steady_clock::now().time_since_epoch()).count();
}

// copy `count` chunks of `words` u64 between a pointer list and a contiguous buffer
__global__ void gather_kernel(uint64_t* const* ptrs, uint64_t* contig, size_t words, size_t count, int scatter) {
    const size_t total = words * count;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t c = i / words, w = i % words;
        if (scatter)
            ptrs[c][w] = contig[i];
        else
            contig[i] = ptrs[c][w];
    }
}

struct Key {
    int kind;  // PG_REQ_EXT_PRODUCT or PG_REQ_KEY_SWITCH
    const pg_ntt_table* table;
    const pg_gadget_basis* basis;  // NULL for a hybrid key switch key
    const pg_hybrid_ks* hks;       // hybrid key switch context, or NULL
    uint32_t k_in, k_out;
    const uint64_t* d_key;
    size_t in_words, out_words;
};

struct Req {
    pg_request r;
    uint64_t ticket;
    double t_submit;
};

struct TicketState {
    std::atomic<int> done{0};
    int status = PG_OK;
    double t_submit = 0, t_done = 0;
};

}  // namespace

struct pg_server;

namespace {
struct Slot {
    pg_server* server = nullptr;
    int index = 0;
    cudaStream_t stream = nullptr;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    uint64_t** h_ptrs = nullptr;  // pinned pointer list for gather/scatter
    uint64_t** d_ptrs = nullptr;
    size_t ptr_cap = 0;
    pg_polymul_batch* polymul = nullptr;
    cudaEvent_t done_ev = nullptr;  // recorded after the batch's last launch
    bool busy = false;
    bool in_flight = false;  // on the GPU, watched by the completion thread
    std::vector<uint64_t> tickets;  // requests of the batch in flight
    int status = PG_OK;
};
}  // namespace

struct pg_server {
    pg_server_config cfg{};
    std::vector<const pg_ntt_table*> polymul_tables;
    std::vector<Key> keys;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_poll;
    std::atomic<int> pending_n{0}, free_n{0};  // mirrors of pending.size() and idle slots (written under mu)
    std::deque<Req> pending;
    std::vector<TicketState*> tickets;  // index = ticket
    std::thread worker, poller;
    bool stop = false;
    int device = 0;
    // statistics
    uint64_t submitted = 0, completed = 0, rejected = 0, batches = 0, batched_requests = 0;
    double enqueue_total_us = 0, enqueue_max_us = 0;
    std::vector<double> latencies;
    std::string worker_error;
};

namespace {

// completes the batch of slot s: timestamps its requests and frees the slot
void on_batch_done(Slot* s) {
    pg_server* srv = s->server;
    const double t = now_us();
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        for (uint64_t tk : s->tickets) {
            TicketState* ts = srv->tickets[tk];
            ts->status = s->status;
            ts->t_done = t;
            ts->done.store(1);
            srv->latencies.push_back(t - ts->t_submit);
            ++srv->completed;
        }
        s->tickets.clear();
        s->busy = false;
        s->in_flight = false;
        srv->free_n.fetch_add(1);
    }
    srv->cv_done.notify_all();
    srv->cv_work.notify_all();
}

// Completion thread: polls the events of the batches on the GPU (no device-side
// waiting, no driver callback thread in the path), so a finished batch frees
// its slot a few microseconds after its last kernel.
void poller_loop(pg_server* srv) {
    cudaSetDevice(srv->device);
    std::vector<Slot*> watch;
    std::unique_lock<std::mutex> lock(srv->mu);
    for (;;) {
        srv->cv_poll.wait(lock, [&] {
            if (srv->stop) return true;
            for (auto& s : srv->slots)
                if (s.in_flight) return true;
            return false;
        });
        if (srv->stop) return;
        watch.clear();
        for (auto& s : srv->slots)
            if (s.in_flight) watch.push_back(&s);
        lock.unlock();
        bool any = false;
        for (Slot* s : watch) {
            const cudaError_t e = cudaEventQuery(s->done_ev);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) {
                s->status = cuda_status(e, "server batch");
                std::lock_guard<std::mutex> g(srv->mu);
                srv->worker_error = pg_last_error();
            }
            on_batch_done(s);
            any = true;
        }
        if (!any) std::this_thread::yield();
        lock.lock();
    }
}

size_t request_scratch(const pg_server* srv, const pg_request& r) {
    if (r.kind == PG_REQ_POLYMUL) return 0;
    const Key& k = srv->keys[r.key];
    const size_t io = (k.in_words + k.out_words) * sizeof(uint64_t);
    if (k.kind == PG_REQ_EXT_PRODUCT) return io + pg_ext_product_workspace_size(k.table, k.basis, k.k_in, 1);
    if (k.hks) return io + pg_hybrid_ks_workspace_size(k.hks, k.k_in, k.k_out, 1);
    return io + pg_key_switch_workspace_size(k.table, k.basis, k.k_in, k.k_out, 1);
}

bool same_class(const pg_request& a, const pg_request& b) {
    if (a.kind != b.kind) return false;
    if (a.kind == PG_REQ_POLYMUL) return true;  // the polymul batch groups ring degrees itself
    return a.key == b.key;
}

int ensure_ptrs(Slot& s, size_t n) {
    if (n <= s.ptr_cap) return PG_OK;
    cudaFreeHost(s.h_ptrs);
    cudaFree(s.d_ptrs);
    s.h_ptrs = nullptr;
    s.d_ptrs = nullptr;
    s.ptr_cap = 0;
    size_t cap = std::max<size_t>(n, 256);
    PG_CUDA(cudaMallocHost(&s.h_ptrs, cap * sizeof(uint64_t*)));
    PG_CUDA(cudaMalloc(&s.d_ptrs, cap * sizeof(uint64_t*)));
    s.ptr_cap = cap;
    return PG_OK;
}

int gather(Slot& s, const std::vector<Req>& batch, bool outputs, uint64_t* contig, size_t words) {
    const size_t n = batch.size();
    for (size_t i = 0; i < n; ++i)
        s.h_ptrs[(outputs ? n : 0) + i] = outputs ? batch[i].r.d_out : const_cast<uint64_t*>(batch[i].r.d_in);
    uint64_t** d = s.d_ptrs + (outputs ? n : 0);
    PG_CUDA(cudaMemcpyAsync(d, s.h_ptrs + (outputs ? n : 0), n * sizeof(uint64_t*), cudaMemcpyHostToDevice,
                            s.stream));
    const size_t total = words * n;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 8);
    gather_kernel<<<blocks, 256, 0, s.stream>>>(d, contig, words, n, outputs ? 1 : 0);
    count_launch();
    PG_LAUNCH_CHECK("gather_kernel launch");
    return PG_OK;
}

// enqueue one batch on slot s (called without the server lock held)
int run_batch(pg_server* srv, Slot& s, const std::vector<Req>& batch) {
    const pg_request& r0 = batch[0].r;
    if (r0.kind == PG_REQ_POLYMUL) {
        std::vector<pg_polymul_job> jobs(batch.size());
        for (size_t i = 0; i < batch.size(); ++i)
            jobs[i] = pg_polymul_job{batch[i].r.d_a, batch[i].r.d_b, batch[i].r.log_n, batch[i].r.moduli_count};
        return pg_polymul_batch_run(s.polymul, jobs.data(), jobs.size(), 0, s.stream);
    }
    const Key& k = srv->keys[r0.key];
    const size_t n = batch.size();
    int rc = ensure_ptrs(s, 2 * n);
    if (rc) return rc;
    uint64_t* in = (uint64_t*)s.scratch;
    uint64_t* out = in + n * k.in_words;
    uint8_t* ws = (uint8_t*)(out + n * k.out_words);
    const size_t ws_bytes = s.scratch_bytes - (size_t)(ws - (uint8_t*)s.scratch);
    rc = gather(s, batch, false, in, k.in_words);
    if (rc) return rc;
    if (k.kind == PG_REQ_EXT_PRODUCT)
        rc = pg_ext_product(k.table, k.basis, k.k_in, in, k.d_key, out, n, ws, ws_bytes, s.stream);
    else if (k.hks)
        rc = pg_key_switch_hybrid(k.hks, k.k_in, k.k_out, k.d_key, in, out, n, ws, ws_bytes, s.stream);
    else
        rc = pg_key_switch(k.table, k.basis, k.k_in, k.k_out, k.d_key, in, out, n, ws, ws_bytes, s.stream);
    if (rc) return rc;
    return gather(s, batch, true, out, k.out_words);
}

void worker_loop(pg_server* srv) {
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lock(srv->mu);
    for (;;) {
        Slot* slot = nullptr;
        if (!srv->stop && (srv->pending.empty() || srv->free_n.load() == 0)) {
            // idle: spin briefly on the lock-free mirrors before sleeping, so a
            // request arriving right after a batch does not pay a thread wake-up
            lock.unlock();
            const double t0 = now_us();
            while (now_us() - t0 < 100.0 && (srv->pending_n.load() == 0 || srv->free_n.load() == 0))
                std::this_thread::yield();
            lock.lock();
        }
        srv->cv_work.wait(lock, [&] {
            if (srv->stop) return true;
            if (srv->pending.empty()) return false;
            for (auto& s : srv->slots)
                if (!s.busy) {
                    slot = &s;
                    return true;
                }
            return false;
        });
        if (srv->stop) return;
        // form a batch: the oldest request's class, every pending request of that
        // class that fits the slot's scratch, up to max_batch
        std::vector<Req> batch;
        const pg_request first = srv->pending.front().r;
        size_t used = 0;
        for (auto it = srv->pending.begin(); it != srv->pending.end() && batch.size() < srv->cfg.max_batch;) {
            if (same_class(it->r, first)) {
                const size_t need = request_scratch(srv, it->r);
                if (used + need <= slot->scratch_bytes) {
                    used += need;
                    batch.push_back(*it);
                    it = srv->pending.erase(it);
                    srv->pending_n.fetch_sub(1);
                    continue;
                }
                if (need > slot->scratch_bytes) {  // cannot ever fit (checked at submit)
                    ++it;
                    continue;
                }
                break;  // the slot is full; later requests of this class wait
            }
            ++it;
        }
        if (batch.empty()) continue;
        slot->busy = true;
        srv->free_n.fetch_sub(1);
        slot->tickets.clear();
        for (auto& b : batch) slot->tickets.push_back(b.ticket);
        ++srv->batches;
        srv->batched_requests += batch.size();
        lock.unlock();
        const double t_enq = now_us();
        int rc = run_batch(srv, *slot, batch);
        slot->status = rc;
        if (rc == PG_OK) {
            cudaError_t e = cudaEventRecord(slot->done_ev, slot->stream);
            if (e != cudaSuccess) rc = cuda_status(e, "server: completion event");
        }
        const double enq = now_us() - t_enq;
        if (rc == PG_OK) {
            {
                std::lock_guard<std::mutex> g(srv->mu);
                slot->in_flight = true;
            }
            srv->cv_poll.notify_one();
        }
        if (rc != PG_OK) {
            // the batch never reached the GPU: fail its requests now
            slot->status = rc;
            {
                std::lock_guard<std::mutex> g(srv->mu);
                srv->worker_error = pg_last_error();
            }
            cudaStreamSynchronize(slot->stream);
            on_batch_done(slot);
        }
        lock.lock();
        srv->enqueue_total_us += enq;
        srv->enqueue_max_us = std::max(srv->enqueue_max_us, enq);
    }
}

}  // namespace

extern "C" {

int pg_server_create(const pg_server_config* cfg, const pg_ntt_table* const* polymul_tables, uint32_t table_count,
                     pg_server** out) {
    if (!out || !cfg) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (cfg->slots == 0 || cfg->slots > 64 || cfg->max_batch == 0)
        return set_error(PG_ERR_INVALID_ARGUMENT, "slots must be in [1, 64] and max_batch >= 1");
    pg_server* srv = new (std::nothrow) pg_server();
    if (!srv) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    srv->cfg = *cfg;
    if (srv->cfg.max_queue == 0) srv->cfg.max_queue = 1u << 20;
    PG_CUDA(cudaGetDevice(&srv->device));
    srv->polymul_tables.assign(polymul_tables, polymul_tables + table_count);
    srv->slots.resize(cfg->slots);
    const size_t share = (cfg->memory_budget_bytes / cfg->slots) & ~(size_t)255;
    for (uint32_t i = 0; i < cfg->slots; ++i) {
        Slot& s = srv->slots[i];
        s.server = srv;
        s.index = (int)i;
        cudaError_t e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done_ev, cudaEventDisableTiming);
        if (e == cudaSuccess && share) e = cudaMalloc(&s.scratch, share);
        if (e != cudaSuccess) {
            pg_server_destroy(srv);
            return cuda_status(e, "pg_server_create: slot");
        }
        s.scratch_bytes = share;
        // everything a batch needs on the host side is allocated here, so that
        // forming batches never allocates (allocations synchronize the device)
        int rc = ensure_ptrs(s, 2 * (size_t)srv->cfg.max_batch);
        if (rc == PG_OK && table_count) {
            rc = pg_polymul_batch_create(polymul_tables, table_count, &s.polymul);
            uint32_t max_l = 0;
            for (uint32_t t = 0; t < table_count; ++t) max_l = std::max(max_l, polymul_tables[t]->L);
            if (rc == PG_OK) rc = pg_polymul_batch_reserve(s.polymul, 3 * (size_t)max_l * srv->cfg.max_batch);
        }
        if (rc) {
            pg_server_destroy(srv);
            return rc;
        }
    }
    srv->tickets.reserve(1 << 16);
    srv->free_n.store((int)srv->slots.size());
    srv->worker = std::thread(worker_loop, srv);
    srv->poller = std::thread(poller_loop, srv);
    *out = srv;
    return PG_OK;
}

int pg_server_destroy(pg_server* srv) {
    if (!srv) return PG_OK;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    srv->cv_poll.notify_all();
    if (srv->worker.joinable()) srv->worker.join();
    if (srv->poller.joinable()) srv->poller.join();
    for (auto& s : srv->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        pg_polymul_batch_destroy(s.polymul);
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.done_ev) cudaEventDestroy(s.done_ev);
        cudaFree(s.scratch);
        cudaFreeHost(s.h_ptrs);
        cudaFree(s.d_ptrs);
    }
    for (TicketState* t : srv->tickets) delete t;
    delete srv;
    return PG_OK;
}

int pg_server_register_key(pg_server* srv, int kind, const pg_ntt_table* table, const pg_gadget_basis* basis,
                           uint32_t k_in, uint32_t k_out, const uint64_t* d_key, uint32_t* key_id) {
    if (!srv || !table || !basis || !d_key || !key_id) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (kind != PG_REQ_EXT_PRODUCT && kind != PG_REQ_KEY_SWITCH)
        return set_error(PG_ERR_INVALID_ARGUMENT, "key kind must be PG_REQ_EXT_PRODUCT or PG_REQ_KEY_SWITCH");
    Key k{};
    k.kind = kind;
    k.table = table;
    k.basis = basis;
    k.k_in = k_in;
    k.k_out = kind == PG_REQ_EXT_PRODUCT ? k_in : k_out;
    k.d_key = d_key;
    const size_t LN = (size_t)table->L * table->n;
    k.in_words = (size_t)(k_in + 1) * LN;
    k.out_words = (size_t)(k.k_out + 1) * LN;
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->keys.push_back(k);
    *key_id = (uint32_t)(srv->keys.size() - 1);
    return PG_OK;
}

int pg_server_register_hybrid_key(pg_server* srv, const pg_hybrid_ks* ks, uint32_t k_in, uint32_t k_out,
                                  const uint64_t* d_key, uint32_t* key_id) {
    if (!srv || !ks || !d_key || !key_id) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (k_in == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k_in must be at least 1");
    Key k{};
    k.kind = PG_REQ_KEY_SWITCH;
    k.hks = ks;
    k.k_in = k_in;
    k.k_out = k_out;
    k.d_key = d_key;
    const size_t LN = (size_t)hybrid_q_limbs(ks) * hybrid_n(ks);
    k.in_words = (size_t)(k_in + 1) * LN;
    k.out_words = (size_t)(k_out + 1) * LN;
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->keys.push_back(k);
    *key_id = (uint32_t)(srv->keys.size() - 1);
    return PG_OK;
}

int pg_server_submit(pg_server* srv, const pg_request* req, uint64_t* ticket) {
    if (!srv || !req || !ticket) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    // validate the request (a malformed request is refused, never queued)
    if (req->kind == PG_REQ_POLYMUL) {
        bool ok = false;
        for (const pg_ntt_table* t : srv->polymul_tables)
            if (t->log_n == req->log_n && req->moduli_count >= 1 && req->moduli_count <= t->L) ok = true;
        if (!ok || !req->d_a || !req->d_b)
            return set_error(PG_ERR_INVALID_ARGUMENT, "polymul request: no table for this degree / limb count");
        const uintptr_t a0 = (uintptr_t)req->d_a, b0 = (uintptr_t)req->d_b;
        const uintptr_t bytes = ((uintptr_t)req->moduli_count << req->log_n) * sizeof(uint64_t);
        if (a0 < b0 + bytes && b0 < a0 + bytes)
            return set_error(PG_ERR_INVALID_ARGUMENT, "polymul request: a and b overlap (both are transformed in place)");
    } else if (req->kind == PG_REQ_EXT_PRODUCT || req->kind == PG_REQ_KEY_SWITCH) {
        if (req->key >= srv->keys.size() || srv->keys[req->key].kind != req->kind || !req->d_in || !req->d_out)
            return set_error(PG_ERR_INVALID_ARGUMENT, "request names an unknown key or NULL buffers");
    } else {
        return set_error(PG_ERR_INVALID_ARGUMENT, "unknown request kind");
    }
    std::unique_lock<std::mutex> lock(srv->mu);
    if (req->kind != PG_REQ_POLYMUL && request_scratch(srv, *req) > srv->slots[0].scratch_bytes) {
        ++srv->rejected;
        return set_error(PG_ERR_REJECTED, "request needs more scratch than one slot of the memory budget holds");
    }
    if (srv->pending.size() >= srv->cfg.max_queue) {
        ++srv->rejected;
        return set_error(PG_ERR_REJECTED, "request queue is full");
    }
    const uint64_t tk = srv->tickets.size();
    TicketState* ts = new (std::nothrow) TicketState();
    if (!ts) return set_error(PG_ERR_OUT_OF_MEMORY, "ticket allocation failed");
    ts->t_submit = now_us();
    srv->tickets.push_back(ts);
    srv->pending.push_back(Req{*req, tk, ts->t_submit});
    srv->pending_n.fetch_add(1);
    ++srv->submitted;
    *ticket = tk;
    lock.unlock();
    srv->cv_work.notify_one();
    return PG_OK;
}

int pg_server_wait(pg_server* srv, uint64_t ticket, int64_t timeout_us, double* latency_us) {
    if (!srv) return set_error(PG_ERR_INVALID_ARGUMENT, "server is NULL");
    std::unique_lock<std::mutex> lock(srv->mu);
    if (ticket >= srv->tickets.size()) return set_error(PG_ERR_INVALID_ARGUMENT, "unknown ticket");
    TicketState* ts = srv->tickets[ticket];
    auto done = [&] { return ts->done.load() != 0; };
    if (timeout_us < 0)
        srv->cv_done.wait(lock, done);
    else if (!srv->cv_done.wait_for(lock, std::chrono::microseconds(timeout_us), done))
        return set_error(PG_ERR_TIMEOUT, "request not finished within the timeout");
    if (latency_us) *latency_us = ts->t_done - ts->t_submit;
    if (ts->status != PG_OK) return set_error(ts->status, "request failed: " + srv->worker_error);
    return PG_OK;
}

int pg_server_drain(pg_server* srv, int64_t timeout_us) {
    if (!srv) return set_error(PG_ERR_INVALID_ARGUMENT, "server is NULL");
    std::unique_lock<std::mutex> lock(srv->mu);
    auto idle = [&] {
        if (!srv->pending.empty()) return false;
        for (auto& s : srv->slots)
            if (s.busy) return false;
        return true;
    };
    if (timeout_us < 0)
        srv->cv_done.wait(lock, idle);
    else if (!srv->cv_done.wait_for(lock, std::chrono::microseconds(timeout_us), idle))
        return set_error(PG_ERR_TIMEOUT, "server not drained within the timeout");
    return PG_OK;
}

int pg_server_stats(pg_server* srv, pg_server_stats_t* out, int reset) {
    if (!srv || !out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lock(srv->mu);
    out->submitted = srv->submitted;
    out->completed = srv->completed;
    out->rejected = srv->rejected;
    out->batches = srv->batches;
    out->mean_batch = srv->batches ? (double)srv->batched_requests / srv->batches : 0.0;
    std::vector<double> l = srv->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
    out->p50_us = pct(0.50);
    out->p99_us = pct(0.99);
    out->max_us = l.empty() ? 0.0 : l.back();
    out->enqueue_mean_us = srv->batches ? srv->enqueue_total_us / srv->batches : 0.0;
    out->enqueue_max_us = srv->enqueue_max_us;
    if (reset) {
        srv->enqueue_total_us = srv->enqueue_max_us = 0;
        srv->submitted = srv->completed = srv->rejected = srv->batches = srv->batched_requests = 0;
        srv->latencies.clear();
    }
    return PG_OK;
}

// Load replay: submit requests at the given arrival offsets (microseconds from
// the call) from this thread, then wait for every one.  latency_us[i] is the
// time from request i's scheduled arrival to its completion, so a submitter
// that falls behind the schedule is charged to the server, not hidden;
// rejected requests get -1.
int pg_server_replay(pg_server* srv, const pg_request* reqs, const double* arrival_us, size_t count,
                     double* latency_us) {
    if (!srv || (count && (!reqs || !arrival_us || !latency_us)))
        return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::vector<uint64_t> tickets(count);
    std::vector<char> ok(count, 0);
    const double t0 = now_us();
    for (size_t i = 0; i < count; ++i) {
        const double target = t0 + arrival_us[i];
        for (;;) {
            const double gap = target - now_us();
            if (gap <= 0) break;
            if (gap > 200) std::this_thread::sleep_for(std::chrono::microseconds((int64_t)(gap - 100)));
        }
        ok[i] = pg_server_submit(srv, &reqs[i], &tickets[i]) == PG_OK;
    }
    int rc = PG_OK;
    for (size_t i = 0; i < count; ++i) {
        latency_us[i] = -1.0;
        if (!ok[i]) continue;
        int st = pg_server_wait(srv, tickets[i], -1, nullptr);
        if (st != PG_OK) rc = st;
        std::lock_guard<std::mutex> lock(srv->mu);
        latency_us[i] = srv->tickets[tickets[i]]->t_done - (t0 + arrival_us[i]);
    }
    return rc;
}

}  // extern "C"
