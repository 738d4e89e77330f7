// Uneven batches of negacyclic polynomial products in one graph launch.
//
// Each job is a product a <- a * b of two coefficient-form DCRT polynomials of
// its own ring degree N_j and limb count L_j (the first L_j primes of the table
// for that degree), i.e. per limb: transform_slice(a), transform_slice(b),
// mul_assign, inverse_transform_slice (primus_ntt/src/ntt/primitive.rs:234-296,
// primus_poly/src/dcrt/mul.rs:97-110) -- the reference's three calls.
//
// Schedule: jobs are grouped by ring degree.  Each degree class gets two
// descriptor-driven launches: one forward NTT over every a- and b-row of the
// class, then one fused (multiply by the b-row, inverse NTT) over every a-row.
// Classes of N <= 2^12 on the FP64 schedule take one launch instead, whose CTAs
// transform the b-row, then the a-row, multiply and run the inverse (the pair
// form of the block kernel).
// Rows are listed limb-major so that concurrently running CTAs share a prime's
// twiddles.  The classes run on forked streams, and the whole set of launches
// is captured once into a CUDA graph that later calls replay (a job set with
// the same shape only rewrites the device descriptors).  Within a launch the
// hardware block scheduler hands rows to CTAs as they free up.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace pg;

namespace {
constexpr int kClasses = 17;  // log_n 0..16
}

struct pg_polymul_batch {
    const pg_ntt_table* tables[kClasses] = {};
    int device = 0;
    cudaStream_t streams[kClasses] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t joins[kClasses] = {};
    // two pinned descriptor slots used in turn, so that a call only waits for the
    // copy of the call before the previous one (the host runs a call ahead)
    cudaEvent_t copied[2] = {};      // slot s may be rewritten once copied[s] completes
    cudaEvent_t finished = nullptr;  // the last call's launches (and so its descriptor reads) are done
    RowDesc* h_desc[2] = {};         // pinned
    int slot = 0;
    RowDesc* d_desc = nullptr;
    size_t cap = 0;
    // launch plan of the last call: per class (forward rows, inverse rows) at offsets
    struct Cls {
        int log_n;
        size_t fwd_off, fwd_n, inv_off, inv_n;
    };
    std::vector<Cls> plan;
    std::vector<Cls> graph_plan;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    RowDesc* graph_desc = nullptr;
};

namespace {

void destroy_graph(pg_polymul_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_plan.clear();
}

bool same_plan(const std::vector<pg_polymul_batch::Cls>& x, const std::vector<pg_polymul_batch::Cls>& y) {
    if (x.size() != y.size()) return false;
    for (size_t i = 0; i < x.size(); ++i)
        if (x[i].log_n != y[i].log_n || x[i].fwd_off != y[i].fwd_off || x[i].fwd_n != y[i].fwd_n ||
            x[i].inv_off != y[i].inv_off || x[i].inv_n != y[i].inv_n)
            return false;
    return true;
}

// kernel launches of the last call's plan: one per class in the pair form, else two
size_t plan_launches(const pg_polymul_batch* b) {
    size_t n = 0;
    for (const auto& c : b->plan) {
        NttArgs ia = make_args(b->tables[c.log_n], nullptr, c.inv_n, 0);
        ia.desc = b->d_desc + c.inv_off;
        n += pair_ok(ia, (uint32_t)c.log_n) ? 1 : 2;
    }
    return n;
}

// the per-class launches, forked off `st` and joined back into it (a batch of
// one ring degree runs on `st` itself: no cross-stream dependencies to pay for)
int enqueue(pg_polymul_batch* b, cudaStream_t st) {
    const bool fork = b->plan.size() > 1;
    if (fork) PG_CUDA(cudaEventRecord(b->fork, st));
    for (const auto& c : b->plan) {
        cudaStream_t cs = fork ? b->streams[c.log_n] : st;
        if (fork) PG_CUDA(cudaStreamWaitEvent(cs, b->fork, 0));
        const pg_ntt_table* t = b->tables[c.log_n];
        NttArgs ia = make_args(t, nullptr, c.inv_n, 0);
        ia.desc = b->d_desc + c.inv_off;
        int rc;
        if (pair_ok(ia, t->log_n)) {
            // one CTA transforms b, multiplies and runs the inverse of a: one launch,
            // and a's forward never goes through HBM
            rc = launch_pair(ia, t->log_n, cs);
        } else {
            NttArgs fa = make_args(t, nullptr, c.fwd_n, 0);
            fa.desc = b->d_desc + c.fwd_off;
            rc = launch_ntt(fa, t->log_n, MODE_FWD, cs);
            if (rc) return rc;
            rc = launch_ntt(ia, t->log_n, MODE_INV, cs);
        }
        if (rc) return rc;
        if (fork) {
            PG_CUDA(cudaEventRecord(b->joins[c.log_n], cs));
            PG_CUDA(cudaStreamWaitEvent(st, b->joins[c.log_n], 0));
        }
    }
    return PG_OK;
}

}  // namespace

extern "C" {

int pg_polymul_batch_create(const pg_ntt_table* const* tables, uint32_t table_count, pg_polymul_batch** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!tables || table_count == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "need at least one table");
    pg_polymul_batch* b = new (std::nothrow) pg_polymul_batch();
    if (!b) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    for (uint32_t i = 0; i < table_count; ++i) {
        const pg_ntt_table* t = tables[i];
        if (!t || t->log_n >= kClasses || b->tables[t->log_n]) {
            delete b;
            return set_error(PG_ERR_INVALID_ARGUMENT, "tables must be non-NULL with distinct log_n <= 16");
        }
        b->tables[t->log_n] = t;
    }
    cudaError_t e = cudaGetDevice(&b->device);
    for (int c = 0; c < kClasses && e == cudaSuccess; ++c) {
        if (!b->tables[c]) continue;
        e = cudaStreamCreateWithFlags(&b->streams[c], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->joins[c], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&b->copied[k], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->finished, cudaEventDisableTiming);
    // room for 4096 rows up front, so that typical calls never allocate
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = cudaMallocHost(&b->h_desc[k], 4096 * sizeof(RowDesc));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_desc, 4096 * sizeof(RowDesc));
    if (e == cudaSuccess) b->cap = 4096;
    if (e != cudaSuccess) {
        pg_polymul_batch_destroy(b);
        return cuda_status(e, "pg_polymul_batch_create");
    }
    *out = b;
    return PG_OK;
}

int pg_polymul_batch_destroy(pg_polymul_batch* b) {
    if (!b) return PG_OK;
    destroy_graph(b);
    for (int c = 0; c < kClasses; ++c) {
        if (b->streams[c]) cudaStreamDestroy(b->streams[c]);
        if (b->joins[c]) cudaEventDestroy(b->joins[c]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    for (int k = 0; k < 2; ++k)
        if (b->copied[k]) cudaEventDestroy(b->copied[k]);
    if (b->finished) cudaEventDestroy(b->finished);
    for (int k = 0; k < 2; ++k) cudaFreeHost(b->h_desc[k]);
    cudaFree(b->d_desc);
    delete b;
    return PG_OK;
}

int pg_polymul_batch_reserve(pg_polymul_batch* b, size_t rows) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (rows <= b->cap) return PG_OK;
    destroy_graph(b);  // captured launches point at the old descriptor buffer
    for (int k = 0; k < 2; ++k) PG_CUDA(cudaEventSynchronize(b->copied[k]));
    PG_CUDA(cudaEventSynchronize(b->finished));
    for (int k = 0; k < 2; ++k) {
        cudaFreeHost(b->h_desc[k]);
        b->h_desc[k] = nullptr;
    }
    cudaFree(b->d_desc);
    b->d_desc = nullptr;
    b->cap = 0;
    for (int k = 0; k < 2; ++k) PG_CUDA(cudaMallocHost(&b->h_desc[k], rows * sizeof(RowDesc)));
    PG_CUDA(cudaMalloc(&b->d_desc, rows * sizeof(RowDesc)));
    b->cap = rows;
    return PG_OK;
}

int pg_polymul_batch_run(pg_polymul_batch* b, const pg_polymul_job* jobs, size_t count, int use_graph,
                         void* stream) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (count == 0) return PG_OK;
    if (!jobs) return set_error(PG_ERR_INVALID_ARGUMENT, "jobs is NULL");
    cudaStream_t st = (cudaStream_t)stream;
    size_t rows[kClasses] = {};
    uint32_t maxL[kClasses] = {};
    for (size_t j = 0; j < count; ++j) {
        const pg_polymul_job& jb = jobs[j];
        if (jb.log_n >= kClasses || !b->tables[jb.log_n])
            return set_error(PG_ERR_INVALID_ARGUMENT, "job ring degree has no table in this batch");
        if (jb.moduli_count == 0 || jb.moduli_count > b->tables[jb.log_n]->L)
            return set_error(PG_ERR_INVALID_ARGUMENT, "job moduli_count exceeds its table");
        if (!jb.d_a || !jb.d_b) return set_error(PG_ERR_INVALID_ARGUMENT, "job buffer is NULL");
        {
            // a and b are transformed in place: the two rows of a job must not overlap
            const uintptr_t a0 = (uintptr_t)jb.d_a, b0 = (uintptr_t)jb.d_b;
            const uintptr_t bytes = ((uintptr_t)jb.moduli_count << jb.log_n) * sizeof(uint64_t);
            if (a0 < b0 + bytes && b0 < a0 + bytes)
                return set_error(PG_ERR_INVALID_ARGUMENT, "job buffers a and b overlap (both are transformed in place)");
        }
        rows[jb.log_n] += jb.moduli_count;
        maxL[jb.log_n] = std::max(maxL[jb.log_n], jb.moduli_count);
    }
    // plan: per class [fwd rows (a and b)] then [inverse rows (a, multiplied by b)]
    b->plan.clear();
    size_t total = 0;
    for (int c = 0; c < kClasses; ++c) {
        if (!rows[c]) continue;
        pg_polymul_batch::Cls k{c, total, 2 * rows[c], total + 2 * rows[c], rows[c]};
        b->plan.push_back(k);
        total += 3 * rows[c];
    }
    // this call's pinned slot was last read by the copy of the call before the
    // previous one; that copy must have completed before the slot is rewritten
    b->slot ^= 1;
    PG_CUDA(cudaEventSynchronize(b->copied[b->slot]));
    if (total > b->cap) {
        // grow geometrically (rare: the batch starts with room for 4096 rows and
        // callers can reserve more); freeing waits for launches still reading
        int rc = pg_polymul_batch_reserve(b, std::max<size_t>(total, 2 * b->cap));
        if (rc) return rc;
    }
    for (const auto& k : b->plan) {
        const size_t n = (size_t)1 << k.log_n;
        size_t f = k.fwd_off, i = k.inv_off;
        for (uint32_t l = 0; l < maxL[k.log_n]; ++l) {  // limb-major across the class's jobs
            for (size_t j = 0; j < count; ++j) {
                const pg_polymul_job& jb = jobs[j];
                if ((int)jb.log_n != k.log_n || l >= jb.moduli_count) continue;
                uint64_t* a = jb.d_a + (size_t)l * n;
                uint64_t* bb = jb.d_b + (size_t)l * n;
                RowDesc* hd = b->h_desc[b->slot];
                hd[f++] = RowDesc{a, nullptr, l, 0};
                hd[f++] = RowDesc{bb, nullptr, l, 0};
                hd[i++] = RowDesc{a, bb, l, 0};
            }
        }
    }
    PG_CUDA(cudaMemcpyAsync(b->d_desc, b->h_desc[b->slot], total * sizeof(RowDesc), cudaMemcpyHostToDevice, st));
    PG_CUDA(cudaEventRecord(b->copied[b->slot], st));
    if (!use_graph) {
        int rc = enqueue(b, st);
        if (rc) return rc;
        PG_CUDA(cudaEventRecord(b->finished, st));
        return PG_OK;
    }
    if (b->exec && same_plan(b->plan, b->graph_plan) && b->graph_desc == b->d_desc) {
        PG_CUDA(cudaGraphLaunch(b->exec, st));
        count_launch(plan_launches(b));
        PG_CUDA(cudaEventRecord(b->finished, st));
        return PG_OK;
    }
    // first call of this shape: run it directly (this also performs each kernel's
    // one-time attribute setup outside any capture), then capture it for replay
    int rc = enqueue(b, st);
    if (rc) return rc;
    PG_CUDA(cudaEventRecord(b->finished, st));
    destroy_graph(b);
    cudaStream_t cap;
    PG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        const uint64_t before = pg_launch_count();
        rc = enqueue(b, cap);
        g_launches.fetch_sub(pg_launch_count() - before);  // captured, not executed
        e = cudaStreamEndCapture(cap, &b->graph);
        if (rc == PG_OK && e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    }
    cudaStreamDestroy(cap);
    if (rc) return rc;
    if (e != cudaSuccess) {
        destroy_graph(b);
        return cuda_status(e, "pg_polymul_batch_run: graph capture");
    }
    b->graph_plan = b->plan;
    b->graph_desc = b->d_desc;
    return PG_OK;
}

}  // extern "C"
