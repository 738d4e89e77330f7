// Alternative NTT kernel shapes and the autotuner that picks among them.
//
// For each ring degree the default dispatch (ntt.cu) uses one shape: rows per
// CTA, elements per thread (the radix of a round) and, for N >= 2^14, the
// cluster size.  The shapes below split the same transform differently: more
// or fewer threads per row, two rows per CTA, a cluster of another size, or a
// whole 2^14 row in one CTA.  Every shape evaluates the same butterflies on
// the same operands stage by stage, so all of them return identical values;
// only their speed differs with (N, L, batch).  pg_ntt_autotune times each
// shape on the table's own moduli and keeps the fastest per mode (canonical
// forward, inverse, fused round trip) in the table.
#include <algorithm>

#include "ntt_kernels.cuh"

namespace pg {

namespace {

struct VariantInfo {
    uint32_t log_n;
    int variant;
    const char* name;
    bool fp;  // FP64 schedule: every q < 2^50, canonical outputs
};

// variant 0 is the default of each degree (ntt.cu); these are 1, 2, ...
constexpr VariantInfo kVariants[] = {
    {10, 1, "block E=8, 2 rows per CTA", false},  {10, 2, "block E=4, 256 threads", false},
    {10, 3, "fp64 block E=8", true},              {10, 4, "fp64 block E=8, 2 rows per CTA", true},
    {11, 1, "block E=16, 128 threads", false},    {11, 2, "block E=16, 2 rows per CTA", false},
    {11, 3, "fp64 block E=8", true},              {11, 4, "fp64 block E=16, 128 threads", true},
    {12, 1, "block E=8, 512 threads", false},     {12, 2, "block E=16, 2 rows per CTA", false},
    {12, 3, "cluster of 2 x 2048", false},        {12, 4, "fp64 block E=16", true},
    {12, 5, "fp64 cluster of 2 x 2048", true},
    {13, 1, "block E=8, 1024 threads", false},    {13, 2, "block E=16, 512 threads", false},
    {13, 3, "cluster of 4 x 2048", false},        {13, 4, "fp64 cluster of 2 x 4096", true},
    {13, 5, "fp64 cluster of 4 x 2048", true},
    {14, 1, "cluster of 2 x 8192", false},        {14, 2, "block E=16, 1024 threads", false},
    {14, 3, "cluster of 8 x 2048", false},        {14, 4, "fp64 cluster of 4 x 4096", true},
    {14, 5, "fp64 cluster of 2 x 8192", true},
    {15, 1, "cluster of 4 x 8192", false},        {15, 2, "cluster of 16 x 2048", false},
    {15, 3, "fp64 cluster of 8 x 4096", true},    {15, 4, "fp64 cluster of 4 x 8192", true},
    {16, 1, "cluster of 8 x 8192", false},        {16, 2, "fp64 cluster of 16 x 4096", true},
    {16, 3, "fp64 cluster of 8 x 8192", true},
    // the same clusters with the spread placement policy (the default is load balancing)
    {14, 6, "fp64 cluster of 4 x 4096, spread placement", true},
    {15, 5, "fp64 cluster of 8 x 4096, spread placement", true},
    {16, 4, "fp64 cluster of 16 x 4096, spread placement", true},
    {16, 5, "fp64 cluster of 8 x 8192, spread placement", true},
};

}  // namespace

// the shape instantiations live in ntt_shapes_*.cu (one family per translation unit)
int run_ntt_shape_lo(const NttArgs& a, uint32_t log_n, int mode, int v, cudaStream_t st);
int run_ntt_shape_mid(const NttArgs& a, uint32_t log_n, int mode, int v, cudaStream_t st);
int run_ntt_shape_hi(const NttArgs& a, uint32_t log_n, int mode, int v, cudaStream_t st);

int ntt_variant_count(uint32_t log_n) {
    int c = 1;
    for (const auto& v : kVariants)
        if (v.log_n == log_n) ++c;
    return c;
}

bool ntt_variant_fp(uint32_t log_n, int variant) {
    for (const auto& v : kVariants)
        if (v.log_n == log_n && v.variant == variant) return v.fp;
    return false;
}

const char* ntt_variant_name(uint32_t log_n, int variant) {
    if (variant == 0) return "default";
    for (const auto& v : kVariants)
        if (v.log_n == log_n && v.variant == variant) return v.name;
    return nullptr;
}

int launch_ntt_variant(const NttArgs& a, uint32_t log_n, int mode, int variant, cudaStream_t st) {
    if (log_n <= 13) return run_ntt_shape_lo(a, log_n, mode, variant, st);
    if (log_n <= 15) return run_ntt_shape_mid(a, log_n, mode, variant, st);
    return run_ntt_shape_hi(a, log_n, mode, variant, st);
}

}  // namespace pg

using namespace pg;

namespace {

// time `reps` launches of one shape; the first launch (untimed) also performs
// the kernel's one-time attribute setup and reports launch errors
int time_variant(NttArgs a, uint32_t log_n, int mode, int v, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                 float* us) {
    a.variant[mode] = v;
    const int reps = 3;
    int rc = v ? launch_ntt_variant(a, log_n, mode, v, st) : launch_ntt(a, log_n, mode, st);
    if (rc) return rc;
    PG_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < reps && rc == PG_OK; ++r)
        rc = v ? launch_ntt_variant(a, log_n, mode, v, st) : launch_ntt(a, log_n, mode, st);
    if (rc) return rc;
    PG_CUDA(cudaEventRecord(e1, st));
    PG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *us = ms * 1000.0f / reps;
    return PG_OK;
}

struct TuneBuffers {
    int prev_device = -1;  // the caller's current device, restored on exit
    uint64_t* data = nullptr;
    uint64_t* plain = nullptr;
    uint64_t* plain_q = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~TuneBuffers() {
        if (st) cudaStreamSynchronize(st);
        cudaFree(data);
        cudaFree(plain);
        cudaFree(plain_q);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
        if (prev_device >= 0) cudaSetDevice(prev_device);
    }
};

}  // namespace

extern "C" {

int pg_ntt_variant_count(uint32_t log_n) { return ntt_variant_count(log_n); }

const char* pg_ntt_variant_name(uint32_t log_n, int variant) { return ntt_variant_name(log_n, variant); }

int pg_ntt_set_variant(pg_ntt_table* t, int mode, int variant) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (mode < 0 || mode > 2) return set_error(PG_ERR_INVALID_ARGUMENT, "mode must be 0 (forward), 1 or 2");
    if (variant < 0 || variant >= ntt_variant_count(t->log_n))
        return set_error(PG_ERR_INVALID_ARGUMENT, "no such NTT kernel variant for this ring degree");
    t->variant[mode] = variant;
    return PG_OK;
}

int pg_ntt_autotune(pg_ntt_table* t, size_t polys, pg_ntt_tuning* out) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (polys == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "polys must be at least 1");
    const size_t row_bytes = t->n * sizeof(uint64_t);
    // time on at most 1 GiB of rows: enough to fill the GPU, bounded in memory
    const size_t max_rows = std::max<size_t>(t->L, ((size_t)1 << 30) / row_bytes);
    size_t rows = polys * t->L;
    if (rows > max_rows) rows = (max_rows / t->L) * t->L;
    TuneBuffers b;
    PG_CUDA(cudaGetDevice(&b.prev_device));
    PG_CUDA(cudaSetDevice(t->device));
    PG_CUDA(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
    PG_CUDA(cudaEventCreate(&b.e0));
    PG_CUDA(cudaEventCreate(&b.e1));
    PG_CUDA(cudaMalloc(&b.data, rows * row_bytes));
    PG_CUDA(cudaMalloc(&b.plain, t->L * row_bytes));
    PG_CUDA(cudaMalloc(&b.plain_q, t->L * row_bytes));
    int rc = pg_fill_uniform(t, b.data, rows / t->L, 0x7A11, 0, b.st);
    if (rc == PG_OK) rc = pg_fill_uniform(t, b.plain, 1, 0x7A12, 0, b.st);
    if (rc == PG_OK) rc = pg_dcrt_shoup_prepare(t, b.plain, b.plain_q, 1, b.st);
    if (rc) return rc;
    NttArgs a = make_args(t, b.data, rows, 0);
    a.plain = b.plain;
    a.plain_q = b.plain_q;
    const bool ffwd = fast_fwd_ok(a), finv = fast_inv_ok(a);
    const int count = ntt_variant_count(t->log_n);
    pg_ntt_tuning res{};
    for (int mode = 0; mode < 3; ++mode) {
        int best = 0;
        float best_us = 0;
        for (int v = 0; v < count; ++v) {
            // alternative shapes exist on the fast schedules only (FP64: every q < 2^50)
            if (v > 0 && !(ntt_variant_fp(t->log_n, v) ? finv && a.fwd_fp : (mode == MODE_FWD ? ffwd : finv)))
                continue;
            float us = 0;
            rc = time_variant(a, t->log_n, mode, v, b.st, b.e0, b.e1, &us);
            if (rc) return rc;
            if (v == 0) res.default_us[mode] = us;
            if (v == 0 || us < best_us) {
                best = v;
                best_us = us;
            }
        }
        t->variant[mode] = best;
        res.variant[mode] = best;
        res.us[mode] = best_us;
    }
    res.rows = rows;
    if (out) *out = res;
    return PG_OK;
}

}  // extern "C"
