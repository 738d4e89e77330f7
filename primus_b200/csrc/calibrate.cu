// Built-in measurements of the ceilings the lattice kernels are held against
// (no counterpart in the reference): a streaming copy through HBM and the
// register-only rate of the forward butterfly on each schedule, measured on the
// current device.  The butterfly kernels run the exact butterflies of the NTT
// kernels (ntt_kernels.cuh) over values held in registers, so their rate is the
// arithmetic ceiling of a transform with no memory traffic at all.
#include <cstring>

#include "ntt_kernels.cuh"

using namespace pg;

namespace {

constexpr int kCalE = 16;          // values per thread, as in the NTT rounds
constexpr int kCalIters = 256;     // rounds of 4 stages per launch
constexpr unsigned kCalThreads = 256;
constexpr unsigned kCalBlocks = 148 * 8;

__global__ void __launch_bounds__(256) copy_kernel(const ulonglong2* __restrict__ src, ulonglong2* __restrict__ dst,
                                                   size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// one round = 4 radix-2 stages over 16 register values (32 butterflies); K as in fwd_round
template <int K>
__global__ void __launch_bounds__(kCalThreads) butterfly_rate_kernel(uint64_t* out, const ulonglong2* tw,
                                                                      uint64_t q, int iters) {
    const FpMod fm = fp_mod(q);
    const uint64_t mA = K == 2 ? as_u(fm.q) : 2 * q, mB = K == 2 ? as_u(fm.qinv) : 0 - q;
    uint64_t x[kCalE];
    for (int i = 0; i < kCalE; ++i) {
        const uint64_t v = (threadIdx.x * 131 + i * 977 + blockIdx.x) % q;
        x[i] = K == 2 ? as_u(u52_to_f(v)) : v;
    }
    ulonglong2 w[8];
    for (int i = 0; i < 8; ++i) w[i] = tw[i];
    for (int it = 0; it < iters; ++it) {
        static_for<0, 4>([&](auto st) {
            constexpr int s = decltype(st)::value, h = 8 >> s;
            static_for<0, kCalE>([&](auto ii) {
                constexpr int i = decltype(ii)::value;
                if constexpr ((i & h) == 0) {
                    if constexpr (K == 2)
                        fwd_bfly_fp<(s & 1) == 0>(x[i], x[i + h], w[(i + s) & 7], as_f(mA), as_f(mB));
                    else
                        fwd_bfly_fast(x[i], x[i + h], w[(i + s) & 7], mA, mB);
                }
            });
        });
        if constexpr (K != 2) {  // keep the integer values bounded as the schedule's reductions do
#pragma unroll
            for (int i = 0; i < kCalE; ++i) x[i] = x[i] >= 16 * q ? x[i] - 16 * q : x[i];
        }
    }
    uint64_t acc = 0;
    for (int i = 0; i < kCalE; ++i) acc ^= x[i];
    out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = acc;
}

template <int K>
int time_butterflies(uint64_t* out, const ulonglong2* tw, uint64_t q, cudaEvent_t e0, cudaEvent_t e1, double* gps) {
    float best = 0;
    for (int rep = 0; rep < 3; ++rep) {
        PG_CUDA(cudaEventRecord(e0));
        butterfly_rate_kernel<K><<<kCalBlocks, kCalThreads>>>(out, tw, q, kCalIters);
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cudaEventRecord(e1));
        PG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        PG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep == 0 || ms < best) best = ms;
    }
    const double bfly = (double)kCalBlocks * kCalThreads * kCalIters * 32;
    *gps = bfly / (best * 1e-3) / 1e9;
    return PG_OK;
}

struct CalBuffers {
    void* a = nullptr;
    void* b = nullptr;
    uint64_t* out = nullptr;
    ulonglong2* tw = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~CalBuffers() {
        cudaDeviceSynchronize();
        cudaFree(a);
        cudaFree(b);
        cudaFree(out);
        cudaFree(tw);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

}  // namespace

extern "C" {

int pg_calibrate(pg_calibration* out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = pg_calibration{};
    CalBuffers b;
    const size_t bytes = (size_t)512 << 20;  // per buffer: 4x the L2
    PG_CUDA(cudaMalloc(&b.a, bytes));
    PG_CUDA(cudaMalloc(&b.b, bytes));
    PG_CUDA(cudaMemset(b.a, 1, bytes));
    PG_CUDA(cudaMalloc(&b.out, (size_t)kCalBlocks * kCalThreads * sizeof(uint64_t)));
    PG_CUDA(cudaMalloc(&b.tw, 8 * sizeof(ulonglong2)));
    PG_CUDA(cudaEventCreate(&b.e0));
    PG_CUDA(cudaEventCreate(&b.e1));
    // streaming copy: read + write bytes per launch over the best of 5
    const size_t n = bytes / sizeof(ulonglong2);
    float best = 0;
    for (int rep = 0; rep < 6; ++rep) {
        PG_CUDA(cudaEventRecord(b.e0));
        copy_kernel<<<148 * 8, 256>>>((const ulonglong2*)b.a, (ulonglong2*)b.b, n);
        PG_CUDA(cudaGetLastError());
        PG_CUDA(cudaEventRecord(b.e1));
        PG_CUDA(cudaEventSynchronize(b.e1));
        float ms = 0;
        PG_CUDA(cudaEventElapsedTime(&ms, b.e0, b.e1));
        if (rep == 1 || (rep > 1 && ms < best)) best = ms;  // launch 0 is the warm-up
    }
    out->hbm_copy_gbs = 2.0 * bytes / (best * 1e-3) / 1e9;
    // butterflies: a prime just below 2^50 (the workloads' size) and twiddles below it
    const uint64_t q = 1125899906826241ull;  // largest prime below 2^50 with q = 1 mod 2^14
    ulonglong2 htw[8], hfp[8];
    for (int i = 0; i < 8; ++i) {
        const uint64_t w = (q / 3 + 1234567ull * (i + 1)) % q;
        htw[i] = make_ulonglong2(w, h_shoup_quotient(w, q));
        const double wd = (double)w, wq = wd / (double)q;
        uint64_t u0, u1;
        memcpy(&u0, &wd, 8);
        memcpy(&u1, &wq, 8);
        hfp[i] = make_ulonglong2(u0, u1);
    }
    PG_CUDA(cudaMemcpy(b.tw, htw, sizeof htw, cudaMemcpyHostToDevice));
    int rc = time_butterflies<1>(b.out, b.tw, q, b.e0, b.e1, &out->int_butterflies_gps);
    if (rc) return rc;
    PG_CUDA(cudaMemcpy(b.tw, hfp, sizeof hfp, cudaMemcpyHostToDevice));
    rc = time_butterflies<2>(b.out, b.tw, q, b.e0, b.e1, &out->fp64_butterflies_gps);
    if (rc) return rc;
    count_launch(6 + 6);
    return PG_OK;
}

}  // extern "C"
