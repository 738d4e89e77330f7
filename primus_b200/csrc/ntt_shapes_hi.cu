// Kernel shapes the autotuner times for ring degree 2^16: the instantiations
// behind launch_ntt_variant (ntt_variants.cu), kept in a translation unit of
// their own so that the shape families compile in parallel.
#include "ntt_kernels.cuh"

namespace pg {

namespace {

template <int MODE>
int run(const NttArgs& a, uint32_t log_n, int v, cudaStream_t st) {
    // the integer shapes run the fast schedules: the forward every q < 2^58,
    // the inverse and the round trip every q < 2^50; the FP64 shapes every q < 2^50
    constexpr int F = MODE == MODE_FWD ? kSchedFastFwd : kSchedFastBoth;
    constexpr int D = kSchedFp64;
    (void)F;
    (void)D;
    switch (log_n * 16 + (uint32_t)v) {
        case 16 * 16 + 1: return launch_cluster<16, 13, 4, MODE, F>(a, st);
        case 16 * 16 + 2: return launch_cluster<16, 12, 4, MODE, D>(a, st);
        case 16 * 16 + 3: return launch_cluster<16, 13, 4, MODE, D>(a, st);
        case 16 * 16 + 4: return launch_cluster<16, 12, 4, MODE, D>(a, st, true);
        case 16 * 16 + 5: return launch_cluster<16, 13, 4, MODE, D>(a, st, true);
    }
    return set_error(PG_ERR_INVALID_ARGUMENT, "no such NTT kernel variant for this ring degree");
}

}  // namespace

int run_ntt_shape_hi(const NttArgs& a, uint32_t log_n, int mode, int v, cudaStream_t st) {
    switch (mode) {
        case MODE_FWD: return run<MODE_FWD>(a, log_n, v, st);
        case MODE_INV: return run<MODE_INV>(a, log_n, v, st);
        case MODE_RT: return run<MODE_RT>(a, log_n, v, st);
    }
    return set_error(PG_ERR_INVALID_ARGUMENT, "bad NTT mode");
}

}  // namespace pg
