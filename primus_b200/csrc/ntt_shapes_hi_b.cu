// Kernel shapes the autotuner times for ring degree 2^16 (register budgets and
// the two-pipe kernel): the instantiations behind launch_ntt_variant
// (ntt_variants.cu), kept in a translation unit of their own so that the shape
// families compile in parallel.
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
        case 16 * 16 + 7: return launch_cluster<16, 12, 4, MODE, D, 3>(a, st);
        case 16 * 16 + 8: return launch_cluster<16, 12, 4, MODE, D, 5>(a, st);
        case 16 * 16 + 9: return launch_cluster<16, 12, 4, MODE, D, 0, 0x11>(a, st);
        case 16 * 16 + 10: return launch_cluster<16, 12, 4, MODE, D, 0, 0x4A>(a, st);
        case 16 * 16 + 11: return launch_cluster<16, 12, 4, MODE, D, 0, 0x55>(a, st);
        case 16 * 16 + 12: return launch_cluster<16, 12, 5, MODE, D, 4>(a, st);
        case 16 * 16 + 13: return launch_cluster<16, 12, 5, MODE, D, 5>(a, st);
        case 16 * 16 + 14: return launch_cluster<16, 12, 5, MODE, D, 6>(a, st);
        case 16 * 16 + 15: return launch_cluster<16, 13, 5, MODE, D, 3>(a, st);
    }
    return set_error(PG_ERR_INVALID_ARGUMENT, "no such NTT kernel variant for this ring degree");
}

}  // namespace

int run_ntt_shape_hi_b(const NttArgs& a, uint32_t log_n, int mode, int v, cudaStream_t st) {
    switch (mode) {
        case MODE_FWD: return run<MODE_FWD>(a, log_n, v, st);
        case MODE_INV: return run<MODE_INV>(a, log_n, v, st);
        case MODE_RT: return run<MODE_RT>(a, log_n, v, st);
    }
    return set_error(PG_ERR_INVALID_ARGUMENT, "bad NTT mode");
}

}  // namespace pg
