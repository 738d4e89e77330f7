// Internal declarations shared by the translation units of libprimus_gpu.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "primus_gpu.h"
#include "common.cuh"

namespace pg {

// ---- error handling: every entry point returns a status and records a message
int set_error(int status, const std::string& msg);
int cuda_status(cudaError_t err, const char* what);
void clear_error();
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ---- launch geometry for elementwise kernels
// 1D grid-stride launch: enough CTAs of `threads` for `work` items, at most 2048
// resident threads' worth per SM (148 SMs)
inline unsigned grid_for(size_t work, unsigned threads) {
    const size_t cap = 148ull * 2048 / threads;
    const size_t b = (work + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : (b < cap ? b : cap));
}
// 2D launch: x covers `inner` elements with 256 threads per CTA, y covers
// `outer` rows (polys, ciphertexts); both loop inside the kernel when capped
inline dim3 grid2(size_t inner, size_t outer) {
    size_t bx = (inner + 255) / 256, by = outer;
    bx = bx < 1 ? 1 : (bx > 4096 ? 4096 : bx);
    by = by < 1 ? 1 : (by > 65535 ? 65535 : by);
    return dim3((unsigned)bx, (unsigned)by);
}

// ---- scratch: stream-ordered allocations from a library-owned pool per device
// that keeps freed memory (release threshold = unlimited), so a call that needs
// scratch does not map fresh memory after every synchronize
cudaMemPool_t scratch_pool(int dev);
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st);
cudaError_t scratch_free(void* p, cudaStream_t st);

#define PG_CUDA(expr)                                              \
    do {                                                           \
        cudaError_t _e = (expr);                                   \
        if (_e != cudaSuccess) return ::pg::cuda_status(_e, #expr); \
    } while (0)

#define PG_LAUNCH_CHECK(what)                                        \
    do {                                                             \
        cudaError_t _e = cudaGetLastError();                         \
        if (_e != cudaSuccess) return ::pg::cuda_status(_e, what);   \
    } while (0)

// ---- host number theory (exact, unsigned __int128)
using u128 = unsigned __int128;
uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t h_invmod(uint64_t a, uint64_t q);
bool h_is_prime(uint64_t n);
inline uint64_t h_shoup_quotient(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }
inline uint64_t h_shoup_mul(uint64_t w, uint64_t wq, uint64_t b, uint64_t q) {
    uint64_t hw = (uint64_t)(((u128)wq * b) >> 64);
    uint64_t t = w * b - q * hw;
    return t >= q ? t - q : t;
}
Barrett h_barrett(uint64_t q);

// Host copy of one prime's tables (UintNttTable, primus_ntt/src/ntt/primitive.rs:34-46)
struct HostNttTable {
    uint64_t q = 0, root = 0, inv_root = 0, inv_n = 0, inv_n_q = 0;
    uint32_t log_n = 0;
    std::vector<uint64_t> root_powers, root_powers_q;          // [N] bit-reversed
    std::vector<uint64_t> inv_root_powers, inv_root_powers_q;  // [N] scrambled
    std::vector<uint64_t> ordinal, ordinal_q;                  // [2N]
};
int build_host_table(uint32_t log_n, uint64_t q, HostNttTable& t);

}  // namespace pg

// Device-resident table set for L primes of degree N = 2^log_n.
struct pg_ntt_table {
    uint32_t log_n = 0, L = 0;
    size_t n = 0;
    int device = 0;
    bool view = false;                 // device arrays belong to another table
    std::vector<uint64_t> moduli;
    std::vector<pg::HostNttTable> host;
    uint64_t* d_moduli = nullptr;      // [L]
    ulonglong2* d_fwd = nullptr;       // [L][N] (w, w') bit-reversed root powers
    ulonglong2* d_inv = nullptr;       // [L][N] (w, w') scrambled inverse powers, slot j = index j + 1
    ulonglong2* d_ordinal = nullptr;   // [L][2N] psi^k
    ulonglong2* d_inv_n = nullptr;     // [L] N^-1
    ulonglong2* d_inv_last = nullptr;  // [L] inv_root_powers[N-1] * N^-1
    pg::Barrett* d_barrett = nullptr;  // [L]
    // FP64-schedule copies of the four twiddle tables, allocated when every
    // modulus is below 2^50: the forward and inverse tables as w / q only (a
    // double per twiddle, w = rint(wq q) recovered in the kernels), the two
    // N^-1 factors as (w, w / q) pairs of doubles
    double* d_fwd_fp = nullptr;
    double* d_inv_fp = nullptr;
    ulonglong2* d_inv_n_fp = nullptr;
    ulonglong2* d_inv_last_fp = nullptr;
    int fp64 = 0;                       // FP64 schedule in use (tables present and not switched off)
    int variant[3] = {0, 0, 0};        // NTT kernel shape per mode (forward, inverse, round trip)
};

namespace pg {
// one row of a descriptor-driven (ragged) NTT launch: the row's data, its limb
// in the table and, for inverse launches, an optional NTT-domain multiplicand
// applied before the transform
struct RowDesc {
    uint64_t* data;
    uint64_t* mul;  // NTT-domain multiplicand (read); the pair form transforms it in place
    uint32_t limb;
    uint32_t pad;
};

// kernel argument block for the NTT family
struct NttArgs {
    uint64_t* data;
    const ulonglong2* fwd;
    const ulonglong2* inv;
    const uint64_t* moduli;
    const ulonglong2* inv_n;
    const ulonglong2* inv_last;
    const uint64_t* plain;
    const uint64_t* plain_q;
    const Barrett* bar;
    // FP64-schedule twiddles: w / q per twiddle (fwd, inv), (w, w / q) pairs (N^-1 factors)
    const double* fwd_fp;
    const double* inv_fp;
    const ulonglong2* inv_n_fp;
    const ulonglong2* inv_last_fp;
    const RowDesc* desc;  // NULL: rows are [polys][L][N] at data
    // forward launches only: when set, row pd * L + limb reads gadget digit row
    // pd ([N] words at lift_src + pd * N) and lifts each digit mod q_limb on the
    // fly (digit < lift_half stays, else q - lift_basis + digit), writing the
    // transform to data; NULL: rows are read from data
    const uint64_t* lift_src;
    uint64_t lift_basis, lift_half;
    uint64_t rows;
    uint64_t max_modulus;
    uint32_t L;
    int lazy;
    int variant[3];  // kernel shape per mode (0 = default), chosen by the autotuner
};

// MODE_PAIR (descriptor rows, block kernel, FP64 schedule): per row b <- NTT(b)
// and a <- INTT(NTT(a) * NTT(b)) in one pass, b being the descriptor's multiplicand
enum NttMode { MODE_FWD = 0, MODE_INV = 1, MODE_RT = 2, MODE_PAIR = 3 };

// one gadget digit's window in the BigUint value: bits [shr, ...) of limb
// `index`, continued by `mask1` bits of limb index + 1 when the digit straddles
struct DigitMask {
    uint32_t index, shr, shl, pad;
    uint64_t mask0, mask1;
};

// gadget decomposition parameters of a basis whose values fit one word (W = 1)
struct GadgetWord {
    uint64_t bm1, carry_mask, basis, split, npq, init_mask;
    int has_split, has_init;
    uint32_t d, log_basis;
    const DigitMask* masks;  // device [d]
};

// fused GLWE x GGSW external product for single-prime, single-word shapes
// (k = 1): decomposition, forward NTT of every digit row, MAC and optionally the
// inverse NTT of the outputs in one kernel, one CTA per ciphertext
bool ext_fused_eligible(const pg_ntt_table* t, const GadgetWord& gw, uint32_t k);
int launch_ext_fused(const pg_ntt_table* t, const GadgetWord& gw, const uint64_t* in, const uint64_t* key,
                     uint64_t* out, size_t batch, bool out_coeff, cudaStream_t st);

inline NttArgs make_args(const pg_ntt_table* t, uint64_t* data, uint64_t rows, int lazy) {
    NttArgs a{};
    a.data = data;
    a.fwd = t->d_fwd;
    a.inv = t->d_inv;
    a.moduli = t->d_moduli;
    a.inv_n = t->d_inv_n;
    a.inv_last = t->d_inv_last;
    a.plain = nullptr;
    a.plain_q = nullptr;
    a.bar = t->d_barrett;
    a.fwd_fp = t->fp64 ? t->d_fwd_fp : nullptr;  // null: integer schedules only
    a.inv_fp = t->d_inv_fp;
    a.inv_n_fp = t->d_inv_n_fp;
    a.inv_last_fp = t->d_inv_last_fp;
    a.desc = nullptr;
    a.lift_src = nullptr;
    a.lift_basis = a.lift_half = 0;
    a.rows = rows;
    a.max_modulus = 0;
    for (uint64_t m : t->moduli) a.max_modulus = m > a.max_modulus ? m : a.max_modulus;
    a.L = t->L;
    a.lazy = lazy;
    for (int m = 0; m < 3; ++m) a.variant[m] = t->variant[m];
    return a;
}

int launch_ntt(const NttArgs& a, uint32_t log_n, int mode, cudaStream_t stream);
// the pair form over descriptor rows (log_n <= kPairMaxLogN, every modulus below
// 2^50 with FP64 tables): one launch instead of a forward and an inverse one
constexpr uint32_t kPairMaxLogN = 12;
bool pair_ok(const NttArgs& a, uint32_t log_n);
int launch_pair(const NttArgs& a, uint32_t log_n, cudaStream_t stream);
// alternative kernel shapes (ntt_variants.cu): variant 1 .. ntt_variant_count(log_n) - 1
// of the canonical forward, the inverse and the round trip; identical results
int ntt_variant_count(uint32_t log_n);
const char* ntt_variant_name(uint32_t log_n, int variant);
bool ntt_variant_fp(uint32_t log_n, int variant);  // FP64 schedule: every q < 2^50
int launch_ntt_variant(const NttArgs& a, uint32_t log_n, int mode, int variant, cudaStream_t stream);

// hybrid key switch context accessors (Q limb count, ring degree)
uint32_t hybrid_q_limbs(const pg_hybrid_ks* ks);
size_t hybrid_n(const pg_hybrid_ks* ks);

// out[b][c] = base + sign * sum_{i < kin, j < d} key[i][j][c] (.) dig[b][i][j] over the
// table's L limbs (NTT domain, canonical); base = acc (accumulate) or, with
// negate, add_last on the last output poly.  With out_hi, limbs >= l_split are
// written to out_hi as [B][kout][L - l_split][N] and the rest to out as
// [B][kout][l_split][N].
int launch_mac(const pg_ntt_table* t, uint32_t d, uint64_t* out, const uint64_t* acc, const uint64_t* add_last,
               const uint64_t* key, const uint64_t* dig, size_t B, uint32_t kin, uint32_t kout, int negate,
               cudaStream_t st, uint64_t* out_hi = nullptr, uint32_t l_split = 0);
}  // namespace pg
