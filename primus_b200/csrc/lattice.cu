// GLev multiply-accumulate, GLWE x GGSW external product and RNS key switch.
//
//   DcrtGlwe::add_dcrt_glev_mul_crt_poly_assign     primus_lattice/src/glwe/dcrt.rs:170-247
//   DcrtGlwe::add_dcrt_glev_mul_big_uint_poly_assign primus_lattice/src/glwe/dcrt.rs:249-325
//   CrtGlwe::mul_dcrt_ggsw_inplace                  primus_lattice/src/glwe/crt.rs:202-229
//   CrtGlweKeySwitchingKey::key_swithching_inplace  primus_fhe_core/src/key_switch.rs:79-128
//
// Layouts (all uint64, limb-major polys [L][N]):
//   GLWE  = (k+1) polys [a_1 .. a_k, b]             (glwe/dcrt.rs:19-27)
//   GLev  = d GLWEs, one per gadget digit            (glev/dcrt.rs:16-24)
//   GGSW  = (k+1) GLevs, one per input component     (ggsw/dcrt.rs:10-21)
//   key-switching key = k_in GLevs over k_out+1 output polys (key_switch.rs:17-24)
//
// Batched pipeline (one launch per step for the whole batch): CRT compose of
// every input poly -> signed gadget digits -> forward NTT of every digit row
// lifted into each limb of the RNS base as the transform loads it -> one
// multiply-accumulate kernel that forms every
// output coefficient as sum_{i,j} key[i][j][c] * digit[i][j] with a 128-bit
// accumulator.  Outputs are canonical NTT-domain residues, equal to the
// reference's sequential per-digit MAC.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

#include "internal.hpp"

namespace pg {
uint32_t rns_L(const pg_rns_base* b);
uint32_t rns_W(const pg_rns_base* b);
const uint64_t* rns_moduli(const pg_rns_base* b);
const pg_rns_base* gadget_base(const pg_gadget_basis* g);
uint32_t gadget_d(const pg_gadget_basis* g);
uint64_t gadget_basis_value(const pg_gadget_basis* g);
bool gadget_word(const pg_gadget_basis* g, GadgetWord* out);
int launch_compose(const pg_rns_base* b, const uint64_t* res, uint64_t* out, size_t count, size_t n, uint32_t ppg,
                   size_t group_stride, cudaStream_t st);
int launch_gadget(const pg_gadget_basis* g, const uint64_t* vals, uint64_t* out, size_t count, size_t n, bool lift,
                  cudaStream_t st);
}  // namespace pg

using namespace pg;

namespace {

PG_DEV void mac128(uint64_t& lo, uint64_t& hi, uint64_t a, uint64_t b) {
    uint64_t pl = a * b, ph = mulhi64(a, b);
    lo += pl;
    hi += ph + (lo < pl);
}

// out[b][c][l][x] = base + sign * sum_{i<KIN, j<d} key[i][j][c][l][x] * dig[b][i][j][l][x]
//   base = acc[b][c][l][x] (accumulate form) or, for the key switch,
//   add_last[b][l][x] on the last component and 0 elsewhere; sign = -1 there.
struct MacArgs {
    uint64_t* out;
    const uint64_t* acc;       // may alias out, or NULL
    const uint64_t* add_last;  // [B][L][N] or NULL
    const uint64_t* key;       // [KIN][d][KOUT][L][N]
    const uint64_t* dig;       // [B][KIN][d][L][N]
    const Barrett* bar;        // [L]
    uint64_t* out_hi;          // optional: limbs >= l_split go to [B][KOUT][L - l_split][N] here
    size_t B, N;
    uint32_t KIN, KOUT, d, L, log_n, l_split;
    int negate;
};

// One thread per (chunk of kMacChunk ciphertexts -- one for a single ciphertext
// --, pair of output polys, limb l, coefficient x); lanes run over consecutive
// coefficients (coalesced).  Each
// digit element is loaded once for both output polys of the pair and each key
// element once for the whole chunk, so a batch reads the digits once per pair
// of output polys and the key ceil(B / kMacChunk) times.  Grid: x over
// (chunk, output pair), y over 256-coefficient tiles (32-bit index).
constexpr uint32_t kMacChunk = 4;
constexpr uint32_t kMacOut = 2;

// NEG: the key-switch form (base - sum, base = add_last on the last output); SPLIT:
// limbs >= l_split written to out_hi (hybrid key switch).  Compile-time, so that
// each launch carries only its own epilogue.
template <bool FOLD, bool NEG, bool SPLIT, uint32_t CHUNK>
__global__ void __launch_bounds__(256, CHUNK == 1 ? 4 : 3) mac_kernel(MacArgs a) {
    // terms whose key and digit loads are issued together: each thread has few
    // terms (4 for a hybrid key switch), so one load round per term would leave
    // the kernel waiting on memory latency instead of bandwidth
    constexpr uint32_t U = CHUNK == 1 ? 4 : 1;
    const uint32_t LN = a.L * (uint32_t)a.N;
    const uint32_t pairs = (a.KOUT + kMacOut - 1) / kMacOut;
    const size_t outer = ((a.B + CHUNK - 1) / CHUNK) * pairs;
    const size_t kstride = (size_t)a.KOUT * LN;
    const size_t dstride = (size_t)a.KIN * a.d * LN;  // one ciphertext's digits
    const uint32_t nterms = a.KIN * a.d;
    // grid x runs over (chunk, output pair) and y over coefficient tiles: CTAs
    // launched next to each other share one tile of the key, which then comes
    // from L2 for every chunk after the first
    for (uint32_t lx0 = blockIdx.y * blockDim.x; lx0 < LN; lx0 += gridDim.y * blockDim.x) {
        const uint32_t lx = lx0 + threadIdx.x;
        if (lx >= LN) break;
        const uint32_t l = lx >> a.log_n;
        const Barrett m = a.bar[l];
        for (size_t o = blockIdx.x; o < outer; o += gridDim.x) {
            const uint32_t c0 = (uint32_t)(o % pairs) * kMacOut;
            const uint32_t nc = min(kMacOut, a.KOUT - c0);
            const size_t b0 = (o / pairs) * CHUNK;
            const uint32_t nb = (uint32_t)min((size_t)CHUNK, a.B - b0);
            uint64_t lo[kMacOut][CHUNK], hi[kMacOut][CHUNK];
#pragma unroll
            for (uint32_t cc = 0; cc < kMacOut; ++cc)
#pragma unroll
                for (uint32_t bb = 0; bb < CHUNK; ++bb) lo[cc][bb] = hi[cc][bb] = 0;
            const uint64_t* kp = a.key + (size_t)c0 * LN + lx;
            const uint64_t* dp = a.dig + b0 * dstride + lx;
            for (uint32_t ij0 = 0; ij0 < nterms; ij0 += U) {
                uint64_t kv[U][kMacOut], dv[U][CHUNK];
#pragma unroll
                for (uint32_t u = 0; u < U; ++u) {
                    const uint32_t ij = ij0 + u;
                    const bool live = ij < nterms;
#pragma unroll
                    for (uint32_t cc = 0; cc < kMacOut; ++cc)
                        kv[u][cc] = live && cc < nc ? __ldg(kp + ij * kstride + cc * LN) : 0;
#pragma unroll
                    for (uint32_t bb = 0; bb < CHUNK; ++bb)
                        dv[u][bb] = live && bb < nb ? __ldg(dp + bb * dstride + ij * LN) : 0;
                }
#pragma unroll
                for (uint32_t u = 0; u < U; ++u) {
                    const uint32_t ij = ij0 + u;
                    if (ij >= nterms) break;
                    if (FOLD && ij && (ij & 7) == 0) {  // products < 2^124: fold before the sum can reach 2^128
#pragma unroll
                        for (uint32_t cc = 0; cc < kMacOut; ++cc)
#pragma unroll
                            for (uint32_t bb = 0; bb < CHUNK; ++bb) {
                                lo[cc][bb] = barrett_reduce_128(lo[cc][bb], hi[cc][bb], m);
                                hi[cc][bb] = 0;
                            }
                    }
#pragma unroll
                    for (uint32_t cc = 0; cc < kMacOut; ++cc)
#pragma unroll
                        for (uint32_t bb = 0; bb < CHUNK; ++bb)
                            if (bb < nb) mac128(lo[cc][bb], hi[cc][bb], kv[u][cc], dv[u][bb]);  // nb is uniform per CTA
                }
            }
#pragma unroll
            for (uint32_t cc = 0; cc < kMacOut; ++cc) {
                if (cc >= nc) break;
                const uint32_t c = c0 + cc;
#pragma unroll
                for (uint32_t bb = 0; bb < CHUNK; ++bb) {
                    if (bb >= nb) break;
                    const size_t b = b0 + bb;
                    const size_t bc = b * a.KOUT + c;
                    const uint64_t s = barrett_reduce_128(lo[cc][bb], hi[cc][bb], m);
                    uint64_t r;
                    if constexpr (NEG) {
                        const uint64_t base = (a.add_last && c == a.KOUT - 1) ? a.add_last[b * LN + lx] : 0;
                        r = sub_mod(base, s, m.q);
                    } else {
                        const uint64_t base = a.acc ? a.acc[bc * LN + lx] : 0;
                        r = add_mod(base, s, m.q);
                    }
                    if constexpr (SPLIT) {  // split output: [B][KOUT][l_split][N] and [B][KOUT][L - l_split][N]
                        const bool lo_part = l < a.l_split;
                        uint64_t* dst = lo_part ? a.out : a.out_hi;
                        const size_t limbs = lo_part ? a.l_split : a.L - a.l_split;
                        const uint32_t lrow = lo_part ? l : l - a.l_split;
                        dst[(bc * limbs + lrow) * a.N + (lx & ((uint32_t)a.N - 1))] = r;
                    } else {
                        a.out[bc * LN + lx] = r;
                    }
                }
            }
        }
    }
}

// NTT-domain automorphism X -> X^degree (generate_ntt_permutation,
// primus_fhe_core/src/automorphism/glwe/dcrt.rs:43-63): bit-reversed slot d
// holds the evaluation at psi^(2 rev(d) + 1); the result's slot d takes the
// input's slot rev(((degree (2 rev(d) + 1) mod 2N) - 1) / 2).  Grid: y over the
// (k+1) polys of each ciphertext, x over their L*N residues; the k masks go to
// out_a, the body to out_b.
__global__ void __launch_bounds__(256) auto_perm_kernel(const uint64_t* __restrict__ in, uint64_t* out_a,
                                                        uint64_t* out_b, size_t batch, uint32_t k, uint32_t L,
                                                        uint32_t log_n, uint64_t degree) {
    const uint32_t N = 1u << log_n, LN = L << log_n;
    const size_t outer = batch * (k + 1);
    for (size_t o = blockIdx.y; o < outer; o += gridDim.y) {
        const size_t b = o / (k + 1);
        const uint32_t c = (uint32_t)(o % (k + 1));
        const uint64_t* src = in + o * LN;
        uint64_t* dst = c < k ? out_a + (b * k + c) * LN : out_b + b * LN;
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < LN; lx += gridDim.x * blockDim.x) {
            const uint32_t d = lx & (N - 1);
            const uint32_t i = __brev(d) >> (32 - log_n);
            const uint64_t j = (degree * (2ull * i + 1)) & (2ull * N - 1);
            const uint32_t from = __brev((uint32_t)((j - 1) >> 1)) >> (32 - log_n);
            dst[lx] = src[(lx - d) + from];
        }
    }
}



int check_compat(const pg_ntt_table* t, const pg_gadget_basis* g) {
    if (!t || !g) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL table or basis");
    const pg_rns_base* b = gadget_base(g);
    if (rns_L(b) != t->L) return set_error(PG_ERR_INVALID_ARGUMENT, "table and RNS base have different moduli counts");
    const uint64_t* m = rns_moduli(b);
    for (uint32_t l = 0; l < t->L; ++l)
        if (m[l] != t->moduli[l]) return set_error(PG_ERR_INVALID_ARGUMENT, "table and RNS base moduli differ");
    if (t->log_n > 16) return set_error(PG_ERR_UNSUPPORTED, "ring degree above 2^16");
    return PG_OK;
}

// workspace: BigUint values [P][N][W] + digits [P][d][N] + NTT-domain digit
// rows [P][d][L][N] (+ extra).
// Every product and sum is overflow-checked: a size that does not fit size_t
// returns SIZE_MAX, which no workspace, pool or fixed array satisfies, so a
// huge batch is refused on the host instead of wrapping to a small size.
size_t ws_bytes(const pg_ntt_table* t, const pg_gadget_basis* g, size_t polys, size_t extra_words) {
    const pg_rns_base* b = gadget_base(g);
    size_t per = 0, words = 0, bytes = 0;
    // words per poly: N * W (BigUint values) + d * N (digits) + d * L * N (digit
    // rows); (N <= 2^16, W <= 64 limbs, d <= 4096 digits, L <= 64 moduli: below 2^36)
    const size_t per_poly = t->n * rns_W(b) + (size_t)gadget_d(g) * t->n + (size_t)gadget_d(g) * t->L * t->n;
    if (__builtin_mul_overflow(polys, per_poly, &per)) return SIZE_MAX;
    if (__builtin_add_overflow(per, extra_words, &words)) return SIZE_MAX;
    if (__builtin_mul_overflow(words, sizeof(uint64_t), &bytes)) return SIZE_MAX;
    if (__builtin_add_overflow(bytes, (size_t)256, &bytes)) return SIZE_MAX;
    return bytes;
}

// checked a * b for the callers' extra-word counts (SIZE_MAX on overflow)
size_t mul_sat(size_t a, size_t b) {
    size_t r = 0;
    return __builtin_mul_overflow(a, b, &r) ? SIZE_MAX : r;
}

struct Workspace {
    void* ptr = nullptr;
    bool owned = false;
    cudaStream_t st = 0;
    ~Workspace() {
        if (owned && ptr) scratch_free(ptr, st);
    }
};

int get_workspace(Workspace& w, void* given, size_t given_bytes, size_t need, cudaStream_t st) {
    w.st = st;
    if (given) {
        if (given_bytes < need) return set_error(PG_ERR_INVALID_ARGUMENT, "workspace too small");
        w.ptr = given;
        return PG_OK;
    }
    cudaError_t e = scratch_alloc(&w.ptr, need, st);
    if (e != cudaSuccess) return cuda_status(e, "workspace allocation");
    w.owned = true;
    return PG_OK;
}

// compose (when the input is CRT residues) + signed gadget digits + forward NTT
// of every digit row lifted into every limb; returns the NTT-domain digit rows
// [P][d][L][N] inside the workspace.  The digits are written once per
// coefficient ([P][d][N]) and the forward NTT lifts them mod each q_l as it
// loads them, so the L-fold lifted rows never pass through HBM before the
// transform.
int digits_pipeline(const pg_ntt_table* t, const pg_gadget_basis* g, const uint64_t* in, bool in_is_crt,
                    size_t polys, uint32_t ppg, size_t group_stride, uint64_t* ws, uint64_t** digits_out,
                    cudaStream_t st) {
    const pg_rns_base* b = gadget_base(g);
    const size_t n = t->n;
    const size_t count = polys * n;
    const uint32_t d = gadget_d(g);
    uint64_t* big = ws;
    uint64_t* small = ws + count * rns_W(b);
    uint64_t* dig = small + count * d;
    const uint64_t* vals = in;
    if (in_is_crt) {
        int rc = launch_compose(b, in, big, count, n, ppg, group_stride, st);
        if (rc) return rc;
        vals = big;
    }
    int rc = launch_gadget(g, vals, small, count, n, false, st);
    if (rc) return rc;
    NttArgs a = make_args(t, dig, polys * d * (size_t)t->L, 0);
    a.lift_src = small;
    a.lift_basis = gadget_basis_value(g);
    a.lift_half = a.lift_basis == 2 ? 2 : (a.lift_basis + 1) / 2;
    rc = launch_ntt(a, t->log_n, MODE_FWD, st);
    if (rc) return rc;
    *digits_out = dig;
    return PG_OK;
}

}  // namespace

namespace {
template <uint32_t CHUNK>
void launch_mac_t(const MacArgs& a, uint32_t kout, size_t LN, bool fold, bool split, bool negate, cudaStream_t st) {
    const size_t outer = ((a.B + CHUNK - 1) / CHUNK) * ((kout + kMacOut - 1) / kMacOut);
    const dim3 grid((unsigned)std::min<size_t>(outer, 0x7fffffff),
                    (unsigned)std::min<size_t>((LN + 255) / 256, 65535));
    if (split) {
        fold ? mac_kernel<true, false, true, CHUNK><<<grid, 256, 0, st>>>(a)
             : mac_kernel<false, false, true, CHUNK><<<grid, 256, 0, st>>>(a);
    } else if (negate) {
        fold ? mac_kernel<true, true, false, CHUNK><<<grid, 256, 0, st>>>(a)
             : mac_kernel<false, true, false, CHUNK><<<grid, 256, 0, st>>>(a);
    } else {
        fold ? mac_kernel<true, false, false, CHUNK><<<grid, 256, 0, st>>>(a)
             : mac_kernel<false, false, false, CHUNK><<<grid, 256, 0, st>>>(a);
    }
}
}  // namespace

int pg::launch_mac(const pg_ntt_table* t, uint32_t d, uint64_t* out, const uint64_t* acc, const uint64_t* add_last,
                   const uint64_t* key, const uint64_t* dig, size_t B, uint32_t kin, uint32_t kout, int negate,
                   cudaStream_t st, uint64_t* out_hi, uint32_t l_split) {
    MacArgs a{};
    a.out_hi = out_hi;
    a.l_split = l_split;
    a.out = out;
    a.acc = acc;
    a.add_last = add_last;
    a.key = key;
    a.dig = dig;
    a.bar = t->d_barrett;
    a.B = B;
    a.N = t->n;
    a.KIN = kin;
    a.KOUT = kout;
    a.d = d;
    a.L = t->L;
    a.log_n = t->log_n;
    a.negate = negate;
    if ((size_t)t->L * t->n > 0xffffffffull) return set_error(PG_ERR_UNSUPPORTED, "poly too large");
    const size_t LN = (size_t)t->L * t->n;
    const bool fold = kin * d > 8;  // more than 8 products per output: fold the 128-bit sums every 8
    if (out_hi && negate) return set_error(PG_ERR_INVALID_ARGUMENT, "split MAC output has no key-switch form");
    // one ciphertext: the single-ciphertext form (fewer registers, more terms' loads in flight)
    if (B == 1) {
        launch_mac_t<1>(a, kout, LN, fold, out_hi != nullptr, negate != 0, st);
    } else {
        launch_mac_t<kMacChunk>(a, kout, LN, fold, out_hi != nullptr, negate != 0, st);
    }
    count_launch();
    PG_LAUNCH_CHECK("mac_kernel launch");
    return PG_OK;
}

namespace {


constexpr size_t kExtFusedMinBatch = 64;

// GLWE x GGSW for a batch: the fused one-kernel form where the shape allows it
// (k = 1, one prime, single-word values, N = 2^10..2^12), else the pipeline of
// compose -> lifted digits -> batched NTT -> MAC (-> inverse NTT of the outputs)
int ext_product(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, const uint64_t* d_in,
                const uint64_t* d_ggsw, uint64_t* d_out, size_t batch, void* d_ws, size_t ws_size, cudaStream_t st,
                bool out_coeff) {
    GadgetWord gw;
    // the fused kernel reads key rows and writes outputs with 16-byte vector accesses
    const bool aligned = ((uintptr_t)d_ggsw % 16 == 0) && ((uintptr_t)d_out % 16 == 0);
    // one CTA per ciphertext: small batches leave most SMs idle, and the
    // pipeline's per-digit parallelism finishes them sooner
    if (batch >= kExtFusedMinBatch && aligned && gadget_word(g, &gw) && ext_fused_eligible(t, gw, k))
        return launch_ext_fused(t, gw, d_in, d_ggsw, d_out, batch, out_coeff, st);
    const size_t polys = batch * (k + 1);
    Workspace w;
    int rc = get_workspace(w, d_ws, ws_size, ws_bytes(t, g, mul_sat(batch, k + 1), 0), st);
    if (rc) return rc;
    uint64_t* dig = nullptr;
    rc = digits_pipeline(t, g, d_in, true, polys, k + 1, (size_t)(k + 1) * t->L * t->n, (uint64_t*)w.ptr, &dig, st);
    if (rc) return rc;
    rc = launch_mac(t, gadget_d(g), d_out, nullptr, nullptr, d_ggsw, dig, batch, k + 1, k + 1, 0, st);
    if (rc || !out_coeff) return rc;
    return launch_ntt(make_args(t, d_out, polys * t->L, 0), t->log_n, MODE_INV, st);
}

// ---------------------------------------------------------------------------
// External product without any device allocation.
//
// Some callers cannot allocate device memory at the moment they call: hosts
// that only receive device pointers from another runtime and hold no CUDA
// allocator of their own (FFI wrappers around buffers someone else owns), and
// serving processes that reserve their HBM budget at start-up and forbid
// allocations afterwards, because cudaMalloc / cudaFree synchronize the device
// and can fail under memory pressure in the middle of a request.  For them the
// scratch of the external product lives in the file-scope array below: a fixed
// 32 MiB that every GPU which loads this library holds until the process exits.
// Host code cannot use the array's name as a device address (it is a host-side
// stand-in), so the device address is fetched once per device with
// cudaGetSymbolAddress, with that device current.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = 32ull << 20;
static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocScratchBytes / sizeof(uint64_t)];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[128] = {};

// device address of g_noalloc_scratch on the current device (set up on first use)
static int noalloc_scratch(void** out) {
    int dev = 0;
    PG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return set_error(PG_ERR_UNSUPPORTED, "device ordinal above 127");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return PG_OK;
}
}  // namespace

extern "C" {

size_t pg_ext_product_workspace_size(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, size_t batch) {
    if (!t || !g) return 0;
    return ws_bytes(t, g, mul_sat(batch, k + 1), 0);
}

int pg_ext_product(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, const uint64_t* d_in,
                   const uint64_t* d_ggsw, uint64_t* d_out, size_t batch, void* d_ws, size_t ws_size, void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (batch == 0) return PG_OK;
    if (!d_in || !d_ggsw || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    return ext_product(t, g, k, d_in, d_ggsw, d_out, batch, d_ws, ws_size, (cudaStream_t)stream, false);
}

int pg_ext_product_coeff(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, const uint64_t* d_in,
                         const uint64_t* d_ggsw, uint64_t* d_out, size_t batch, void* d_ws, size_t ws_size,
                         void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (batch == 0) return PG_OK;
    if (!d_in || !d_ggsw || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    return ext_product(t, g, k, d_in, d_ggsw, d_out, batch, d_ws, ws_size, (cudaStream_t)stream, true);
}

int pg_glev_mac_crt_poly(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, uint64_t* d_acc,
                         const uint64_t* d_glev, const uint64_t* d_crt_poly, void* d_ws, size_t ws_size,
                         void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (!d_acc || !d_glev || !d_crt_poly) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t st = (cudaStream_t)stream;
    Workspace w;
    rc = get_workspace(w, d_ws, ws_size, ws_bytes(t, g, 1, 0), st);
    if (rc) return rc;
    uint64_t* dig = nullptr;
    rc = digits_pipeline(t, g, d_crt_poly, true, 1, 1, (size_t)t->L * t->n, (uint64_t*)w.ptr, &dig, st);
    if (rc) return rc;
    return launch_mac(t, gadget_d(g), d_acc, d_acc, nullptr, d_glev, dig, 1, 1, k + 1, 0, st);
}

int pg_glev_mac_big_uint_poly(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, uint64_t* d_acc,
                              const uint64_t* d_glev, const uint64_t* d_big_poly, void* d_ws, size_t ws_size,
                              void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (!d_acc || !d_glev || !d_big_poly) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t st = (cudaStream_t)stream;
    Workspace w;
    rc = get_workspace(w, d_ws, ws_size, ws_bytes(t, g, 1, 0), st);
    if (rc) return rc;
    uint64_t* dig = nullptr;
    rc = digits_pipeline(t, g, d_big_poly, false, 1, 1, 0, (uint64_t*)w.ptr, &dig, st);
    if (rc) return rc;
    return launch_mac(t, gadget_d(g), d_acc, d_acc, nullptr, d_glev, dig, 1, 1, k + 1, 0, st);
}

size_t pg_key_switch_workspace_size(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k_in, uint32_t k_out,
                                    size_t batch) {
    (void)k_out;
    if (!t || !g) return 0;
    return ws_bytes(t, g, mul_sat(batch, k_in), mul_sat(batch, (size_t)t->L * t->n));
}

int pg_key_switch(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k_in, uint32_t k_out,
                  const uint64_t* d_key, const uint64_t* d_in, uint64_t* d_out, size_t batch, void* d_ws,
                  size_t ws_size, void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (batch == 0) return PG_OK;
    if (!d_key || !d_in || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (k_in == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k_in must be at least 1");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t LN = (size_t)t->L * t->n;
    const size_t polys = batch * k_in;
    Workspace w;
    rc = get_workspace(w, d_ws, ws_size, ws_bytes(t, g, mul_sat(batch, k_in), mul_sat(batch, LN)), st);
    if (rc) return rc;
    uint64_t* ws = (uint64_t*)w.ptr;
    uint64_t* dig = nullptr;
    rc = digits_pipeline(t, g, d_in, true, polys, k_in, (size_t)(k_in + 1) * LN, ws, &dig, st);
    if (rc) return rc;
    // b of every input, moved to the NTT domain (key_switch.rs:118-121)
    uint64_t* bt = dig + polys * gadget_d(g) * LN;
    PG_CUDA(cudaMemcpy2DAsync(bt, LN * 8, d_in + (size_t)k_in * LN, (size_t)(k_in + 1) * LN * 8, LN * 8, batch,
                              cudaMemcpyDeviceToDevice, st));
    rc = launch_ntt(make_args(t, bt, batch * t->L, 0), t->log_n, MODE_FWD, st);
    if (rc) return rc;
    // c_out = -(sum_i GLev_i (x) a_i) + (0, .., NTT(b))  (key_switch.rs:96-127)
    return launch_mac(t, gadget_d(g), d_out, nullptr, bt, d_key, dig, batch, k_in, k_out + 1, 1, st);
}

size_t pg_glwe_automorphism_workspace_size(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k,
                                           size_t batch) {
    if (!t || !g) return 0;
    return ws_bytes(t, g, mul_sat(batch, k), mul_sat(batch, (k + 1) * (size_t)t->L * t->n));
}

// DcrtGlweAutoKey::automorphism_inplace (primus_fhe_core/src/automorphism/glwe/dcrt.rs:269-331):
// permute every poly in the NTT domain, inverse-transform the masks, then the
// key-switch MAC with the permuted body added on the last output poly:
// c_out = -(sum_i key_i (x) sigma(a_i)) + (0, .., sigma(b)).
int pg_glwe_automorphism(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, uint64_t degree,
                         const uint64_t* d_key, const uint64_t* d_in, uint64_t* d_out, size_t batch, void* d_ws,
                         size_t ws_size, void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (batch == 0) return PG_OK;
    if (!d_key || !d_in || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (k == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k must be at least 1");
    if ((degree & 1) == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "automorphism degree must be odd");
    if (d_in == d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "input and output must not overlap");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t LN = (size_t)t->L * t->n;
    Workspace w;
    rc = get_workspace(w, d_ws, ws_size, pg_glwe_automorphism_workspace_size(t, g, k, batch), st);
    if (rc) return rc;
    uint64_t* pa = (uint64_t*)w.ptr;        // [batch][k][L][N] permuted masks
    uint64_t* pb = pa + batch * k * LN;     // [batch][L][N] permuted bodies
    uint64_t* ws = pb + batch * LN;         // digits pipeline scratch
    auto_perm_kernel<<<grid2(LN, batch * (k + 1)), 256, 0, st>>>(d_in, pa, pb, batch, k, t->L, t->log_n,
                                                                 degree & (2 * t->n - 1));
    count_launch();
    PG_LAUNCH_CHECK("auto_perm_kernel launch");
    rc = launch_ntt(make_args(t, pa, batch * k * t->L, 0), t->log_n, MODE_INV, st);
    if (rc) return rc;
    uint64_t* dig = nullptr;
    rc = digits_pipeline(t, g, pa, true, batch * k, k, (size_t)k * LN, ws, &dig, st);
    if (rc) return rc;
    return launch_mac(t, gadget_d(g), d_out, nullptr, pb, d_key, dig, batch, k, k + 1, 1, st);
}

// Same computation and outputs as pg_ext_product, without any device
// allocation.  The shapes the fused kernel takes (k = 1, one prime, single-word
// gadget values, N = 2^10..2^12, at least kExtFusedMinBatch ciphertexts) run
// there and use no scratch at all, so their batch is bounded only by one
// launch; every other shape runs the pipeline with its scratch in the
// library's fixed device array and is refused, before anything is launched,
// when that array is too small.
int pg_ext_product_noalloc(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, const uint64_t* d_in,
                           const uint64_t* d_ggsw, uint64_t* d_out, size_t batch, void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (batch == 0) return PG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    GadgetWord gw;
    const bool aligned = ((uintptr_t)d_ggsw % 16 == 0) && ((uintptr_t)d_out % 16 == 0);
    const bool fused = batch >= kExtFusedMinBatch && aligned && gadget_word(g, &gw) && ext_fused_eligible(t, gw, k);
    if (!fused) {
        // the size check comes first, so that an oversized batch is refused on
        // the host whatever the buffers are
        const size_t need = ws_bytes(t, g, mul_sat(batch, k + 1), 0);
        if (need > kNoAllocScratchBytes) {
            // ws_bytes adds one fixed 256-byte pad per call: the largest batch b
            // has b * (per - 256) + 256 <= the array
            const size_t per = ws_bytes(t, g, (size_t)(k + 1), 0);
            const size_t max_batch = per > 256 ? (kNoAllocScratchBytes - 256) / (per - 256) : 0;
            char buf[320];
            snprintf(buf, sizeof buf,
                     "pg_ext_product_noalloc: this batch needs %s bytes of scratch, above the fixed %zu bytes; "
                     "submit at most %zu ciphertexts of this shape per call",
                     need == SIZE_MAX ? "more than SIZE_MAX" : std::to_string(need).c_str(), kNoAllocScratchBytes,
                     max_batch);
            return set_error(PG_ERR_UNSUPPORTED, buf);
        }
    }
    if (!d_in || !d_ggsw || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (fused) return launch_ext_fused(t, gw, d_in, d_ggsw, d_out, batch, false, st);
    void* ws = nullptr;
    rc = noalloc_scratch(&ws);
    if (rc) return rc;
    uint64_t* dig = nullptr;
    rc = digits_pipeline(t, g, d_in, true, batch * (k + 1), k + 1, (size_t)(k + 1) * t->L * t->n, (uint64_t*)ws,
                         &dig, st);
    if (rc) return rc;
    return launch_mac(t, gadget_d(g), d_out, nullptr, nullptr, d_ggsw, dig, batch, k + 1, k + 1, 0, st);
}

}  // extern "C"

// ---- field trace and coefficient expansion: sums of automorphisms
// (primus_fhe_core/src/trace, primus_fhe_core/src/expand_coeff)
namespace {

// one automorphism key: k GLevs [k][d][k+1][L][N]
size_t auto_key_words(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k) {
    return (size_t)k * gadget_d(g) * (k + 1) * t->L * t->n;
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// ciphertexts per automorphism call inside an expansion level, bounding the
// workspace of the late levels (2^i ciphertexts each)
constexpr size_t kExpandChunk = 256;

size_t expand_chunk(size_t count) { return std::max<size_t>(1, std::min(count / 2, kExpandChunk)); }

bool ranges_overlap(const uint64_t* a, size_t na, const uint64_t* b, size_t nb) { return a < b + nb && b < a + na; }

}  // namespace

extern "C" {

size_t pg_glwe_trace_workspace_size(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, size_t batch) {
    if (!t || !g) return 0;
    const size_t sums = mul_sat(mul_sat(batch, (k + 1) * (size_t)t->L * t->n), sizeof(uint64_t));
    const size_t autos = pg_glwe_automorphism_workspace_size(t, g, k, batch);
    // saturate: a batch whose size does not fit size_t gets SIZE_MAX, which no workspace satisfies
    if (sums > SIZE_MAX / 2 || autos > SIZE_MAX / 2) return SIZE_MAX;
    return round256(sums) + autos;
}

// DcrtGlweTraceKey::trace_inplace (primus_fhe_core/src/trace/glwe/dcrt.rs:84-108):
// out = in, then out += sigma_d(out) for d = N+1, N/2+1, .., 3; with reverse,
// DcrtGlweRevTraceKey::trace_inplace (trace/glwe/rev.rs:79-115): d = 3, 5, ..,
// N+1 and out *= 2^-1 before each automorphism.  Each step is one batched
// automorphism and one batched add over every ciphertext.
int pg_glwe_trace(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, const uint64_t* d_keys, int reverse,
                  const uint64_t* d_in, uint64_t* d_out, size_t batch, void* d_ws, size_t ws_size, void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (batch == 0) return PG_OK;
    if (!d_keys || !d_in || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (k == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k must be at least 1");
    const size_t glwe = (size_t)(k + 1) * t->L * t->n, polys = batch * (k + 1);
    if (d_in != d_out && ranges_overlap(d_in, batch * glwe, d_out, batch * glwe))
        return set_error(PG_ERR_INVALID_ARGUMENT, "input and output must be the same buffer or not overlap");
    cudaStream_t st = (cudaStream_t)stream;
    Workspace w;
    rc = get_workspace(w, d_ws, ws_size, pg_glwe_trace_workspace_size(t, g, k, batch), st);
    if (rc) return rc;
    uint64_t* tmp = (uint64_t*)w.ptr;
    void* aws = (char*)w.ptr + round256(batch * glwe * 8);
    const size_t aws_size = pg_glwe_automorphism_workspace_size(t, g, k, batch);
    if (d_in != d_out) PG_CUDA(cudaMemcpyAsync(d_out, d_in, batch * glwe * 8, cudaMemcpyDeviceToDevice, st));
    std::vector<uint64_t> half(t->L);
    for (uint32_t l = 0; l < t->L; ++l) half[l] = (t->moduli[l] + 1) >> 1;  // 2^-1 mod q_l (rev.rs:47-53)
    const size_t kw = auto_key_words(t, g, k);
    for (uint32_t r = 0; r < t->log_n; ++r) {
        const uint64_t degree = reverse ? ((uint64_t)2 << r) + 1 : (uint64_t)(t->n >> r) + 1;
        if (reverse && (rc = pg_dcrt_mul_scalar(t, d_out, half.data(), polys, stream))) return rc;
        rc = pg_glwe_automorphism(t, g, k, degree, d_keys + r * kw, d_out, tmp, batch, aws, aws_size, stream);
        if (rc) return rc;
        rc = pg_dcrt_add(t, d_out, tmp, polys, polys, stream);
        if (rc) return rc;
    }
    return PG_OK;
}

size_t pg_glwe_expand_workspace_size(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, size_t count) {
    if (!t || !g) return 0;
    const size_t c = expand_chunk(count), LN = (size_t)t->L * t->n;
    return round256(c * (k + 1) * LN * 8) + round256(2 * LN * 8) + pg_glwe_automorphism_workspace_size(t, g, k, c);
}

// DcrtGlweExpandCoeffKey::expand_partial_coefficients_inplace
// (primus_fhe_core/src/expand_coeff/glwe/dcrt.rs:235-287): out[0] = in *
// count^-1 (:209-232); level i < log2(count) applies the key of degree
// N/2^i + 1 to out[0 .. 2^i) as batched automorphisms (at most 256 per call)
// and one batched butterfly (out[j], out[j + 2^i]) = (a + sigma(a),
// (a - sigma(a)) * NTT(X^(2N - 2^i))) (:181-207).  The reference's levels
// run their 2^i pairs one by one on rayon workers (:341-412); here each level
// is a handful of launches over all of its ciphertexts.
int pg_glwe_expand_coefficients(const pg_ntt_table* t, const pg_gadget_basis* g, uint32_t k, const uint64_t* d_keys,
                                size_t count, const uint64_t* d_in, uint64_t* d_out, void* d_ws, size_t ws_size,
                                void* stream) {
    int rc = check_compat(t, g);
    if (rc) return rc;
    if (!d_keys || !d_in || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (k == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k must be at least 1");
    if (count == 0 || (count & (count - 1)) || count > t->n)
        return set_error(PG_ERR_INVALID_ARGUMENT, "count must be a power of two no larger than N");
    const size_t LN = (size_t)t->L * t->n, glwe = (size_t)(k + 1) * LN;
    if (d_in != d_out && ranges_overlap(d_in, glwe, d_out, count * glwe))
        return set_error(PG_ERR_INVALID_ARGUMENT, "input must be the first output slot or not overlap the output");
    cudaStream_t st = (cudaStream_t)stream;
    Workspace w;
    rc = get_workspace(w, d_ws, ws_size, pg_glwe_expand_workspace_size(t, g, k, count), st);
    if (rc) return rc;
    const size_t chunk = expand_chunk(count);
    uint64_t* tmp = (uint64_t*)w.ptr;
    uint64_t* fw = (uint64_t*)((char*)w.ptr + round256(chunk * glwe * 8));
    uint64_t* fwq = fw + LN;
    void* aws = (char*)fw + round256(2 * LN * 8);
    const size_t aws_size = pg_glwe_automorphism_workspace_size(t, g, k, chunk);
    if (d_in != d_out) PG_CUDA(cudaMemcpyAsync(d_out, d_in, glwe * 8, cudaMemcpyDeviceToDevice, st));
    std::vector<uint64_t> inv(t->L);
    for (uint32_t l = 0; l < t->L; ++l) inv[l] = h_invmod(count % t->moduli[l], t->moduli[l]);
    rc = pg_dcrt_mul_scalar(t, d_out, inv.data(), k + 1, stream);
    if (rc) return rc;
    const size_t kw = auto_key_words(t, g, k);
    for (uint32_t lev = 0; (size_t(1) << lev) < count; ++lev) {
        const size_t half = (size_t)1 << lev;
        if ((rc = pg_ntt_coeff_one_monomial(t, 2 * t->n - half, fw, stream))) return rc;
        if ((rc = pg_dcrt_shoup_prepare(t, fw, fwq, 1, stream))) return rc;
        const uint64_t degree = (uint64_t)(t->n >> lev) + 1;
        for (size_t c0 = 0; c0 < half; c0 += chunk) {
            const size_t m = std::min(chunk, half - c0);
            rc = pg_glwe_automorphism(t, g, k, degree, d_keys + lev * kw, d_out + c0 * glwe, tmp, m, aws, aws_size,
                                      stream);
            if (rc) return rc;
            rc = pg_dcrt_butterfly_mul_factor(t, d_out + c0 * glwe, tmp, fw, fwq, d_out + (half + c0) * glwe,
                                              m * (k + 1), stream);
            if (rc) return rc;
        }
    }
    return PG_OK;
}

}  // extern "C"
