// NTT entry points, default kernel dispatch, fused external product and
// monomial transforms.  The kernel templates live in ntt_kernels.cuh.
#include "ntt_kernels.cuh"


namespace pg {

// ============================================================================
// Fused external product (GLWE x GGSW, k = 1, one prime, single-word values):
// CrtGlwe::mul_dcrt_ggsw_inplace (primus_lattice/src/glwe/crt.rs:202-229) and,
// for OUT_COEFF, inverse_transform_slice of both output polys.  One CTA per
// ciphertext.  For each input poly i the CTA decomposes its coefficients into
// d gadget digits (digits of one poly kept in shared memory), then for each
// digit j lifts the digit row to residues mod q, runs the forward NTT in
// shared memory and multiply-accumulates the NTT-domain row against the
// GGSW rows key[i][j][c] into 128-bit accumulators in shared memory, one per
// output element, each touched only by its own thread.  Outputs are canonical residues (NTT domain, or coefficient form
// after the in-kernel inverse NTT): the same residues as the reference's
// per-digit sequence, since every step is exact arithmetic mod q.
// ============================================================================
struct ExtFusedArgs {
    const uint64_t* in;   // [B][2][N] coefficient form
    const uint64_t* key;  // [2][d][2][N] NTT domain
    uint64_t* out;        // [B][2][N]
    const ulonglong2* fwd;
    const ulonglong2* inv;
    const ulonglong2* inv_n;
    const ulonglong2* inv_last;
    Barrett bar;
    GadgetWord gw;
    uint64_t B;
    int out_coeff;
};

// d digits of one word v (init_value_carry_slice_inplace, basis.rs:307-331, and
// unsigned_decompose, common.rs:150-160, with W = 1), written to dst[j * N]
template <typename DT, int N>
PG_DEV void decompose_word(uint64_t v, const GadgetWord& g, DT* dst) {
    if (g.has_split && v >= g.split) v += g.npq;
    uint64_t carry = g.has_init ? ((v & g.init_mask) != 0) : 0;
    for (uint32_t j = 0; j < g.d; ++j) {
        const DigitMask m = g.masks[j];
        // limb 1 is the zero guard limb: only limb 0 contributes bits
        uint64_t temp = m.index == 0 ? (v & m.mask0) >> m.shr : 0;
        temp += carry;
        carry = (temp & g.carry_mask) != 0;
        dst[(size_t)j * N] = (DT)(temp & g.bm1);
    }
}

// TAB (small bases, fast forward schedule): the first forward stage pairs element
// i with i + N/2 under the one twiddle w = root_powers[1], and its product operand
// is a lifted digit, one of `basis` values, so the products w * lift(digit) mod q
// come from a table of `basis` words in shared memory instead of Shoup products.
template <int LOG_N, int LOG_E, typename DT, bool FAST, bool TAB>
__global__ void __launch_bounds__(1 << (LOG_N - LOG_E), LOG_N == 11 ? 2 : 1) ext_fused_kernel(ExtFusedArgs a) {
    constexpr int N = 1 << LOG_N, E = 1 << LOG_E, T = N / E, KP = 2;
    static_assert(!TAB || FAST, "the table form feeds the fast forward schedule");
    extern __shared__ uint64_t smem_ext[];
    // shared memory: NTT exchange buffer | 128-bit accumulators [KP][E][T] | digits [d][N]
    // | (TAB) first-stage products [basis]
    uint64_t* sm = smem_ext;
    ulonglong2* acc = reinterpret_cast<ulonglong2*>(smem_ext + padded(N));
    DT* dg = reinterpret_cast<DT*>(acc + KP * N);
    const uint32_t tid = threadIdx.x;
    const uint64_t b = blockIdx.x;
    const Barrett bar = a.bar;
    const uint64_t q = bar.q, q2 = q << 1, nq = 0 - q;
    const uint32_t d = a.gw.d;
    const uint64_t basis = a.gw.basis, half = (basis + 1) / 2, lift = q - basis;
    uint64_t* tab = reinterpret_cast<uint64_t*>(dg + (size_t)d * N);
    if constexpr (TAB) {
        const ulonglong2 w1 = a.fwd[1];
        for (uint32_t v = tid; v < basis; v += T) {
            const uint64_t lv = (basis == 2 || v < half) ? v : lift + v;
            tab[v] = shoup_mul(w1.x, w1.y, lv, q);
        }
        __syncthreads();
    }
    using R0 = FwdRounds<LOG_N, LOG_E, 0>;
    static_assert(R0::G == LOG_N - LOG_E, "first forward group is the column tid + jj*T");
    static_assert(!TAB || R0::P_HI > R0::P_LO, "the table stage leaves at least one stage in the first round");
    // each thread owns accumulator entries (c, e, tid): no other thread touches them
#pragma unroll
    for (int ce = 0; ce < KP * E; ++ce) acc[ce * T + tid] = make_ulonglong2(0, 0);
    uint32_t terms = 0;
    for (int i = 0; i < KP; ++i) {
        // this thread's coefficients tid + jj*T; it alone reads their digits back
        const uint64_t* src = a.in + (b * KP + i) * N;
        // every global load is issued before the digits' shared-memory stores
        uint64_t v[E];
#pragma unroll
        for (int jj = 0; jj < E; ++jj) v[jj] = ld_stream(src + tid + jj * T);
#pragma unroll
        for (int jj = 0; jj < E; ++jj) decompose_word<DT, N>(v[jj], a.gw, dg + tid + jj * T);
        for (uint32_t j = 0; j < d; ++j) {
            uint64_t x[E];
            if constexpr (TAB) {
                // stage LOG_N - 1: (u + w y, u - w y) with w y = tab[digit of y], u = the
                // lifted digit of x; outputs below 2q, inside the fast schedule's bounds
#pragma unroll
                for (int jj = 0; jj < E / 2; ++jj) {
                    const uint64_t v = dg[(size_t)j * N + tid + jj * T];
                    const uint64_t u = (basis == 2 || v < half) ? v : lift + v;
                    const uint64_t t = tab[dg[(size_t)j * N + tid + (jj + E / 2) * T]];
                    x[jj] = u + t;
                    x[jj + E / 2] = u + q - t;
                }
                fwd_round<LOG_N, LOG_E, R0::G, R0::P_HI - 1, R0::P_LO, FAST>(x, tid, 1, a.fwd, q2, nq);
            } else {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) {
                    const uint64_t v = dg[(size_t)j * N + tid + jj * T];
                    x[jj] = (basis == 2 || v < half) ? v : lift + v;  // wrapping_decompose_small_values
                }
                fwd_round<LOG_N, LOG_E, R0::G, R0::P_HI, R0::P_LO, FAST>(x, tid, 1, a.fwd, q2, nq);
            }
            __syncthreads();  // the previous row's last shared-memory reads are done
            fwd_rest<LOG_N, LOG_N, LOG_E, 1, FAST>(x, sm, tid, 1, a.fwd, q2, nq);
            if constexpr (!FAST) {
#pragma unroll
                for (int e = 0; e < E; ++e) x[e] = canon4(x[e], q, q2);
            }
            // x = NTT-domain elements tid*E .. tid*E+E-1 of digit row (i, j); products
            // are below 2^122, so 8 of them plus a folded value stay below 2^128
            const bool fold = terms == 8;
            terms = fold ? 1 : terms + 1;
            const uint64_t* kp = a.key + ((size_t)(i * d + j) * KP) * N + tid * E;
#pragma unroll
            for (int c = 0; c < KP; ++c)
#pragma unroll
                for (int e = 0; e < E; e += 2) {
                    ulonglong2 w;
                    asm("ld.global.nc.v2.u64 {%0, %1}, [%2];" : "=l"(w.x), "=l"(w.y) : "l"(kp + c * N + e));
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        ulonglong2 s = acc[(c * E + e + h) * T + tid];
                        if (fold) {
                            s.x = barrett_reduce_128(s.x, s.y, bar);
                            s.y = 0;
                        }
                        const uint64_t kv = h ? w.y : w.x;
                        const uint64_t pl = kv * x[e + h], ph = mulhi64(kv, x[e + h]);
                        s.x += pl;
                        s.y += ph + (s.x < pl);
                        acc[(c * E + e + h) * T + tid] = s;
                    }
                }
        }
    }
    uint64_t* out = a.out + b * KP * N;
    if (!a.out_coeff) {
#pragma unroll
        for (int c = 0; c < KP; ++c)
#pragma unroll
            for (int e = 0; e < E; e += 2) {
                const ulonglong2 s0 = acc[(c * E + e) * T + tid], s1 = acc[(c * E + e + 1) * T + tid];
                const uint64_t r0 = barrett_reduce_128(s0.x, s0.y, bar);
                const uint64_t r1 = barrett_reduce_128(s1.x, s1.y, bar);
                asm volatile("st.global.v2.u64 [%0], {%1, %2};" ::"l"(out + c * N + tid * E + e), "l"(r0), "l"(r1)
                             : "memory");
            }
        return;
    }
    // coefficient form: inverse NTT of each output poly; the first inverse group
    // is the contiguous tid*E .. tid*E+E-1, so the accumulators feed it directly
    using I0 = InvRounds<LOG_N, LOG_E, 0>;
    static_assert(I0::G == 0, "first inverse group is contiguous");
#pragma unroll 1
    for (int c = 0; c < KP; ++c) {
        uint64_t x[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const ulonglong2 s = acc[(c * E + e) * T + tid];
            x[e] = barrett_reduce_128(s.x, s.y, bar);
        }
        __syncthreads();  // earlier shared-memory reads of the exchange buffer are done
        inv_round<LOG_N, LOG_N, LOG_E, I0::G, I0::P_LO, I0::P_HI>(x, tid * E, 0, a.inv, a.inv_n, a.inv_last, q, nq);
        inv_range<LOG_N, LOG_N, LOG_N, LOG_E, 1, I0::COUNT>(x, sm, tid, 0, a.inv, a.inv_n, a.inv_last, q, nq);
#pragma unroll
        for (int jj = 0; jj < E; ++jj) out[c * N + tid + jj * T] = x[jj];
    }
}

}  // namespace pg

// ============================================================================
// Launch dispatch
// ============================================================================
namespace pg {

// block size (2^PG_NTT_LOG_M elements) each CTA of a cluster owns
#ifndef PG_NTT_LOG_M
#define PG_NTT_LOG_M 12
#endif

template <int MODE, int FAST>
static int launch_mode(const NttArgs& a, uint32_t log_n, cudaStream_t st) {
    switch (log_n) {
        case 1: return launch_block<1, 1, 128, MODE, FAST>(a, st);
        case 2: return launch_block<2, 2, 128, MODE, FAST>(a, st);
        case 3: return launch_block<3, 3, 128, MODE, FAST>(a, st);
        case 4: return launch_block<4, 3, 64, MODE, FAST>(a, st);
        case 5: return launch_block<5, 3, 32, MODE, FAST>(a, st);
        case 6: return launch_block<6, 3, 16, MODE, FAST>(a, st);
        case 7: return launch_block<7, 3, 8, MODE, FAST>(a, st);
        case 8: return launch_block<8, 3, 4, MODE, FAST>(a, st);
        case 9: return launch_block<9, 3, 2, MODE, FAST>(a, st);
        case 10: return launch_block<10, 3, 1, MODE, FAST>(a, st);
        case 11: return launch_block<11, 3, 1, MODE, FAST>(a, st);
        case 12: return launch_block<12, 4, 1, MODE, FAST>(a, st);
        // 2^13: a 2-CTA cluster beats one 512-thread CTA per row by 20-35%
        case 13: return launch_cluster<13, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        case 14: return launch_cluster<14, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        case 15: return launch_cluster<15, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        case 16: return launch_cluster<16, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        default: return set_error(PG_ERR_UNSUPPORTED, "this build runs NTTs for log_n in [1, 16]");
    }
}



// the opt-in maximum of dynamic shared memory per CTA on sm_100 (227 KiB)
constexpr size_t kExtFusedMaxSmem = 227 * 1024;

template <int LOG_N, int LOG_E, typename DT, bool FAST, bool TAB>
static int launch_ext_fused_t(const ExtFusedArgs& a, size_t smem, cudaStream_t st) {
    constexpr int T = 1 << (LOG_N - LOG_E);
    auto kern = ext_fused_kernel<LOG_N, LOG_E, DT, FAST, TAB>;
    // shared memory grows with the digit count; raise the limit to the largest allowed once
    static const cudaError_t attr =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kExtFusedMaxSmem);
    if (attr != cudaSuccess) return cuda_status(attr, "ext_fused_kernel: shared memory attribute");
    kern<<<(unsigned)a.B, T, smem, st>>>(a);
    count_launch();
    PG_LAUNCH_CHECK("ext_fused_kernel launch");
    return PG_OK;
}

template <typename DT, bool FAST, bool TAB = false>
static int launch_ext_fused_n(const ExtFusedArgs& a, uint32_t log_n, size_t smem, cudaStream_t st) {
    switch (log_n) {
        case 10: return launch_ext_fused_t<10, 3, DT, FAST, TAB>(a, smem, st);
        // 2^11: E = 4 (512 threads, 64 registers, two CTAs per SM) beats E = 8 by 4.5%
        case 11: return launch_ext_fused_t<11, 2, DT, FAST, TAB>(a, smem, st);
        case 12: return launch_ext_fused_t<12, 3, DT, FAST, TAB>(a, smem, st);
        default: return set_error(PG_ERR_UNSUPPORTED, "fused external product: log_n outside 10..12");
    }
}

// first-stage product tables for bases up to this size (2 KiB of shared memory)
constexpr uint64_t kExtTabMaxBasis = 256;

static bool ext_fused_tab(const pg_ntt_table* t, const GadgetWord& gw) {
    return gw.basis <= kExtTabMaxBasis && gw.log_basis <= 16 && t->moduli[0] < (1ull << 58);
}

static size_t ext_fused_smem(const pg_ntt_table* t, const GadgetWord& gw) {
    const size_t dt = gw.log_basis <= 16 ? 2 : 8;
    return (size_t)padded((int)t->n) * 8 + 2 * t->n * 16 + (size_t)gw.d * t->n * dt +
           (ext_fused_tab(t, gw) ? gw.basis * 8 : 0);
}

bool ext_fused_eligible(const pg_ntt_table* t, const GadgetWord& gw, uint32_t k) {
    if (k != 1 || t->L != 1 || t->log_n < 10 || t->log_n > 12) return false;
    if (gw.basis < 2 || gw.basis > t->moduli[0] || gw.d == 0) return false;
    return ext_fused_smem(t, gw) <= kExtFusedMaxSmem;
}

int launch_ext_fused(const pg_ntt_table* t, const GadgetWord& gw, const uint64_t* in, const uint64_t* key,
                     uint64_t* out, size_t batch, bool out_coeff, cudaStream_t st) {
    if (batch == 0) return PG_OK;
    if (batch > 0x7fffffffull) return set_error(PG_ERR_UNSUPPORTED, "too many ciphertexts for one launch");
    ExtFusedArgs a{};
    a.in = in;
    a.key = key;
    a.out = out;
    a.fwd = t->d_fwd;
    a.inv = t->d_inv;
    a.inv_n = t->d_inv_n;
    a.inv_last = t->d_inv_last;
    a.bar = h_barrett(t->moduli[0]);
    a.gw = gw;
    a.B = batch;
    a.out_coeff = out_coeff ? 1 : 0;
    const size_t smem = ext_fused_smem(t, gw);
    const bool fast = t->moduli[0] < (1ull << 58);
    if (ext_fused_tab(t, gw)) return launch_ext_fused_n<uint16_t, true, true>(a, t->log_n, smem, st);
    if (gw.log_basis <= 16)
        return fast ? launch_ext_fused_n<uint16_t, true>(a, t->log_n, smem, st)
                    : launch_ext_fused_n<uint16_t, false>(a, t->log_n, smem, st);
    return fast ? launch_ext_fused_n<uint64_t, true>(a, t->log_n, smem, st)
                : launch_ext_fused_n<uint64_t, false>(a, t->log_n, smem, st);
}

int launch_ntt(const NttArgs& a, uint32_t log_n, int mode, cudaStream_t st) {
    if (a.rows == 0) return PG_OK;
    const bool ffwd = fast_fwd_ok(a), finv = fast_inv_ok(a);
    // a tuned shape runs the fast schedules: canonical forward, inverse and round trip
    if (mode >= 0 && mode < 3 && a.variant[mode] > 0) {
        const bool ok = ntt_variant_fp(log_n, a.variant[mode])
                            ? finv && a.fwd_fp && (mode != MODE_FWD || !a.lazy)
                            : (mode == MODE_FWD ? (!a.lazy && ffwd) : finv);
        if (ok) return launch_ntt_variant(a, log_n, mode, a.variant[mode], st);
    }
    // the FP64 schedule (every q < 2^50, tables present) is the fastest on every shape
    const bool ffp = finv && a.fwd_fp;
    switch (mode) {
        case MODE_FWD:
            if (!a.lazy && ffp) return launch_mode<MODE_FWD, kSchedFp64>(a, log_n, st);
            if (!a.lazy && ffwd) return launch_mode<MODE_FWD, kSchedFastFwd>(a, log_n, st);
            return launch_mode<MODE_FWD, kSchedExact>(a, log_n, st);
        case MODE_INV:
            // the inverse's outputs are canonical on every schedule (lazy included)
            if (ffp) return launch_mode<MODE_INV, kSchedFp64>(a, log_n, st);
            if (finv) return launch_mode<MODE_INV, kSchedFastBoth>(a, log_n, st);
            return launch_mode<MODE_INV, kSchedExact>(a, log_n, st);
        case MODE_RT:
            if (ffp) return launch_mode<MODE_RT, kSchedFp64>(a, log_n, st);
            if (finv) return launch_mode<MODE_RT, kSchedFastBoth>(a, log_n, st);
            if (ffwd) return launch_mode<MODE_RT, kSchedFastFwd>(a, log_n, st);
            return launch_mode<MODE_RT, kSchedExact>(a, log_n, st);
    }
    return set_error(PG_ERR_INVALID_ARGUMENT, "bad NTT mode");
}

bool pair_ok(const NttArgs& a, uint32_t log_n) {
    return log_n >= 1 && log_n <= kPairMaxLogN && a.desc && fast_inv_ok(a) && a.fwd_fp;
}

// the default block shapes of launch_mode, in the pair form
int launch_pair(const NttArgs& a, uint32_t log_n, cudaStream_t st) {
    if (a.rows == 0) return PG_OK;
    if (!pair_ok(a, log_n)) return set_error(PG_ERR_UNSUPPORTED, "pair form: needs descriptor rows, log_n <= 12 "
                                                                 "and every modulus below 2^50");
    constexpr int M = MODE_PAIR, S = kSchedFp64;
    switch (log_n) {
        case 1: return launch_block<1, 1, 128, M, S>(a, st);
        case 2: return launch_block<2, 2, 128, M, S>(a, st);
        case 3: return launch_block<3, 3, 128, M, S>(a, st);
        case 4: return launch_block<4, 3, 64, M, S>(a, st);
        case 5: return launch_block<5, 3, 32, M, S>(a, st);
        case 6: return launch_block<6, 3, 16, M, S>(a, st);
        case 7: return launch_block<7, 3, 8, M, S>(a, st);
        case 8: return launch_block<8, 3, 4, M, S>(a, st);
        case 9: return launch_block<9, 3, 2, M, S>(a, st);
        case 10: return launch_block<10, 3, 1, M, S>(a, st);
        case 11: return launch_block<11, 3, 1, M, S>(a, st);
        case 12: return launch_block<12, 4, 1, M, S>(a, st);
    }
    return set_error(PG_ERR_UNSUPPORTED, "pair form: log_n outside 1..12");
}

// ---------------------------------------------------------------- monomials
// transform_monomial (primus_ntt/src/ntt/primitive.rs:298-349): out[i] =
// coeff * psi^((2 rev(i) + 1) * degree mod 2N); kind 0 = general coeff,
// 1 = X^degree, 2 = -X^degree (index XOR N selects -psi^k).
__global__ void monomial_kernel(uint64_t* out, const ulonglong2* __restrict__ ordinal, const uint64_t* __restrict__ moduli,
                                uint32_t log_n, uint32_t L, uint64_t coeff, uint64_t degree, int kind) {
    const size_t n = (size_t)1 << log_n;
    const size_t total = n * L;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
        const uint32_t l = (uint32_t)(idx >> log_n);
        const uint32_t i = (uint32_t)(idx & (n - 1));
        const uint64_t q = moduli[l];
        uint64_t v;
        if (kind == 0 && coeff == 0) {
            v = 0;
        } else if (degree == 0) {
            v = kind == 0 ? coeff : (kind == 1 ? 1 : q - 1);
        } else {
            const uint32_t rev = __brev(i) >> (32 - log_n);
            size_t e = ((2 * (size_t)rev + 1) * degree) & (2 * n - 1);
            const ulonglong2* o = ordinal + (size_t)l * 2 * n;
            if (kind == 2 || (kind == 0 && coeff == q - 1)) {
                v = o[e ^ n].x;
            } else if (kind == 1 || coeff == 1) {
                v = o[e].x;
            } else {
                v = shoup_mul(o[e].x, o[e].y, coeff, q);
            }
        }
        out[idx] = v;
    }
}

static int launch_monomial(const pg_ntt_table* t, uint64_t coeff, size_t degree, uint64_t* d_out, int kind,
                           cudaStream_t st) {
    if (!t || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL table or output");
    // any degree: exponents are taken mod 2N (X^N = -1), as primitive.rs:319 masks them
    const size_t total = t->n * t->L;
    const unsigned threads = 256;
    const unsigned blocks = (unsigned)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    monomial_kernel<<<blocks, threads, 0, st>>>(d_out, t->d_ordinal, t->d_moduli, t->log_n, t->L, coeff, degree, kind);
    count_launch();
    PG_LAUNCH_CHECK("monomial_kernel launch");
    return PG_OK;
}

static int check_table_data(const pg_ntt_table* t, const void* d, size_t polys) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (!d && polys) return set_error(PG_ERR_INVALID_ARGUMENT, "data is NULL");
    if (t->log_n > 16) return set_error(PG_ERR_UNSUPPORTED, "this build runs NTTs for log_n in [1, 16]");
    return PG_OK;
}

#ifndef PG_PIPE_STREAMS
#define PG_PIPE_STREAMS 3
#endif
#ifndef PG_PIPE_CHUNK_MB
#define PG_PIPE_CHUNK_MB 64
#endif

// Host slices through a copy / compute pipeline: chunks of whole polys are
// copied in on one of kPipeStreams streams, transformed there and copied back,
// so that the two copy engines (host->device and device->host) and the SMs work
// at the same time.  With pinned host memory the copies overlap; with pageable
// memory the same calls run at the speed of the driver's staged copies.
// Synchronous, like the reference's &mut [u64] calls.
static int host_pipeline(const pg_ntt_table* t, uint64_t* h, size_t polys, int lazy, int mode,
                         const uint64_t* d_plain, const uint64_t* d_plain_q, cudaStream_t user = nullptr) {
    int rc = check_table_data(t, h, polys);
    if (rc) return rc;
    if (polys == 0) return PG_OK;
    constexpr int kPipeStreams = PG_PIPE_STREAMS;
    constexpr size_t kChunkBytes = (size_t)PG_PIPE_CHUNK_MB << 20;
    const size_t poly_words = (size_t)t->L * t->n;
    const size_t chunk = std::max<size_t>(1, kChunkBytes / (poly_words * sizeof(uint64_t)));
    const size_t nchunks = (polys + chunk - 1) / chunk;
    const int ns = (int)std::min<size_t>(kPipeStreams, nchunks);
    cudaStream_t st[kPipeStreams] = {};
    cudaEvent_t ev[kPipeStreams + 1] = {};
    for (int i = 0; i < ns; ++i) PG_CUDA(cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking));
    for (int i = 0; i <= ns && user; ++i) PG_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    if (user) {  // the pipeline starts after the caller's stream and rejoins it at the end
        PG_CUDA(cudaEventRecord(ev[ns], user));
        for (int i = 0; i < ns; ++i) PG_CUDA(cudaStreamWaitEvent(st[i], ev[ns], 0));
    }
    auto cleanup = [&](void* buf) {
        for (int i = 0; i < ns && user; ++i) {
            cudaEventRecord(ev[i], st[i]);
            cudaStreamWaitEvent(user, ev[i], 0);
        }
        for (int i = 0; i < ns; ++i) cudaStreamSynchronize(st[i]);
        if (buf) {
            scratch_free(buf, st[0]);
            cudaStreamSynchronize(st[0]);
        }
        for (int i = 0; i < ns; ++i) cudaStreamDestroy(st[i]);
        for (int i = 0; i <= ns; ++i)
            if (ev[i]) cudaEventDestroy(ev[i]);
    };
    void* buf = nullptr;
    cudaError_t e = scratch_alloc(&buf, (size_t)ns * chunk * poly_words * sizeof(uint64_t), st[0]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st[0]);
    if (e != cudaSuccess) {
        cleanup(nullptr);
        return cuda_status(e, "host transform: staging buffers");
    }
    for (size_t c = 0; c < nchunks && rc == PG_OK; ++c) {
        const int si = (int)(c % ns);
        const size_t p0 = c * chunk, np = std::min(chunk, polys - p0);
        uint64_t* d = (uint64_t*)buf + (size_t)si * chunk * poly_words;
        uint64_t* hp = h + p0 * poly_words;
        const size_t bytes = np * poly_words * sizeof(uint64_t);
        e = cudaMemcpyAsync(d, hp, bytes, cudaMemcpyHostToDevice, st[si]);
        if (e != cudaSuccess) {
            rc = cuda_status(e, "host transform: copy in");
            break;
        }
        NttArgs a = make_args(t, d, np * t->L, lazy);
        a.plain = d_plain;
        a.plain_q = d_plain_q;
        rc = launch_ntt(a, t->log_n, mode, st[si]);
        if (rc) break;
        e = cudaMemcpyAsync(hp, d, bytes, cudaMemcpyDeviceToHost, st[si]);
        if (e != cudaSuccess) rc = cuda_status(e, "host transform: copy out");
    }
    cleanup(buf);
    if (rc == PG_OK) {
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_status(e, "host transform");
    }
    return rc;
}

}  // namespace pg

using namespace pg;

extern "C" {

int pg_ntt_forward(const pg_ntt_table* t, uint64_t* d_data, size_t polys, int lazy, void* stream) {
    int rc = check_table_data(t, d_data, polys);
    if (rc) return rc;
    return launch_ntt(make_args(t, d_data, polys * t->L, lazy), t->log_n, MODE_FWD, (cudaStream_t)stream);
}

int pg_ntt_inverse(const pg_ntt_table* t, uint64_t* d_data, size_t polys, int lazy, void* stream) {
    int rc = check_table_data(t, d_data, polys);
    if (rc) return rc;
    return launch_ntt(make_args(t, d_data, polys * t->L, lazy), t->log_n, MODE_INV, (cudaStream_t)stream);
}

int pg_ntt_forward_host(const pg_ntt_table* t, uint64_t* h_data, size_t polys, int lazy) {
    return host_pipeline(t, h_data, polys, lazy, MODE_FWD, nullptr, nullptr);
}

int pg_ntt_inverse_host(const pg_ntt_table* t, uint64_t* h_data, size_t polys, int lazy) {
    return host_pipeline(t, h_data, polys, lazy, MODE_INV, nullptr, nullptr);
}

int pg_ntt_monomial(const pg_ntt_table* t, uint64_t coeff, size_t degree, uint64_t* d_out, void* stream) {
    return launch_monomial(t, coeff, degree, d_out, 0, (cudaStream_t)stream);
}

int pg_ntt_coeff_one_monomial(const pg_ntt_table* t, size_t degree, uint64_t* d_out, void* stream) {
    return launch_monomial(t, 1, degree, d_out, 1, (cudaStream_t)stream);
}

int pg_ntt_coeff_minus_one_monomial(const pg_ntt_table* t, size_t degree, uint64_t* d_out, void* stream) {
    return launch_monomial(t, 1, degree, d_out, 2, (cudaStream_t)stream);
}

int pg_dcrt_polymul_ntt_plain(const pg_ntt_table* t, uint64_t* d_data, const uint64_t* d_plain,
                              const uint64_t* d_plain_q, size_t polys, void* stream) {
    int rc = check_table_data(t, d_data, polys);
    if (rc) return rc;
    if (!d_plain || !d_plain_q) return set_error(PG_ERR_INVALID_ARGUMENT, "plaintext is NULL");
    NttArgs a = make_args(t, d_data, polys * t->L, 0);
    a.plain = d_plain;
    a.plain_q = d_plain_q;
    return launch_ntt(a, t->log_n, MODE_RT, (cudaStream_t)stream);
}

int pg_dcrt_polymul_ntt_plain_host(const pg_ntt_table* t, uint64_t* h_data, const uint64_t* d_plain,
                                   const uint64_t* d_plain_q, size_t polys, void* stream) {
    if (!d_plain || !d_plain_q) return set_error(PG_ERR_INVALID_ARGUMENT, "plaintext is NULL");
    return host_pipeline(t, h_data, polys, 0, MODE_RT, d_plain, d_plain_q, (cudaStream_t)stream);
}

}  // extern "C"
