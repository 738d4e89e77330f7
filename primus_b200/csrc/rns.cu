// RNS base (CRT compose / decompose), fast base conversion and gadget
// (approximate signed) decomposition on the device.
//
//   RNSBase            primus_rns/src/base.rs:24-90, 201-231, 285-309, 396-449
//   BaseConverter      primus_rns/src/converter.rs:12-175
//   BigUintApproxSignedBasis  primus_decompose/src/big_integer/basis.rs:34-342
//   OnceBigUintSignedDecomposer primus_decompose/src/big_integer/common.rs:8-200
//
// Every output here is unique (canonical residues, the canonical CRT value in
// [0, Q), digits defined bit by bit), so the device kernels reproduce the
// reference's values with their own schedules: one thread per coefficient,
// BigUint limbs in registers (compose) or in a per-thread shared-memory row
// (decomposition, where the digit position moves through the limbs).
#include <algorithm>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace pg;

// ============================================================== host BigUint
namespace {

using Big = std::vector<uint64_t>;  // little-endian limbs

int big_cmp(const uint64_t* a, const uint64_t* b, size_t w) {
    for (size_t i = w; i-- > 0;)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

bool big_sub(uint64_t* a, const uint64_t* b, size_t w) {
    uint64_t borrow = 0;
    for (size_t i = 0; i < w; ++i) {
        u128 t = (u128)a[i] - b[i] - borrow;
        a[i] = (uint64_t)t;
        borrow = (t >> 64) ? 1 : 0;
    }
    return borrow != 0;
}

bool big_add(uint64_t* a, const uint64_t* b, size_t w) {
    uint64_t carry = 0;
    for (size_t i = 0; i < w; ++i) {
        u128 t = (u128)a[i] + b[i] + carry;
        a[i] = (uint64_t)t;
        carry = (uint64_t)(t >> 64);
    }
    return carry != 0;
}

// shift left by bits (< 64 per call), returns bits shifted out
uint64_t big_shl(uint64_t* a, size_t w, uint32_t bits) {
    if (bits == 0) return 0;
    uint64_t carry = 0;
    for (size_t i = 0; i < w; ++i) {
        uint64_t nc = a[i] >> (64 - bits);
        a[i] = (a[i] << bits) | carry;
        carry = nc;
    }
    return carry;
}

bool big_shl_any(uint64_t* a, size_t w, uint32_t bits) {
    bool overflow = false;
    while (bits >= 63) {
        overflow |= big_shl(a, w, 63) != 0;
        bits -= 63;
    }
    overflow |= big_shl(a, w, bits) != 0;
    return overflow;
}

uint64_t big_mod(const uint64_t* a, size_t w, uint64_t q) {
    u128 r = 0;
    for (size_t i = w; i-- > 0;) r = ((r << 64) | a[i]) % q;
    return (uint64_t)r;
}

uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

struct pg_rns_base {
    uint32_t L = 0, W = 0;
    std::vector<uint64_t> moduli, product, punctured, inv, inv_q;
    uint64_t* d_moduli = nullptr;
    uint64_t* d_product = nullptr;   // [W]
    uint64_t* d_punctured = nullptr; // [L][W]
    ulonglong2* d_inv = nullptr;     // [L] (value, Shoup quotient)
    Barrett* d_bar = nullptr;        // [L]
};

struct pg_gadget_basis {
    const pg_rns_base* base = nullptr;
    uint32_t W = 0, L = 0, d = 0, log_basis = 0, drop_bits = 0;
    uint64_t basis = 0, bm1 = 0, carry_mask = 0;
    bool has_split = false, has_init = false;
    uint32_t init_index = 0;
    uint64_t init_mask = 0;
    Big split, npq, scalars, scalar_residues;
    std::vector<DigitMask> masks;
    uint64_t* d_split = nullptr;  // [W]
    uint64_t* d_npq = nullptr;    // [W] next_pow_of_2_sub_modulus
    DigitMask* d_masks = nullptr; // [d]
};

struct pg_base_converter {
    const pg_rns_base* ibase = nullptr;
    const pg_rns_base* obase = nullptr;
    uint64_t* d_matrix = nullptr;  // [Lout][Lin]: (Q/q_i) mod p_j
};

namespace pg {
// accessors for lattice.cu
uint32_t rns_L(const pg_rns_base* b) { return b->L; }
uint32_t rns_W(const pg_rns_base* b) { return b->W; }
const pg_rns_base* gadget_base(const pg_gadget_basis* g) { return g->base; }
uint32_t gadget_d(const pg_gadget_basis* g) { return g->d; }
uint64_t gadget_basis_value(const pg_gadget_basis* g) { return g->basis; }
// the basis as single-word parameters; false when its values need more than one word
bool gadget_word(const pg_gadget_basis* g, GadgetWord* out) {
    if (g->W != 1) return false;
    GadgetWord w{};
    w.bm1 = g->bm1;
    w.carry_mask = g->carry_mask;
    w.basis = g->basis;
    w.split = g->has_split ? g->split[0] : 0;
    w.npq = g->has_split ? g->npq[0] : 0;
    w.init_mask = g->init_mask;
    w.has_split = g->has_split;
    w.has_init = g->has_init && g->init_index == 0;
    w.d = g->d;
    w.log_basis = g->log_basis;
    w.masks = g->d_masks;
    if (g->has_init && g->init_index != 0) return false;
    *out = w;
    return true;
}
const uint64_t* rns_moduli(const pg_rns_base* b) { return b->moduli.data(); }
}  // namespace pg

// =================================================================== kernels
namespace {

// 64x64 -> 128 multiply-add into (lo, hi) with carry
PG_DEV void mac128(uint64_t& lo, uint64_t& hi, uint64_t a, uint64_t b) {
    uint64_t pl = a * b, ph = mulhi64(a, b);
    lo += pl;
    hi += ph + (lo < pl);
}

// compose_inplace (base.rs:396-420) for one coefficient per thread.  W is the
// limb count; the running value stays in [0, Q) after every step exactly as in
// the reference (conditional subtraction of Q on carry or value >= Q).
// Coefficient x of the launch is column x % n of poly p = x / n; poly p's
// residue row i starts at (p / ppg) * group_stride + (p % ppg) * L * n + i * n
// (ppg polys per group, e.g. the a-part of a GLWE ciphertext).
struct ComposeArgs {
    const uint64_t* res;
    uint64_t* out;
    size_t count, n, group_stride;
    uint32_t L, ppg;
    const uint64_t* moduli;
    const ulonglong2* inv;
    const uint64_t* punct;
    const uint64_t* prod;
};

template <int W>
__global__ void __launch_bounds__(128) compose_kernel(ComposeArgs a) {
    const uint32_t L = a.L;
    const uint64_t* __restrict__ moduli = a.moduli;
    const ulonglong2* __restrict__ inv = a.inv;
    const uint64_t* __restrict__ punct = a.punct;
    const uint64_t* __restrict__ prod = a.prod;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < a.count; x += (size_t)gridDim.x * blockDim.x) {
        const size_t p = x / a.n, c = x % a.n;
        const uint64_t* rp = a.res + (p / a.ppg) * a.group_stride + (p % a.ppg) * (size_t)L * a.n + c;
        uint64_t v[W];
#pragma unroll
        for (int k = 0; k < W; ++k) v[k] = 0;
        for (uint32_t i = 0; i < L; ++i) {
            const uint64_t q = moduli[i];
            const ulonglong2 f = inv[i];
            const uint64_t y = shoup_mul(f.x, f.y, rp[(size_t)i * a.n], q);
            const uint64_t* P = punct + (size_t)i * W;
            uint64_t carry = 0;
            if (y != 0) {
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    uint64_t lo = v[k], hi = 0;
                    mac128(lo, hi, y, P[k]);
                    lo += carry;
                    hi += (lo < carry);
                    v[k] = lo;
                    carry = hi;
                }
            }
            // value >= Q ? (lexicographic from the top limb)
            int cmp = 0;
#pragma unroll
            for (int k = W - 1; k >= 0; --k)
                if (cmp == 0 && v[k] != prod[k]) cmp = v[k] < prod[k] ? -1 : 1;
            if (carry != 0 || cmp >= 0) {
                uint64_t borrow = 0;
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    uint64_t t = v[k] - prod[k];
                    uint64_t b1 = v[k] < prod[k];
                    uint64_t t2 = t - borrow;
                    uint64_t b2 = t < borrow;
                    v[k] = t2;
                    borrow = b1 | b2;
                }
            }
        }
        uint64_t* o = a.out + x * W;
#pragma unroll
        for (int k = 0; k < W; ++k) o[k] = v[k];
    }
}

// decompose_big_uint_values_inplace (base.rs:285-309): value mod q_i by Horner
// over the limbs with a 2-limb Barrett step
__global__ void __launch_bounds__(256) decompose_kernel(const uint64_t* __restrict__ vals, uint64_t* __restrict__ res,
                                                        size_t count, uint32_t L, uint32_t W,
                                                        const Barrett* __restrict__ bar) {
    const size_t total = count * L;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(t / count);
        const size_t x = t % count;
        const Barrett m = bar[i];
        const uint64_t* v = vals + x * W;
        uint64_t r = 0;
        for (uint32_t k = W; k-- > 0;) r = barrett_reduce_2limb(v[k], r, m);
        res[t] = r;
    }
}

// wrapping_decompose_small_values_inplace (base.rs:201-231)
__global__ void __launch_bounds__(256) wrap_small_kernel(const uint64_t* __restrict__ small, uint64_t* __restrict__ res,
                                                         size_t count, uint32_t L, const uint64_t* __restrict__ moduli,
                                                         uint64_t sm) {
    const size_t total = count * L;
    const uint64_t half = (sm + 1) / 2;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(t / count);
        const uint64_t v = small[t % count];
        res[t] = (sm == 2 || v < half) ? v : moduli[i] - sm + v;
    }
}

// add_wrapping_decompose_small_values_scaled (base.rs:238-283): dest[l][x] +=
// factor_l * lift_l(small[x]) mod q_l, the lift as in wrap_small_kernel and the
// product by the Shoup-prepared factor (f, f') canonical, so the sum is too.
// Grid-stride over [L][count], one 16-byte factor load per element.
__global__ void __launch_bounds__(256) add_wrap_scaled_kernel(const uint64_t* __restrict__ small,
                                                              uint64_t* __restrict__ dest, size_t count, uint32_t L,
                                                              const uint64_t* __restrict__ moduli,
                                                              const ulonglong2* __restrict__ factor, uint64_t sm) {
    const size_t total = count * L;
    const uint64_t half = (sm + 1) / 2;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(t / count);
        const uint64_t q = moduli[i], v = small[t % count];
        const uint64_t lifted = (sm == 2 || v < half) ? v : q - sm + v;
        const ulonglong2 f = factor[i];
        dest[t] = add_mod(dest[t], shoup_mul(f.x, f.y, lifted, q), q);
    }
}

// fast_convert_array (converter.rs:147-175): y_j = sum_i buf_i * M[j][i] mod p_j,
// buf_i = [x_i * (Q/q_i)^-1]_{q_i}; 128-bit accumulation folded every 8 terms
__global__ void __launch_bounds__(256) fast_convert_kernel(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                                           size_t n, uint32_t Li, uint32_t Lo,
                                                           const uint64_t* __restrict__ qi,
                                                           const ulonglong2* __restrict__ inv,
                                                           const Barrett* __restrict__ bar_o,
                                                           const uint64_t* __restrict__ matrix) {
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n; x += (size_t)gridDim.x * blockDim.x) {
        uint64_t buf[64];
        for (uint32_t i = 0; i < Li; ++i) {
            const ulonglong2 f = inv[i];
            const uint64_t v = in[(size_t)i * n + x];
            buf[i] = f.x == 1 ? (v >= qi[i] ? v % qi[i] : v) : shoup_mul(f.x, f.y, v, qi[i]);
        }
        for (uint32_t j = 0; j < Lo; ++j) {
            const Barrett m = bar_o[j];
            const uint64_t* row = matrix + (size_t)j * Li;
            uint64_t lo = 0, hi = 0;
            for (uint32_t i = 0; i < Li; ++i) {
                mac128(lo, hi, buf[i], row[i]);
                if ((i & 7) == 7) {  // keep the sum below 2^128 (terms < 2^124)
                    lo = barrett_reduce_128(lo, hi, m);
                    hi = 0;
                }
            }
            out[(size_t)j * n + x] = barrett_reduce_128(lo, hi, m);
        }
    }
}

// Gadget decomposition of one BigUint per thread.  The value lives in a
// per-thread shared-memory row (the digit window moves through the limbs).
// init_value_carry_slice_inplace (basis.rs:307-331), then per level
// unsigned_decompose (common.rs:150-160): temp = bits + carry,
// carry = temp & (B | B/2) != 0, digit = temp & (B - 1); LIFT writes
// wrapping_decompose_small_values (digit < B/2 ? digit : q_l - B + digit).
// Value x of the launch is column x % n of poly x / n; LIFT writes digit j,
// limb l of it at ((x / n) * d + j) * L * n + l * n + x % n, the plain form at
// ((x / n) * d + j) * n + x % n.
struct GadgetArgs {
    const uint64_t* vals;
    uint64_t* out;
    size_t count, n;
    uint32_t W, L, d;
    uint64_t bm1, carry_mask, basis;
    int has_split, has_init;
    uint32_t init_index;
    uint64_t init_mask;
    const uint64_t* split;
    const uint64_t* npq;
    const DigitMask* masks;
    const uint64_t* moduli;
};

template <bool LIFT>
__global__ void __launch_bounds__(128) gadget_kernel(GadgetArgs a) {
    extern __shared__ uint64_t gsm[];
    uint64_t* v = gsm + threadIdx.x * (a.W + 1);
    const uint64_t half = (a.basis + 1) / 2;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < a.count; x += (size_t)gridDim.x * blockDim.x) {
        const uint64_t* src = a.vals + x * a.W;
        // global loads (not generic ones, which would wait for each preceding
        // shared-memory store), so the W limbs are requested back to back
        for (uint32_t k = 0; k < a.W; ++k) v[k] = ld_cached(src + k);
        v[a.W] = 0;  // guard limb for the straddling mask read (its mask is 0 there)
        if (a.has_split) {
            int cmp = 0;
            for (uint32_t k = a.W; k-- > 0;) {
                const uint64_t sk = ld_table(a.split + k);
                if (cmp == 0 && v[k] != sk) cmp = v[k] < sk ? -1 : 1;
            }
            if (cmp >= 0) {
                uint64_t carry = 0;
                for (uint32_t k = 0; k < a.W; ++k) {
                    uint64_t s = v[k] + ld_table(a.npq + k);
                    uint64_t c1 = s < v[k];
                    uint64_t s2 = s + carry;
                    uint64_t c2 = s2 < s;
                    v[k] = s2;
                    carry = c1 | c2;
                }
            }
        }
        uint64_t carry = a.has_init ? ((v[a.init_index] & a.init_mask) != 0) : 0;
        for (uint32_t j = 0; j < a.d; ++j) {
            DigitMask m;  // read-only path (the generic load would wait for the stores above)
            {
                const ulonglong2 m0 = __ldg(reinterpret_cast<const ulonglong2*>(a.masks + j));
                const ulonglong2 m1 = __ldg(reinterpret_cast<const ulonglong2*>(a.masks + j) + 1);
                m.index = (uint32_t)m0.x;
                m.shr = (uint32_t)(m0.x >> 32);
                m.shl = (uint32_t)m0.y;
                m.pad = (uint32_t)(m0.y >> 32);
                m.mask0 = m1.x;
                m.mask1 = m1.y;
            }
            uint64_t temp = (v[m.index] & m.mask0) >> m.shr;
            if (m.mask1 != 0) temp |= (v[m.index + 1] & m.mask1) << m.shl;
            temp += carry;
            carry = (temp & a.carry_mask) != 0;
            const uint64_t digit = temp & a.bm1;
            const size_t p = x / a.n, c = x % a.n;
            if constexpr (LIFT) {
                uint64_t* o = a.out + ((p * a.d + j) * a.L) * a.n + c;
                for (uint32_t l = 0; l < a.L; ++l)
                    o[(size_t)l * a.n] = (a.basis == 2 || digit < half) ? digit : ld_table(a.moduli + l) - a.basis + digit;
            } else {
                a.out[(p * a.d + j) * a.n + c] = digit;
            }
        }
    }
}

void free_base(pg_rns_base* b) {
    if (!b) return;
    cudaFree(b->d_moduli);
    cudaFree(b->d_product);
    cudaFree(b->d_punctured);
    cudaFree(b->d_inv);
    cudaFree(b->d_bar);
    delete b;
}

void free_basis(pg_gadget_basis* g) {
    if (!g) return;
    cudaFree(g->d_split);
    cudaFree(g->d_npq);
    cudaFree(g->d_masks);
    delete g;
}

template <typename T>
cudaError_t upload(T** d, const T* h, size_t n) {
    cudaError_t e = cudaMalloc((void**)d, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess && n) e = cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

template <int W>
int launch_compose_w(const ComposeArgs& a, cudaStream_t st) {
    compose_kernel<W><<<grid_for(a.count, 128), 128, 0, st>>>(a);
    count_launch();
    PG_LAUNCH_CHECK("compose_kernel launch");
    return PG_OK;
}

}  // namespace

namespace pg {
// compose `count` coefficients laid out as described at ComposeArgs
int launch_compose(const pg_rns_base* b, const uint64_t* res, uint64_t* out, size_t count, size_t n, uint32_t ppg,
                   size_t group_stride, cudaStream_t st) {
    ComposeArgs a{};
    a.res = res;
    a.out = out;
    a.count = count;
    a.n = n;
    a.ppg = ppg;
    a.group_stride = group_stride;
    a.L = b->L;
    a.moduli = b->d_moduli;
    a.inv = b->d_inv;
    a.punct = b->d_punctured;
    a.prod = b->d_product;
    switch (b->W) {
#define PG_W(w) \
    case w: return launch_compose_w<w>(a, st);
        PG_W(1) PG_W(2) PG_W(3) PG_W(4) PG_W(5) PG_W(6) PG_W(7) PG_W(8) PG_W(9) PG_W(10) PG_W(11) PG_W(12)
        PG_W(13) PG_W(14) PG_W(15) PG_W(16) PG_W(17) PG_W(18) PG_W(19) PG_W(20) PG_W(21) PG_W(22) PG_W(23) PG_W(24)
#undef PG_W
        default: return set_error(PG_ERR_UNSUPPORTED, "RNS compose supports products of up to 24 limbs");
    }
}

int launch_gadget(const pg_gadget_basis* g, const uint64_t* vals, uint64_t* out, size_t count, size_t n, bool lift,
                  cudaStream_t st) {
    if (count == 0) return PG_OK;
    GadgetArgs a{};
    a.vals = vals;
    a.out = out;
    a.count = count;
    a.n = n;
    a.W = g->W;
    a.L = g->L;
    a.d = g->d;
    a.bm1 = g->bm1;
    a.carry_mask = g->carry_mask;
    a.basis = g->basis;
    a.has_split = g->has_split;
    a.has_init = g->has_init;
    a.init_index = g->init_index;
    a.init_mask = g->init_mask;
    a.split = g->d_split;
    a.npq = g->d_npq;
    a.masks = g->d_masks;
    a.moduli = g->base->d_moduli;
    const size_t smem = 128 * (g->W + 1) * sizeof(uint64_t);
    if (lift)
        gadget_kernel<true><<<grid_for(count, 128), 128, smem, st>>>(a);
    else
        gadget_kernel<false><<<grid_for(count, 128), 128, smem, st>>>(a);
    count_launch();
    PG_LAUNCH_CHECK("gadget_kernel launch");
    return PG_OK;
}
}  // namespace pg

// ===================================================================== C ABI
extern "C" {

// RNSBase::new (base.rs:50-90) with multiply_many_values / _except_inplace
// (primus_integer/src/big_integer.rs:647-706)
int pg_rns_base_create(const uint64_t* h_moduli, uint32_t L, pg_rns_base** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!h_moduli || L == 0 || L > 64) return set_error(PG_ERR_INVALID_ARGUMENT, "need 1..64 moduli");
    for (uint32_t i = 0; i < L; ++i) {
        if (h_moduli[i] < 2 || (h_moduli[i] >> 62) != 0)
            return set_error(PG_ERR_INVALID_ARGUMENT, "moduli must be in [2, 2^62)");
        for (uint32_t j = i + 1; j < L; ++j)
            if (gcd64(h_moduli[i], h_moduli[j]) != 1) return set_error(PG_ERR_NOT_COPRIME, "moduli are not co-prime");
    }
    pg_rns_base* b = new (std::nothrow) pg_rns_base();
    if (!b) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    b->L = L;
    b->moduli.assign(h_moduli, h_moduli + L);
    Big prod(L + 1, 0);
    size_t len = 1;
    prod[0] = h_moduli[0];
    for (uint32_t i = 1; i < L; ++i) {
        uint64_t c = 0;
        for (size_t k = 0; k < len; ++k) {
            u128 t = (u128)prod[k] * h_moduli[i] + c;
            prod[k] = (uint64_t)t;
            c = (uint64_t)(t >> 64);
        }
        if (c) prod[len++] = c;
    }
    b->W = (uint32_t)len;
    prod.resize(len);
    b->product = prod;
    b->punctured.assign((size_t)L * len, 0);
    b->inv.resize(L);
    b->inv_q.resize(L);
    std::vector<Barrett> bar(L);
    std::vector<ulonglong2> inv2(L);
    for (uint32_t i = 0; i < L; ++i) {
        uint64_t* r = &b->punctured[(size_t)i * len];
        r[0] = 1;
        size_t rl = 1;
        for (uint32_t j = 0; j < L; ++j) {
            if (j == i) continue;
            uint64_t c = 0;
            for (size_t k = 0; k < rl; ++k) {
                u128 t = (u128)r[k] * h_moduli[j] + c;
                r[k] = (uint64_t)t;
                c = (uint64_t)(t >> 64);
            }
            if (c) r[rl++] = c;
        }
        uint64_t iv = h_invmod(big_mod(r, len, h_moduli[i]), h_moduli[i]);
        b->inv[i] = iv;
        b->inv_q[i] = h_shoup_quotient(iv, h_moduli[i]);
        inv2[i] = make_ulonglong2(iv, b->inv_q[i]);
        bar[i] = h_barrett(h_moduli[i]);
    }
    cudaError_t e = upload(&b->d_moduli, h_moduli, L);
    if (e == cudaSuccess) e = upload(&b->d_product, b->product.data(), len);
    if (e == cudaSuccess) e = upload(&b->d_punctured, b->punctured.data(), (size_t)L * len);
    if (e == cudaSuccess) e = upload(&b->d_inv, inv2.data(), L);
    if (e == cudaSuccess) e = upload(&b->d_bar, bar.data(), L);
    if (e != cudaSuccess) {
        free_base(b);
        return cuda_status(e, "pg_rns_base_create: device upload");
    }
    *out = b;
    return PG_OK;
}

int pg_rns_base_destroy(pg_rns_base* base) {
    free_base(base);
    return PG_OK;
}

int pg_rns_base_info(const pg_rns_base* b, uint32_t* L, uint32_t* W, uint64_t* h_product) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "base is NULL");
    if (L) *L = b->L;
    if (W) *W = b->W;
    if (h_product) std::copy(b->product.begin(), b->product.end(), h_product);
    return PG_OK;
}

int pg_rns_compose(const pg_rns_base* b, const uint64_t* d_res, uint64_t* d_vals, size_t count, void* stream) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "base is NULL");
    if (count == 0) return PG_OK;
    if (!d_res || !d_vals) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    return launch_compose(b, d_res, d_vals, count, count, 1, (size_t)b->L * count, (cudaStream_t)stream);
}

int pg_rns_decompose(const pg_rns_base* b, const uint64_t* d_vals, uint64_t* d_res, size_t count, void* stream) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "base is NULL");
    if (count == 0) return PG_OK;
    if (!d_res || !d_vals) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    decompose_kernel<<<grid_for(count * b->L, 256), 256, 0, (cudaStream_t)stream>>>(d_vals, d_res, count, b->L, b->W,
                                                                                    b->d_bar);
    count_launch();
    PG_LAUNCH_CHECK("decompose_kernel launch");
    return PG_OK;
}

int pg_rns_wrapping_decompose_small(const pg_rns_base* b, const uint64_t* d_small, uint64_t* d_res, size_t count,
                                    uint64_t small_modulus, void* stream) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "base is NULL");
    if (count == 0) return PG_OK;
    if (!d_small || !d_res) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    for (uint64_t q : b->moduli)
        if (q <= small_modulus) return set_error(PG_ERR_INVALID_ARGUMENT, "every modulus must exceed small_modulus");
    wrap_small_kernel<<<grid_for(count * b->L, 256), 256, 0, (cudaStream_t)stream>>>(d_small, d_res, count, b->L,
                                                                                     b->d_moduli, small_modulus);
    count_launch();
    PG_LAUNCH_CHECK("wrap_small_kernel launch");
    return PG_OK;
}

int pg_rns_add_wrapping_decompose_small_scaled(const pg_rns_base* b, const uint64_t* d_small, uint64_t* d_dest,
                                               size_t count, uint64_t small_modulus, const uint64_t* h_factor,
                                               void* stream) {
    if (!b) return set_error(PG_ERR_INVALID_ARGUMENT, "base is NULL");
    if (count == 0) return PG_OK;
    if (!d_small || !d_dest || !h_factor) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (small_modulus < 2) return set_error(PG_ERR_INVALID_ARGUMENT, "small_modulus must be at least 2");
    std::vector<ulonglong2> f(b->L);
    for (uint32_t l = 0; l < b->L; ++l) {
        const uint64_t q = b->moduli[l];
        if (q <= small_modulus) return set_error(PG_ERR_INVALID_ARGUMENT, "every modulus must exceed small_modulus");
        if (h_factor[l] >= q) return set_error(PG_ERR_INVALID_ARGUMENT, "factor not below its modulus");
        f[l] = make_ulonglong2(h_factor[l], h_shoup_quotient(h_factor[l], q));
    }
    cudaStream_t st = (cudaStream_t)stream;
    void* d_f = nullptr;
    PG_CUDA(scratch_alloc(&d_f, b->L * sizeof(ulonglong2), st));
    // pageable source: the copy below completes before the call returns
    cudaError_t e = cudaMemcpyAsync(d_f, f.data(), b->L * sizeof(ulonglong2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        add_wrap_scaled_kernel<<<grid_for(count * b->L, 256), 256, 0, st>>>(d_small, d_dest, count, b->L,
                                                                             b->d_moduli, (const ulonglong2*)d_f,
                                                                             small_modulus);
        count_launch();
        e = cudaGetLastError();
    }
    scratch_free(d_f, st);
    if (e != cudaSuccess) return cuda_status(e, "add_wrap_scaled_kernel");
    return PG_OK;
}

// BaseConverter::new (converter.rs:22-47)
int pg_base_converter_create(const pg_rns_base* ib, const pg_rns_base* ob, pg_base_converter** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!ib || !ob) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL base");
    pg_base_converter* c = new (std::nothrow) pg_base_converter();
    if (!c) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    c->ibase = ib;
    c->obase = ob;
    std::vector<uint64_t> m((size_t)ib->L * ob->L);
    for (uint32_t j = 0; j < ob->L; ++j)
        for (uint32_t i = 0; i < ib->L; ++i)
            m[(size_t)j * ib->L + i] = big_mod(&ib->punctured[(size_t)i * ib->W], ib->W, ob->moduli[j]);
    cudaError_t e = upload(&c->d_matrix, m.data(), m.size());
    if (e != cudaSuccess) {
        cudaFree(c->d_matrix);
        delete c;
        return cuda_status(e, "pg_base_converter_create: device upload");
    }
    *out = c;
    return PG_OK;
}

int pg_base_converter_destroy(pg_base_converter* c) {
    if (c) {
        cudaFree(c->d_matrix);
        delete c;
    }
    return PG_OK;
}

int pg_fast_convert_array(const pg_base_converter* c, const uint64_t* d_in, uint64_t* d_out, size_t n, void* stream) {
    if (!c) return set_error(PG_ERR_INVALID_ARGUMENT, "converter is NULL");
    if (n == 0) return PG_OK;
    if (!d_in || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    fast_convert_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        d_in, d_out, n, c->ibase->L, c->obase->L, c->ibase->d_moduli, c->ibase->d_inv, c->obase->d_bar, c->d_matrix);
    count_launch();
    PG_LAUNCH_CHECK("fast_convert_kernel launch");
    return PG_OK;
}

// BigUintApproxSignedBasis::new (primus_decompose/src/big_integer/basis.rs:34-193)
int pg_gadget_basis_create(const pg_rns_base* base, uint32_t log_basis, int32_t reverse_length,
                           pg_gadget_basis** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!base) return set_error(PG_ERR_INVALID_ARGUMENT, "base is NULL");
    if (log_basis == 0 || log_basis >= 64) return set_error(PG_ERR_INVALID_ARGUMENT, "log_basis must be in [1, 63]");
    const uint32_t W = base->W;
    const uint64_t* Q = base->product.data();
    pg_gadget_basis* g = new (std::nothrow) pg_gadget_basis();
    if (!g) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    g->base = base;
    g->W = W;
    g->L = base->L;
    g->log_basis = log_basis;
    const uint32_t unused = (uint32_t)__builtin_clzll(Q[W - 1]);
    g->basis = 1ull << log_basis;
    g->bm1 = g->basis - 1;
    const uint32_t bits = 64 * W - unused;
    uint32_t d = bits / log_basis;
    uint32_t drop = bits - d * log_basis;
    if (reverse_length >= 0) {
        if ((uint32_t)reverse_length > d || reverse_length == 0) {
            free_basis(g);
            return set_error(PG_ERR_INVALID_ARGUMENT, "reverse_length must be in [1, floor(bits(Q)/log_basis)]");
        }
        d = (uint32_t)reverse_length;
        drop = bits - d * log_basis;
    }
    g->d = d;
    g->drop_bits = drop;
    if (drop > 0) {
        g->has_init = true;
        g->init_index = (drop - 1) / 64;
        g->init_mask = 1ull << ((drop - 1) % 64);
    }
    g->carry_mask = log_basis == 1 ? 2ull : ((1ull << log_basis) | (1ull << (log_basis - 1)));
    // split value
    Big v(W, 0);
    bool has_split = false;
    if (log_basis == 1) {
        if (drop != 0) {
            for (uint32_t i = 0; i < d; ++i) {
                big_shl(v.data(), W, 1);
                v[0] |= 1;
            }
            big_shl(v.data(), W, 1);
            v[0] |= 1;
            big_shl_any(v.data(), W, drop - 1);
            has_split = big_cmp(v.data(), Q, W) < 0;
        }
    } else {
        for (uint32_t i = 0; i < d; ++i) {
            big_shl(v.data(), W, log_basis);
            v[0] |= g->bm1 >> 1;
        }
        if (drop > 0) {
            big_shl(v.data(), W, 1);
            v[0] |= 1;
            big_shl_any(v.data(), W, drop - 1);
        } else {
            Big one(W, 0);
            one[0] = 1;
            big_add(v.data(), one.data(), W);
        }
        has_split = big_cmp(v.data(), Q, W) < 0;
    }
    g->has_split = has_split;
    g->split = v;
    // next_pow_of_2_sub_modulus = (2^bits - 1) - (Q - 1)
    g->npq.assign(W, ~0ull);
    g->npq[W - 1] = unused == 64 ? 0 : (~0ull >> unused);
    Big qm1(Q, Q + W), one(W, 0);
    one[0] = 1;
    big_sub(qm1.data(), one.data(), W);
    big_sub(g->npq.data(), qm1.data(), W);
    // gadget scalars 2^(drop + j*log_basis) and their residues
    g->scalars.assign((size_t)d * W, 0);
    g->scalar_residues.assign((size_t)d * base->L, 0);
    Big cur(W, 0);
    cur[0] = 1;
    big_shl_any(cur.data(), W, drop);
    for (uint32_t j = 0; j < d; ++j) {
        if (j > 0) big_shl(cur.data(), W, log_basis);
        std::copy(cur.begin(), cur.end(), g->scalars.begin() + (size_t)j * W);
        for (uint32_t l = 0; l < base->L; ++l)
            g->scalar_residues[(size_t)j * base->L + l] = big_mod(cur.data(), W, base->moduli[l]);
    }
    // value masks (common.rs:16-53)
    g->masks.resize(d);
    uint32_t index = drop / 64, shr = drop % 64;
    for (uint32_t j = 0; j < d; ++j) {
        if (j > 0) {
            uint32_t ns = log_basis + shr;
            if (ns >= 64) {
                index += 1;
                ns -= 64;
            }
            shr = ns;
        }
        DigitMask m{};
        m.index = index;
        m.shr = shr;
        m.shl = 64 - shr;
        m.mask0 = g->bm1 << shr;
        m.mask1 = shr == 0 ? 0 : (g->bm1 >> (64 - shr));
        g->masks[j] = m;
    }
    cudaError_t e = upload(&g->d_split, g->split.data(), W);
    if (e == cudaSuccess) e = upload(&g->d_npq, g->npq.data(), W);
    if (e == cudaSuccess) e = upload(&g->d_masks, g->masks.data(), d);
    if (e != cudaSuccess) {
        free_basis(g);
        return cuda_status(e, "pg_gadget_basis_create: device upload");
    }
    *out = g;
    return PG_OK;
}

int pg_gadget_basis_destroy(pg_gadget_basis* g) {
    free_basis(g);
    return PG_OK;
}

int pg_gadget_basis_info(const pg_gadget_basis* g, uint32_t* d, uint32_t* drop, uint64_t* h_scalar_residues) {
    if (!g) return set_error(PG_ERR_INVALID_ARGUMENT, "basis is NULL");
    if (d) *d = g->d;
    if (drop) *drop = g->drop_bits;
    if (h_scalar_residues) std::copy(g->scalar_residues.begin(), g->scalar_residues.end(), h_scalar_residues);
    return PG_OK;
}

int pg_gadget_decompose(const pg_gadget_basis* g, const uint64_t* d_vals, uint64_t* d_digits, size_t count,
                        void* stream) {
    if (!g) return set_error(PG_ERR_INVALID_ARGUMENT, "basis is NULL");
    if (count && (!d_vals || !d_digits)) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    return launch_gadget(g, d_vals, d_digits, count, count, false, (cudaStream_t)stream);
}

int pg_gadget_decompose_lift(const pg_gadget_basis* g, const uint64_t* d_vals, uint64_t* d_res, size_t count,
                             void* stream) {
    if (!g) return set_error(PG_ERR_INVALID_ARGUMENT, "basis is NULL");
    if (count && (!d_vals || !d_res)) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    for (uint64_t q : g->base->moduli)
        if (q <= g->basis) return set_error(PG_ERR_INVALID_ARGUMENT, "every modulus must exceed the gadget basis");
    return launch_gadget(g, d_vals, d_res, count, count, true, (cudaStream_t)stream);
}

}  // extern "C"
