// Hybrid RNS key switch with special primes.
//
// The reference's key switch decomposes each mask poly into BigUint gadget
// digits (primus_fhe_core/src/key_switch.rs:79-128).  This is the other standard
// form, over a modulus chain Q (L primes) extended by K special primes P, with
// digit groups of `alpha` consecutive Q limbs (dnum = ceil(L / alpha) groups).
// The reference has no such path, so its definition is this build's own, stated
// once more here:
//
//   for each input mask a_i (coefficient form over Q) and group g:
//     ModUp:  ext = a_i's residues on the limbs of D_g, and on every other limb
//             of QP the fast base conversion of those residues
//             (fast_convert_array semantics, primus_rns/src/converter.rs:147-175)
//     acc[c] += NTT(ext) (.) key[i][g][c]              (over QP, NTT domain)
//   ModDown of acc[c]: inverse NTT of its P limbs, fast conversion P -> Q,
//     forward NTT, then (acc_Q - conv) * P^-1 mod q_l
//   c_out = -ModDown(acc) + (0, .., NTT(b))           (the reference's sign form)
//
// Evaluated through the linearity of the NTT as
//   c_out[c] = NTT(P^-1 conv[c] + [c = last] b) - P^-1 acc_Q[c]
// (P^-1 folded into the conversion matrix, b added in coefficient form), so b
// needs no transform of its own; the residues are the same.
//
// The key row [i][g] encrypts P * (Q/Q_g) * ((Q/Q_g)^-1 mod Q_g) * s_in_i under
// s_out over QP, i.e. [P]_{q_l} * s_in_i on the limbs of D_g and 0 elsewhere.
//
// Launch sequence for a batch: modup_kernel -> forward NTT of every extended
// row -> the MAC kernel (Q and P limbs written apart) -> inverse NTT of the P
// limbs -> pconv_kernel (P -> Q, scaled by P^-1, b added on the last output)
// -> forward NTT of the converted rows -> finish_kernel.  Each step runs over
// the whole batch in one launch.  On the FP64 schedule at N = 2^13 .. 2^16 the
// conversions run inside the transforms' loads and stores instead (the fused
// form below): scale -> forward(ModUp on load) -> MAC -> inverse(P scaling on
// store) -> forward(P -> Q on load, final combination on store).
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "ntt_kernels.cuh"

using namespace pg;

namespace {
constexpr uint32_t kMaxAlpha = 8;  // residues held per thread in ModUp
constexpr uint32_t kMaxK = 8;      // special primes held per thread in ModDown
}  // namespace

struct pg_hybrid_ks {
    const pg_ntt_table* t = nullptr;  // L + K primes: Q then P
    pg_ntt_table tq, tp;              // views of the Q and P limbs (no ownership)
    uint32_t L = 0, K = 0, alpha = 0, dnum = 0;
    ulonglong2* d_ginv = nullptr;  // [L] Shoup pair of ((Q_g/q_i)^-1 mod q_i), q_i in group g
    ulonglong2* d_gmat = nullptr;  // per group g: [L+K-alpha_g][alpha_g] Shoup pair of (Q_g/q_i) mod r_j, at gmat_off[g]
    uint32_t* d_gout = nullptr;    // per group g: [L+K-alpha_g] output limb indices, at gout_off[g]
    std::vector<uint32_t> gmat_off, gout_off;
    ulonglong2* d_pinv_k = nullptr;  // [K] Shoup pair of ((P/p_k)^-1 mod p_k)
    ulonglong2* d_pmat = nullptr;    // [L][K] Shoup pair of (P/p_k) * P^-1 mod q_l
    ulonglong2* d_pinv = nullptr;    // [L] Shoup pair of (P^-1 mod q_l)
    uint32_t* d_offs = nullptr;      // [2 * dnum]: gmat_off then gout_off
    // FP64 copies for moduli below 2^50: (w, w / r) as doubles, and (q, 1/q) per limb
    ulonglong2* d_gmat_fp = nullptr;
    ulonglong2* d_pmat_fp = nullptr;
    ulonglong2* d_fmod = nullptr;  // [L+K]
};

namespace {

// v mod q for v < 16 q
PG_DEV uint64_t reduce_below_16q(uint64_t v, uint64_t q) {
    v = v >= 8 * q ? v - 8 * q : v;
    v = v >= 4 * q ? v - 4 * q : v;
    v = v >= 2 * q ? v - 2 * q : v;
    return v >= q ? v - q : v;
}

struct ModUpArgs {
    const uint64_t* in;  // [B][k_in+1][L][N]
    uint64_t* ext;       // [B*k_in][dnum][L+K][N]
    const ulonglong2* ginv;
    const ulonglong2* gmat;
    const ulonglong2* gmat_fp;  // FP64 form of gmat (FP kernels)
    const ulonglong2* fmod;     // [L+K] (q, 1/q) as doubles (FP kernels)
    const uint32_t* gout;
    const uint32_t* gmat_off;  // [dnum]
    const uint32_t* gout_off;  // [dnum]
    const uint64_t* moduli;    // [L+K]
    const Barrett* bar;        // [L+K]
    size_t polys, N;           // polys = B * k_in
    uint32_t k_in, L, K, alpha, dnum, log_n;
};

// one thread per (input mask, group, coefficient); grid y = mask * dnum + group.
// AMAX bounds the group size (registers held per thread).  FP: the dot products
// run on the FP64 pipe (fmulmod, every modulus below 2^50): each product lies in
// (-0.75 r, 0.75 r), a sum of at most 8 below 6 r < 2^53, reduced exactly to [0, r).
template <uint32_t AMAX, bool FP>
__global__ void __launch_bounds__(256, 3) modup_kernel(ModUpArgs a) {
    const uint32_t LK = a.L + a.K;
    const size_t outer = a.polys * a.dnum;
    for (size_t o = blockIdx.y; o < outer; o += gridDim.y) {
        const uint32_t g = (uint32_t)(o % a.dnum);
        const size_t p = o / a.dnum;  // b * k_in + i
        const size_t b = p / a.k_in, i = p % a.k_in;
        const uint64_t* src0 = a.in + ((b * (a.k_in + 1) + i) * a.L) * a.N;
        uint64_t* dst0 = a.ext + (o * LK) * a.N;
        const uint32_t lo = g * a.alpha, hi = min(a.L, lo + a.alpha), ag = hi - lo;
        const ulonglong2* mat = a.gmat + a.gmat_off[g];
        const uint32_t* outl = a.gout + a.gout_off[g];
        // two coefficients per thread (x and x + blockDim.x): twice the independent
        // work per loaded matrix entry
        for (uint32_t x0 = blockIdx.x * 2 * blockDim.x + threadIdx.x; x0 < a.N; x0 += gridDim.x * 2 * blockDim.x) {
            const uint32_t x1 = x0 + blockDim.x;
            const bool two = x1 < a.N;
            uint64_t tv0[AMAX], tv1[AMAX];
#pragma unroll
            for (uint32_t m = 0; m < AMAX; ++m) {
                tv0[m] = tv1[m] = 0;
                if (m < ag) {
                    const uint32_t l = lo + m;
                    const ulonglong2 f = a.ginv[l];
                    const uint64_t ql = a.moduli[l];
                    const uint64_t v0 = src0[(size_t)l * a.N + x0];
                    dst0[(size_t)l * a.N + x0] = v0;
                    tv0[m] = shoup_mul(f.x, f.y, v0, ql);
                    if (two) {
                        const uint64_t v1 = src0[(size_t)l * a.N + x1];
                        dst0[(size_t)l * a.N + x1] = v1;
                        tv1[m] = shoup_mul(f.x, f.y, v1, ql);
                    }
                }
            }
            if constexpr (FP) {
                double td0[AMAX], td1[AMAX];
#pragma unroll
                for (uint32_t m = 0; m < AMAX; ++m) {
                    td0[m] = u52_to_f(tv0[m]);
                    td1[m] = u52_to_f(tv1[m]);
                }
                const ulonglong2* matf = a.gmat_fp + a.gmat_off[g];
#pragma unroll 2
                for (uint32_t j = 0; j < LK - ag; ++j) {
                    const uint32_t r = outl[j];
                    const ulonglong2 fm = a.fmod[r];
                    const double rd = as_f(fm.x), rinv = as_f(fm.y);
                    double y0 = 0.0, y1 = 0.0;
#pragma unroll
                    for (uint32_t m = 0; m < AMAX; ++m)
                        if (m < ag) {
                            const ulonglong2 w = matf[j * ag + m];
                            y0 = __dadd_rn(y0, fmulmod(td0[m], as_f(w.x), as_f(w.y), rd));
                            y1 = __dadd_rn(y1, fmulmod(td1[m], as_f(w.x), as_f(w.y), rd));
                        }
                    uint64_t* d = dst0 + (size_t)r * a.N;
                    d[x0] = f_to_u52(fcanon(freduce(y0, rd, rinv), rd));
                    if (two) d[x1] = f_to_u52(fcanon(freduce(y1, rd, rinv), rd));
                }
            } else {
#pragma unroll 2
                for (uint32_t j = 0; j < LK - ag; ++j) {
                    const uint32_t r = outl[j];
                    const uint64_t rq = a.moduli[r], nq = 0 - rq;
                    // sums of at most 8 lazy products in [0, 2 r): below 16 r < 2^64
                    uint64_t y0 = 0, y1 = 0;
#pragma unroll
                    for (uint32_t m = 0; m < AMAX; ++m)
                        if (m < ag) {
                            const ulonglong2 w = mat[j * ag + m];
                            y0 += shoup_lazy_nq(w.x, w.y, tv0[m], nq);
                            y1 += shoup_lazy_nq(w.x, w.y, tv1[m], nq);
                        }
                    // [0, 4 r) is enough: the forward NTT that follows accepts inputs below
                    // 4q and returns canonical values of the same residues
                    if (AMAX > 4) {
                        y0 = y0 >= 8 * rq ? y0 - 8 * rq : y0;
                        y1 = y1 >= 8 * rq ? y1 - 8 * rq : y1;
                    }
                    uint64_t* d = dst0 + (size_t)r * a.N;
                    d[x0] = y0 >= 4 * rq ? y0 - 4 * rq : y0;
                    if (two) d[x1] = y1 >= 4 * rq ? y1 - 4 * rq : y1;
                }
            }
        }
    }
}

struct PConvArgs {
    const uint64_t* accp;  // [PC][K][N], coefficient form
    uint64_t* conv;        // [PC][L][N]
    const uint64_t* bsrc;  // b of ciphertext j at bsrc + j * bstride ([L][N], coefficient form)
    size_t bstride;
    uint32_t ko;           // output polys per ciphertext (b goes to the last)
    const ulonglong2* pinv_k;
    const ulonglong2* pmat;     // [L][K]
    const ulonglong2* pmat_fp;  // FP64 form of pmat (FP kernels)
    const ulonglong2* fmod;     // [L+K] (q, 1/q) as doubles (FP kernels)
    const uint64_t* moduli;     // [L+K]
    const Barrett* bar;         // [L+K]
    size_t pc, N;
    uint32_t L, K, log_n;
};

// fast conversion of the P limbs to the Q limbs, one thread per (poly, coefficient); grid y = poly.
// KMAX bounds the special prime count (registers held per thread).  FP: the dot
// products on the FP64 pipe, as in modup_kernel.
template <uint32_t KMAX, bool FP>
__global__ void __launch_bounds__(256) pconv_kernel(PConvArgs a) {
    for (size_t p = blockIdx.y; p < a.pc; p += gridDim.y) {
        const uint64_t* src = a.accp + (p * a.K) * a.N;
        uint64_t* dst = a.conv + (p * a.L) * a.N;
        // the last output poly of each ciphertext also takes b (coefficient form)
        const uint64_t* bp = (p % a.ko) == a.ko - 1 ? a.bsrc + (p / a.ko) * a.bstride : nullptr;
        // two coefficients per thread (x and x + blockDim.x)
        for (uint32_t x0 = blockIdx.x * 2 * blockDim.x + threadIdx.x; x0 < a.N; x0 += gridDim.x * 2 * blockDim.x) {
            const uint32_t x1 = x0 + blockDim.x;
            const bool two = x1 < a.N;
            uint64_t tv0[KMAX], tv1[KMAX];
#pragma unroll
            for (uint32_t k = 0; k < KMAX; ++k) {
                tv0[k] = tv1[k] = 0;
                if (k < a.K) {
                    const ulonglong2 f = a.pinv_k[k];
                    const uint64_t pk = a.moduli[a.L + k];
                    tv0[k] = shoup_mul(f.x, f.y, src[(size_t)k * a.N + x0], pk);
                    if (two) tv1[k] = shoup_mul(f.x, f.y, src[(size_t)k * a.N + x1], pk);
                }
            }
            if constexpr (FP) {
                double td0[KMAX], td1[KMAX];
#pragma unroll
                for (uint32_t k = 0; k < KMAX; ++k) {
                    td0[k] = u52_to_f(tv0[k]);
                    td1[k] = u52_to_f(tv1[k]);
                }
#pragma unroll 2
                for (uint32_t l = 0; l < a.L; ++l) {
                    const ulonglong2 fm = a.fmod[l];
                    const double qd = as_f(fm.x), qinv = as_f(fm.y);
                    double y0 = 0.0, y1 = 0.0;
#pragma unroll
                    for (uint32_t k = 0; k < KMAX; ++k)
                        if (k < a.K) {
                            const ulonglong2 w = a.pmat_fp[l * a.K + k];
                            y0 = __dadd_rn(y0, fmulmod(td0[k], as_f(w.x), as_f(w.y), qd));
                            y1 = __dadd_rn(y1, fmulmod(td1[k], as_f(w.x), as_f(w.y), qd));
                        }
                    uint64_t r0 = f_to_u52(fcanon(freduce(y0, qd, qinv), qd));
                    uint64_t r1 = two ? f_to_u52(fcanon(freduce(y1, qd, qinv), qd)) : 0;
                    if (bp) {
                        const uint64_t ql = a.moduli[l];
                        r0 = add_mod(r0, bp[(size_t)l * a.N + x0], ql);
                        if (two) r1 = add_mod(r1, bp[(size_t)l * a.N + x1], ql);
                    }
                    dst[(size_t)l * a.N + x0] = r0;
                    if (two) dst[(size_t)l * a.N + x1] = r1;
                }
            } else {
#pragma unroll 2
                for (uint32_t l = 0; l < a.L; ++l) {
                    const uint64_t ql = a.moduli[l], nq = 0 - ql;
                    // sums of at most 8 lazy products in [0, 2 q_l): below 16 q_l < 2^64
                    uint64_t y0 = 0, y1 = 0;
#pragma unroll
                    for (uint32_t k = 0; k < KMAX; ++k)
                        if (k < a.K) {
                            const ulonglong2 w = a.pmat[l * a.K + k];
                            y0 += shoup_lazy_nq(w.x, w.y, tv0[k], nq);
                            y1 += shoup_lazy_nq(w.x, w.y, tv1[k], nq);
                        }
                    uint64_t r0 = reduce_below_16q(y0, ql);
                    uint64_t r1 = two ? reduce_below_16q(y1, ql) : 0;
                    if (bp) {
                        r0 = add_mod(r0, bp[(size_t)l * a.N + x0], ql);
                        if (two) r1 = add_mod(r1, bp[(size_t)l * a.N + x1], ql);
                    }
                    dst[(size_t)l * a.N + x0] = r0;
                    if (two) dst[(size_t)l * a.N + x1] = r1;
                }
            }
        }
    }
}

struct FinishArgs {
    const uint64_t* accq;  // [B][KO][L][N]
    const uint64_t* conv;  // [B][KO][L][N] NTT(P^-1 conv + [last] b)
    uint64_t* out;         // [B][KO][L][N]
    const ulonglong2* pinv;
    const uint64_t* moduli;
    size_t B, N;
    uint32_t KO, L, log_n;
};

// out = NTT(P^-1 conv + [c = last] b) - acc_Q * P^-1; grid y = b * KO + c
__global__ void __launch_bounds__(256) finish_kernel(FinishArgs a) {
    const uint32_t LN = a.L * (uint32_t)a.N;
    const size_t outer = a.B * a.KO;
    for (size_t o = blockIdx.y; o < outer; o += gridDim.y) {
        const uint64_t* aq = a.accq + o * LN;
        const uint64_t* cv = a.conv + o * LN;
        uint64_t* out = a.out + o * LN;
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < LN; lx += gridDim.x * blockDim.x) {
            const uint32_t l = lx >> a.log_n;
            const uint64_t q = a.moduli[l];
            const ulonglong2 f = a.pinv[l];
            out[lx] = sub_mod(cv[lx], shoup_mul(f.x, f.y, aq[lx], q), q);
        }
    }
}



// ---------------------------------------------------------------------------
// Fused form (FP64 tables, N = 2^13 .. 2^16: the cluster transform).  The base
// conversions move into the transforms' loads and stores, so the extended rows
// and the converted rows never make a separate pass through HBM:
//   scale_kernel: tv[p][l] = [a_p]_{q_l} * ((Q_g / q_l)^-1 mod q_l) for every Q limb
//   forward NTT of the extended rows with ModUpIO: own-group limbs load a_p, the
//     others load sum_m tv[p][lo + m] * ((Q_g / q_m) mod r) (ModUp on the integer
//     pipe)
//   MAC (unchanged)
//   inverse NTT of the P limbs with PScaleIO: stores [acc_P]_{p_k} * ((P / p_k)^-1 mod p_k)
//   forward NTT of the Q limbs with PConvIO: loads sum_k tvp[k] * ((P / p_k) P^-1 mod q_l)
//     (+ b on the last output), stores NTT(..) - P^-1 acc_Q straight to the output
// Same residues as the unfused sequence: every step is the same exact modular
// arithmetic, and the transforms return canonical values for any input below 4q.
// It runs for batches of at most kFusedMaxBatch key switches (see pg_key_switch_hybrid).
// ---------------------------------------------------------------------------
struct ScaleArgs {
    const uint64_t* in;  // [B][k_in+1][L][N]
    uint64_t* tv;        // [B * k_in][L][N]
    const ulonglong2* ginv;
    const uint64_t* moduli;
    size_t polys, N;
    uint32_t k_in, L, log_n;
};

// one thread per (mask, limb, coefficient); grid y = mask
__global__ void __launch_bounds__(256) scale_kernel(ScaleArgs a) {
    const uint32_t LN = a.L * (uint32_t)a.N;
    for (size_t p = blockIdx.y; p < a.polys; p += gridDim.y) {
        const size_t b = p / a.k_in, i = p % a.k_in;
        const uint64_t* src = a.in + (b * (a.k_in + 1) + i) * LN;
        uint64_t* dst = a.tv + p * LN;
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < LN; lx += gridDim.x * blockDim.x) {
            const uint32_t l = lx >> a.log_n;
            const ulonglong2 f = __ldg(a.ginv + l);
            dst[lx] = shoup_mul(f.x, f.y, ld_stream(src + lx), ld_table(a.moduli + l));
        }
    }
}

// the extended rows ext[o][r] of o = (b k_in + i) dnum + g over the L + K limbs
struct ModUpIO {
    static constexpr bool kLoad = true, kStore = false;
    const uint64_t* in;          // [B][k_in+1][L][N]
    const uint64_t* tv;          // [B * k_in][L][N]
    const ulonglong2* gmat;      // per group: [L+K-alpha_g][alpha_g] Shoup pairs
    uint32_t k_in, L, K, alpha, dnum, log_n;

    template <int E>
    PG_DEV void load(uint64_t o, uint32_t r, uint64_t q, uint32_t i0, uint32_t stride, uint64_t (&x)[E]) const {
        const uint32_t g = (uint32_t)(o % dnum);
        const uint64_t p = o / dnum;
        const uint32_t lo = g * alpha, hi = min(L, lo + alpha), ag = hi - lo;
        if (r >= lo && r < hi) {  // the group's own limbs keep a_p's residues
            const uint64_t* src = in + (((p / k_in) * (k_in + 1) + p % k_in) * L + r) * ((uint64_t)1 << log_n) + i0;
#pragma unroll
            for (int jj = 0; jj < E; ++jj) x[jj] = ld_stream(src + (size_t)jj * stride);
            return;
        }
        // row j of the group's conversion matrix (every group before the last
        // has alpha limbs, so the group's matrix starts at g (L + K - alpha) alpha)
        const uint32_t j = r < lo ? r : r - ag;
        const ulonglong2* mat = gmat + (size_t)g * (L + K - alpha) * alpha + (size_t)j * ag;
        const uint64_t nq = 0 - q;
#pragma unroll
        for (int jj = 0; jj < E; ++jj) x[jj] = 0;
        for (uint32_t m = 0; m < ag; ++m) {
            const ulonglong2 w = __ldg(mat + m);
            const uint64_t* t = tv + (p * L + lo + m) * ((uint64_t)1 << log_n) + i0;
            // sums of at most 8 lazy products in [0, 2q): below 16q < 2^64
#pragma unroll
            for (int jj = 0; jj < E; ++jj) x[jj] += shoup_lazy_nq(w.x, w.y, ld_cached(t + (size_t)jj * stride), nq);
        }
#pragma unroll
        for (int jj = 0; jj < E; ++jj) {  // [0, 4q): a valid forward input
            uint64_t v = x[jj];
            v = v >= 8 * q ? v - 8 * q : v;
            x[jj] = v >= 4 * q ? v - 4 * q : v;
        }
    }
};

// inverse transform of the P limbs of acc[p] (p = b KO + c, rows p * K + k):
// stores [acc_P]_{p_k} * ((P / p_k)^-1 mod p_k), the scaled residues of the P -> Q conversion
struct PScaleIO {
    static constexpr bool kLoad = false, kStore = true;
    uint64_t* accp;              // [B*KO][K][N]
    const ulonglong2* pinv_k;    // [K]
    uint32_t K, log_n;

    template <int E, class V>
    PG_DEV void store(uint64_t p, uint32_t k, uint64_t q, uint32_t i0, uint32_t stride, V value) const {
        const ulonglong2 f = __ldg(pinv_k + k);
        uint64_t* dst = accp + ((p * K + k) << log_n) + i0;
#pragma unroll
        for (int jj = 0; jj < E; ++jj) dst[(size_t)jj * stride] = shoup_mul(f.x, f.y, value(jj), q);
    }
};

// forward transform of the converted Q rows (p = b KO + c, rows p * L + l):
// loads sum_k tvp[p][k] * ((P / p_k) P^-1 mod q_l) (+ b of ciphertext b on the
// last output), stores NTT(..) - P^-1 acc_Q[p][l] to the output
struct PConvIO {
    static constexpr bool kLoad = true, kStore = true;
    const uint64_t* tvp;         // [B*KO][K][N] (PScaleIO's stores)
    const ulonglong2* pmat;      // [L][K]
    const uint64_t* bsrc;        // b of ciphertext j at bsrc + j * bstride
    size_t bstride;
    const uint64_t* accq;        // [B*KO][L][N]
    const ulonglong2* pinv;      // [L]
    uint64_t* out;               // [B*KO][L][N]
    uint32_t K, L, ko, log_n;

    template <int E>
    PG_DEV void load(uint64_t p, uint32_t l, uint64_t q, uint32_t i0, uint32_t stride, uint64_t (&x)[E]) const {
        const uint64_t nq = 0 - q;
#pragma unroll
        for (int jj = 0; jj < E; ++jj) x[jj] = 0;
        for (uint32_t k = 0; k < K; ++k) {
            const ulonglong2 w = __ldg(pmat + (size_t)l * K + k);
            const uint64_t* t = tvp + ((p * K + k) << log_n) + i0;
            // sums of at most 8 lazy products in [0, 2q): below 16q
#pragma unroll
            for (int jj = 0; jj < E; ++jj) x[jj] += shoup_lazy_nq(w.x, w.y, ld_cached(t + (size_t)jj * stride), nq);
        }
        const uint64_t* bp = (p % ko) == ko - 1 ? bsrc + (p / ko) * bstride + ((uint64_t)l << log_n) + i0 : nullptr;
#pragma unroll
        for (int jj = 0; jj < E; ++jj) {
            uint64_t v = reduce_below_16q(x[jj], q);
            if (bp) v += ld_stream(bp + (size_t)jj * stride);  // below 2q: a valid forward input
            x[jj] = v;
        }
    }

    template <int E, class V>
    PG_DEV void store(uint64_t p, uint32_t l, uint64_t q, uint32_t i0, uint32_t stride, V value) const {
        const size_t base = ((p * L + l) << log_n) + i0;
        // every acc_Q load is issued before the first output store (out may
        // alias acc_Q as far as the compiler knows, which would serialise them)
        uint64_t acc[E];
#pragma unroll
        for (int jj = 0; jj < E; ++jj) acc[jj] = ld_stream(accq + base + (size_t)jj * stride);
        const ulonglong2 f = __ldg(pinv + l);
#pragma unroll
        for (int jj = 0; jj < E; ++jj)
            out[base + (size_t)jj * stride] = sub_mod(value(jj), shoup_mul(f.x, f.y, acc[jj], q), q);
    }
};

// a table view over limbs [first, first + count) of t (device arrays shared)
void make_view(const pg_ntt_table* t, uint32_t first, uint32_t count, pg_ntt_table& v) {
    v.log_n = t->log_n;
    v.L = count;
    v.n = t->n;
    v.device = t->device;
    v.moduli.assign(t->moduli.begin() + first, t->moduli.begin() + first + count);
    v.d_moduli = t->d_moduli + first;
    v.d_fwd = t->d_fwd + (size_t)first * t->n;
    v.d_inv = t->d_inv + (size_t)first * t->n;
    v.d_ordinal = t->d_ordinal + (size_t)first * 2 * t->n;
    v.d_inv_n = t->d_inv_n + first;
    v.d_inv_last = t->d_inv_last + first;
    v.d_barrett = t->d_barrett + first;
    v.fp64 = t->fp64;
    if (t->d_fwd_fp) {  // FP64 tables (every modulus below 2^50)
        v.d_fwd_fp = t->d_fwd_fp + (size_t)first * t->n;
        v.d_inv_fp = t->d_inv_fp + (size_t)first * t->n;
        v.d_inv_n_fp = t->d_inv_n_fp + first;
        v.d_inv_last_fp = t->d_inv_last_fp + first;
    }
    for (int m = 0; m < 3; ++m) v.variant[m] = t->variant[m];
}

template <typename T>
cudaError_t upload(T** d, const std::vector<T>& h) {
    cudaError_t e = cudaMalloc((void**)d, std::max<size_t>(h.size(), 1) * sizeof(T));
    if (e == cudaSuccess && !h.empty()) e = cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

ulonglong2 shoup_pair(uint64_t w, uint64_t q) { return make_ulonglong2(w, h_shoup_quotient(w, q)); }

// (a, b) as the bit patterns of two doubles
ulonglong2 fp_bits(double a, double b) {
    uint64_t x, y;
    memcpy(&x, &a, 8);
    memcpy(&y, &b, 8);
    return make_ulonglong2(x, y);
}

// FP64 form of a Shoup pair (w, w') mod q: (w, w / q) as doubles
ulonglong2 fp_pair(const ulonglong2& p, uint64_t q) { return fp_bits((double)p.x, (double)p.x / (double)q); }

// product of moduli[idx] over idx in [lo, hi) except `skip`, mod r
uint64_t prod_except(const std::vector<uint64_t>& m, uint32_t lo, uint32_t hi, uint32_t skip, uint64_t r) {
    uint64_t p = 1 % r;
    for (uint32_t i = lo; i < hi; ++i)
        if (i != skip) p = h_mulmod(p, m[i] % r, r);
    return p;
}

// scratch words: ext | accQ | accP | conv | tv (the fused form's scaled masks)
struct HybridWs {
    size_t ext, accq, accp, conv, tv;
    size_t total() const { return ext + accq + accp + conv + tv; }
};

HybridWs hybrid_ws(const pg_hybrid_ks* h, uint32_t k_in, uint32_t k_out, size_t batch) {
    const size_t n = h->t->n, KO = k_out + 1;
    HybridWs w;
    w.ext = batch * k_in * h->dnum * (size_t)(h->L + h->K) * n;
    w.accq = batch * KO * h->L * n;
    w.accp = batch * KO * h->K * n;
    w.conv = batch * KO * h->L * n;
    w.tv = batch * k_in * h->L * n;
    return w;
}

// the fused transforms run the cluster kernel's default shape of each degree
constexpr uint64_t kFusedNarrowRows = 32;

template <int MODE, class IO>
int launch_fused_ntt(const NttArgs& a, uint32_t log_n, const IO& io, cudaStream_t st) {
    switch (log_n) {
        case 13: return launch_cluster<13, 12, 4, MODE, kSchedFp64, IO>(a, st, false, io);
        case 14: return launch_cluster<14, 12, 4, MODE, kSchedFp64, IO>(a, st, false, io);
        case 15:
            // a launch of a few rows (a single key switch's P rows and converted
            // rows) runs 8 elements per thread: twice the threads per row, so each
            // thread's chain of loads and butterflies is half as long, and all of
            // its clusters still fit one wave (2 CTAs of 512 threads per SM)
            if (a.rows <= kFusedNarrowRows) return launch_cluster<15, 12, 3, MODE, kSchedFp64, IO>(a, st, false, io);
            return launch_cluster<15, 12, 4, MODE, kSchedFp64, IO>(a, st, false, io);
        case 16: return launch_cluster<16, 12, 4, MODE, kSchedFp64, IO>(a, st, false, io);
    }
    return set_error(PG_ERR_UNSUPPORTED, "fused key switch: ring degree outside 2^13 .. 2^16");
}

// largest batch that runs the fused form
constexpr size_t kFusedMaxBatch = 8;

// ModUp of every mask of every ciphertext, all groups, into ext (the separate kernel)
int modup(const pg_hybrid_ks* h, uint32_t k_in, size_t batch, const uint64_t* d_in, uint64_t* ext, bool fp,
          cudaStream_t st) {
    const pg_ntt_table* t = h->t;
    ModUpArgs ma{};
    ma.in = d_in;
    ma.ext = ext;
    ma.ginv = h->d_ginv;
    ma.gmat = h->d_gmat;
    ma.gout = h->d_gout;
    ma.gmat_off = h->d_offs;
    ma.gout_off = h->d_offs + h->dnum;
    ma.moduli = t->d_moduli;
    ma.bar = t->d_barrett;
    ma.polys = batch * k_in;
    ma.N = t->n;
    ma.k_in = k_in;
    ma.L = h->L;
    ma.K = h->K;
    ma.alpha = h->alpha;
    ma.dnum = h->dnum;
    ma.log_n = t->log_n;
    ma.gmat_fp = h->d_gmat_fp;
    ma.fmod = h->d_fmod;
    const dim3 mgrid = grid2((t->n + 1) / 2, ma.polys * h->dnum);
    if (h->alpha <= 4)
        fp ? modup_kernel<4, true><<<mgrid, 256, 0, st>>>(ma) : modup_kernel<4, false><<<mgrid, 256, 0, st>>>(ma);
    else
        fp ? modup_kernel<kMaxAlpha, true><<<mgrid, 256, 0, st>>>(ma)
           : modup_kernel<kMaxAlpha, false><<<mgrid, 256, 0, st>>>(ma);
    count_launch();
    PG_LAUNCH_CHECK("modup_kernel launch");
    return PG_OK;
}

struct OwnedWs {
    void* ptr = nullptr;
    cudaStream_t st = 0;
    ~OwnedWs() {
        if (ptr) scratch_free(ptr, st);
    }
};

}  // namespace

uint32_t pg::hybrid_q_limbs(const pg_hybrid_ks* ks) { return ks->L; }
size_t pg::hybrid_n(const pg_hybrid_ks* ks) { return ks->t->n; }

extern "C" {

int pg_hybrid_ks_create(const pg_ntt_table* t, uint32_t L, uint32_t K, uint32_t alpha, pg_hybrid_ks** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (L == 0 || K == 0 || L + K != t->L) return set_error(PG_ERR_INVALID_ARGUMENT, "table must hold L + K primes");
    if (alpha == 0 || alpha > L || alpha > kMaxAlpha)
        return set_error(PG_ERR_INVALID_ARGUMENT, "alpha must be in [1, min(L, 8)]");
    if (K > kMaxK) return set_error(PG_ERR_UNSUPPORTED, "at most 8 special primes");
    const std::vector<uint64_t>& m = t->moduli;
    for (uint32_t i = 0; i < L + K; ++i)
        if (m[i] >= (1ull << 59)) return set_error(PG_ERR_UNSUPPORTED, "hybrid key switch moduli must be below 2^59");
    for (uint32_t i = 0; i < L + K; ++i)
        for (uint32_t j = i + 1; j < L + K; ++j)
            if (m[i] == m[j]) return set_error(PG_ERR_NOT_COPRIME, "moduli must be distinct primes");
    pg_hybrid_ks* h = new (std::nothrow) pg_hybrid_ks();
    if (!h) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    h->t = t;
    h->L = L;
    h->K = K;
    h->alpha = alpha;
    h->dnum = (L + alpha - 1) / alpha;
    make_view(t, 0, L, h->tq);
    make_view(t, L, K, h->tp);
    std::vector<ulonglong2> ginv(L), pinv_k(K), pinv(L);
    std::vector<ulonglong2> gmat, pmat((size_t)L * K);
    std::vector<uint32_t> gout;
    for (uint32_t g = 0; g < h->dnum; ++g) {
        const uint32_t lo = g * alpha, hi = std::min(L, lo + alpha);
        for (uint32_t i = lo; i < hi; ++i) ginv[i] = shoup_pair(h_invmod(prod_except(m, lo, hi, i, m[i]), m[i]), m[i]);
        h->gmat_off.push_back((uint32_t)gmat.size());
        h->gout_off.push_back((uint32_t)gout.size());
        for (uint32_t r = 0; r < L + K; ++r) {
            if (r >= lo && r < hi) continue;
            gout.push_back(r);
            for (uint32_t i = lo; i < hi; ++i) gmat.push_back(shoup_pair(prod_except(m, lo, hi, i, m[r]), m[r]));
        }
    }
    for (uint32_t k = 0; k < K; ++k)
        pinv_k[k] = shoup_pair(h_invmod(prod_except(m, L, L + K, L + k, m[L + k]), m[L + k]), m[L + k]);
    for (uint32_t l = 0; l < L; ++l) {
        const uint64_t pi = h_invmod(prod_except(m, L, L + K, UINT32_MAX, m[l]), m[l]);  // P^-1 mod q_l
        pinv[l] = shoup_pair(pi, m[l]);
        for (uint32_t k = 0; k < K; ++k)
            pmat[(size_t)l * K + k] = shoup_pair(h_mulmod(prod_except(m, L, L + K, L + k, m[l]), pi, m[l]), m[l]);
    }
    // FP64 copies (every modulus below 2^50): matrices as (w, w / r), moduli as (q, 1/q)
    uint64_t maxq = 0;
    for (uint64_t q : m) maxq = std::max(maxq, q);
    const bool fp = maxq < (1ull << 50);
    std::vector<ulonglong2> gmat_fp, pmat_fp, fmod;
    if (fp) {
        for (uint32_t g = 0; g < h->dnum; ++g) {
            const uint32_t lo = g * alpha, hi = std::min(L, lo + alpha), ag = hi - lo;
            size_t idx = h->gmat_off[g], j = h->gout_off[g];
            for (uint32_t r = 0; r < L + K; ++r) {
                if (r >= lo && r < hi) continue;
                for (uint32_t i = 0; i < ag; ++i, ++idx) gmat_fp.push_back(fp_pair(gmat[idx], m[gout[j]]));
                ++j;
            }
        }
        for (uint32_t l = 0; l < L; ++l)
            for (uint32_t k = 0; k < K; ++k) pmat_fp.push_back(fp_pair(pmat[(size_t)l * K + k], m[l]));
        for (uint32_t i = 0; i < L + K; ++i) fmod.push_back(fp_bits((double)m[i], 1.0 / (double)m[i]));
    }
    std::vector<uint32_t> offs(h->gmat_off);
    offs.insert(offs.end(), h->gout_off.begin(), h->gout_off.end());
    cudaError_t e = upload(&h->d_ginv, ginv);
    if (e == cudaSuccess) e = upload(&h->d_gmat, gmat);
    if (e == cudaSuccess) e = upload(&h->d_gout, gout);
    if (e == cudaSuccess) e = upload(&h->d_pinv_k, pinv_k);
    if (e == cudaSuccess) e = upload(&h->d_pmat, pmat);
    if (e == cudaSuccess) e = upload(&h->d_pinv, pinv);
    if (e == cudaSuccess) e = upload(&h->d_offs, offs);
    if (e == cudaSuccess && fp) e = upload(&h->d_gmat_fp, gmat_fp);
    if (e == cudaSuccess && fp) e = upload(&h->d_pmat_fp, pmat_fp);
    if (e == cudaSuccess && fp) e = upload(&h->d_fmod, fmod);
    if (e != cudaSuccess) {
        pg_hybrid_ks_destroy(h);
        return cuda_status(e, "pg_hybrid_ks_create: upload");
    }
    *out = h;
    return PG_OK;
}

int pg_hybrid_ks_destroy(pg_hybrid_ks* h) {
    if (!h) return PG_OK;
    cudaFree(h->d_ginv);
    cudaFree(h->d_gmat);
    cudaFree(h->d_gout);
    cudaFree(h->d_pinv_k);
    cudaFree(h->d_pmat);
    cudaFree(h->d_pinv);
    cudaFree(h->d_offs);
    cudaFree(h->d_gmat_fp);
    cudaFree(h->d_pmat_fp);
    cudaFree(h->d_fmod);
    delete h;
    return PG_OK;
}

uint32_t pg_hybrid_ks_dnum(const pg_hybrid_ks* h) { return h ? h->dnum : 0; }

size_t pg_hybrid_ks_workspace_size(const pg_hybrid_ks* h, uint32_t k_in, uint32_t k_out, size_t batch) {
    if (!h) return 0;
    return hybrid_ws(h, k_in, k_out, batch).total() * sizeof(uint64_t) + 256;
}

int pg_key_switch_hybrid(const pg_hybrid_ks* h, uint32_t k_in, uint32_t k_out, const uint64_t* d_key,
                         const uint64_t* d_in, uint64_t* d_out, size_t batch, void* d_ws, size_t ws_size,
                         void* stream) {
    if (!h) return set_error(PG_ERR_INVALID_ARGUMENT, "key switch context is NULL");
    if (batch == 0) return PG_OK;
    if (!d_key || !d_in || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (k_in == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k_in must be at least 1");
    cudaStream_t st = (cudaStream_t)stream;
    const pg_ntt_table* t = h->t;
    const size_t n = t->n, KO = k_out + 1, L = h->L, K = h->K;
    const HybridWs w = hybrid_ws(h, k_in, k_out, batch);
    const size_t need = w.total() * sizeof(uint64_t);
    OwnedWs owned;
    uint64_t* ws = (uint64_t*)d_ws;
    if (ws) {
        if (ws_size < need) return set_error(PG_ERR_INVALID_ARGUMENT, "workspace too small");
    } else {
        owned.st = st;
        cudaError_t e = scratch_alloc(&owned.ptr, need, st);
        if (e != cudaSuccess) return cuda_status(e, "key switch workspace");
        ws = (uint64_t*)owned.ptr;
    }
    uint64_t* ext = ws;
    uint64_t* accq = ext + w.ext;
    uint64_t* accp = accq + w.accq;
    uint64_t* conv = accp + w.accp;
    uint64_t* tv = conv + w.conv;
    // the FP64 dot products when the table runs the FP64 schedule (every modulus below 2^50)
    const bool fp = h->d_fmod && t->fp64;
    // the fused form's last transform reads b from the input while it stores the
    // outputs, so an output that overlaps the input takes the unfused sequence
    const size_t in_words = batch * (k_in + 1) * L * n, out_words = batch * KO * L * n;
    const bool overlap = d_in < d_out + out_words && d_out < d_in + in_words;
    // The fused form pays off while launches and the serial chain of kernels
    // dominate (N = 2^15, L = 16, K = 4: 150 -> 134 us for one key switch, 71 ->
    // 70 us each in batches of 8); on a full GPU its integer dot products compete
    // with the FP64 transforms, and the separate kernels are faster (batches of
    // 32: 62.8 us separate, 65.0 us with only the P -> Q side fused, 70.3 us fused)
    const bool fused = fp && !overlap && t->log_n >= 13 && t->log_n <= 16 && batch <= kFusedMaxBatch;
    if (fused) {
        ScaleArgs sa{};
        sa.in = d_in;
        sa.tv = tv;
        sa.ginv = h->d_ginv;
        sa.moduli = t->d_moduli;
        sa.polys = batch * k_in;
        sa.N = n;
        sa.k_in = k_in;
        sa.L = h->L;
        sa.log_n = t->log_n;
        scale_kernel<<<grid2(L * n, sa.polys), 256, 0, st>>>(sa);
        count_launch();
        PG_LAUNCH_CHECK("scale_kernel launch");
        ModUpIO mio{};
        mio.in = d_in;
        mio.tv = tv;
        mio.gmat = h->d_gmat;
        mio.k_in = k_in;
        mio.L = h->L;
        mio.K = h->K;
        mio.alpha = h->alpha;
        mio.dnum = h->dnum;
        mio.log_n = t->log_n;
        int rc = launch_fused_ntt<MODE_FWD>(make_args(t, ext, batch * k_in * h->dnum * (L + K), 0), t->log_n, mio,
                                            st);
        if (rc) return rc;
    } else {
        int rc = modup(h, k_in, batch, d_in, ext, fp, st);
        if (rc) return rc;
        rc = launch_ntt(make_args(t, ext, batch * k_in * h->dnum * (L + K), 0), t->log_n, MODE_FWD, st);
        if (rc) return rc;
    }
    // sum over masks and groups, Q limbs to accq, P limbs to accp
    int rc = launch_mac(t, h->dnum, accq, nullptr, nullptr, d_key, ext, batch, k_in, (uint32_t)KO, 0, st, accp,
                        h->L);
    if (rc) return rc;
    if (fused) {
        // ModDown with the P -> Q conversion and the final combination inside the transforms
        PScaleIO pio{};
        pio.accp = accp;
        pio.pinv_k = h->d_pinv_k;
        pio.K = h->K;
        pio.log_n = t->log_n;
        rc = launch_fused_ntt<MODE_INV>(make_args(&h->tp, accp, batch * KO * K, 0), t->log_n, pio, st);
        if (rc) return rc;
        PConvIO cio{};
        cio.tvp = accp;
        cio.pmat = h->d_pmat;
        cio.bsrc = d_in + (size_t)k_in * L * n;  // b of ciphertext j: after its k_in masks
        cio.bstride = (size_t)(k_in + 1) * L * n;
        cio.accq = accq;
        cio.pinv = h->d_pinv;
        cio.out = d_out;
        cio.K = h->K;
        cio.L = h->L;
        cio.ko = (uint32_t)KO;
        cio.log_n = t->log_n;
        // the rows' own storage is never touched: the policy loads and stores
        return launch_fused_ntt<MODE_FWD>(make_args(&h->tq, conv, batch * KO * L, 0), t->log_n, cio, st);
    }
    // ModDown: P limbs to coefficients, convert to Q, back to the NTT domain
    rc = launch_ntt(make_args(&h->tp, accp, batch * KO * K, 0), t->log_n, MODE_INV, st);
    if (rc) return rc;
    PConvArgs pa{};
    pa.accp = accp;
    pa.conv = conv;
    pa.pinv_k = h->d_pinv_k;
    pa.pmat = h->d_pmat;
    pa.moduli = t->d_moduli;
    pa.bar = t->d_barrett;
    pa.pc = batch * KO;
    pa.N = n;
    pa.L = h->L;
    pa.K = h->K;
    pa.log_n = t->log_n;
    pa.pmat_fp = h->d_pmat_fp;
    pa.fmod = h->d_fmod;
    pa.bsrc = d_in + (size_t)k_in * L * n;  // b of ciphertext j: after its k_in masks
    pa.bstride = (size_t)(k_in + 1) * L * n;
    pa.ko = (uint32_t)KO;
    const dim3 pgrid = grid2((n + 1) / 2, pa.pc);
    if (h->K <= 4)
        fp ? pconv_kernel<4, true><<<pgrid, 256, 0, st>>>(pa) : pconv_kernel<4, false><<<pgrid, 256, 0, st>>>(pa);
    else
        fp ? pconv_kernel<kMaxK, true><<<pgrid, 256, 0, st>>>(pa) : pconv_kernel<kMaxK, false><<<pgrid, 256, 0, st>>>(pa);
    count_launch();
    PG_LAUNCH_CHECK("pconv_kernel launch");
    // NTT(P^-1 conv + [last] b): b reaches the NTT domain through the same transform
    rc = launch_ntt(make_args(&h->tq, conv, batch * KO * L, 0), t->log_n, MODE_FWD, st);
    if (rc) return rc;
    FinishArgs fa{};
    fa.accq = accq;
    fa.conv = conv;
    fa.out = d_out;
    fa.pinv = h->d_pinv;
    fa.moduli = t->d_moduli;
    fa.B = batch;
    fa.N = n;
    fa.KO = (uint32_t)KO;
    fa.L = h->L;
    fa.log_n = t->log_n;
    if (L * n > 0xffffffffull) return set_error(PG_ERR_UNSUPPORTED, "poly too large");
    finish_kernel<<<grid2(L * n, batch * KO), 256, 0, st>>>(fa);
    count_launch();
    PG_LAUNCH_CHECK("finish_kernel launch");
    return PG_OK;
}

}  // extern "C"
