// Secret-key GLWE encryption on the device with a reproducible sampler:
// DcrtGlweSecretKey::encrypt_inplace (primus_fhe_core/src/secret_key/glwe.rs:386-424)
// and, with a gadget scale in place of Delta, the GLev / key-switching-key rows
// (encrypt_crt_msg_to_dcrt_glev_inplace, :683-708).
//
// Samplers (the reference draws from an unseeded rng; here every value is a
// pure function of (seed, stream, index), identical on host and device):
//   masks  a_i limb l of ciphertext j: uniform_at(seed, stream0 + (j k + i) L + l, x, q_l)
//   noise  e of ciphertext j: discrete Gaussian over [-B, B], B = ceil(24 sigma)
//          (the reference's bound, primus_distr/src/common.rs:282), by a
//          cumulative table cdt[m] = floor(2^63 P(|e| <= m)) searched with the
//          top 63 bits of hash64(seed, stream0 + 2^32 + j, x, 0); bit 0 is the sign
//   b = NTT(e + scale_l * msg) + sum_i a_i s_i        (NTT domain)
// Launches: noise_kernel -> forward NTT -> mask_body_kernel.
//
// Public-key encryption (DcrtGlwePublicKey, primus_fhe_core/src/public_key/glwe.rs):
// the public key is a secret-key encryption of zero (pk = (a, NTT(e) + sum a_i s_i),
// DcrtGlwePublicKey::new :33-71), so pg_glwe_encrypt with no message makes one.
// Encryption of ciphertext j (:74-126), samplers as above:
//   v      ternary, two hash bits per coefficient (P(0) = 1/2, P(+-1) = 1/4):
//          bits 2(x mod 16) of hash64(seed, stream0 + 2^33 + j, x / 16, 0): 0,1 -> 0, 2 -> 1, 3 -> -1
//   e_c    discrete Gaussian as above, stream stream0 + 2^32 + j (k+1) + c
//   ct_c = NTT(e_c + message part) + NTT(v) pk_c
// The message part is scale_l * msg in the body (GLWE) or, for GGSW row
// r = i d + j of coeff * X^degree (encrypt_monomial_ggsw_inplace, :128-263),
// coeff_l * g_{j,l} at coefficient `degree` of component i.
// Launches: pk_noise_kernel -> forward NTT of the noise and of v -> pk_combine_kernel.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace pg;

struct pg_glwe_encryptor {
    const pg_ntt_table* t = nullptr;
    double sigma = 0;
    uint32_t entries = 0;
    uint64_t* d_cdt = nullptr;
};

namespace {

constexpr uint32_t kMaxCdt = 4096;

// the cumulative table (same arithmetic as the oracle's orc_cdt_table)
uint32_t cdt_table(double sigma, std::vector<uint64_t>& cdt) {
    const uint32_t B = (uint32_t)std::ceil(24.0 * sigma);
    if (B + 1 > kMaxCdt) return 0;
    cdt.assign(B + 1, 0);
    double total = 0;
    for (int64_t m = -(int64_t)B; m <= (int64_t)B; ++m) total += std::exp(-(double)(m * m) / (2.0 * sigma * sigma));
    double acc = 0;
    for (uint32_t m = 0; m <= B; ++m) {
        const double rho = std::exp(-(double)m * m / (2.0 * sigma * sigma));
        acc += (m == 0 ? rho : 2.0 * rho) / total;
        const double v = acc * 9223372036854775808.0;
        cdt[m] = v >= 9223372036854775808.0 ? (1ull << 63) : (uint64_t)v;
    }
    cdt[B] = 1ull << 63;
    return B + 1;
}

PG_DEV int64_t cdt_sample(const uint64_t* __restrict__ cdt, uint32_t entries, uint64_t seed, uint64_t stream,
                          uint64_t x) {
    const uint64_t u = hash64(seed, stream, x, 0);
    const uint64_t v = u >> 1;
    uint32_t lo = 0, hi = entries - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (v < __ldg(cdt + mid))
            hi = mid;
        else
            lo = mid + 1;
    }
    return (lo > 0 && (u & 1)) ? -(int64_t)lo : (int64_t)lo;
}

struct NoiseArgs {
    uint64_t* out;        // [B][L][N] coefficient form
    const uint64_t* msg;  // [B][L][N] or NULL
    const uint64_t* cdt;
    const uint64_t* scale;  // [L] device
    const uint64_t* moduli;
    const Barrett* bar;
    uint64_t seed, stream0;
    size_t B;
    uint32_t entries, L, log_n;
};

// e + scale_l msg, grid y = ciphertext, x over N
__global__ void __launch_bounds__(256) noise_kernel(NoiseArgs a) {
    const uint32_t N = 1u << a.log_n;
    for (size_t j = blockIdx.y; j < a.B; j += gridDim.y) {
        for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < N; x += gridDim.x * blockDim.x) {
            const int64_t e = cdt_sample(a.cdt, a.entries, a.seed, a.stream0 + (1ull << 32) + j, x);
            for (uint32_t l = 0; l < a.L; ++l) {
                const uint64_t q = a.moduli[l];
                uint64_t v = e >= 0 ? (uint64_t)e % q : q - (uint64_t)(-e) % q;
                const size_t o = (j * a.L + l) * (size_t)N + x;
                if (a.msg) v = barrett_mul_add(a.msg[o], a.scale[l], v, a.bar[l]);
                a.out[o] = v;
            }
        }
    }
}

struct BodyArgs {
    uint64_t* ct;         // [B][k+1][L][N]
    const uint64_t* eb;   // [B][L][N] NTT(e + scale msg)
    const uint64_t* sk;   // [k][L][N]
    const uint64_t* moduli;
    const Barrett* bar;
    uint64_t seed, stream0;
    size_t B;
    uint32_t k, L, log_n;
};

// masks and body, grid y = ciphertext, x over L*N
__global__ void __launch_bounds__(256) mask_body_kernel(BodyArgs a) {
    const uint32_t N = 1u << a.log_n, LN = a.L << a.log_n;
    for (size_t j = blockIdx.y; j < a.B; j += gridDim.y) {
        uint64_t* ct = a.ct + j * (a.k + 1) * (size_t)LN;
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < LN; lx += gridDim.x * blockDim.x) {
            const uint32_t l = lx >> a.log_n, x = lx & (N - 1);
            const Barrett m = a.bar[l];
            uint64_t lo = 0, hi = 0;
            for (uint32_t i = 0; i < a.k; ++i) {
                if (i && (i & 7) == 0) {  // products < 2^124: fold before the sum can reach 2^128
                    lo = barrett_reduce_128(lo, hi, m);
                    hi = 0;
                }
                const uint64_t av = uniform_at(a.seed, a.stream0 + (j * a.k + i) * a.L + l, x, m.q);
                ct[(size_t)i * LN + lx] = av;
                const uint64_t s = a.sk[(size_t)i * LN + lx];
                const uint64_t pl = av * s, ph = mulhi64(av, s);
                lo += pl;
                hi += ph + (lo < pl);
            }
            ct[(size_t)a.k * LN + lx] = add_mod(a.eb[j * LN + lx], barrett_reduce_128(lo, hi, m), m.q);
        }
    }
}


struct PkNoiseArgs {
    uint64_t* ct;            // [B][k+1][L][N]: noise plus message part, coefficient form
    uint64_t* v;             // [B][L][N] ternary
    const uint64_t* msg;     // GLWE: [B][L][N] or NULL
    const uint64_t* scale;   // GLWE: [L]
    const uint64_t* mono;    // GGSW: coefficient residues [L], or NULL
    const uint64_t* gsc;     // GGSW: gadget scalar residues [d][L]
    const uint64_t* cdt;
    const uint64_t* moduli;
    const Barrett* bar;
    uint64_t seed, stream0;
    size_t B, degree;
    uint32_t entries, L, log_n, k, d;
};

// grid y = ciphertext, x over N
__global__ void __launch_bounds__(256) pk_noise_kernel(PkNoiseArgs a) {
    const uint32_t N = 1u << a.log_n;
    for (size_t j = blockIdx.y; j < a.B; j += gridDim.y) {
        const uint32_t mc = a.mono ? (uint32_t)(j / a.d) : a.k;  // component carrying the message
        for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < N; x += gridDim.x * blockDim.x) {
            const uint32_t r = (uint32_t)(hash64(a.seed, a.stream0 + (2ull << 32) + j, x >> 4, 0) >> (2 * (x & 15))) & 3;
            for (uint32_t l = 0; l < a.L; ++l) {
                const uint64_t q = a.moduli[l];
                a.v[(j * a.L + l) * (size_t)N + x] = r <= 1 ? 0 : (r == 2 ? 1 : q - 1);
            }
            for (uint32_t c = 0; c <= a.k; ++c) {
                const int64_t e = cdt_sample(a.cdt, a.entries, a.seed, a.stream0 + (1ull << 32) + j * (a.k + 1) + c, x);
                for (uint32_t l = 0; l < a.L; ++l) {
                    const uint64_t q = a.moduli[l];
                    uint64_t val = e >= 0 ? (uint64_t)e % q : q - (uint64_t)(-e) % q;
                    if (c == mc) {
                        if (a.msg) val = barrett_mul_add(a.msg[(j * a.L + l) * (size_t)N + x], a.scale[l], val, a.bar[l]);
                        if (a.mono && x == a.degree)
                            val = barrett_mul_add(a.mono[l], a.gsc[(size_t)(j % a.d) * a.L + l], val, a.bar[l]);
                    }
                    a.ct[((j * (a.k + 1) + c) * a.L + l) * (size_t)N + x] = val;
                }
            }
        }
    }
}

// ct_c += v pk_c (all NTT domain); grid y = ciphertext component, x over L*N
__global__ void __launch_bounds__(256) pk_combine_kernel(uint64_t* __restrict__ ct, const uint64_t* __restrict__ v,
                                                         const uint64_t* __restrict__ pk, const Barrett* __restrict__ bar,
                                                         size_t comps, uint32_t k, uint32_t L, uint32_t log_n) {
    const uint32_t LN = L << log_n;
    for (size_t rc = blockIdx.y; rc < comps; rc += gridDim.y) {
        const size_t j = rc / (k + 1), c = rc % (k + 1);
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < LN; lx += gridDim.x * blockDim.x) {
            const size_t o = rc * LN + lx;
            ct[o] = barrett_mul_add(v[j * LN + lx], pk[c * LN + lx], ct[o], bar[lx >> log_n]);
        }
    }
}

}  // namespace

namespace pg {
uint32_t rns_L(const pg_rns_base* b);
const uint64_t* rns_moduli(const pg_rns_base* b);
const pg_rns_base* gadget_base(const pg_gadget_basis* g);
}  // namespace pg

namespace {

// noise + v -> forward NTTs -> ct_c += v pk_c, for B ciphertexts
int pk_encrypt_launch(const pg_glwe_encryptor* h, PkNoiseArgs na, const uint64_t* d_pk, cudaStream_t st) {
    const pg_ntt_table* t = h->t;
    const size_t LN = (size_t)t->L * t->n;
    pk_noise_kernel<<<grid2(t->n, na.B), 256, 0, st>>>(na);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "pk_noise_kernel launch");
    int rc = launch_ntt(make_args(t, na.ct, na.B * (na.k + 1) * t->L, 0), t->log_n, MODE_FWD, st);
    if (rc == PG_OK) rc = launch_ntt(make_args(t, na.v, na.B * t->L, 0), t->log_n, MODE_FWD, st);
    if (rc) return rc;
    pk_combine_kernel<<<grid2(LN, na.B * (na.k + 1)), 256, 0, st>>>(na.ct, na.v, d_pk, t->d_barrett,
                                                                     na.B * (na.k + 1), na.k, t->L, t->log_n);
    count_launch();
    e = cudaGetLastError();
    return e == cudaSuccess ? PG_OK : cuda_status(e, "pk_combine_kernel launch");
}

}  // namespace

extern "C" {

int pg_glwe_pk_encrypt(const pg_glwe_encryptor* h, uint32_t k, const uint64_t* d_pk, const uint64_t* d_msg,
                       const uint64_t* h_scale, uint64_t seed, uint64_t stream0, uint64_t* d_ct, size_t batch,
                       void* stream) {
    if (!h) return set_error(PG_ERR_INVALID_ARGUMENT, "encryptor is NULL");
    if (batch == 0) return PG_OK;
    if (!d_pk || !d_ct || (d_msg && !h_scale)) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (k == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k must be at least 1");
    const pg_ntt_table* t = h->t;
    const size_t LN = (size_t)t->L * t->n;
    if (LN > 0xffffffffull) return set_error(PG_ERR_UNSUPPORTED, "poly too large");
    if (d_msg)
        for (uint32_t l = 0; l < t->L; ++l)
            if (h_scale[l] >= t->moduli[l]) return set_error(PG_ERR_INVALID_ARGUMENT, "scale not below its modulus");
    cudaStream_t st = (cudaStream_t)stream;
    void* ws = nullptr;
    PG_CUDA(scratch_alloc(&ws, (batch * LN + t->L) * sizeof(uint64_t) + 256, st));
    uint64_t* v = (uint64_t*)ws;
    uint64_t* d_scale = v + batch * LN;
    int rc = PG_OK;
    if (d_msg) {
        cudaError_t e = cudaMemcpyAsync(d_scale, h_scale, t->L * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) rc = cuda_status(e, "pg_glwe_pk_encrypt: scale copy");
    }
    if (rc == PG_OK) {
        PkNoiseArgs na{d_ct, v, d_msg, d_msg ? d_scale : nullptr, nullptr, nullptr, h->d_cdt, t->d_moduli,
                       t->d_barrett, seed, stream0, batch, 0, h->entries, t->L, t->log_n, k, 1};
        rc = pk_encrypt_launch(h, na, d_pk, st);
    }
    scratch_free(ws, st);
    return rc;
}

int pg_ggsw_pk_encrypt_monomial(const pg_glwe_encryptor* h, const pg_gadget_basis* g, uint32_t k,
                                const uint64_t* d_pk, const uint64_t* h_coeff_residues, size_t degree, uint64_t seed,
                                uint64_t stream0, uint64_t* d_ggsw, void* stream) {
    if (!h || !g) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL encryptor or basis");
    if (!d_pk || !d_ggsw || !h_coeff_residues) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (k == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k must be at least 1");
    const pg_ntt_table* t = h->t;
    if (degree >= t->n) return set_error(PG_ERR_INVALID_ARGUMENT, "degree must be below N");  // public_key/glwe.rs:250
    const pg_rns_base* base = gadget_base(g);
    if (rns_L(base) != t->L) return set_error(PG_ERR_INVALID_ARGUMENT, "table and basis have different moduli counts");
    for (uint32_t l = 0; l < t->L; ++l) {
        if (rns_moduli(base)[l] != t->moduli[l]) return set_error(PG_ERR_INVALID_ARGUMENT, "table and basis moduli differ");
        if (h_coeff_residues[l] >= t->moduli[l])
            return set_error(PG_ERR_INVALID_ARGUMENT, "coefficient residue not below its modulus");
    }
    uint32_t d = 0, drop = 0;
    int rc = pg_gadget_basis_info(g, &d, &drop, nullptr);
    if (rc) return rc;
    std::vector<uint64_t> host((size_t)d * t->L + t->L);
    rc = pg_gadget_basis_info(g, &d, &drop, host.data());
    if (rc) return rc;
    std::copy(h_coeff_residues, h_coeff_residues + t->L, host.begin() + (size_t)d * t->L);
    const size_t LN = (size_t)t->L * t->n, rows = (size_t)(k + 1) * d;
    cudaStream_t st = (cudaStream_t)stream;
    void* ws = nullptr;
    PG_CUDA(scratch_alloc(&ws, (rows * LN + host.size()) * sizeof(uint64_t) + 256, st));
    uint64_t* v = (uint64_t*)ws;
    uint64_t* d_host = v + rows * LN;
    cudaError_t e = cudaMemcpyAsync(d_host, host.data(), host.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
    rc = e == cudaSuccess ? PG_OK : cuda_status(e, "pg_ggsw_pk_encrypt_monomial: constants copy");
    if (rc == PG_OK) {
        PkNoiseArgs na{d_ggsw, v, nullptr, nullptr, d_host + (size_t)d * t->L, d_host, h->d_cdt, t->d_moduli,
                       t->d_barrett, seed, stream0, rows, degree, h->entries, t->L, t->log_n, k, d};
        rc = pk_encrypt_launch(h, na, d_pk, st);
    }
    scratch_free(ws, st);
    return rc;
}

int pg_glwe_encryptor_create(const pg_ntt_table* t, double sigma, pg_glwe_encryptor** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (!(sigma > 0) || sigma > 100) return set_error(PG_ERR_INVALID_ARGUMENT, "sigma must be in (0, 100]");
    std::vector<uint64_t> cdt;
    const uint32_t entries = cdt_table(sigma, cdt);
    if (!entries) return set_error(PG_ERR_UNSUPPORTED, "noise table too large");
    pg_glwe_encryptor* h = new (std::nothrow) pg_glwe_encryptor();
    if (!h) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    h->t = t;
    h->sigma = sigma;
    h->entries = entries;
    cudaError_t e = cudaMalloc(&h->d_cdt, entries * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMemcpy(h->d_cdt, cdt.data(), entries * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        pg_glwe_encryptor_destroy(h);
        return cuda_status(e, "pg_glwe_encryptor_create");
    }
    *out = h;
    return PG_OK;
}

int pg_glwe_encryptor_destroy(pg_glwe_encryptor* h) {
    if (!h) return PG_OK;
    cudaFree(h->d_cdt);
    delete h;
    return PG_OK;
}

int pg_glwe_encrypt(const pg_glwe_encryptor* h, uint32_t k, const uint64_t* d_sk_ntt, const uint64_t* d_msg,
                    const uint64_t* h_scale, uint64_t seed, uint64_t stream0, uint64_t* d_ct, size_t batch,
                    void* stream) {
    if (!h) return set_error(PG_ERR_INVALID_ARGUMENT, "encryptor is NULL");
    if (batch == 0) return PG_OK;
    if (!d_sk_ntt || !d_ct || (d_msg && !h_scale)) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL argument");
    const pg_ntt_table* t = h->t;
    const size_t LN = (size_t)t->L * t->n;
    if (LN > 0xffffffffull) return set_error(PG_ERR_UNSUPPORTED, "poly too large");
    if (d_msg)
        for (uint32_t l = 0; l < t->L; ++l)
            if (h_scale[l] >= t->moduli[l]) return set_error(PG_ERR_INVALID_ARGUMENT, "scale not below its modulus");
    cudaStream_t st = (cudaStream_t)stream;
    void* ws = nullptr;
    const size_t scale_words = d_msg ? t->L : 0;
    PG_CUDA(scratch_alloc(&ws, (batch * LN + scale_words) * sizeof(uint64_t) + 256, st));
    uint64_t* eb = (uint64_t*)ws;
    uint64_t* d_scale = eb + batch * LN;
    cudaError_t e = cudaSuccess;
    if (d_msg) e = cudaMemcpyAsync(d_scale, h_scale, t->L * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
    int rc = e == cudaSuccess ? PG_OK : cuda_status(e, "pg_glwe_encrypt: scale copy");
    if (rc == PG_OK) {
        NoiseArgs na{eb, d_msg, h->d_cdt, d_scale, t->d_moduli, t->d_barrett, seed, stream0, batch, h->entries, t->L,
                     t->log_n};
        noise_kernel<<<grid2(t->n, batch), 256, 0, st>>>(na);
        count_launch();
        e = cudaGetLastError();
        rc = e == cudaSuccess ? launch_ntt(make_args(t, eb, batch * t->L, 0), t->log_n, MODE_FWD, st)
                              : cuda_status(e, "noise_kernel launch");
    }
    if (rc == PG_OK) {
        BodyArgs ba{d_ct, eb, d_sk_ntt, t->d_moduli, t->d_barrett, seed, stream0, batch, k, t->L, t->log_n};
        mask_body_kernel<<<grid2(LN, batch), 256, 0, st>>>(ba);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_status(e, "mask_body_kernel launch");
    }
    scratch_free(ws, st);
    return rc;
}

}  // extern "C"
