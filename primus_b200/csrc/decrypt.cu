// BFV-style GLWE decryption through fast base conversion, on the device:
// DcrtGlweSecretKey::decrypt_inplace (primus_fhe_core/src/secret_key/glwe.rs:782-837).
//
//   phase = b - sum_i a_i s_i                 (NTT domain, phase_inplace :713-737)
//   inverse NTT of the phase                   (canonical residues mod each q_l)
//   y_{t,gamma} = fast_convert(phase * [t gamma]_q)   (converter.rs:147-175)
//   y_{t,gamma} *= -Q^-1 mod {t, gamma}
//   m = gamma^-1 (gamma - y_gamma + y_t mod gamma) mod t
//
// Launches per batch: phase_kernel -> inverse NTT -> convert_kernel (the
// scaling, the fast conversion to {t, gamma} and the gamma correction of one
// coefficient per thread, every limb read once).
#include <algorithm>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace pg;

struct pg_bfv_decryptor {
    const pg_ntt_table* t = nullptr;
    uint64_t pt = 0, gamma = 0;
    ulonglong2* d_scale = nullptr;  // [L] Shoup pair of ([t gamma]_{q_l} * (Q/q_l)^-1) mod q_l
    uint64_t* d_hat = nullptr;      // [2][L] (Q/q_l) mod t, (Q/q_l) mod gamma
    Barrett bt{}, bg{};             // t and gamma
    uint64_t minus_inv_q_t = 0, minus_inv_q_g = 0;
    uint64_t inv_gamma_t = 0, inv_gamma_t_q = 0;
};

namespace {

struct PhaseArgs {
    const uint64_t* ct;  // [B][k+1][L][N]
    const uint64_t* sk;  // [k][L][N]
    uint64_t* ph;        // [B][L][N]
    const Barrett* bar;
    size_t B;
    uint32_t k, L, log_n;
};

// phase = b - sum_i a_i s_i (canonical); grid y = ciphertext, x over L*N
__global__ void __launch_bounds__(256) phase_kernel(PhaseArgs a) {
    const uint32_t LN = a.L << a.log_n;
    for (size_t b = blockIdx.y; b < a.B; b += gridDim.y) {
        const uint64_t* ct = a.ct + b * (a.k + 1) * (size_t)LN;
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < LN; lx += gridDim.x * blockDim.x) {
            const Barrett m = a.bar[lx >> a.log_n];
            uint64_t lo = 0, hi = 0;
            for (uint32_t i = 0; i < a.k; ++i) {
                if (i && (i & 7) == 0) {  // products < 2^124: fold before the sum can reach 2^128
                    lo = barrett_reduce_128(lo, hi, m);
                    hi = 0;
                }
                const uint64_t x = ct[(size_t)i * LN + lx], s = a.sk[(size_t)i * LN + lx];
                const uint64_t pl = x * s, phi = mulhi64(x, s);
                lo += pl;
                hi += phi + (lo < pl);
            }
            a.ph[b * LN + lx] = sub_mod(ct[(size_t)a.k * LN + lx], barrett_reduce_128(lo, hi, m), m.q);
        }
    }
}

struct ConvertArgs {
    const uint64_t* ph;  // [B][L][N] coefficient form
    uint64_t* msg;       // [B][N]
    const ulonglong2* scale;
    const uint64_t* moduli;
    const uint64_t* hat;  // [2][L]
    Barrett bt, bg;
    uint64_t minus_inv_q_t, minus_inv_q_g, inv_gamma_t, inv_gamma_t_q;
    size_t B;
    uint32_t L, log_n;
};

// one coefficient per thread; grid y = ciphertext, x over N
__global__ void __launch_bounds__(256) convert_kernel(ConvertArgs a) {
    const uint32_t N = 1u << a.log_n;
    for (size_t b = blockIdx.y; b < a.B; b += gridDim.y) {
        const uint64_t* ph = a.ph + b * (size_t)a.L * N;
        for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < N; x += gridDim.x * blockDim.x) {
            uint64_t lt = 0, ht = 0, lg = 0, hg = 0;
            for (uint32_t l = 0; l < a.L; ++l) {
                if (l && (l & 7) == 0) {  // keep the sums below 2^128
                    lt = barrett_reduce_128(lt, ht, a.bt);
                    ht = 0;
                    lg = barrett_reduce_128(lg, hg, a.bg);
                    hg = 0;
                }
                const ulonglong2 f = a.scale[l];
                const uint64_t v = shoup_mul(f.x, f.y, ph[(size_t)l * N + x], a.moduli[l]);
                const uint64_t wt = a.hat[l], wg = a.hat[a.L + l];
                uint64_t pl = v * wt, phi = mulhi64(v, wt);
                lt += pl;
                ht += phi + (lt < pl);
                pl = v * wg;
                phi = mulhi64(v, wg);
                lg += pl;
                hg += phi + (lg < pl);
            }
            const uint64_t yt = barrett_mul(barrett_reduce_128(lt, ht, a.bt), a.minus_inv_q_t, a.bt);
            const uint64_t yg = barrett_mul(barrett_reduce_128(lg, hg, a.bg), a.minus_inv_q_g, a.bg);
            uint64_t temp = a.bg.q - yg + yt;
            if (temp >= a.bg.q) temp -= a.bg.q;
            a.msg[b * N + x] = shoup_mul(a.inv_gamma_t, a.inv_gamma_t_q, temp, a.bt.q);
        }
    }
}


// product of moduli[i] for i != skip, mod r
uint64_t prod_except(const std::vector<uint64_t>& m, size_t skip, uint64_t r) {
    uint64_t p = 1 % r;
    for (size_t i = 0; i < m.size(); ++i)
        if (i != skip) p = h_mulmod(p, m[i] % r, r);
    return p;
}

}  // namespace

extern "C" {

int pg_bfv_decryptor_create(const pg_ntt_table* t, uint64_t plain_modulus, uint64_t gamma, pg_bfv_decryptor** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (plain_modulus < 2 || gamma < 2 || plain_modulus >= (1ull << 62) || gamma >= (1ull << 62))
        return set_error(PG_ERR_INVALID_ARGUMENT, "t and gamma must be in [2, 2^62)");
    if (plain_modulus >= gamma) return set_error(PG_ERR_INVALID_ARGUMENT, "t must be below gamma");
    const std::vector<uint64_t>& m = t->moduli;
    const size_t L = m.size();
    const uint64_t q_t = prod_except(m, SIZE_MAX, plain_modulus), q_g = prod_except(m, SIZE_MAX, gamma);
    const uint64_t iq_t = h_invmod(q_t, plain_modulus), iq_g = h_invmod(q_g, gamma);
    const uint64_t ig_t = h_invmod(gamma % plain_modulus, plain_modulus);
    if (iq_t == 0 || iq_g == 0 || ig_t == 0)
        return set_error(PG_ERR_NOT_COPRIME, "t, gamma and the moduli must be pairwise coprime");
    pg_bfv_decryptor* d = new (std::nothrow) pg_bfv_decryptor();
    if (!d) return set_error(PG_ERR_OUT_OF_MEMORY, "allocation failed");
    d->t = t;
    d->pt = plain_modulus;
    d->gamma = gamma;
    d->bt = h_barrett(plain_modulus);
    d->bg = h_barrett(gamma);
    d->minus_inv_q_t = plain_modulus - iq_t;
    d->minus_inv_q_g = gamma - iq_g;
    d->inv_gamma_t = ig_t;
    d->inv_gamma_t_q = h_shoup_quotient(ig_t, plain_modulus);
    std::vector<ulonglong2> scale(L);
    std::vector<uint64_t> hat(2 * L);
    const unsigned __int128 tg = (unsigned __int128)plain_modulus * gamma;
    for (size_t l = 0; l < L; ++l) {
        const uint64_t tg_l = (uint64_t)(tg % m[l]);
        const uint64_t inv_hat = h_invmod(prod_except(m, l, m[l]), m[l]);
        const uint64_t w = h_mulmod(tg_l, inv_hat, m[l]);
        scale[l] = make_ulonglong2(w, h_shoup_quotient(w, m[l]));
        hat[l] = prod_except(m, l, plain_modulus);
        hat[L + l] = prod_except(m, l, gamma);
    }
    cudaError_t e = cudaMalloc(&d->d_scale, L * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMemcpy(d->d_scale, scale.data(), L * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&d->d_hat, 2 * L * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMemcpy(d->d_hat, hat.data(), 2 * L * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        pg_bfv_decryptor_destroy(d);
        return cuda_status(e, "pg_bfv_decryptor_create");
    }
    *out = d;
    return PG_OK;
}

int pg_bfv_decryptor_destroy(pg_bfv_decryptor* d) {
    if (!d) return PG_OK;
    cudaFree(d->d_scale);
    cudaFree(d->d_hat);
    delete d;
    return PG_OK;
}

size_t pg_bfv_decrypt_workspace_size(const pg_bfv_decryptor* d, size_t batch) {
    if (!d) return 0;
    return batch * (size_t)d->t->L * d->t->n * sizeof(uint64_t) + 256;
}

int pg_bfv_decrypt(const pg_bfv_decryptor* d, uint32_t k, const uint64_t* d_sk_ntt, const uint64_t* d_ct,
                   uint64_t* d_msg, size_t batch, void* d_ws, size_t ws_size, void* stream) {
    if (!d) return set_error(PG_ERR_INVALID_ARGUMENT, "decryptor is NULL");
    if (batch == 0) return PG_OK;
    if (!d_sk_ntt || !d_ct || !d_msg) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (k == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "k must be at least 1");
    const pg_ntt_table* t = d->t;
    const size_t LN = (size_t)t->L * t->n;
    if (LN > 0xffffffffull) return set_error(PG_ERR_UNSUPPORTED, "poly too large");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t need = pg_bfv_decrypt_workspace_size(d, batch);
    void* owned = nullptr;
    uint64_t* ph = (uint64_t*)d_ws;
    if (ph) {
        if (ws_size < need) return set_error(PG_ERR_INVALID_ARGUMENT, "workspace too small");
    } else {
        PG_CUDA(scratch_alloc(&owned, need, st));
        ph = (uint64_t*)owned;
    }
    PhaseArgs pa{d_ct, d_sk_ntt, ph, t->d_barrett, batch, k, t->L, t->log_n};
    phase_kernel<<<grid2(LN, batch), 256, 0, st>>>(pa);
    count_launch();
    cudaError_t e = cudaGetLastError();
    int rc = e == cudaSuccess ? launch_ntt(make_args(t, ph, batch * t->L, 0), t->log_n, MODE_INV, st)
                              : cuda_status(e, "phase_kernel launch");
    if (rc == PG_OK) {
        ConvertArgs ca{};
        ca.ph = ph;
        ca.msg = d_msg;
        ca.scale = d->d_scale;
        ca.moduli = t->d_moduli;
        ca.hat = d->d_hat;
        ca.bt = d->bt;
        ca.bg = d->bg;
        ca.minus_inv_q_t = d->minus_inv_q_t;
        ca.minus_inv_q_g = d->minus_inv_q_g;
        ca.inv_gamma_t = d->inv_gamma_t;
        ca.inv_gamma_t_q = d->inv_gamma_t_q;
        ca.B = batch;
        ca.L = t->L;
        ca.log_n = t->log_n;
        convert_kernel<<<grid2(t->n, batch), 256, 0, st>>>(ca);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_status(e, "convert_kernel launch");
    }
    if (owned) scratch_free(owned, st);
    return rc;
}

}  // extern "C"
