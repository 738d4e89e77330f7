// Element-wise DCRT polynomial operations (primus_poly/src/dcrt, primus_poly/src/array).
//
// Every op reads and writes canonical residues, so the outputs are unique and
// equal the reference's for any exact reduction; products use Barrett with
// ratio floor(2^128/q) (BarrettModulus) or the Shoup path when the right-hand
// side carries precomputed quotients.  The kernels are HBM-bound streams:
// 16-byte vector accesses, grid sized to a multiple of the SM count.
#include <algorithm>
#include <vector>

#include "internal.hpp"

namespace pg {

enum PwOp {
    PW_MUL = 0,
    PW_ADD_MUL,
    PW_ADD,
    PW_SUB,
    PW_NEG,
    PW_MUL_SCALAR,
    PW_ADD_MUL_SCALAR,
    PW_MUL_PREPARED,
    PW_SHOUP_PREPARE
};

struct PwArgs {
    uint64_t* x;         // in/out
    const uint64_t* y;   // rhs
    const uint64_t* z;   // second rhs / quotients
    const Barrett* bar;  // [L]
    const uint64_t* scalars;  // [2L] (device copy): scalars, then their Shoup quotients
    uint64_t pairs;      // element pairs in x
    uint64_t rhs_pairs;  // element pairs in one rhs period (L*N/2 when broadcast)
    uint32_t log_n, L;
};

// floor(w * 2^64 / q) for w < q: Barrett estimate, then at most two corrections
PG_DEV uint64_t shoup_quotient(uint64_t w, const Barrett& m) {
    // est = floor(w * ratio / 2^64) with ratio = r1*2^64 + r0
    uint64_t est = w * m.r1 + mulhi64(w, m.r0);
    // rem = w*2^64 - est*q  (128-bit, non-negative)
    uint64_t lo = est * m.q, hi = mulhi64(est, m.q);
    uint64_t rlo = 0 - lo;
    uint64_t rhi = w - hi - (lo != 0 ? 1 : 0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (rhi != 0 || rlo >= m.q) {
            ++est;
            uint64_t nlo = rlo - m.q;
            rhi -= (rlo < m.q);
            rlo = nlo;
        }
    }
    return est;
}

template <int OP>
PG_DEV void pw_elem(uint64_t& x, uint64_t y, uint64_t z, const Barrett& m, uint64_t sc, uint64_t scq) {
    const uint64_t q = m.q;
    if constexpr (OP == PW_MUL) x = barrett_mul(x, y, m);
    if constexpr (OP == PW_ADD_MUL) x = barrett_mul_add(y, z, x, m);
    if constexpr (OP == PW_ADD) x = add_mod(x, y, q);
    if constexpr (OP == PW_SUB) x = sub_mod(x, y, q);
    if constexpr (OP == PW_NEG) x = neg_mod(x, q);
    if constexpr (OP == PW_MUL_SCALAR) x = shoup_mul(sc, scq, x, q);
    if constexpr (OP == PW_ADD_MUL_SCALAR) x = add_mod(x, shoup_mul(sc, scq, y, q), q);
    if constexpr (OP == PW_MUL_PREPARED) x = shoup_mul(y, z, x, q);
    if constexpr (OP == PW_SHOUP_PREPARE) x = shoup_quotient(y, m);
}

// pairs per thread: the multiplying ops hold more registers (fewer resident
// threads), so each thread issues the loads of two pairs before computing to
// keep as many bytes in flight per SM as the light ops do
template <int OP>
__host__ __device__ constexpr int pw_per_thread() {
    return (OP == PW_MUL || OP == PW_ADD_MUL || OP == PW_MUL_PREPARED || OP == PW_SHOUP_PREPARE) ? 2 : 1;
}

// grid: y over polys, x over the L*N/2 element pairs of one poly (32-bit
// index); CTA b covers pairs [b*256*PER, (b+1)*256*PER), thread t of it the
// pairs t, t+256, ... (coalesced)
template <int OP>
__global__ void __launch_bounds__(256) pw_kernel(PwArgs a) {
    constexpr int PER = pw_per_thread<OP>();
    constexpr bool SC = OP == PW_MUL_SCALAR || OP == PW_ADD_MUL_SCALAR;
    const uint32_t pp = (uint32_t)((a.L << a.log_n) >> 1);  // pairs per poly
    const uint64_t polys = a.pairs / pp;
    for (uint64_t p = blockIdx.y; p < polys; p += gridDim.y) {
        ulonglong2* xp = reinterpret_cast<ulonglong2*>(a.x) + p * pp;
        const uint64_t roff = a.rhs_pairs ? 0 : p * pp;
        for (uint32_t i0 = blockIdx.x * (256 * PER) + threadIdx.x; i0 < pp; i0 += gridDim.x * (256 * PER)) {
            ulonglong2 x[PER], y[PER], z[PER];
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const uint32_t ix = i0 + 256 * k;
                x[k] = y[k] = z[k] = make_ulonglong2(0, 0);
                if (ix < pp) {
                    x[k] = xp[ix];
                    if constexpr (OP != PW_NEG && OP != PW_MUL_SCALAR)
                        y[k] = __ldg(reinterpret_cast<const ulonglong2*>(a.y) + roff + ix);
                    if constexpr (OP == PW_ADD_MUL || OP == PW_MUL_PREPARED)
                        z[k] = __ldg(reinterpret_cast<const ulonglong2*>(a.z) + roff + ix);
                }
            }
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const uint32_t ix = i0 + 256 * k;
                if (ix >= pp) break;
                const uint32_t limb = (2 * ix) >> a.log_n;
                const Barrett m = a.bar[limb];
                const uint64_t sc = SC ? a.scalars[limb] : 0, scq = SC ? a.scalars[a.L + limb] : 0;
                uint64_t x0 = x[k].x, x1 = x[k].y;
                pw_elem<OP>(x0, y[k].x, z[k].x, m, sc, scq);
                pw_elem<OP>(x1, y[k].y, z[k].y, m, sc, scq);
                xp[ix] = make_ulonglong2(x0, x1);
            }
        }
    }
}

// butterfly_mul_factor_inplace (primus_poly/src/dcrt/mul.rs:119-155):
// a' = a + s, b = (a - s) * w with w Shoup-prepared (values w, quotients wq);
// grid: y over polys, x over the L*N elements of one poly
__global__ void __launch_bounds__(256) butterfly_kernel(uint64_t* __restrict__ a, const uint64_t* __restrict__ s,
                                                        const uint64_t* __restrict__ w, const uint64_t* __restrict__ wq,
                                                        uint64_t* __restrict__ b, const uint64_t* __restrict__ moduli,
                                                        uint64_t polys, uint32_t log_n, uint32_t L) {
    const uint32_t ln = L << log_n;
    for (uint64_t p = blockIdx.y; p < polys; p += gridDim.y) {
        const uint64_t off = p * ln;
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < ln; lx += gridDim.x * blockDim.x) {
            const uint64_t q = moduli[lx >> log_n];
            const uint64_t av = a[off + lx], sv = s[off + lx];
            a[off + lx] = add_mod(av, sv, q);
            b[off + lx] = shoup_mul(__ldg(w + lx), __ldg(wq + lx), sub_mod(av, sv, q), q);
        }
    }
}

// seeded uniform fill: row r (= poly*L + limb) uses stream stream0 + r
__global__ void __launch_bounds__(256) fill_uniform_kernel(uint64_t* out, const uint64_t* __restrict__ moduli,
                                                           uint64_t polys, uint32_t log_n, uint32_t L, uint64_t seed,
                                                           uint64_t stream0) {
    const uint32_t ln = L << log_n;
    const uint32_t mask = (1u << log_n) - 1;
    for (uint64_t p = blockIdx.y; p < polys; p += gridDim.y) {
        for (uint32_t lx = blockIdx.x * blockDim.x + threadIdx.x; lx < ln; lx += gridDim.x * blockDim.x) {
            const uint32_t limb = lx >> log_n;
            out[p * ln + lx] = uniform_at(seed, stream0 + p * L + limb, lx & mask, moduli[limb]);
        }
    }
}



template <int OP>
static int launch_pw(const pg_ntt_table* t, uint64_t* x, const uint64_t* y, const uint64_t* z,
                     const uint64_t* h_scalars, size_t polys, size_t rhs_polys, cudaStream_t st) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (polys == 0) return PG_OK;
    if (!x) return set_error(PG_ERR_INVALID_ARGUMENT, "x is NULL");
    const bool needs_y = !(OP == PW_NEG || OP == PW_MUL_SCALAR);
    if (needs_y && !y) return set_error(PG_ERR_INVALID_ARGUMENT, "rhs is NULL");
    if ((OP == PW_ADD_MUL || OP == PW_MUL_PREPARED) && !z) return set_error(PG_ERR_INVALID_ARGUMENT, "rhs is NULL");
    if (needs_y && rhs_polys != 1 && rhs_polys != polys)
        return set_error(PG_ERR_INVALID_ARGUMENT, "rhs_polys must be 1 or polys");
    PwArgs a{};
    a.x = x;
    a.y = y;
    a.z = z;
    a.bar = t->d_barrett;
    a.log_n = t->log_n;
    a.L = t->L;
    a.pairs = (uint64_t)polys * t->L * t->n / 2;
    a.rhs_pairs = (needs_y && rhs_polys == 1 && polys > 1) ? (uint64_t)t->L * t->n / 2 : 0;
    uint64_t* d_sc = nullptr;
    if (OP == PW_MUL_SCALAR || OP == PW_ADD_MUL_SCALAR) {
        if (!h_scalars) return set_error(PG_ERR_INVALID_ARGUMENT, "scalars is NULL");
        // pageable source: the copy below completes before the call returns
        std::vector<uint64_t> sq(2 * (size_t)t->L);
        for (uint32_t l = 0; l < t->L; ++l) {
            if (h_scalars[l] >= t->moduli[l]) return set_error(PG_ERR_INVALID_ARGUMENT, "scalar not below its modulus");
            sq[l] = h_scalars[l];
            sq[t->L + l] = h_shoup_quotient(h_scalars[l], t->moduli[l]);
        }
        PG_CUDA(scratch_alloc((void**)&d_sc, sq.size() * sizeof(uint64_t), st));
        PG_CUDA(cudaMemcpyAsync(d_sc, sq.data(), sq.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        a.scalars = d_sc;
    }
    pw_kernel<OP><<<grid2((uint64_t)t->L * t->n / 2 / pw_per_thread<OP>(), polys), 256, 0, st>>>(a);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (d_sc) scratch_free(d_sc, st);
    if (e != cudaSuccess) return cuda_status(e, "pointwise kernel launch");
    return PG_OK;
}

}  // namespace pg

using namespace pg;

extern "C" {

int pg_dcrt_mul(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* d_y, size_t polys, size_t rhs_polys,
                void* stream) {
    return launch_pw<PW_MUL>(t, d_x, d_y, nullptr, nullptr, polys, rhs_polys, (cudaStream_t)stream);
}

int pg_dcrt_add_mul(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* d_y, const uint64_t* d_z, size_t polys,
                    size_t rhs_polys, void* stream) {
    return launch_pw<PW_ADD_MUL>(t, d_x, d_y, d_z, nullptr, polys, rhs_polys, (cudaStream_t)stream);
}

int pg_dcrt_add(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* d_y, size_t polys, size_t rhs_polys,
                void* stream) {
    return launch_pw<PW_ADD>(t, d_x, d_y, nullptr, nullptr, polys, rhs_polys, (cudaStream_t)stream);
}

int pg_dcrt_sub(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* d_y, size_t polys, size_t rhs_polys,
                void* stream) {
    return launch_pw<PW_SUB>(t, d_x, d_y, nullptr, nullptr, polys, rhs_polys, (cudaStream_t)stream);
}

int pg_dcrt_neg(const pg_ntt_table* t, uint64_t* d_x, size_t polys, void* stream) {
    return launch_pw<PW_NEG>(t, d_x, nullptr, nullptr, nullptr, polys, polys, (cudaStream_t)stream);
}

int pg_dcrt_mul_scalar(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* h_scalars, size_t polys,
                       void* stream) {
    return launch_pw<PW_MUL_SCALAR>(t, d_x, nullptr, nullptr, h_scalars, polys, polys, (cudaStream_t)stream);
}

int pg_dcrt_add_mul_scalar(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* d_y, const uint64_t* h_scalars,
                           size_t polys, void* stream) {
    return launch_pw<PW_ADD_MUL_SCALAR>(t, d_x, d_y, nullptr, h_scalars, polys, polys, (cudaStream_t)stream);
}

int pg_dcrt_mul_prepared(const pg_ntt_table* t, uint64_t* d_x, const uint64_t* d_w, const uint64_t* d_wq,
                         size_t polys, size_t rhs_polys, void* stream) {
    return launch_pw<PW_MUL_PREPARED>(t, d_x, d_w, d_wq, nullptr, polys, rhs_polys, (cudaStream_t)stream);
}

int pg_dcrt_shoup_prepare(const pg_ntt_table* t, const uint64_t* d_values, uint64_t* d_quotients, size_t polys,
                          void* stream) {
    // x = quotient(y): the output buffer doubles as x
    return launch_pw<PW_SHOUP_PREPARE>(t, d_quotients, d_values, nullptr, nullptr, polys, polys,
                                       (cudaStream_t)stream);
}

int pg_dcrt_butterfly_mul_factor(const pg_ntt_table* t, uint64_t* d_a, const uint64_t* d_s, const uint64_t* d_w,
                                 const uint64_t* d_wq, uint64_t* d_b, size_t polys, void* stream) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (polys == 0) return PG_OK;
    if (!d_a || !d_s || !d_w || !d_wq || !d_b) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL operand");
    const uint64_t total = (uint64_t)polys * t->L * t->n;
    (void)total;
    butterfly_kernel<<<grid2((uint64_t)t->L * t->n, polys), 256, 0, (cudaStream_t)stream>>>(
        d_a, d_s, d_w, d_wq, d_b, t->d_moduli, polys, t->log_n, t->L);
    count_launch();
    PG_LAUNCH_CHECK("butterfly_kernel launch");
    return PG_OK;
}

int pg_fill_uniform(const pg_ntt_table* t, uint64_t* d_out, size_t polys, uint64_t seed, uint64_t stream0,
                    void* stream) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (polys == 0) return PG_OK;
    if (!d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "output is NULL");
    const uint64_t total = (uint64_t)polys * t->L * t->n;
    (void)total;
    fill_uniform_kernel<<<grid2((uint64_t)t->L * t->n, polys), 256, 0, (cudaStream_t)stream>>>(
        d_out, t->d_moduli, polys, t->log_n, t->L, seed, stream0);
    count_launch();
    PG_LAUNCH_CHECK("fill_uniform_kernel launch");
    return PG_OK;
}

}  // extern "C"
