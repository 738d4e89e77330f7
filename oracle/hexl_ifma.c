/* CPU baseline, not the parity oracle: the reference's fastest CPU transform
 * path restated, i.e. the HEXL-style NTT with AVX-512 IFMA52 Harvey butterflies
 * that primus_ntt dispatches to when q < 2^50 and the host has avx512ifma
 * (primus_ntt/src/ntt/hexl/mod.rs:473-540; butterflies hexl/fwd.rs,
 * hexl/inv.rs).  Algorithm: Harvey's lazy butterflies (arXiv 1205.2926,
 * Algorithm 4) on eight 64-bit lanes, with the Shoup quotient of each twiddle
 * taken at 2^52 so that vpmadd52huq / vpmadd52luq form W*Y - Q*q exactly; the
 * three stages whose butterfly gap is below 8 pair lanes through two-vector
 * permutes.  Roots and their order are those of the scalar restatement
 * (UintNttTable), so the canonical outputs are the same values; the test suite
 * checks that.  Only bench.py's CPU-baseline leg times it.
 *
 * Test infrastructure: used only by tests/ and bench.py's cpu_baseline /
 * reference arm. */
#include <immintrin.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "primus_oracle.h"

#define HX_TARGET __attribute__((target("avx512f,avx512dq,avx512vl,avx512ifma")))

struct orc_hexl_table {
    const orc_ntt_table *t;
    size_t n;
    uint64_t q;
    uint64_t *wp;  /* [n] 52-bit Shoup quotients of the forward roots */
    uint64_t *iwp; /* [n] 52-bit Shoup quotients of the inverse roots */
    uint64_t inv_n, inv_n_p, last, last_p; /* N^-1 and w_last * N^-1 with quotients */
};

static uint64_t precon52(uint64_t w, uint64_t q) { return (uint64_t)(((unsigned __int128)w << 52) / q); }

int orc_hexl_available(void) {
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx512ifma") && __builtin_cpu_supports("avx512dq") &&
           __builtin_cpu_supports("avx512vl");
}

orc_hexl_table *orc_hexl_table_new(const orc_ntt_table *t) {
    if (!t || t->q >= (1ull << 50) || t->n < 16) return NULL;
    orc_hexl_table *h = calloc(1, sizeof *h);
    h->t = t;
    h->n = t->n;
    h->q = t->q;
    h->wp = malloc(t->n * 8);
    h->iwp = malloc(t->n * 8);
    for (size_t i = 0; i < t->n; ++i) {
        h->wp[i] = precon52(t->root_powers[i], t->q);
        h->iwp[i] = precon52(t->inv_root_powers[i], t->q);
    }
    h->inv_n = t->inv_n;
    h->inv_n_p = precon52(t->inv_n, t->q);
    h->last = orc_mulmod(t->inv_root_powers[t->n - 1], t->inv_n, t->q);
    h->last_p = precon52(h->last, t->q);
    return h;
}

void orc_hexl_table_delete(orc_hexl_table *h) {
    if (!h) return;
    free(h->wp);
    free(h->iwp);
    free(h);
}

/* W*Y mod q in [0, 2q) for Y < 2^52: Q = hi52(Wp*Y), T = (W*Y - Q*q) mod 2^52 */
HX_TARGET static inline __m512i mul_lazy52(__m512i y, __m512i w, __m512i wp, __m512i negq, __m512i mask) {
    const __m512i zero = _mm512_setzero_si512();
    __m512i qq = _mm512_madd52hi_epu64(zero, wp, y);
    __m512i t = _mm512_madd52lo_epu64(zero, w, y);
    t = _mm512_madd52lo_epu64(t, qq, negq);
    return _mm512_and_si512(t, mask);
}

/* x mod m for x < 2m: min(x, x - m) with unsigned wrap */
HX_TARGET static inline __m512i small_mod(__m512i x, __m512i m) { return _mm512_min_epu64(x, _mm512_sub_epi64(x, m)); }

/* forward Harvey butterfly, x, y in [0, 4q) -> [0, 4q) */
HX_TARGET static inline void fwd_bf(__m512i *x, __m512i *y, __m512i w, __m512i wp, __m512i negq, __m512i q2,
                                    __m512i mask) {
    __m512i u = small_mod(*x, q2);
    __m512i t = mul_lazy52(*y, w, wp, negq, mask);
    *y = _mm512_add_epi64(u, _mm512_sub_epi64(q2, t));
    *x = _mm512_add_epi64(u, t);
}

/* inverse Gentleman-Sande butterfly, x, y in [0, 2q) -> [0, 2q) */
HX_TARGET static inline void inv_bf(__m512i *x, __m512i *y, __m512i w, __m512i wp, __m512i negq, __m512i q2,
                                    __m512i mask) {
    __m512i u = *x, v = *y;
    *x = small_mod(_mm512_add_epi64(u, v), q2);
    *y = mul_lazy52(_mm512_add_epi64(u, _mm512_sub_epi64(q2, v)), w, wp, negq, mask);
}

/* lane patterns for gaps 4, 2, 1 over two consecutive vectors a = v0 | v1 */
#define IDX(a, b, c, d, e, f, g, h) _mm512_set_epi64(h, g, f, e, d, c, b, a)

HX_TARGET static void fwd_impl(const orc_hexl_table *h, uint64_t *a) {
    const size_t n = h->n;
    const uint64_t *w = h->t->root_powers, *wp = h->wp;
    const __m512i q1 = _mm512_set1_epi64((long long)h->q), q2 = _mm512_set1_epi64((long long)(2 * h->q));
    const __m512i negq = _mm512_set1_epi64((long long)((1ull << 52) - h->q));
    const __m512i mask = _mm512_set1_epi64((long long)((1ull << 52) - 1));
    /* stages with gap >= 8: one twiddle per group, broadcast */
    for (size_t gap = n >> 1, m = 1; gap >= 8; gap >>= 1, m <<= 1) {
        for (size_t k = 0; k < m; ++k) {
            const __m512i vw = _mm512_set1_epi64((long long)w[m + k]), vwp = _mm512_set1_epi64((long long)wp[m + k]);
            uint64_t *x = a + 2 * k * gap, *y = x + gap;
            for (size_t j = 0; j < gap; j += 8) {
                __m512i vx = _mm512_loadu_si512(x + j), vy = _mm512_loadu_si512(y + j);
                fwd_bf(&vx, &vy, vw, vwp, negq, q2, mask);
                _mm512_storeu_si512(x + j, vx);
                _mm512_storeu_si512(y + j, vy);
            }
        }
    }
    /* gaps 4, 2, 1: 16 elements at a time */
    const size_t m4 = n / 8, m2 = n / 4, m1 = n / 2;
    const __m512i i4x = IDX(0, 1, 2, 3, 8, 9, 10, 11), i4y = IDX(4, 5, 6, 7, 12, 13, 14, 15);
    const __m512i i2x = IDX(0, 1, 4, 5, 8, 9, 12, 13), i2y = IDX(2, 3, 6, 7, 10, 11, 14, 15);
    const __m512i i2b0 = IDX(0, 1, 8, 9, 2, 3, 10, 11), i2b1 = IDX(4, 5, 12, 13, 6, 7, 14, 15);
    const __m512i i1x = IDX(0, 2, 4, 6, 8, 10, 12, 14), i1y = IDX(1, 3, 5, 7, 9, 11, 13, 15);
    const __m512i i1b0 = IDX(0, 8, 1, 9, 2, 10, 3, 11), i1b1 = IDX(4, 12, 5, 13, 6, 14, 7, 15);
    for (size_t o = 0; o < n; o += 16) {
        __m512i v0 = _mm512_loadu_si512(a + o), v1 = _mm512_loadu_si512(a + o + 8);
        /* gap 4: groups o/8, o/8 + 1 */
        {
            const size_t k = o / 8;
            __m512i vw = IDX(w[m4 + k], w[m4 + k], w[m4 + k], w[m4 + k], w[m4 + k + 1], w[m4 + k + 1],
                             w[m4 + k + 1], w[m4 + k + 1]);
            __m512i vwp = IDX(wp[m4 + k], wp[m4 + k], wp[m4 + k], wp[m4 + k], wp[m4 + k + 1], wp[m4 + k + 1],
                              wp[m4 + k + 1], wp[m4 + k + 1]);
            __m512i x = _mm512_permutex2var_epi64(v0, i4x, v1), y = _mm512_permutex2var_epi64(v0, i4y, v1);
            fwd_bf(&x, &y, vw, vwp, negq, q2, mask);
            v0 = _mm512_permutex2var_epi64(x, i4x, y);
            v1 = _mm512_permutex2var_epi64(x, i4y, y);
        }
        /* gap 2: groups o/4 .. o/4 + 3 */
        {
            const size_t k = o / 4;
            __m512i vw = IDX(w[m2 + k], w[m2 + k], w[m2 + k + 1], w[m2 + k + 1], w[m2 + k + 2], w[m2 + k + 2],
                             w[m2 + k + 3], w[m2 + k + 3]);
            __m512i vwp = IDX(wp[m2 + k], wp[m2 + k], wp[m2 + k + 1], wp[m2 + k + 1], wp[m2 + k + 2],
                              wp[m2 + k + 2], wp[m2 + k + 3], wp[m2 + k + 3]);
            __m512i x = _mm512_permutex2var_epi64(v0, i2x, v1), y = _mm512_permutex2var_epi64(v0, i2y, v1);
            fwd_bf(&x, &y, vw, vwp, negq, q2, mask);
            v0 = _mm512_permutex2var_epi64(x, i2b0, y);
            v1 = _mm512_permutex2var_epi64(x, i2b1, y);
        }
        /* gap 1: groups o/2 .. o/2 + 7, twiddles contiguous */
        {
            const size_t k = o / 2;
            __m512i vw = _mm512_loadu_si512(w + m1 + k), vwp = _mm512_loadu_si512(wp + m1 + k);
            __m512i x = _mm512_permutex2var_epi64(v0, i1x, v1), y = _mm512_permutex2var_epi64(v0, i1y, v1);
            fwd_bf(&x, &y, vw, vwp, negq, q2, mask);
            /* canonical output */
            x = small_mod(small_mod(x, q2), q1);
            y = small_mod(small_mod(y, q2), q1);
            v0 = _mm512_permutex2var_epi64(x, i1b0, y);
            v1 = _mm512_permutex2var_epi64(x, i1b1, y);
        }
        _mm512_storeu_si512(a + o, v0);
        _mm512_storeu_si512(a + o + 8, v1);
    }
}

HX_TARGET static void inv_impl(const orc_hexl_table *h, uint64_t *a) {
    const size_t n = h->n;
    const uint64_t *w = h->t->inv_root_powers, *wp = h->iwp;
    const __m512i q1 = _mm512_set1_epi64((long long)h->q), q2 = _mm512_set1_epi64((long long)(2 * h->q));
    const __m512i negq = _mm512_set1_epi64((long long)((1ull << 52) - h->q));
    const __m512i mask = _mm512_set1_epi64((long long)((1ull << 52) - 1));
    /* stage s (gap 2^s) uses inv_root_powers[base_s + group], base_0 = 1,
     * base_{s+1} = base_s + n / 2^(s+1) */
    const size_t b1 = 1, b2 = b1 + n / 2, b4 = b2 + n / 4;
    const __m512i i4x = IDX(0, 1, 2, 3, 8, 9, 10, 11), i4y = IDX(4, 5, 6, 7, 12, 13, 14, 15);
    const __m512i i2x = IDX(0, 1, 4, 5, 8, 9, 12, 13), i2y = IDX(2, 3, 6, 7, 10, 11, 14, 15);
    const __m512i i2b0 = IDX(0, 1, 8, 9, 2, 3, 10, 11), i2b1 = IDX(4, 5, 12, 13, 6, 7, 14, 15);
    const __m512i i1x = IDX(0, 2, 4, 6, 8, 10, 12, 14), i1y = IDX(1, 3, 5, 7, 9, 11, 13, 15);
    const __m512i i1b0 = IDX(0, 8, 1, 9, 2, 10, 3, 11), i1b1 = IDX(4, 12, 5, 13, 6, 14, 7, 15);
    for (size_t o = 0; o < n; o += 16) {
        __m512i v0 = _mm512_loadu_si512(a + o), v1 = _mm512_loadu_si512(a + o + 8);
        {
            const size_t k = o / 2;
            __m512i vw = _mm512_loadu_si512(w + b1 + k), vwp = _mm512_loadu_si512(wp + b1 + k);
            __m512i x = _mm512_permutex2var_epi64(v0, i1x, v1), y = _mm512_permutex2var_epi64(v0, i1y, v1);
            inv_bf(&x, &y, vw, vwp, negq, q2, mask);
            v0 = _mm512_permutex2var_epi64(x, i1b0, y);
            v1 = _mm512_permutex2var_epi64(x, i1b1, y);
        }
        {
            const size_t k = o / 4;
            __m512i vw = IDX(w[b2 + k], w[b2 + k], w[b2 + k + 1], w[b2 + k + 1], w[b2 + k + 2], w[b2 + k + 2],
                             w[b2 + k + 3], w[b2 + k + 3]);
            __m512i vwp = IDX(wp[b2 + k], wp[b2 + k], wp[b2 + k + 1], wp[b2 + k + 1], wp[b2 + k + 2],
                              wp[b2 + k + 2], wp[b2 + k + 3], wp[b2 + k + 3]);
            __m512i x = _mm512_permutex2var_epi64(v0, i2x, v1), y = _mm512_permutex2var_epi64(v0, i2y, v1);
            inv_bf(&x, &y, vw, vwp, negq, q2, mask);
            v0 = _mm512_permutex2var_epi64(x, i2b0, y);
            v1 = _mm512_permutex2var_epi64(x, i2b1, y);
        }
        {
            const size_t k = o / 8;
            __m512i vw = IDX(w[b4 + k], w[b4 + k], w[b4 + k], w[b4 + k], w[b4 + k + 1], w[b4 + k + 1],
                             w[b4 + k + 1], w[b4 + k + 1]);
            __m512i vwp = IDX(wp[b4 + k], wp[b4 + k], wp[b4 + k], wp[b4 + k], wp[b4 + k + 1], wp[b4 + k + 1],
                              wp[b4 + k + 1], wp[b4 + k + 1]);
            __m512i x = _mm512_permutex2var_epi64(v0, i4x, v1), y = _mm512_permutex2var_epi64(v0, i4y, v1);
            inv_bf(&x, &y, vw, vwp, negq, q2, mask);
            v0 = _mm512_permutex2var_epi64(x, i4x, y);
            v1 = _mm512_permutex2var_epi64(x, i4y, y);
        }
        _mm512_storeu_si512(a + o, v0);
        _mm512_storeu_si512(a + o + 8, v1);
    }
    /* stages with gap 8 .. n/4, then the N^-1-scaled last stage (gap n/2) */
    size_t base = b4 + n / 8;
    for (size_t gap = 8; gap < n / 2; gap <<= 1) {
        const size_t groups = n / (2 * gap);
        for (size_t k = 0; k < groups; ++k) {
            const __m512i vw = _mm512_set1_epi64((long long)w[base + k]);
            const __m512i vwp = _mm512_set1_epi64((long long)wp[base + k]);
            uint64_t *x = a + 2 * k * gap, *y = x + gap;
            for (size_t j = 0; j < gap; j += 8) {
                __m512i vx = _mm512_loadu_si512(x + j), vy = _mm512_loadu_si512(y + j);
                inv_bf(&vx, &vy, vw, vwp, negq, q2, mask);
                _mm512_storeu_si512(x + j, vx);
                _mm512_storeu_si512(y + j, vy);
            }
        }
        base += groups;
    }
    const size_t gap = n / 2;
    const __m512i s = _mm512_set1_epi64((long long)h->inv_n), sp = _mm512_set1_epi64((long long)h->inv_n_p);
    const __m512i sr = _mm512_set1_epi64((long long)h->last), srp = _mm512_set1_epi64((long long)h->last_p);
    for (size_t j = 0; j < gap; j += 8) {
        __m512i u = _mm512_loadu_si512(a + j), v = _mm512_loadu_si512(a + gap + j);
        __m512i x = mul_lazy52(_mm512_add_epi64(u, v), s, sp, negq, mask);
        __m512i y = mul_lazy52(_mm512_add_epi64(u, _mm512_sub_epi64(q2, v)), sr, srp, negq, mask);
        _mm512_storeu_si512(a + j, small_mod(x, q1));
        _mm512_storeu_si512(a + gap + j, small_mod(y, q1));
    }
}

/* x = x * y mod q (canonical) with y's 52-bit quotients precomputed */
HX_TARGET static void mul_prepared_impl(uint64_t *x, const uint64_t *y, const uint64_t *yp, size_t n, uint64_t q) {
    const __m512i q1 = _mm512_set1_epi64((long long)q);
    const __m512i negq = _mm512_set1_epi64((long long)((1ull << 52) - q));
    const __m512i mask = _mm512_set1_epi64((long long)((1ull << 52) - 1));
    for (size_t i = 0; i < n; i += 8) {
        __m512i v = mul_lazy52(_mm512_loadu_si512(x + i), _mm512_loadu_si512(y + i), _mm512_loadu_si512(yp + i),
                               negq, mask);
        _mm512_storeu_si512(x + i, small_mod(v, q1));
    }
}

void orc_hexl_forward(const orc_hexl_table *h, uint64_t *a) { fwd_impl(h, a); }
void orc_hexl_inverse(const orc_hexl_table *h, uint64_t *a) { inv_impl(h, a); }

void orc_hexl_precon52(const uint64_t *y, uint64_t *yp, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; ++i) yp[i] = precon52(y[i], q);
}

/* rows [polys][L][n]: forward, x plain (NTT domain, 52-bit quotients in plain_p), inverse */
void orc_hexl_polymul_roundtrip(orc_hexl_table *const *tables, uint32_t L, uint64_t *a, const uint64_t *plain,
                                const uint64_t *plain_p, size_t polys, int threads) {
    const size_t n = tables[0]->n;
    long long r, rows = (long long)polys * L;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (r = 0; r < rows; ++r) {
        const orc_hexl_table *h = tables[r % L];
        uint64_t *row = a + (size_t)r * n;
        fwd_impl(h, row);
        mul_prepared_impl(row, plain + (size_t)(r % L) * n, plain_p + (size_t)(r % L) * n, n, h->q);
        inv_impl(h, row);
    }
}
