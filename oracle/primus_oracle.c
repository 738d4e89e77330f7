/*
 * primus_oracle.c -- CPU restatement of the primus lattice-arithmetic path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity oracle).  Loaded by tests/, by the smoke
 * check and by bench.py's CPU-baseline / reference arm; never by the product.
 *
 * Each function names the reference function it restates as
 * `crate/src/file.rs:line`.  The arithmetic is exact 64/128-bit integer math
 * (unsigned __int128); no floating point is used except in the discrete
 * Gaussian sampler that generates test noise (not part of the path).
 */
#include "primus_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ======================================================================
 * Seeded inputs: a counter-based generator so that any element can be
 * produced independently (the product library generates the same stream on
 * the device).  Uniform values below q use rejection sampling on the top
 * bitlen(q-1) bits of a 64-bit hash.
 * ====================================================================== */
static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t orc_hash64(uint64_t seed, uint64_t stream, uint64_t index, uint64_t attempt) {
    uint64_t h = mix64(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull);
    h = mix64(h ^ (stream * 0xD1B54A32D192ED03ull));
    h = mix64(h ^ (index * 0xA0761D6478BD642Full) ^ (attempt * 0xE7037ED1A0B428DBull));
    return h;
}

uint64_t orc_uniform_at(uint64_t seed, uint64_t stream, uint64_t index, uint64_t q) {
    if (q <= 1) return 0;
    uint64_t top = q - 1;
    int bits = 64 - __builtin_clzll(top);
    /* acceptance probability > 1/2 per attempt; after 64 rejections (p < 2^-64)
       the generator returns 0, exactly as the device generator does */
    for (uint64_t attempt = 0; attempt < 64; ++attempt) {
        uint64_t v = orc_hash64(seed, stream, index, attempt) >> (64 - bits);
        if (v < q) return v;
    }
    return 0;
}

void orc_fill_uniform(uint64_t seed, uint64_t stream, uint64_t q, size_t n, uint64_t *out) {
    for (size_t i = 0; i < n; ++i) out[i] = orc_uniform_at(seed, stream, i, q);
}

void orc_fill_uniform_rns(uint64_t seed, uint64_t stream0, const uint64_t *moduli, uint32_t L,
                          size_t n, uint64_t *out) {
    for (uint32_t l = 0; l < L; ++l) orc_fill_uniform(seed, stream0 + l, moduli[l], n, out + (size_t)l * n);
}

/* ======================================================================
 * Integer helpers
 * ====================================================================== */
uint64_t orc_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

uint64_t orc_powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = orc_mulmod(r, a, q);
        a = orc_mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

uint64_t orc_invmod(uint64_t a, uint64_t q) {
    /* extended Euclid on signed 128-bit */
    __int128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr != 0) {
        __int128 quo = r / nr, tmp;
        tmp = t - quo * nt; t = nt; nt = tmp;
        tmp = r - quo * nr; r = nr; nr = tmp;
    }
    if (r != 1) return 0;
    if (t < 0) t += q;
    return (uint64_t)t;
}

static uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) { uint64_t t = a % b; a = b; b = t; }
    return a;
}

int orc_is_prime(uint64_t n) {
    if (n < 2) return 0;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (int i = 0; i < 12; ++i) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    /* deterministic for all 64-bit n */
    static const uint64_t bases[] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    for (int i = 0; i < 7; ++i) {
        uint64_t a = bases[i] % n;
        if (a == 0) continue;
        uint64_t x = orc_powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; ++r) {
            x = orc_mulmod(x, x, n);
            if (x == n - 1) { comp = 0; break; }
        }
        if (comp) return 0;
    }
    return 1;
}

uint64_t orc_prev_prime_congruent(uint64_t bound, uint64_t m) {
    if (bound < 3 || m == 0) return 0;
    /* largest v < bound with v = 1 mod m */
    uint64_t v = ((bound - 2) / m) * m + 1;
    for (;;) {
        if (v < 2) return 0;
        if (orc_is_prime(v)) return v;
        if (v < m + 1) return 0;
        v -= m;
    }
}

int orc_ntt_primes(uint64_t bound, uint64_t m, uint32_t count, uint64_t *out) {
    uint64_t b = bound;
    for (uint32_t i = 0; i < count; ++i) {
        uint64_t p = orc_prev_prime_congruent(b, m);
        if (!p) return -1;
        out[i] = p;
        b = p;
    }
    return 0;
}

/* ======================================================================
 * Shoup factor: primus_factor/src/shoup_factor/mod.rs
 * ====================================================================== */
/* ShoupFactor::new (mod.rs:44-55): quotient = floor(value * 2^64 / q) */
uint64_t orc_shoup_quotient(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

/* LazyFactorMul::lazy_factor_mul_modulo (mod.rs:108-113): w*b - q*hi(w'*b), in [0,2q) */
uint64_t orc_shoup_lazy_mul(uint64_t w, uint64_t wq, uint64_t b, uint64_t q) {
    uint64_t hw = (uint64_t)(((u128)wq * b) >> 64);
    return w * b - q * hw;
}

/* FactorMul::factor_mul_modulo (mod.rs:120-124) */
uint64_t orc_shoup_mul(uint64_t w, uint64_t wq, uint64_t b, uint64_t q) {
    uint64_t t = orc_shoup_lazy_mul(w, wq, b, q);
    return t >= q ? t - q : t;
}

/* ======================================================================
 * Barrett modulus: primus_modulus/src/barrett
 * ====================================================================== */
/* BarrettModulus::new_unchecked (barrett/mod.rs:66-73): ratio = floor(2^128 / q) */
void orc_barrett_ratio(uint64_t q, uint64_t ratio[2]) {
    /* 2^128 / q computed as ((2^128 - 1) / q) adjusted: q is never a power of two > 1 here
       except in tests; handle exactly with long division on limbs [0,0,1]. */
    u128 hi = 1;          /* top limb */
    u128 rem = hi % q;    /* remainder after top limb */
    uint64_t q1 = (uint64_t)(((rem << 64) | 0) / q);
    rem = ((rem << 64) | 0) % q;
    uint64_t q0 = (uint64_t)(((rem << 64) | 0) / q);
    ratio[0] = q0;
    ratio[1] = q1;
}

/* lazy_reduce_2limb (barrett/ops.rs:41-76), result in [0,2q) */
uint64_t orc_barrett_lazy_reduce_2limb(uint64_t lo, uint64_t hi, uint64_t q, const uint64_t ratio[2]) {
    uint64_t ah = (uint64_t)(((u128)lo * ratio[0]) >> 64);
    u128 b = (u128)lo * ratio[1] + ah;           /* carrying_mul: lo*r1 + ah */
    u128 c = (u128)hi * ratio[0];
    uint64_t d = hi * ratio[1];
    uint64_t b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
    uint64_t c0 = (uint64_t)c, c1 = (uint64_t)(c >> 64);
    uint64_t carry = (uint64_t)(((u128)b0 + c0) >> 64);
    uint64_t bch = b1 + c1 + carry;
    uint64_t qq = d + bch;
    return lo - qq * q;
}

/* ReduceMul::reduce_mul (barrett/ops.rs:310-324): full reduce of the 128-bit product */
uint64_t orc_barrett_reduce_mul(uint64_t a, uint64_t b, uint64_t q, const uint64_t ratio[2]) {
    u128 p = (u128)a * b;
    uint64_t r = orc_barrett_lazy_reduce_2limb((uint64_t)p, (uint64_t)(p >> 64), q, ratio);
    return r >= q ? r - q : r;
}

/* ReduceMulAdd::reduce_mul_add (barrett/ops.rs:342-355): (a*b + c) mod q */
uint64_t orc_barrett_reduce_mul_add(uint64_t a, uint64_t b, uint64_t c, uint64_t q,
                                    const uint64_t ratio[2]) {
    u128 p = (u128)a * b + c;
    uint64_t r = orc_barrett_lazy_reduce_2limb((uint64_t)p, (uint64_t)(p >> 64), q, ratio);
    return r >= q ? r - q : r;
}

/* scalar_reduce_dot_product (barrett/slice.rs:341-372): (sum a_i b_i) mod q */
uint64_t orc_barrett_dot_product(const uint64_t *a, const uint64_t *b, size_t n, uint64_t q) {
    uint64_t acc = 0;
    for (size_t i = 0; i < n; ++i) {
        uint64_t p = (uint64_t)(((u128)a[i] * b[i]) % q);
        acc += p;
        if (acc >= q) acc -= q;
    }
    return acc;
}

/* ======================================================================
 * NTT tables: primus_ntt/src/root.rs, primus_ntt/src/ntt/primitive.rs
 * ====================================================================== */
static uint32_t rev_bits(uint32_t x, uint32_t bits) {
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* try_primitive_root (root.rs:46-87) + try_minimal_primitive_root (root.rs:89-111).
 * The reference draws the first primitive root at random and then takes the
 * minimum over all of its odd powers, so the result is the smallest primitive
 * 2^log_degree-th root; the search here starts from r = 2, 3, ... instead. */
int orc_minimal_primitive_root(uint32_t log_degree, uint64_t q, uint64_t *root) {
    if (log_degree == 0 || log_degree >= 64) return 3;
    uint64_t degree = 1ull << log_degree;
    uint64_t qm1 = q - 1;
    uint64_t quotient = qm1 >> log_degree;
    if (quotient * degree != qm1) return 1;
    uint64_t w = 0;
    int found = 0;
    for (uint64_t r = 2; r < q && r < 100000; ++r) {
        w = orc_powmod(r, quotient, q);
        /* is_primitive_root (root.rs:26-44): w^(degree/2) == q - 1 */
        uint64_t x = w;
        for (uint32_t i = 0; i + 1 < log_degree; ++i) x = orc_mulmod(x, x, q);
        if (w != 0 && x == qm1) { found = 1; break; }
    }
    if (!found) return 1;
    uint64_t best = w;
    uint64_t g2 = orc_mulmod(w, w, q);
    uint64_t cur = w;
    for (uint64_t i = 0; i < degree; ++i) {
        if (cur < best) best = cur;
        cur = orc_mulmod(g2, cur, q);
    }
    *root = best;
    return 0;
}

void orc_ntt_table_free(orc_ntt_table *t) {
    free(t->root_powers); free(t->root_powers_q);
    free(t->inv_root_powers); free(t->inv_root_powers_q);
    free(t->ordinal); free(t->ordinal_q);
    free(t->rev);
    memset(t, 0, sizeof(*t));
}

/* UintNttTable::new (primitive.rs:113-185) */
int orc_ntt_table_init(orc_ntt_table *t, uint32_t log_n, uint64_t q) {
    memset(t, 0, sizeof(*t));
    if (log_n == 0 || log_n > 30 || q < 3) return 3;
    uint64_t root;
    int rc = orc_minimal_primitive_root(log_n + 1, q, &root);
    if (rc) return rc;
    size_t n = (size_t)1 << log_n;
    t->q = q; t->log_n = log_n; t->n = n; t->root = root;
    t->ordinal = malloc(2 * n * 8); t->ordinal_q = malloc(2 * n * 8);
    t->root_powers = malloc(n * 8); t->root_powers_q = malloc(n * 8);
    t->inv_root_powers = malloc(n * 8); t->inv_root_powers_q = malloc(n * 8);
    t->rev = malloc(n * 4);
    if (!t->ordinal || !t->ordinal_q || !t->root_powers || !t->root_powers_q ||
        !t->inv_root_powers || !t->inv_root_powers_q || !t->rev) {
        orc_ntt_table_free(t);
        return 3;
    }
    /* ordinal_root_powers: psi^0 .. psi^(2n-1) (:130-137) */
    uint64_t rq = orc_shoup_quotient(root, q);
    t->ordinal[0] = 1;
    t->ordinal[1] = root;
    uint64_t power = root;
    for (size_t i = 2; i < 2 * n; ++i) {
        power = orc_shoup_mul(root, rq, power, q);
        t->ordinal[i] = power;
    }
    for (size_t i = 0; i < 2 * n; ++i) t->ordinal_q[i] = orc_shoup_quotient(t->ordinal[i], q);
    t->inv_root = t->ordinal[2 * n - 1];
    for (size_t i = 0; i < n; ++i) t->rev[i] = rev_bits((uint32_t)i, log_n);
    /* root_powers[rev(i)] = psi^i (:145-149) */
    for (size_t i = 0; i < n; ++i) {
        t->root_powers[t->rev[i]] = t->ordinal[i];
        t->root_powers_q[t->rev[i]] = t->ordinal_q[i];
    }
    /* inv_root_powers[rev(i)+1] = psi^-(i+1) (:151-159) */
    t->inv_root_powers[0] = 1;
    t->inv_root_powers_q[0] = orc_shoup_quotient(1, q);
    for (size_t i = 0; i + 1 < n; ++i) {
        size_t src = 2 * n - 1 - i;
        t->inv_root_powers[t->rev[i] + 1] = t->ordinal[src];
        t->inv_root_powers_q[t->rev[i] + 1] = t->ordinal_q[src];
    }
    /* inv_n (:161-168) */
    if ((uint64_t)n >= q) { orc_ntt_table_free(t); return 2; }
    t->inv_n = orc_invmod((uint64_t)n, q);
    t->inv_n_q = orc_shoup_quotient(t->inv_n, q);
    return 0;
}

orc_ntt_table *orc_ntt_table_new(uint32_t log_n, uint64_t q) {
    orc_ntt_table *t = calloc(1, sizeof(*t));
    if (!t) return NULL;
    if (orc_ntt_table_init(t, log_n, q)) { free(t); return NULL; }
    return t;
}

void orc_ntt_table_delete(orc_ntt_table *t) {
    if (!t) return;
    orc_ntt_table_free(t);
    free(t);
}

void orc_ntt_table_export(const orc_ntt_table *t, uint64_t *root, uint64_t *inv_root,
                          uint64_t *inv_n, uint64_t *inv_n_q, uint64_t *root_powers,
                          uint64_t *root_powers_q, uint64_t *inv_root_powers,
                          uint64_t *inv_root_powers_q, uint64_t *ordinal, uint64_t *ordinal_q) {
    size_t n = t->n;
    if (root) *root = t->root;
    if (inv_root) *inv_root = t->inv_root;
    if (inv_n) *inv_n = t->inv_n;
    if (inv_n_q) *inv_n_q = t->inv_n_q;
    if (root_powers) memcpy(root_powers, t->root_powers, n * 8);
    if (root_powers_q) memcpy(root_powers_q, t->root_powers_q, n * 8);
    if (inv_root_powers) memcpy(inv_root_powers, t->inv_root_powers, n * 8);
    if (inv_root_powers_q) memcpy(inv_root_powers_q, t->inv_root_powers_q, n * 8);
    if (ordinal) memcpy(ordinal, t->ordinal, 2 * n * 8);
    if (ordinal_q) memcpy(ordinal_q, t->ordinal_q, 2 * n * 8);
}

/* lazy_transform_slice (primitive.rs:211-232): CT/Harvey butterflies, [0,4q) -> [0,4q) */
void orc_ntt_lazy_forward(const orc_ntt_table *t, uint64_t *a) {
    const uint64_t q = t->q, q2 = q << 1;
    size_t idx = 1;
    for (size_t gap = t->n >> 1; gap >= 1; gap >>= 1) {
        for (size_t start = 0; start < t->n; start += 2 * gap) {
            uint64_t w = t->root_powers[idx], wq = t->root_powers_q[idx];
            ++idx;
            for (size_t i = start; i < start + gap; ++i) {
                uint64_t x = a[i], y = a[i + gap];
                uint64_t u = x >= q2 ? x - q2 : x;
                uint64_t v = orc_shoup_lazy_mul(w, wq, y, q);
                a[i] = u + v;
                a[i + gap] = u + q2 - v;
            }
        }
        if (gap == 1) break;
    }
}

/* transform_slice (primitive.rs:234-244) */
void orc_ntt_forward(const orc_ntt_table *t, uint64_t *a) {
    orc_ntt_lazy_forward(t, a);
    const uint64_t q = t->q, q2 = q << 1;
    for (size_t i = 0; i < t->n; ++i) {
        uint64_t v = a[i];
        if (v >= q2) v -= q2;
        if (v >= q) v -= q;
        a[i] = v;
    }
}

/* lazy_inverse_transform_slice (primitive.rs:246-286): GS butterflies; the last
 * stage is fused with the N^-1 scaling.  Input [0,2q), output [0,q). */
void orc_ntt_lazy_inverse(const orc_ntt_table *t, uint64_t *a) {
    const uint64_t q = t->q, q2 = q << 1;
    const size_t n = t->n;
    size_t idx = 1;
    for (size_t gap = 1; gap < n / 2; gap <<= 1) {
        for (size_t start = 0; start < n; start += 2 * gap) {
            uint64_t w = t->inv_root_powers[idx], wq = t->inv_root_powers_q[idx];
            ++idx;
            for (size_t i = start; i < start + gap; ++i) {
                uint64_t u = a[i], v = a[i + gap];
                /* UintModulus::reduce_add (unsigned_integer/ops.rs:34-41) */
                uint64_t diff = q2 - v;
                a[i] = diff > u ? u + v : u - diff;
                a[i + gap] = orc_shoup_lazy_mul(w, wq, u + q2 - v, q);
            }
        }
    }
    size_t gap = n / 2;
    uint64_t s = t->inv_n, sq = t->inv_n_q;
    uint64_t sr = orc_shoup_mul(t->inv_root_powers[idx], t->inv_root_powers_q[idx], s, q);
    uint64_t srq = orc_shoup_quotient(sr, q);
    for (size_t i = 0; i < gap; ++i) {
        uint64_t u = a[i], v = a[i + gap];
        a[i] = orc_shoup_mul(s, sq, u + v, q);
        a[i + gap] = orc_shoup_mul(sr, srq, u + q2 - v, q);
    }
}

/* inverse_transform_slice (primitive.rs:288-296) */
void orc_ntt_inverse(const orc_ntt_table *t, uint64_t *a) {
    orc_ntt_lazy_inverse(t, a);
    const uint64_t q = t->q;
    for (size_t i = 0; i < t->n; ++i)
        if (a[i] >= q) a[i] -= q;
}

/* transform_monomial (primitive.rs:298-349) */
void orc_ntt_monomial(const orc_ntt_table *t, uint64_t coeff, size_t degree, uint64_t *out) {
    const size_t n = t->n;
    if (coeff == 0) { memset(out, 0, n * 8); return; }
    if (degree == 0) { for (size_t i = 0; i < n; ++i) out[i] = coeff; return; }
    const size_t mask = 2 * n - 1;
    for (size_t i = 0; i < n; ++i) {
        size_t index = ((2 * (size_t)t->rev[i] + 1) * degree) & mask;
        if (coeff == 1)
            out[i] = t->ordinal[index];
        else if (coeff == t->q - 1)
            out[i] = t->ordinal[index ^ n];
        else
            out[i] = orc_shoup_mul(t->ordinal[index], t->ordinal_q[index], coeff, t->q);
    }
}

/* transform_coeff_one_monomial (primitive.rs:351-373) */
void orc_ntt_coeff_one_monomial(const orc_ntt_table *t, size_t degree, uint64_t *out) {
    const size_t n = t->n;
    if (degree == 0) { for (size_t i = 0; i < n; ++i) out[i] = 1; return; }
    const size_t mask = 2 * n - 1;
    for (size_t i = 0; i < n; ++i) out[i] = t->ordinal[((2 * (size_t)t->rev[i] + 1) * degree) & mask];
}

/* transform_coeff_minus_one_monomial (primitive.rs:375-397) */
void orc_ntt_coeff_minus_one_monomial(const orc_ntt_table *t, size_t degree, uint64_t *out) {
    const size_t n = t->n;
    if (degree == 0) { for (size_t i = 0; i < n; ++i) out[i] = t->q - 1; return; }
    const size_t mask = 2 * n - 1;
    for (size_t i = 0; i < n; ++i)
        out[i] = t->ordinal[(((2 * (size_t)t->rev[i] + 1) * degree) & mask) ^ n];
}

void orc_ntt_forward_rows(const orc_ntt_table *t, uint64_t *a, size_t rows, int lazy, int threads) {
    long long r;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (r = 0; r < (long long)rows; ++r) {
        if (lazy) orc_ntt_lazy_forward(t, a + (size_t)r * t->n);
        else orc_ntt_forward(t, a + (size_t)r * t->n);
    }
}

void orc_ntt_inverse_rows(const orc_ntt_table *t, uint64_t *a, size_t rows, int lazy, int threads) {
    long long r;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (r = 0; r < (long long)rows; ++r) {
        if (lazy) orc_ntt_lazy_inverse(t, a + (size_t)r * t->n);
        else orc_ntt_inverse(t, a + (size_t)r * t->n);
    }
}

/* The NTT's definition as encoded by transform_monomial (primitive.rs:321-328):
 * out[i] = sum_j a_j psi^((2 rev(i) + 1) j) mod q.  O(N^2), small N only. */
void orc_ntt_by_definition(const orc_ntt_table *t, const uint64_t *a, uint64_t *out) {
    const size_t n = t->n, mask = 2 * n - 1;
    for (size_t i = 0; i < n; ++i) {
        size_t e = 2 * (size_t)t->rev[i] + 1;
        u128 acc = 0;
        for (size_t j = 0; j < n; ++j) {
            acc += (u128)(a[j] % t->q) * t->ordinal[(e * j) & mask];
            acc %= t->q;
        }
        out[i] = (uint64_t)acc;
    }
}

/* ======================================================================
 * DCRT: primus_ntt/src/dcrt/primitive.rs:96-141 (one table per limb)
 * ====================================================================== */
void orc_dcrt_forward(orc_ntt_table *const *tables, uint32_t L, uint64_t *a, size_t polys,
                      int lazy, int threads) {
    const size_t n = tables[0]->n;
    long long r, rows = (long long)polys * L;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (r = 0; r < rows; ++r) {
        const orc_ntt_table *t = tables[r % L];
        if (lazy) orc_ntt_lazy_forward(t, a + (size_t)r * n);
        else orc_ntt_forward(t, a + (size_t)r * n);
    }
}

void orc_dcrt_inverse(orc_ntt_table *const *tables, uint32_t L, uint64_t *a, size_t polys,
                      int lazy, int threads) {
    const size_t n = tables[0]->n;
    long long r, rows = (long long)polys * L;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (r = 0; r < rows; ++r) {
        const orc_ntt_table *t = tables[r % L];
        if (lazy) orc_ntt_lazy_inverse(t, a + (size_t)r * n);
        else orc_ntt_inverse(t, a + (size_t)r * n);
    }
}

/* transform_slice -> DcrtPolynomial::mul_assign (primus_poly/src/dcrt/mul.rs:97-110)
 * -> inverse_transform_slice, for every row of every poly */
void orc_dcrt_polymul_roundtrip(orc_ntt_table *const *tables, uint32_t L, uint64_t *a,
                                const uint64_t *plain, size_t polys, int threads) {
    const size_t n = tables[0]->n;
    long long r, rows = (long long)polys * L;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (r = 0; r < rows; ++r) {
        const orc_ntt_table *t = tables[r % L];
        uint64_t *row = a + (size_t)r * n;
        orc_ntt_forward(t, row);
        orc_mul_assign(row, plain + (size_t)(r % L) * n, n, t->q);
        orc_ntt_inverse(t, row);
    }
}

/* ======================================================================
 * Pointwise ops (canonical in, canonical out)
 * ====================================================================== */
/* ArrayBase::mul_element_wise_assign (primus_poly/src/array/mul.rs:60-69) */
void orc_mul_assign(uint64_t *x, const uint64_t *y, size_t n, uint64_t q) {
    uint64_t ratio[2];
    orc_barrett_ratio(q, ratio);
    for (size_t i = 0; i < n; ++i) x[i] = orc_barrett_reduce_mul(x[i], y[i], q, ratio);
}

/* ArrayBase::add_mul_element_wise_assign (primus_poly/src/array/add.rs:35-48) */
void orc_add_mul_assign(uint64_t *acc, const uint64_t *b, const uint64_t *c, size_t n, uint64_t q) {
    uint64_t ratio[2];
    orc_barrett_ratio(q, ratio);
    for (size_t i = 0; i < n; ++i) acc[i] = orc_barrett_reduce_mul_add(b[i], c[i], acc[i], q, ratio);
}

/* ArrayBase::mul_scalar_assign (used by DcrtPolynomial::mul_scalar_assign, dcrt/mul.rs:27-34) */
void orc_mul_scalar_assign(uint64_t *x, uint64_t s, size_t n, uint64_t q) {
    uint64_t ratio[2];
    orc_barrett_ratio(q, ratio);
    for (size_t i = 0; i < n; ++i) x[i] = orc_barrett_reduce_mul(x[i], s, q, ratio);
}

/* DcrtPolynomial::add_mul_scalar_assign (dcrt/mul.rs:37-58) */
void orc_add_mul_scalar_assign(uint64_t *x, const uint64_t *y, uint64_t s, size_t n, uint64_t q) {
    uint64_t ratio[2];
    orc_barrett_ratio(q, ratio);
    for (size_t i = 0; i < n; ++i) x[i] = orc_barrett_reduce_mul_add(y[i], s, x[i], q, ratio);
}

/* DcrtPolynomial::mul_factor_assign (dcrt/mul.rs:73-83) */
void orc_mul_factor_assign(uint64_t *x, uint64_t w, uint64_t wq, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; ++i) x[i] = orc_shoup_mul(w, wq, x[i], q);
}

/* UintModulus reduce_add / reduce_sub / reduce_neg (unsigned_integer/ops.rs:34,81,105) */
void orc_add_assign(uint64_t *x, const uint64_t *y, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; ++i) {
        uint64_t diff = q - y[i];
        x[i] = diff > x[i] ? x[i] + y[i] : x[i] - diff;
    }
}

void orc_sub_assign(uint64_t *x, const uint64_t *y, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; ++i) x[i] = y[i] > x[i] ? x[i] - y[i] + q : x[i] - y[i];
}

void orc_neg_assign(uint64_t *x, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; ++i) x[i] = x[i] == 0 ? 0 : q - x[i];
}

/* DcrtPolynomial::butterfly_mul_factor_inplace (dcrt/mul.rs:119-155):
 * (a, b) = (a + s, (a - s) * w) */
void orc_butterfly_mul_factor(uint64_t *a, const uint64_t *s, const uint64_t *w,
                              const uint64_t *wq, uint64_t *b, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; ++i) {
        uint64_t orig = a[i];
        uint64_t diff = q - s[i];
        a[i] = diff > orig ? orig + s[i] : orig - diff;
        uint64_t d = s[i] > orig ? orig - s[i] + q : orig - s[i];
        b[i] = orc_shoup_mul(w[i], wq[i], d, q);
    }
}

/* Polynomial::naive_mul_inplace (primus_poly/src/poly/mul.rs:111-142) */
void orc_naive_negacyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t *c, size_t n,
                              uint64_t q) {
    uint64_t ratio[2];
    orc_barrett_ratio(q, ratio);
    for (size_t i = 0; i < n; ++i) c[i] = 0;
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j <= i; ++j) c[i] = orc_barrett_reduce_mul_add(a[j], b[i - j], c[i], q, ratio);
    for (size_t i = n; i + 1 < 2 * n; ++i) {
        size_t k = i - n;
        for (size_t j = i - n + 1; j < n; ++j) {
            uint64_t p = orc_barrett_reduce_mul(a[j], b[i - j], q, ratio);
            c[k] = p > c[k] ? c[k] - p + q : c[k] - p;
        }
    }
}

/* ======================================================================
 * BigUint helpers (primus_integer/src/big_integer.rs), little-endian limbs
 * ====================================================================== */
/* mul_value_add_inplace (big_integer.rs:281-299): dst += src * v, returns carry */
static uint64_t big_mul_value_add(const uint64_t *src, uint64_t v, uint64_t *dst, uint32_t W) {
    if (v == 0) return 0;
    uint64_t carry = 0;
    for (uint32_t i = 0; i < W; ++i) {
        u128 t = (u128)v * src[i] + dst[i] + carry;
        dst[i] = (uint64_t)t;
        carry = (uint64_t)(t >> 64);
    }
    return carry;
}

static int big_cmp(const uint64_t *a, const uint64_t *b, uint32_t W) {
    for (uint32_t i = W; i-- > 0;) {
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}

static int big_sub_assign(uint64_t *a, const uint64_t *b, uint32_t W) {
    uint64_t borrow = 0;
    for (uint32_t i = 0; i < W; ++i) {
        u128 t = (u128)a[i] - b[i] - borrow;
        a[i] = (uint64_t)t;
        borrow = (uint64_t)(t >> 64) ? 1 : 0;
    }
    return (int)borrow;
}

static int big_add_assign(uint64_t *a, const uint64_t *b, uint32_t W) {
    uint64_t carry = 0;
    for (uint32_t i = 0; i < W; ++i) {
        u128 t = (u128)a[i] + b[i] + carry;
        a[i] = (uint64_t)t;
        carry = (uint64_t)(t >> 64);
    }
    return (int)carry;
}

static uint64_t big_shl(uint64_t *a, uint32_t W, uint32_t bits) {
    /* bits < 64; returns the bits shifted out */
    if (bits == 0) return 0;
    uint64_t carry = 0;
    for (uint32_t i = 0; i < W; ++i) {
        uint64_t nc = a[i] >> (64 - bits);
        a[i] = (a[i] << bits) | carry;
        carry = nc;
    }
    return carry;
}

static uint64_t big_mod_value(const uint64_t *a, uint32_t W, uint64_t q) {
    u128 r = 0;
    for (uint32_t i = W; i-- > 0;) r = ((r << 64) | a[i]) % q;
    return (uint64_t)r;
}

/* ======================================================================
 * RNS base: primus_rns/src/base.rs
 * ====================================================================== */
/* RNSBase::new (base.rs:50-90) with multiply_many_values (big_integer.rs:647-658)
 * and multiply_many_values_except_inplace (big_integer.rs:688-706) */
orc_rns_base *orc_rns_base_new(const uint64_t *moduli, uint32_t L) {
    if (L == 0) return NULL;
    for (uint32_t i = 0; i < L; ++i)
        for (uint32_t j = i + 1; j < L; ++j)
            if (gcd64(moduli[i], moduli[j]) != 1) return NULL;
    orc_rns_base *b = calloc(1, sizeof(*b));
    b->L = L;
    b->moduli = malloc(L * 8);
    memcpy(b->moduli, moduli, L * 8);
    uint64_t *prod = calloc(L + 1, 8);
    uint32_t len = 1;
    prod[0] = moduli[0];
    for (uint32_t i = 1; i < L; ++i) {
        uint64_t carry = 0;
        for (uint32_t k = 0; k < len; ++k) {
            u128 t = (u128)prod[k] * moduli[i] + carry;
            prod[k] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        if (carry) prod[len++] = carry;
    }
    b->W = len;
    b->product = prod;
    b->punctured = calloc((size_t)L * len, 8);
    b->inv_punctured = malloc(L * 8);
    b->inv_punctured_q = malloc(L * 8);
    for (uint32_t i = 0; i < L; ++i) {
        uint64_t *r = b->punctured + (size_t)i * len;
        r[0] = 1;
        uint32_t rl = 1;
        for (uint32_t j = 0; j < L; ++j) {
            if (j == i) continue;
            uint64_t carry = 0;
            for (uint32_t k = 0; k < rl; ++k) {
                u128 t = (u128)r[k] * moduli[j] + carry;
                r[k] = (uint64_t)t;
                carry = (uint64_t)(t >> 64);
            }
            if (carry) r[rl++] = carry;
        }
        uint64_t pm = big_mod_value(r, len, moduli[i]);
        uint64_t inv = orc_invmod(pm, moduli[i]);
        b->inv_punctured[i] = inv;
        b->inv_punctured_q[i] = orc_shoup_quotient(inv, moduli[i]);
    }
    return b;
}

void orc_rns_base_delete(orc_rns_base *b) {
    if (!b) return;
    free(b->moduli); free(b->product); free(b->punctured);
    free(b->inv_punctured); free(b->inv_punctured_q);
    free(b);
}

uint32_t orc_rns_base_width(const orc_rns_base *b) { return b->W; }

void orc_rns_base_export(const orc_rns_base *b, uint64_t *product, uint64_t *punctured,
                         uint64_t *inv_punctured) {
    if (product) memcpy(product, b->product, b->W * 8);
    if (punctured) memcpy(punctured, b->punctured, (size_t)b->L * b->W * 8);
    if (inv_punctured) memcpy(inv_punctured, b->inv_punctured, b->L * 8);
}

/* compose_inplace (base.rs:396-420) */
void orc_rns_compose(const orc_rns_base *b, const uint64_t *residues, uint64_t *value) {
    const uint32_t W = b->W;
    memset(value, 0, W * 8);
    for (uint32_t i = 0; i < b->L; ++i) {
        uint64_t product = orc_shoup_mul(b->inv_punctured[i], b->inv_punctured_q[i], residues[i], b->moduli[i]);
        uint64_t carry = big_mul_value_add(b->punctured + (size_t)i * W, product, value, W);
        if (carry != 0 || big_cmp(value, b->product, W) >= 0) big_sub_assign(value, b->product, W);
    }
}

/* compose_multiple_values_inplace (base.rs:422-449): [L][count] -> [count][W] */
void orc_rns_compose_multiple(const orc_rns_base *b, const uint64_t *multi_residues,
                              uint64_t *values, size_t count) {
    uint64_t res[64];
    for (size_t x = 0; x < count; ++x) {
        for (uint32_t i = 0; i < b->L; ++i) res[i] = multi_residues[(size_t)i * count + x];
        orc_rns_compose(b, res, values + x * b->W);
    }
}

/* decompose_inplace (base.rs:171-177) */
void orc_rns_decompose(const orc_rns_base *b, const uint64_t *value, uint64_t *residues) {
    for (uint32_t i = 0; i < b->L; ++i) residues[i] = big_mod_value(value, b->W, b->moduli[i]);
}

/* decompose_big_uint_values_inplace (base.rs:285-309): [count][W] -> [L][count] */
void orc_rns_decompose_multiple(const orc_rns_base *b, const uint64_t *values,
                                uint64_t *multi_residues, size_t count) {
    for (uint32_t i = 0; i < b->L; ++i)
        for (size_t x = 0; x < count; ++x)
            multi_residues[(size_t)i * count + x] = big_mod_value(values + x * b->W, b->W, b->moduli[i]);
}

/* wrapping_decompose_small_values_inplace (base.rs:201-231) */
void orc_rns_wrapping_decompose_small(const orc_rns_base *b, const uint64_t *small,
                                      uint64_t *multi_residues, size_t count,
                                      uint64_t small_modulus) {
    for (uint32_t i = 0; i < b->L; ++i) {
        uint64_t *out = multi_residues + (size_t)i * count;
        if (small_modulus != 2) {
            uint64_t half = (small_modulus + 1) / 2;
            uint64_t temp = b->moduli[i] - small_modulus;
            for (size_t x = 0; x < count; ++x) out[x] = small[x] < half ? small[x] : temp + small[x];
        } else {
            memcpy(out, small, count * 8);
        }
    }
}

/* ======================================================================
 * Fast base conversion: primus_rns/src/converter.rs
 * ====================================================================== */
/* BaseConverter::new (converter.rs:22-47): matrix[j][i] = (Q/q_i) mod p_j */
orc_base_converter *orc_base_converter_new(const orc_rns_base *ibase, const orc_rns_base *obase) {
    orc_base_converter *c = calloc(1, sizeof(*c));
    c->ibase = ibase; c->obase = obase;
    c->matrix = malloc((size_t)ibase->L * obase->L * 8);
    for (uint32_t j = 0; j < obase->L; ++j)
        for (uint32_t i = 0; i < ibase->L; ++i)
            c->matrix[(size_t)j * ibase->L + i] =
                big_mod_value(ibase->punctured + (size_t)i * ibase->W, ibase->W, obase->moduli[j]);
    return c;
}

void orc_base_converter_delete(orc_base_converter *c) {
    if (!c) return;
    free(c->matrix);
    free(c);
}

/* fast_convert_array (converter.rs:147-175) with fill_fast_convert_array_buffer (:103-145) */
void orc_fast_convert_array(const orc_base_converter *c, const uint64_t *in, uint64_t *out,
                            size_t n) {
    const orc_rns_base *ib = c->ibase, *ob = c->obase;
    const uint32_t Li = ib->L;
    uint64_t *buf = malloc((size_t)n * Li * 8);
    for (uint32_t i = 0; i < Li; ++i) {
        const uint64_t qi = ib->moduli[i];
        for (size_t x = 0; x < n; ++x) {
            uint64_t v = in[(size_t)i * n + x];
            buf[x * Li + i] = ib->inv_punctured[i] == 1 ? v % qi
                                                        : orc_shoup_mul(ib->inv_punctured[i], ib->inv_punctured_q[i], v, qi);
        }
    }
    for (uint32_t j = 0; j < ob->L; ++j)
        for (size_t x = 0; x < n; ++x)
            out[(size_t)j * n + x] = orc_barrett_dot_product(buf + x * Li, c->matrix + (size_t)j * Li, Li, ob->moduli[j]);
    free(buf);
}

/* ======================================================================
 * Gadget decomposition: primus_decompose/src/big_integer/{basis,common}.rs
 * ====================================================================== */
/* BigUintApproxSignedBasis::new (basis.rs:34-193) */
orc_gadget_basis *orc_gadget_basis_new(const orc_rns_base *base, uint32_t log_basis,
                                       int32_t reverse_length) {
    const uint32_t W = base->W;
    const uint64_t *Q = base->product;
    if (Q[W - 1] == 0 || log_basis == 0 || log_basis >= 64) return NULL;
    orc_gadget_basis *g = calloc(1, sizeof(*g));
    g->W = W; g->L = base->L; g->log_basis = log_basis;
    uint32_t unused = (uint32_t)__builtin_clzll(Q[W - 1]);
    g->basis = 1ull << log_basis;
    g->basis_minus_one = g->basis - 1;
    uint32_t bits = 64 * W - unused;
    uint32_t d = bits / log_basis;
    uint32_t drop = bits - d * log_basis;
    if (reverse_length >= 0) {
        if ((uint32_t)reverse_length > d || reverse_length == 0) { free(g); return NULL; }
        d = (uint32_t)reverse_length;
        drop = bits - d * log_basis;
    }
    g->decompose_length = d;
    g->drop_bits = drop;
    if (drop > 0) {
        g->has_init_carry = 1;
        g->init_carry_index = (drop - 1) / 64;
        g->init_carry_mask = 1ull << ((drop - 1) % 64);
    }
    g->carry_mask = log_basis == 1 ? 2ull : ((1ull << log_basis) | (1ull << (log_basis - 1)));
    g->modulus = malloc(W * 8);
    memcpy(g->modulus, Q, W * 8);
    /* split value */
    g->split = calloc(W, 8);
    uint64_t *v = g->split;
    if (log_basis == 1) {
        if (drop != 0) {
            for (uint32_t i = 0; i < d; ++i) { big_shl(v, W, 1); v[0] |= 1; }
            big_shl(v, W, 1); v[0] |= 1;
            uint32_t s = drop - 1;
            while (s >= 63) { big_shl(v, W, 63); s -= 63; }
            big_shl(v, W, s);
            g->has_split = big_cmp(v, Q, W) < 0;
        }
    } else {
        for (uint32_t i = 0; i < d; ++i) { big_shl(v, W, log_basis); v[0] |= g->basis_minus_one >> 1; }
        if (drop > 0) {
            big_shl(v, W, 1); v[0] |= 1;
            uint32_t s = drop - 1;
            while (s >= 63) { big_shl(v, W, 63); s -= 63; }
            big_shl(v, W, s);
        } else {
            uint64_t one[64] = {0};
            one[0] = 1;
            big_add_assign(v, one, W);
        }
        g->has_split = big_cmp(v, Q, W) < 0;
    }
    /* next_pow_of_2_sub_modulus = (2^bits - 1) - (Q - 1) */
    g->next_pow2_sub_q = malloc(W * 8);
    for (uint32_t i = 0; i < W; ++i) g->next_pow2_sub_q[i] = ~0ull;
    g->next_pow2_sub_q[W - 1] >>= unused;
    uint64_t qm1[64];
    memcpy(qm1, Q, W * 8);
    {
        uint64_t one[64] = {0};
        one[0] = 1;
        big_sub_assign(qm1, one, W);
    }
    big_sub_assign(g->next_pow2_sub_q, qm1, W);
    /* scalars: 2^drop, 2^(drop+lb), ... */
    g->scalars = calloc((size_t)d * W, 8);
    {
        uint64_t cur[64] = {0};
        cur[0] = 1;
        uint32_t s = drop;
        while (s >= 63) { big_shl(cur, W, 63); s -= 63; }
        big_shl(cur, W, s);
        for (uint32_t j = 0; j < d; ++j) {
            if (j > 0) big_shl(cur, W, log_basis);
            memcpy(g->scalars + (size_t)j * W, cur, W * 8);
        }
    }
    g->scalar_residues = malloc((size_t)d * base->L * 8);
    for (uint32_t j = 0; j < d; ++j) orc_rns_decompose(base, g->scalars + (size_t)j * W, g->scalar_residues + (size_t)j * base->L);
    /* ValueMask::new / next (common.rs:16-53) */
    g->mask_index = malloc(d * 4); g->mask0 = malloc(d * 8); g->mask1 = malloc(d * 8);
    g->mask_shr = malloc(d * 4); g->mask_shl = malloc(d * 4);
    uint32_t index = drop / 64, shr = drop % 64;
    for (uint32_t j = 0; j < d; ++j) {
        if (j > 0) {
            uint32_t ns = log_basis + shr;
            if (ns >= 64) { index += 1; ns -= 64; }
            shr = ns;
        }
        g->mask_index[j] = index;
        g->mask0[j] = g->basis_minus_one << shr;
        g->mask1[j] = shr == 0 ? 0 : (g->basis_minus_one >> (64 - shr));
        g->mask_shr[j] = shr;
        g->mask_shl[j] = 64 - shr;
    }
    return g;
}

void orc_gadget_basis_delete(orc_gadget_basis *g) {
    if (!g) return;
    free(g->split); free(g->next_pow2_sub_q); free(g->modulus); free(g->scalars);
    free(g->scalar_residues); free(g->mask_index); free(g->mask0); free(g->mask1);
    free(g->mask_shr); free(g->mask_shl);
    free(g);
}

void orc_gadget_basis_info(const orc_gadget_basis *g, uint32_t *decompose_length,
                           uint32_t *drop_bits, uint64_t *scalar_residues) {
    if (decompose_length) *decompose_length = g->decompose_length;
    if (drop_bits) *drop_bits = g->drop_bits;
    if (scalar_residues) memcpy(scalar_residues, g->scalar_residues, (size_t)g->decompose_length * g->L * 8);
}

/* init_value_carry_slice_inplace (basis.rs:307-331) */
void orc_gadget_init_carry(const orc_gadget_basis *g, uint64_t *values, uint8_t *carries,
                           size_t count) {
    const uint32_t W = g->W;
    if (g->has_split) {
        for (size_t x = 0; x < count; ++x) {
            uint64_t *v = values + x * W;
            if (big_cmp(v, g->split, W) >= 0) big_add_assign(v, g->next_pow2_sub_q, W);
        }
    }
    for (size_t x = 0; x < count; ++x)
        carries[x] = g->has_init_carry ? ((values[x * W + g->init_carry_index] & g->init_carry_mask) != 0) : 0;
}

/* ValueMask::get_value (common.rs:55-63) */
static inline uint64_t gadget_get_value(const orc_gadget_basis *g, uint32_t j, const uint64_t *v) {
    uint32_t idx = g->mask_index[j];
    uint64_t temp = (v[idx] & g->mask0[j]) >> g->mask_shr[j];
    if (g->mask1[j] != 0) temp |= (v[idx + 1] & g->mask1[j]) << g->mask_shl[j];
    return temp;
}

/* unsigned_decompose_slice_inplace (common.rs:184-200) */
void orc_gadget_unsigned_digit(const orc_gadget_basis *g, uint32_t level, const uint64_t *values,
                               uint64_t *digits, uint8_t *carries, size_t count) {
    for (size_t x = 0; x < count; ++x) {
        uint64_t temp = gadget_get_value(g, level, values + x * g->W) + carries[x];
        carries[x] = (temp & g->carry_mask) != 0;
        digits[x] = temp & g->basis_minus_one;
    }
}

void orc_gadget_decompose_all(const orc_gadget_basis *g, const uint64_t *values, uint64_t *digits,
                              size_t count) {
    uint64_t *adj = malloc(count * g->W * 8);
    uint8_t *carries = malloc(count);
    memcpy(adj, values, count * g->W * 8);
    orc_gadget_init_carry(g, adj, carries, count);
    for (uint32_t j = 0; j < g->decompose_length; ++j)
        orc_gadget_unsigned_digit(g, j, adj, digits + (size_t)j * count, carries, count);
    free(adj);
    free(carries);
}

/* ApproxSignedBasis::new (primitive/basis.rs:41-166) */
orc_approx_basis *orc_approx_basis_new(int has_modulus, uint64_t modulus, uint32_t log_basis,
                                       int32_t reverse_length) {
    if (log_basis == 0 || log_basis > 63) return NULL;
    orc_approx_basis *b = calloc(1, sizeof(*b));
    b->has_modulus = has_modulus; b->modulus = modulus; b->log_basis = log_basis;
    b->basis = 1ull << log_basis;
    b->basis_minus_one = b->basis - 1;
    if (has_modulus) {
        if ((modulus & (modulus - 1)) == 0) {
            b->modulus_is_pow2 = 1;
            b->value_bits = (uint32_t)__builtin_ctzll(modulus);
        } else {
            b->value_bits = 64 - (uint32_t)__builtin_clzll(modulus);
        }
        if (b->value_bits < log_basis) { free(b); return NULL; }
        b->modulus_minus_basis = modulus - b->basis;
    } else {
        b->modulus_is_pow2 = 1;
        b->value_bits = 64;
        b->modulus_minus_basis = ~0ull - b->basis_minus_one;
    }
    uint32_t d = b->value_bits / log_basis;
    uint32_t drop = b->value_bits - d * log_basis;
    if (reverse_length >= 0) {
        if ((uint32_t)reverse_length > d || reverse_length == 0) { free(b); return NULL; }
        d = (uint32_t)reverse_length;
        drop = b->value_bits - d * log_basis;
    }
    b->decompose_length = d; b->drop_bits = drop;
    if (drop > 0) { b->has_init_carry = 1; b->init_carry_mask = 1ull << (drop - 1); }
    b->carry_mask = log_basis == 1 ? 2ull : ((1ull << log_basis) | (1ull << (log_basis - 1)));
    if (!b->modulus_is_pow2) {
        uint64_t value = 0;
        if (log_basis == 1) {
            if (drop != 0) {
                for (uint32_t i = 0; i < d; ++i) { value <<= 1; value |= 1; }
                value <<= 1; value |= 1;
                value <<= drop - 1;
                b->has_split = value < modulus;
                b->split = value;
            }
        } else {
            for (uint32_t i = 0; i < d; ++i) { value <<= log_basis; value |= b->basis_minus_one >> 1; }
            if (drop > 0) { value <<= 1; value |= 1; value <<= drop - 1; }
            else value += 1;
            b->has_split = value < modulus;
            b->split = value;
        }
        b->next_pow2_sub_q = (~0ull >> (64 - b->value_bits)) - (modulus - 1);
    }
    b->scalars = malloc(d * 8);
    b->mask = malloc(d * 8);
    b->shr = malloc(d * 4);
    for (uint32_t j = 0; j < d; ++j) {
        b->scalars[j] = (1ull << drop) << (j * log_basis);
        b->mask[j] = (b->basis_minus_one << drop) << (j * log_basis);
        b->shr[j] = drop + j * log_basis;
    }
    return b;
}

void orc_approx_basis_delete(orc_approx_basis *b) {
    if (!b) return;
    free(b->scalars); free(b->mask); free(b->shr);
    free(b);
}

void orc_approx_basis_info(const orc_approx_basis *b, uint32_t *decompose_length,
                           uint32_t *drop_bits, uint32_t *value_bits, uint64_t *scalars) {
    if (decompose_length) *decompose_length = b->decompose_length;
    if (drop_bits) *drop_bits = b->drop_bits;
    if (value_bits) *value_bits = b->value_bits;
    if (scalars) memcpy(scalars, b->scalars, b->decompose_length * 8);
}

/* init_value_carry (primitive/basis.rs:226-240) + OnceSignedDecompose::decompose
 * (primitive/common.rs:98-112) for every digit */
void orc_approx_decompose(const orc_approx_basis *b, uint64_t value, uint64_t *digits) {
    uint64_t adj = value;
    if (b->has_split && value >= b->split) adj += b->next_pow2_sub_q;
    int carry = b->has_init_carry ? ((adj & b->init_carry_mask) != 0) : 0;
    for (uint32_t j = 0; j < b->decompose_length; ++j) {
        uint64_t temp = ((adj & b->mask[j]) >> b->shr[j]) + (uint64_t)carry;
        carry = (temp & b->carry_mask) != 0;
        if (carry) temp = temp > b->basis_minus_one ? 0 : temp + b->modulus_minus_basis;
        digits[j] = temp;
    }
}

/* ======================================================================
 * GLev MAC, external product, key switch
 * ====================================================================== */
/* the per-digit loop shared by add_dcrt_glev_mul_crt_poly_assign
 * (primus_lattice/src/glwe/dcrt.rs:170-247) and add_dcrt_glev_mul_big_uint_poly_assign
 * (:249-325): adjusted values -> unsigned digit -> wrapping lift -> NTT -> MAC */
static void glev_mac_from_adjusted(const orc_lattice_ctx *c, uint32_t k, uint64_t *acc,
                                   const uint64_t *glev, uint64_t *adj, uint8_t *carries) {
    const size_t n = c->n;
    const uint32_t L = c->L;
    const size_t poly = (size_t)L * n;
    const size_t glwe = (size_t)(k + 1) * poly;
    uint64_t *digits = malloc(n * 8);
    uint64_t *res = malloc(poly * 8);
    for (uint32_t j = 0; j < c->basis->decompose_length; ++j) {
        orc_gadget_unsigned_digit(c->basis, j, adj, digits, carries, n);
        orc_rns_wrapping_decompose_small(c->base, digits, res, n, c->basis->basis);
        for (uint32_t l = 0; l < L; ++l) orc_ntt_forward(c->tables[l], res + (size_t)l * n);
        /* add_dcrt_glwe_mul_dcrt_polynomial_assign (glwe/dcrt.rs:101-119) */
        for (uint32_t p = 0; p <= k; ++p)
            for (uint32_t l = 0; l < L; ++l)
                orc_add_mul_assign(acc + p * poly + (size_t)l * n, glev + (size_t)j * glwe + p * poly + (size_t)l * n,
                                   res + (size_t)l * n, n, c->tables[l]->q);
    }
    free(digits);
    free(res);
}

void orc_glev_mac_crt_poly(const orc_lattice_ctx *c, uint32_t k, uint64_t *acc,
                           const uint64_t *glev, const uint64_t *crt_poly) {
    const uint32_t W = c->base->W;
    uint64_t *adj = malloc(c->n * W * 8);
    uint8_t *carries = malloc(c->n);
    orc_rns_compose_multiple(c->base, crt_poly, adj, c->n);
    orc_gadget_init_carry(c->basis, adj, carries, c->n);
    glev_mac_from_adjusted(c, k, acc, glev, adj, carries);
    free(adj);
    free(carries);
}

void orc_glev_mac_big_uint_poly(const orc_lattice_ctx *c, uint32_t k, uint64_t *acc,
                                const uint64_t *glev, const uint64_t *big_poly) {
    const uint32_t W = c->base->W;
    uint64_t *adj = malloc(c->n * W * 8);
    uint8_t *carries = malloc(c->n);
    memcpy(adj, big_poly, c->n * W * 8);
    orc_gadget_init_carry(c->basis, adj, carries, c->n);
    glev_mac_from_adjusted(c, k, acc, glev, adj, carries);
    free(adj);
    free(carries);
}

/* CrtGlwe::mul_dcrt_ggsw_inplace (primus_lattice/src/glwe/crt.rs:202-229) */
void orc_external_product(const orc_lattice_ctx *c, uint32_t k, const uint64_t *glwe_in,
                          const uint64_t *ggsw, uint64_t *glwe_out) {
    const size_t poly = (size_t)c->L * c->n;
    const size_t glwe = (size_t)(k + 1) * poly;
    const size_t glev = (size_t)c->basis->decompose_length * glwe;
    memset(glwe_out, 0, glwe * 8);
    for (uint32_t i = 0; i <= k; ++i)
        orc_glev_mac_crt_poly(c, k, glwe_out, ggsw + i * glev, glwe_in + i * poly);
}

void orc_external_product_batch(const orc_lattice_ctx *c, uint32_t k, const uint64_t *glwe_in,
                                const uint64_t *ggsw, uint64_t *glwe_out, size_t batch,
                                int threads) {
    const size_t glwe = (size_t)(k + 1) * c->L * c->n;
    long long b;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static) if (threads > 1)
    for (b = 0; b < (long long)batch; ++b)
        orc_external_product(c, k, glwe_in + (size_t)b * glwe, ggsw, glwe_out + (size_t)b * glwe);
}

/* CrtGlweKeySwitchingKey::key_swithching_inplace (primus_fhe_core/src/key_switch.rs:79-128) */
void orc_key_switch(const orc_lattice_ctx *c, uint32_t k_in, uint32_t k_out, const uint64_t *key,
                    const uint64_t *c_in, uint64_t *c_out) {
    const size_t n = c->n;
    const uint32_t L = c->L, W = c->base->W;
    const size_t poly = (size_t)L * n;
    const size_t glwe_out = (size_t)(k_out + 1) * poly;
    const size_t glev = (size_t)c->basis->decompose_length * glwe_out;
    uint64_t *big = malloc(n * W * 8);
    memset(c_out, 0, glwe_out * 8);
    for (uint32_t i = 0; i < k_in; ++i) {
        orc_rns_compose_multiple(c->base, c_in + i * poly, big, n);
        orc_glev_mac_big_uint_poly(c, k_out, c_out, key + i * glev, big);
    }
    uint64_t *b = malloc(poly * 8);
    memcpy(b, c_in + (size_t)k_in * poly, poly * 8);
    for (uint32_t l = 0; l < L; ++l) orc_ntt_forward(c->tables[l], b + (size_t)l * n);
    for (uint32_t p = 0; p <= k_out; ++p)
        for (uint32_t l = 0; l < L; ++l) orc_neg_assign(c_out + p * poly + (size_t)l * n, n, c->tables[l]->q);
    for (uint32_t l = 0; l < L; ++l)
        orc_add_assign(c_out + (size_t)k_out * poly + (size_t)l * n, b + (size_t)l * n, n, c->tables[l]->q);
    free(big);
    free(b);
}

/* ======================================================================
 * Encryption / decryption (test input construction and result checks)
 * ====================================================================== */
/* sample_crt_ternary_values_inplace (primus_distr/src/common.rs:163-215):
 * two bits per coefficient, 0|1 -> 0, 2 -> 1, 3 -> -1 (= q_i - 1) */
void orc_sample_ternary(uint64_t seed, uint64_t stream, const uint64_t *moduli, uint32_t L,
                        size_t n, uint64_t *out) {
    for (size_t x = 0; x < n; ++x) {
        uint64_t r = (orc_hash64(seed, stream, x / 16, 0) >> (2 * (x % 16))) & 3;
        for (uint32_t l = 0; l < L; ++l)
            out[(size_t)l * n + x] = r <= 1 ? 0 : (r == 2 ? 1 : moduli[l] - 1);
    }
}

/* rounded Gaussian noise bounded by 24 sigma (common.rs:282); test inputs only */
void orc_sample_gaussian(uint64_t seed, uint64_t stream, double sigma, const uint64_t *moduli,
                         uint32_t L, size_t n, uint64_t *out) {
    const double bound = 24.0 * sigma;
    for (size_t x = 0; x < n; ++x) {
        double v;
        uint64_t attempt = 0;
        do {
            uint64_t h1 = orc_hash64(seed, stream, x, 2 * attempt);
            uint64_t h2 = orc_hash64(seed, stream, x, 2 * attempt + 1);
            double u1 = ((h1 >> 11) + 1.0) * (1.0 / 9007199254740993.0);
            double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
            v = sigma * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
            ++attempt;
        } while (fabs(v) > bound);
        long long e = llround(v);
        for (uint32_t l = 0; l < L; ++l)
            out[(size_t)l * n + x] = e >= 0 ? (uint64_t)e : moduli[l] - (uint64_t)(-e);
    }
}

/* DcrtGlweSecretKey::encrypt_inplace (secret_key/glwe.rs:386-424) and the
 * custom-delta variant (:639-681) */
void orc_glwe_encrypt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt,
                      const uint64_t *msg, const uint64_t *delta_res, uint64_t seed,
                      double sigma, uint64_t *ct) {
    const size_t n = c->n;
    const uint32_t L = c->L;
    const size_t poly = (size_t)L * n;
    uint64_t *b = ct + (size_t)k * poly;
    orc_sample_gaussian(seed, 1000, sigma, c->base->moduli, L, n, b);
    for (uint32_t l = 0; l < L; ++l) {
        if (msg) orc_add_mul_scalar_assign(b + (size_t)l * n, msg + (size_t)l * n, delta_res[l], n, c->tables[l]->q);
        orc_ntt_forward(c->tables[l], b + (size_t)l * n);
    }
    for (uint32_t i = 0; i < k; ++i) {
        uint64_t *a = ct + (size_t)i * poly;
        orc_fill_uniform_rns(seed, 2000 + 64 * i, c->base->moduli, L, n, a);
        for (uint32_t l = 0; l < L; ++l)
            orc_add_mul_assign(b + (size_t)l * n, a + (size_t)l * n, sk_ntt + i * poly + (size_t)l * n, n, c->tables[l]->q);
    }
}

/* GGSW of coeff*X^degree: row i, digit j adds coeff*g_j*X^degree to component i
 * of a fresh encryption of zero (public_key/glwe.rs:127-195 places the message
 * the same way; the secret-key form of the encryption is used here). */
void orc_ggsw_encrypt_monomial(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt,
                               const uint64_t *coeff_res, size_t degree, uint64_t seed,
                               double sigma, uint64_t *ggsw) {
    const size_t n = c->n;
    const uint32_t L = c->L, d = c->basis->decompose_length;
    const size_t poly = (size_t)L * n, glwe = (size_t)(k + 1) * poly, glev = (size_t)d * glwe;
    uint64_t *mono = malloc(n * 8);
    for (uint32_t i = 0; i <= k; ++i) {
        for (uint32_t j = 0; j < d; ++j) {
            uint64_t *ct = ggsw + i * glev + (size_t)j * glwe;
            orc_glwe_encrypt(c, k, sk_ntt, NULL, NULL, seed * 7919 + (uint64_t)i * 131 + j, sigma, ct);
            for (uint32_t l = 0; l < L; ++l) {
                uint64_t q = c->tables[l]->q;
                uint64_t m = orc_mulmod(coeff_res[l], c->basis->scalar_residues[(size_t)j * L + l], q);
                orc_ntt_monomial(c->tables[l], m, degree, mono);
                orc_add_assign(ct + i * poly + (size_t)l * n, mono, n, q);
            }
        }
    }
    free(mono);
}

/* CrtGlweKeySwitchingKey::new (key_switch.rs:27-73) via
 * encrypt_crt_msg_to_dcrt_glev_inplace (secret_key/glwe.rs:683-708) */
void orc_ksk_generate(const orc_lattice_ctx *c, uint32_t k_in, uint32_t k_out,
                      const uint64_t *sk_in_coeff, const uint64_t *sk_out_ntt, uint64_t seed,
                      double sigma, uint64_t *key) {
    const uint32_t L = c->L, d = c->basis->decompose_length;
    const size_t poly = (size_t)L * c->n, glwe = (size_t)(k_out + 1) * poly, glev = (size_t)d * glwe;
    for (uint32_t i = 0; i < k_in; ++i)
        for (uint32_t j = 0; j < d; ++j)
            orc_glwe_encrypt(c, k_out, sk_out_ntt, sk_in_coeff + i * poly, c->basis->scalar_residues + (size_t)j * L,
                             seed * 104729 + (uint64_t)i * 257 + j, sigma, key + i * glev + (size_t)j * glwe);
}

/* delta = round(Q / t) (parameter/glwe.rs:332-338), reduced mod each q_i */
void orc_bfv_delta(const orc_rns_base *base, uint64_t t, uint64_t *delta_res) {
    const uint32_t W = base->W;
    uint64_t delta[64];
    u128 rem = 0;
    for (uint32_t i = W; i-- > 0;) {
        u128 cur = (rem << 64) | base->product[i];
        delta[i] = (uint64_t)(cur / t);
        rem = cur % t;
    }
    if ((uint64_t)rem * 2 >= t) {
        uint64_t one[64] = {0};
        one[0] = 1;
        big_add_assign(delta, one, W);
    }
    orc_rns_decompose(base, delta, delta_res);
}

/* DcrtGlweSecretKey::decrypt_inplace (secret_key/glwe.rs:782-837) */
void orc_glwe_decrypt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt,
                      const uint64_t *ct, uint64_t t, uint64_t gamma, uint64_t *msg) {
    const size_t n = c->n;
    const uint32_t L = c->L;
    const size_t poly = (size_t)L * n;
    const orc_rns_base *bq = c->base;
    uint64_t *ph = calloc(poly, 8);
    /* phase = b - sum a_i s_i (phase_inplace :713-737) */
    for (uint32_t i = 0; i < k; ++i)
        for (uint32_t l = 0; l < L; ++l)
            orc_add_mul_assign(ph + (size_t)l * n, ct + i * poly + (size_t)l * n, sk_ntt + i * poly + (size_t)l * n, n,
                               c->tables[l]->q);
    for (uint32_t l = 0; l < L; ++l) {
        uint64_t q = c->tables[l]->q;
        const uint64_t *b = ct + (size_t)k * poly + (size_t)l * n;
        uint64_t *p = ph + (size_t)l * n;
        for (size_t x = 0; x < n; ++x) p[x] = b[x] >= p[x] ? b[x] - p[x] : b[x] + q - p[x];
        orc_ntt_inverse(c->tables[l], p);
    }
    /* parameters (parameter/glwe.rs:340-356) */
    uint64_t tg[2] = {t, gamma};
    orc_rns_base *btg = orc_rns_base_new(tg, 2);
    uint64_t q_mod_tg[2] = {big_mod_value(bq->product, bq->W, t), big_mod_value(bq->product, bq->W, gamma)};
    uint64_t minus_inv_q[2];
    for (int i = 0; i < 2; ++i) {
        uint64_t inv = orc_invmod(q_mod_tg[i], tg[i]);
        minus_inv_q[i] = inv == 0 ? 0 : tg[i] - inv;
    }
    uint64_t inv_gamma_t = orc_invmod(gamma % t, t);
    uint64_t inv_gamma_t_q = orc_shoup_quotient(inv_gamma_t, t);
    uint64_t tgv[2];
    {
        u128 prod = (u128)t * gamma;
        tgv[0] = (uint64_t)prod;
        tgv[1] = (uint64_t)(prod >> 64);
    }
    for (uint32_t l = 0; l < L; ++l) {
        uint64_t q = c->tables[l]->q;
        uint64_t tg_mod_q = (uint64_t)((((u128)tgv[1] << 64) | tgv[0]) % q);
        orc_mul_scalar_assign(ph + (size_t)l * n, tg_mod_q, n, q);
    }
    orc_base_converter *conv = orc_base_converter_new(bq, btg);
    uint64_t *y = malloc(2 * n * 8);
    orc_fast_convert_array(conv, ph, y, n);
    orc_mul_scalar_assign(y, minus_inv_q[0], n, t);
    orc_mul_scalar_assign(y + n, minus_inv_q[1], n, gamma);
    for (size_t x = 0; x < n; ++x) {
        uint64_t temp = gamma - y[n + x] + y[x];
        if (temp >= gamma) temp -= gamma;
        msg[x] = orc_shoup_mul(inv_gamma_t, inv_gamma_t_q, temp, t);
    }
    free(y);
    orc_base_converter_delete(conv);
    orc_rns_base_delete(btg);
    free(ph);
}

/* ======================================================================
 * Hybrid RNS key switch with special primes (definition in the header)
 * ====================================================================== */
struct orc_hybrid_ks {
    uint32_t L, K, alpha, dnum, log_n;
    size_t n;
    uint64_t *moduli;            /* [L+K] */
    orc_ntt_table **tables;      /* [L+K] */
    orc_rns_base **gin, **gout;  /* per group: D_g, and the other QP limbs */
    orc_base_converter **gconv;  /* per group: D_g -> others */
    uint32_t **gout_limbs;       /* per group: limb index of each output row */
    orc_rns_base *bp, *bq;
    orc_base_converter *pq;      /* P -> Q */
    uint64_t *p_inv;             /* [L] P^-1 mod q_l */
};

static uint32_t hyb_group_lo(const orc_hybrid_ks *h, uint32_t g) { return g * h->alpha; }
static uint32_t hyb_group_hi(const orc_hybrid_ks *h, uint32_t g) {
    uint32_t e = (g + 1) * h->alpha;
    return e < h->L ? e : h->L;
}

void orc_hybrid_ks_delete(orc_hybrid_ks *h) {
    if (!h) return;
    for (uint32_t l = 0; h->tables && l < h->L + h->K; ++l) orc_ntt_table_delete(h->tables[l]);
    for (uint32_t g = 0; g < h->dnum; ++g) {
        if (h->gconv) orc_base_converter_delete(h->gconv[g]);
        if (h->gin) orc_rns_base_delete(h->gin[g]);
        if (h->gout) orc_rns_base_delete(h->gout[g]);
        if (h->gout_limbs) free(h->gout_limbs[g]);
    }
    free(h->tables);
    free(h->gconv);
    free(h->gin);
    free(h->gout);
    free(h->gout_limbs);
    if (h->pq) orc_base_converter_delete(h->pq);
    if (h->bp) orc_rns_base_delete(h->bp);
    if (h->bq) orc_rns_base_delete(h->bq);
    free(h->moduli);
    free(h->p_inv);
    free(h);
}

orc_hybrid_ks *orc_hybrid_ks_new(uint32_t log_n, const uint64_t *moduli, uint32_t L, uint32_t K,
                                 uint32_t alpha) {
    if (L == 0 || K == 0 || alpha == 0 || alpha > L) return NULL;
    orc_hybrid_ks *h = calloc(1, sizeof *h);
    h->L = L;
    h->K = K;
    h->alpha = alpha;
    h->dnum = (L + alpha - 1) / alpha;
    h->log_n = log_n;
    h->n = (size_t)1 << log_n;
    const uint32_t LK = L + K;
    h->moduli = malloc(LK * 8);
    memcpy(h->moduli, moduli, LK * 8);
    h->tables = calloc(LK, sizeof *h->tables);
    for (uint32_t l = 0; l < LK; ++l)
        if (!(h->tables[l] = orc_ntt_table_new(log_n, moduli[l]))) goto fail;
    h->gin = calloc(h->dnum, sizeof *h->gin);
    h->gout = calloc(h->dnum, sizeof *h->gout);
    h->gconv = calloc(h->dnum, sizeof *h->gconv);
    h->gout_limbs = calloc(h->dnum, sizeof *h->gout_limbs);
    uint64_t *tmp = malloc(LK * 8);
    for (uint32_t g = 0; g < h->dnum; ++g) {
        const uint32_t lo = hyb_group_lo(h, g), hi = hyb_group_hi(h, g);
        h->gin[g] = orc_rns_base_new(moduli + lo, hi - lo);
        uint32_t m = 0;
        h->gout_limbs[g] = malloc(LK * sizeof(uint32_t));
        for (uint32_t l = 0; l < LK; ++l)
            if (l < lo || l >= hi) {
                h->gout_limbs[g][m] = l;
                tmp[m++] = moduli[l];
            }
        h->gout[g] = orc_rns_base_new(tmp, m);
        if (!h->gin[g] || !h->gout[g]) {
            free(tmp);
            goto fail;
        }
        h->gconv[g] = orc_base_converter_new(h->gin[g], h->gout[g]);
    }
    free(tmp);
    h->bq = orc_rns_base_new(moduli, L);
    h->bp = orc_rns_base_new(moduli + L, K);
    if (!h->bq || !h->bp) goto fail;
    h->pq = orc_base_converter_new(h->bp, h->bq);
    h->p_inv = malloc(L * 8);
    for (uint32_t l = 0; l < L; ++l) {
        uint64_t pm = 1;
        for (uint32_t k = 0; k < K; ++k) pm = orc_mulmod(pm, moduli[L + k] % moduli[l], moduli[l]);
        h->p_inv[l] = orc_invmod(pm, moduli[l]);
        if (h->p_inv[l] == 0) goto fail;
    }
    return h;
fail:
    orc_hybrid_ks_delete(h);
    return NULL;
}

uint32_t orc_hybrid_ks_dnum(const orc_hybrid_ks *h) { return h->dnum; }

/* P * (Q/Q_g) * ((Q/Q_g)^-1 mod Q_g) mod r: [P]_{q_l} on the limbs of D_g, 0 elsewhere */
void orc_hybrid_ks_factor(const orc_hybrid_ks *h, uint32_t g, uint64_t *fac) {
    const uint32_t lo = hyb_group_lo(h, g), hi = hyb_group_hi(h, g);
    for (uint32_t l = 0; l < h->L + h->K; ++l) {
        fac[l] = 0;
        if (l >= lo && l < hi) {
            uint64_t pm = 1;
            for (uint32_t k = 0; k < h->K; ++k) pm = orc_mulmod(pm, h->moduli[h->L + k] % h->moduli[l], h->moduli[l]);
            fac[l] = pm;
        }
    }
}

void orc_hybrid_key_switch(const orc_hybrid_ks *h, uint32_t k_in, uint32_t k_out, const uint64_t *key,
                           const uint64_t *c_in, uint64_t *c_out) {
    const size_t n = h->n;
    const uint32_t L = h->L, K = h->K, LK = L + K, KO = k_out + 1;
    const size_t pq = (size_t)L * n, pqp = (size_t)LK * n;
    uint64_t *acc = calloc((size_t)KO * pqp, 8);
    uint64_t *ext = malloc(pqp * 8);
    uint64_t *conv = malloc(pqp * 8);
    for (uint32_t i = 0; i < k_in; ++i) {
        const uint64_t *a = c_in + (size_t)i * pq;
        for (uint32_t g = 0; g < h->dnum; ++g) {
            const uint32_t lo = hyb_group_lo(h, g), hi = hyb_group_hi(h, g);
            /* ModUp: D_g residues kept, the other limbs by fast base conversion */
            memcpy(ext + (size_t)lo * n, a + (size_t)lo * n, (size_t)(hi - lo) * n * 8);
            orc_fast_convert_array(h->gconv[g], a + (size_t)lo * n, conv, n);
            for (uint32_t m = 0; m < h->gout[g]->L; ++m)
                memcpy(ext + (size_t)h->gout_limbs[g][m] * n, conv + (size_t)m * n, n * 8);
            for (uint32_t l = 0; l < LK; ++l) orc_ntt_forward(h->tables[l], ext + (size_t)l * n);
            const uint64_t *row = key + ((size_t)i * h->dnum + g) * KO * pqp;
            for (uint32_t c = 0; c < KO; ++c)
                for (uint32_t l = 0; l < LK; ++l)
                    orc_add_mul_assign(acc + (size_t)c * pqp + (size_t)l * n, ext + (size_t)l * n,
                                       row + (size_t)c * pqp + (size_t)l * n, n, h->moduli[l]);
        }
    }
    /* b of the input, in the NTT domain */
    uint64_t *bt = malloc(pq * 8);
    memcpy(bt, c_in + (size_t)k_in * pq, pq * 8);
    for (uint32_t l = 0; l < L; ++l) orc_ntt_forward(h->tables[l], bt + (size_t)l * n);
    for (uint32_t c = 0; c < KO; ++c) {
        uint64_t *ac = acc + (size_t)c * pqp;
        /* ModDown: P limbs to coefficients, fast-convert to Q, back to NTT */
        for (uint32_t k = 0; k < K; ++k) orc_ntt_inverse(h->tables[L + k], ac + (size_t)(L + k) * n);
        orc_fast_convert_array(h->pq, ac + (size_t)L * n, conv, n);
        for (uint32_t l = 0; l < L; ++l) {
            const uint64_t q = h->moduli[l];
            uint64_t *cv = conv + (size_t)l * n;
            orc_ntt_forward(h->tables[l], cv);
            uint64_t *o = c_out + (size_t)c * pq + (size_t)l * n;
            memcpy(o, ac + (size_t)l * n, n * 8);
            orc_sub_assign(o, cv, n, q);
            orc_mul_scalar_assign(o, h->p_inv[l], n, q);
            orc_neg_assign(o, n, q);
            if (c == k_out) orc_add_assign(o, bt + (size_t)l * n, n, q);
        }
    }
    free(bt);
    free(acc);
    free(ext);
    free(conv);
}

/* ======================================================================
 * NTT-domain automorphism (primus_fhe_core/src/automorphism/glwe/dcrt.rs)
 * ====================================================================== */
/* generate_ntt_permutation (:43-63): natural index i holds the evaluation at
 * psi^(2i+1); sigma_k moves it to psi^(k(2i+1) mod 2N), index (j-1)/2; both in
 * bit-reversed storage */
void orc_ntt_auto_perm(uint32_t log_n, uint64_t degree, uint32_t *perm) {
    const uint64_t n = 1ull << log_n, mask = 2 * n - 1;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t j = (degree * (2 * i + 1)) & mask;
        const uint64_t target = (j - 1) / 2;
        perm[rev_bits((uint32_t)i, log_n)] = rev_bits((uint32_t)target, log_n);
    }
}

/* automorphism_inplace (:269-331): for each a_i: permute, inverse NTT, GLev MAC
 * into the result; then result = (-a', sigma(b) - b') */
void orc_glwe_automorphism(const orc_lattice_ctx *c, uint32_t k, uint64_t degree, const uint64_t *key,
                           const uint64_t *ct_in, uint64_t *ct_out) {
    const size_t n = c->n;
    const uint32_t L = c->L, log_n = (uint32_t)__builtin_ctzll(n);
    const size_t poly = (size_t)L * n;
    const size_t glev = (size_t)c->basis->decompose_length * (k + 1) * poly;
    uint32_t *perm = malloc(n * sizeof(uint32_t));
    orc_ntt_auto_perm(log_n, degree, perm);
    uint64_t *tmp = malloc(poly * 8);
    memset(ct_out, 0, (size_t)(k + 1) * poly * 8);
    for (uint32_t i = 0; i < k; ++i) {
        const uint64_t *a = ct_in + (size_t)i * poly;
        for (uint32_t l = 0; l < L; ++l)
            for (size_t d = 0; d < n; ++d) tmp[(size_t)l * n + d] = a[(size_t)l * n + perm[d]];
        for (uint32_t l = 0; l < L; ++l) orc_ntt_inverse(c->tables[l], tmp + (size_t)l * n);
        orc_glev_mac_crt_poly(c, k, ct_out, key + (size_t)i * glev, tmp);
    }
    const uint64_t *b = ct_in + (size_t)k * poly;
    for (uint32_t l = 0; l < L; ++l)
        for (size_t d = 0; d < n; ++d) tmp[(size_t)l * n + d] = b[(size_t)l * n + perm[d]];
    for (uint32_t i = 0; i < k; ++i)
        for (uint32_t l = 0; l < L; ++l) orc_neg_assign(ct_out + (size_t)i * poly + (size_t)l * n, n, c->tables[l]->q);
    /* sub_to_right: b_out = sigma(b) - b_out */
    for (uint32_t l = 0; l < L; ++l) {
        const uint64_t q = c->tables[l]->q;
        uint64_t *bo = ct_out + (size_t)k * poly + (size_t)l * n;
        const uint64_t *sb = tmp + (size_t)l * n;
        for (size_t x = 0; x < n; ++x) bo[x] = sb[x] >= bo[x] ? sb[x] - bo[x] : sb[x] + q - bo[x];
    }
    free(tmp);
    free(perm);
}

/* DcrtGlweTraceKey::trace_inplace (primus_fhe_core/src/trace/glwe/dcrt.rs:84-108):
 * result = ct; for each key: result += sigma(result), degrees N+1, N/2+1, .., 3
 * (keys built at :66-71).  DcrtGlweRevTraceKey::trace_inplace
 * (trace/glwe/rev.rs:79-115): degrees 3, 5, .., N+1 (:41-45), and before each
 * automorphism the ciphertext is multiplied by 2^-1 = (q+1)/2 mod q (:47-53, :101-107). */
void orc_glwe_trace(const orc_lattice_ctx *c, uint32_t k, const uint64_t *keys, int reverse,
                    const uint64_t *ct_in, uint64_t *ct_out) {
    const size_t n = c->n;
    const uint32_t L = c->L, log_n = (uint32_t)__builtin_ctzll(n);
    const size_t poly = (size_t)L * n, glwe = (size_t)(k + 1) * poly;
    const size_t key_len = (size_t)k * c->basis->decompose_length * glwe;
    uint64_t *tmp = malloc(glwe * 8);
    memmove(ct_out, ct_in, glwe * 8);
    for (uint32_t r = 0; r < log_n; ++r) {
        const uint64_t degree = reverse ? ((uint64_t)2 << r) + 1 : (uint64_t)(n >> r) + 1;
        if (reverse)
            for (uint32_t i = 0; i <= k; ++i)
                for (uint32_t l = 0; l < L; ++l) {
                    const uint64_t q = c->tables[l]->q, h = (q + 1) >> 1;
                    orc_mul_factor_assign(ct_out + (size_t)i * poly + (size_t)l * n, h, orc_shoup_quotient(h, q),
                                          n, q);
                }
        orc_glwe_automorphism(c, k, degree, keys + (size_t)r * key_len, ct_out, tmp);
        for (uint32_t i = 0; i <= k; ++i)
            for (uint32_t l = 0; l < L; ++l)
                orc_add_assign(ct_out + (size_t)i * poly + (size_t)l * n, tmp + (size_t)i * poly + (size_t)l * n,
                               n, c->tables[l]->q);
    }
    free(tmp);
}

/* DcrtGlweExpandCoeffKey::expand_partial_coefficients_inplace
 * (primus_fhe_core/src/expand_coeff/glwe/dcrt.rs:235-287): result[0] = ct *
 * count^-1 mod q_l (inv_count_residues, :209-232), then level i = 0 ..
 * log2(count)-1 with the key of degree N/2^i + 1 and the Shoup factor
 * NTT(X^(2N - 2^i)) (precompute_monomial_factors, :181-207): for j < 2^i,
 * (result[j], result[j + 2^i]) = (a + sigma(a), (a - sigma(a)) * factor), a = result[j]. */
void orc_glwe_expand(const orc_lattice_ctx *c, uint32_t k, const uint64_t *keys, size_t count,
                     const uint64_t *ct_in, uint64_t *out) {
    const size_t n = c->n;
    const uint32_t L = c->L;
    const size_t poly = (size_t)L * n, glwe = (size_t)(k + 1) * poly;
    const size_t key_len = (size_t)k * c->basis->decompose_length * glwe;
    const uint32_t log_d = (uint32_t)__builtin_ctzll(count);
    memmove(out, ct_in, glwe * 8);
    for (uint32_t l = 0; l < L; ++l) {
        const uint64_t q = c->tables[l]->q, inv = orc_invmod(count % q, q), invq = orc_shoup_quotient(inv, q);
        for (uint32_t i = 0; i <= k; ++i) orc_mul_factor_assign(out + (size_t)i * poly + (size_t)l * n, inv, invq, n, q);
    }
    uint64_t *tmp = malloc(glwe * 8), *w = malloc(poly * 8), *wq = malloc(poly * 8);
    for (uint32_t lev = 0; lev < log_d; ++lev) {
        const size_t half = (size_t)1 << lev;
        for (uint32_t l = 0; l < L; ++l) {
            orc_ntt_coeff_one_monomial(c->tables[l], 2 * n - half, w + (size_t)l * n);
            for (size_t x = 0; x < n; ++x) wq[(size_t)l * n + x] = orc_shoup_quotient(w[(size_t)l * n + x], c->tables[l]->q);
        }
        const uint64_t degree = (uint64_t)(n >> lev) + 1;
        for (size_t j = 0; j < half; ++j) {
            uint64_t *a = out + j * glwe, *b = out + (j + half) * glwe;
            orc_glwe_automorphism(c, k, degree, keys + (size_t)lev * key_len, a, tmp);
            for (uint32_t i = 0; i <= k; ++i)
                for (uint32_t l = 0; l < L; ++l) {
                    const size_t o = (size_t)i * poly + (size_t)l * n;
                    orc_butterfly_mul_factor(a + o, tmp + o, w + (size_t)l * n, wq + (size_t)l * n, b + o, n,
                                             c->tables[l]->q);
                }
        }
    }
    free(tmp);
    free(w);
    free(wq);
}

/* ======================================================================
 * Encryption with the CDT Gaussian sampler (reproducible on the device)
 * ====================================================================== */
uint32_t orc_cdt_table(double sigma, uint64_t *cdt, uint32_t cap) {
    const uint32_t B = (uint32_t)ceil(24.0 * sigma);
    if (B + 1 > cap) return 0;
    double total = 0;
    for (int64_t m = -(int64_t)B; m <= (int64_t)B; ++m) total += exp(-(double)(m * m) / (2.0 * sigma * sigma));
    double acc = 0;
    for (uint32_t m = 0; m <= B; ++m) {
        const double rho = exp(-(double)m * m / (2.0 * sigma * sigma));
        acc += (m == 0 ? rho : 2.0 * rho) / total;
        double v = acc * 9223372036854775808.0; /* 2^63 */
        cdt[m] = v >= 9223372036854775808.0 ? (1ull << 63) : (uint64_t)v;
    }
    cdt[B] = 1ull << 63;
    return B + 1;
}

int64_t orc_cdt_sample(const uint64_t *cdt, uint32_t entries, uint64_t seed, uint64_t stream, uint64_t x) {
    const uint64_t u = orc_hash64(seed, stream, x, 0);
    const uint64_t v = u >> 1;
    uint32_t lo = 0, hi = entries - 1; /* least m with v < cdt[m]; cdt[entries-1] = 2^63 > v */
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (v < cdt[mid]) hi = mid; else lo = mid + 1;
    }
    return (lo > 0 && (u & 1)) ? -(int64_t)lo : (int64_t)lo;
}

void orc_glwe_encrypt_cdt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt, const uint64_t *msg,
                          const uint64_t *scale, double sigma, uint64_t seed, uint64_t stream0, uint64_t index,
                          uint64_t *ct) {
    const size_t n = c->n;
    const uint32_t L = c->L;
    const size_t poly = (size_t)L * n;
    uint64_t cdt[512];
    const uint32_t entries = orc_cdt_table(sigma, cdt, 512);
    uint64_t *b = ct + (size_t)k * poly;
    for (size_t x = 0; x < n; ++x) {
        const int64_t e = orc_cdt_sample(cdt, entries, seed, stream0 + (1ull << 32) + index, x);
        for (uint32_t l = 0; l < L; ++l) {
            const uint64_t q = c->tables[l]->q;
            b[(size_t)l * n + x] = e >= 0 ? (uint64_t)e % q : q - (uint64_t)(-e) % q;
        }
    }
    for (uint32_t l = 0; l < L; ++l) {
        if (msg) orc_add_mul_scalar_assign(b + (size_t)l * n, msg + (size_t)l * n, scale[l], n, c->tables[l]->q);
        orc_ntt_forward(c->tables[l], b + (size_t)l * n);
    }
    for (uint32_t i = 0; i < k; ++i) {
        uint64_t *a = ct + (size_t)i * poly;
        for (uint32_t l = 0; l < L; ++l)
            orc_fill_uniform(seed, stream0 + (index * k + i) * L + l, c->tables[l]->q, n, a + (size_t)l * n);
        for (uint32_t l = 0; l < L; ++l)
            orc_add_mul_assign(b + (size_t)l * n, a + (size_t)l * n, sk_ntt + i * poly + (size_t)l * n, n,
                               c->tables[l]->q);
    }
}

/* one public-key encryption: DcrtGlwePublicKey::encrypt
 * (primus_fhe_core/src/public_key/glwe.rs:74-126) with the counter-based
 * samplers: v ternary (stream stream0 + 2^33 + index), e_c discrete Gaussian
 * (stream stream0 + 2^32 + index (k+1) + c); ct_c = NTT(e_c + [c == mc] m_c) + v pk_c.
 * The message enters component mc: a scaled polynomial (GLWE, mc = k) or one
 * coefficient coeff_l * g_l at `degree` (a GGSW row, :128-193). */
static void pk_encrypt_one(const orc_lattice_ctx *c, uint32_t k, const uint64_t *pk, const uint64_t *cdt,
                           uint32_t entries, uint64_t seed, uint64_t stream0, uint64_t index, uint32_t mc,
                           const uint64_t *msg, const uint64_t *scale, const uint64_t *mono_coeff,
                           const uint64_t *mono_scalar, size_t degree, uint64_t *ct) {
    const size_t n = c->n;
    const uint32_t L = c->L;
    const size_t poly = (size_t)L * n;
    uint64_t *v = malloc(poly * 8), *moduli = malloc((size_t)L * 8);
    for (uint32_t l = 0; l < L; ++l) moduli[l] = c->tables[l]->q;
    orc_sample_ternary(seed, stream0 + (1ull << 33) + index, moduli, L, n, v);
    for (uint32_t l = 0; l < L; ++l) orc_ntt_forward(c->tables[l], v + (size_t)l * n);
    for (uint32_t comp = 0; comp <= k; ++comp) {
        uint64_t *e = ct + (size_t)comp * poly;
        for (size_t x = 0; x < n; ++x) {
            const int64_t g = orc_cdt_sample(cdt, entries, seed, stream0 + (1ull << 32) + index * (k + 1) + comp, x);
            for (uint32_t l = 0; l < L; ++l) {
                const uint64_t q = moduli[l];
                e[(size_t)l * n + x] = g >= 0 ? (uint64_t)g % q : q - (uint64_t)(-g) % q;
            }
        }
        for (uint32_t l = 0; l < L; ++l) {
            const uint64_t q = moduli[l];
            if (comp == mc && msg) orc_add_mul_scalar_assign(e + (size_t)l * n, msg + (size_t)l * n, scale[l], n, q);
            if (comp == mc && mono_coeff) {
                uint64_t ratio[2];
                orc_barrett_ratio(q, ratio);
                e[(size_t)l * n + degree] =
                    orc_barrett_reduce_mul_add(mono_coeff[l], mono_scalar[l], e[(size_t)l * n + degree], q, ratio);
            }
            orc_ntt_forward(c->tables[l], e + (size_t)l * n);
            orc_add_mul_assign(e + (size_t)l * n, v + (size_t)l * n, pk + (size_t)comp * poly + (size_t)l * n, n, q);
        }
    }
    free(v);
    free(moduli);
}

void orc_glwe_pk_encrypt_cdt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *pk, const uint64_t *msg,
                             const uint64_t *scale, double sigma, uint64_t seed, uint64_t stream0, uint64_t index,
                             uint64_t *ct) {
    uint64_t cdt[512];
    const uint32_t entries = orc_cdt_table(sigma, cdt, 512);
    pk_encrypt_one(c, k, pk, cdt, entries, seed, stream0, index, k, msg, scale, NULL, NULL, 0, ct);
}

/* DcrtGlwePublicKey::encrypt_monomial_ggsw_inplace (public_key/glwe.rs:214-263):
 * row r = i d + j (GLev i = 0..k, digit j) is a public-key encryption whose
 * component i carries coeff_l * g_{j,l} at `degree` (:128-193). */
void orc_ggsw_pk_encrypt_monomial(const orc_lattice_ctx *c, uint32_t k, const uint64_t *pk,
                                  const uint64_t *coeff_res, size_t degree, double sigma, uint64_t seed,
                                  uint64_t stream0, uint64_t *ggsw) {
    uint64_t cdt[512];
    const uint32_t entries = orc_cdt_table(sigma, cdt, 512);
    const uint32_t d = c->basis->decompose_length, L = c->L;
    const size_t glwe = (size_t)(k + 1) * L * c->n;
    const uint64_t *g = c->basis->scalar_residues; /* [d][L] */
    for (uint32_t i = 0; i <= k; ++i)
        for (uint32_t j = 0; j < d; ++j) {
            const uint64_t r = (uint64_t)i * d + j;
            pk_encrypt_one(c, k, pk, cdt, entries, seed, stream0, r, i, NULL, NULL, coeff_res, g + (size_t)j * L,
                           degree, ggsw + r * glwe);
        }
}
