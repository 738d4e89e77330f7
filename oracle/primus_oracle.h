/*
 * primus_oracle.h -- CPU restatement of the primus lattice-arithmetic path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: tests/, the smoke
 * check and bench.py's CPU-baseline / reference arm may load it; the product
 * library (primus_b200/libprimus_gpu.so) never links, loads or calls it.
 *
 * Every function restates one reference function (Rust crate path:line in the
 * comment above its definition in primus_oracle.c).  The reference is a Rust
 * workspace that is not compiled or run next to this library, so the
 * restatement is pinned by the reference's own known-answer tests and
 * property tests (tests/test_oracle_pins.py) rather than by running it.
 *
 * All values are uint64_t.  Polynomials are limb-major [L][N]; BigUint values
 * are little-endian limbs, coefficient-major [N][W].
 */
#ifndef PRIMUS_ORACLE_H
#define PRIMUS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- seeded input generation (counter based, identical to the product's) */
uint64_t orc_hash64(uint64_t seed, uint64_t stream, uint64_t index, uint64_t attempt);
uint64_t orc_uniform_at(uint64_t seed, uint64_t stream, uint64_t index, uint64_t q);
void orc_fill_uniform(uint64_t seed, uint64_t stream, uint64_t q, size_t n, uint64_t *out);
/* fill [L][n] with limb l uniform below moduli[l], stream = stream0 + l */
void orc_fill_uniform_rns(uint64_t seed, uint64_t stream0, const uint64_t *moduli, uint32_t L,
                          size_t n, uint64_t *out);

/* ---- integer helpers */
uint64_t orc_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t orc_invmod(uint64_t a, uint64_t q); /* 0 if not invertible */
int orc_is_prime(uint64_t n);
/* largest prime p < bound with p = 1 mod m; 0 if none */
uint64_t orc_prev_prime_congruent(uint64_t bound, uint64_t m);
/* count descending primes < bound with p = 1 mod m */
int orc_ntt_primes(uint64_t bound, uint64_t m, uint32_t count, uint64_t *out);

/* ---- Shoup factor (primus_factor/src/shoup_factor/mod.rs) */
uint64_t orc_shoup_quotient(uint64_t w, uint64_t q);
uint64_t orc_shoup_lazy_mul(uint64_t w, uint64_t wq, uint64_t b, uint64_t q);
uint64_t orc_shoup_mul(uint64_t w, uint64_t wq, uint64_t b, uint64_t q);

/* ---- Barrett modulus (primus_modulus/src/barrett) */
void orc_barrett_ratio(uint64_t q, uint64_t ratio[2]);
uint64_t orc_barrett_lazy_reduce_2limb(uint64_t lo, uint64_t hi, uint64_t q, const uint64_t ratio[2]);
uint64_t orc_barrett_reduce_mul(uint64_t a, uint64_t b, uint64_t q, const uint64_t ratio[2]);
uint64_t orc_barrett_reduce_mul_add(uint64_t a, uint64_t b, uint64_t c, uint64_t q,
                                    const uint64_t ratio[2]);
uint64_t orc_barrett_dot_product(const uint64_t *a, const uint64_t *b, size_t n, uint64_t q);

/* ---- NTT table (primus_ntt/src/ntt/primitive.rs) */
typedef struct orc_ntt_table {
    uint64_t q;
    uint32_t log_n;
    size_t n;
    uint64_t root, inv_root;
    uint64_t inv_n, inv_n_q;
    uint64_t *root_powers, *root_powers_q;       /* [n] bit-reversed order */
    uint64_t *inv_root_powers, *inv_root_powers_q; /* [n] scrambled order */
    uint64_t *ordinal, *ordinal_q;               /* [2n] psi^0..psi^(2n-1) */
    uint32_t *rev;                               /* [n] */
} orc_ntt_table;

/* 0 ok; 1 no primitive root; 2 degree too large; 3 bad argument / alloc */
int orc_minimal_primitive_root(uint32_t log_degree, uint64_t q, uint64_t *root);
int orc_ntt_table_init(orc_ntt_table *t, uint32_t log_n, uint64_t q);
void orc_ntt_table_free(orc_ntt_table *t);
orc_ntt_table *orc_ntt_table_new(uint32_t log_n, uint64_t q); /* NULL on error */
void orc_ntt_table_delete(orc_ntt_table *t);
/* accessors for ctypes */
void orc_ntt_table_export(const orc_ntt_table *t, uint64_t *root, uint64_t *inv_root,
                          uint64_t *inv_n, uint64_t *inv_n_q, uint64_t *root_powers,
                          uint64_t *root_powers_q, uint64_t *inv_root_powers,
                          uint64_t *inv_root_powers_q, uint64_t *ordinal, uint64_t *ordinal_q);

void orc_ntt_lazy_forward(const orc_ntt_table *t, uint64_t *a);
void orc_ntt_forward(const orc_ntt_table *t, uint64_t *a);
void orc_ntt_lazy_inverse(const orc_ntt_table *t, uint64_t *a);
void orc_ntt_inverse(const orc_ntt_table *t, uint64_t *a);
void orc_ntt_monomial(const orc_ntt_table *t, uint64_t coeff, size_t degree, uint64_t *out);
void orc_ntt_coeff_one_monomial(const orc_ntt_table *t, size_t degree, uint64_t *out);
void orc_ntt_coeff_minus_one_monomial(const orc_ntt_table *t, size_t degree, uint64_t *out);
/* batched helpers: rows laid out back to back, OpenMP over rows when threads > 1 */
void orc_ntt_forward_rows(const orc_ntt_table *t, uint64_t *a, size_t rows, int lazy, int threads);
void orc_ntt_inverse_rows(const orc_ntt_table *t, uint64_t *a, size_t rows, int lazy, int threads);
/* definition check: out[i] = sum_j a_j psi^((2 rev(i)+1) j) */
void orc_ntt_by_definition(const orc_ntt_table *t, const uint64_t *a, uint64_t *out);

/* ---- DCRT (primus_ntt/src/dcrt/primitive.rs): tables[L], data [polys][L][n] */
void orc_dcrt_forward(orc_ntt_table *const *tables, uint32_t L, uint64_t *a, size_t polys,
                      int lazy, int threads);
void orc_dcrt_inverse(orc_ntt_table *const *tables, uint32_t L, uint64_t *a, size_t polys,
                      int lazy, int threads);
/* fused round trip used by the batched workload: fwd, x *= plain (NTT domain), inv */
void orc_dcrt_polymul_roundtrip(orc_ntt_table *const *tables, uint32_t L, uint64_t *a,
                                const uint64_t *plain, size_t polys, int threads);

/* ---- pointwise (primus_poly/src/dcrt/{mod.rs,mul.rs}), canonical in/out */
void orc_mul_assign(uint64_t *x, const uint64_t *y, size_t n, uint64_t q);
void orc_add_mul_assign(uint64_t *acc, const uint64_t *b, const uint64_t *c, size_t n, uint64_t q);
void orc_mul_scalar_assign(uint64_t *x, uint64_t s, size_t n, uint64_t q);
void orc_add_mul_scalar_assign(uint64_t *x, const uint64_t *y, uint64_t s, size_t n, uint64_t q);
void orc_mul_factor_assign(uint64_t *x, uint64_t w, uint64_t wq, size_t n, uint64_t q);
void orc_add_assign(uint64_t *x, const uint64_t *y, size_t n, uint64_t q);
void orc_sub_assign(uint64_t *x, const uint64_t *y, size_t n, uint64_t q);
void orc_neg_assign(uint64_t *x, size_t n, uint64_t q);
void orc_butterfly_mul_factor(uint64_t *a, const uint64_t *s, const uint64_t *w,
                              const uint64_t *wq, uint64_t *b, size_t n, uint64_t q);

/* ---- schoolbook negacyclic product (primus_poly/src/poly/mul.rs:111-142) */
void orc_naive_negacyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t *c, size_t n,
                              uint64_t q);

/* ---- RNS base (primus_rns/src/base.rs) */
typedef struct orc_rns_base {
    uint32_t L;
    uint32_t W; /* BigUint limbs of Q */
    uint64_t *moduli;
    uint64_t *product;            /* [W] */
    uint64_t *punctured;          /* [L][W] */
    uint64_t *inv_punctured;      /* [L] */
    uint64_t *inv_punctured_q;    /* [L] */
} orc_rns_base;
orc_rns_base *orc_rns_base_new(const uint64_t *moduli, uint32_t L); /* NULL if not coprime */
void orc_rns_base_delete(orc_rns_base *b);
uint32_t orc_rns_base_width(const orc_rns_base *b);
void orc_rns_base_export(const orc_rns_base *b, uint64_t *product, uint64_t *punctured,
                         uint64_t *inv_punctured);
void orc_rns_compose(const orc_rns_base *b, const uint64_t *residues, uint64_t *value);
void orc_rns_compose_multiple(const orc_rns_base *b, const uint64_t *multi_residues,
                              uint64_t *values, size_t count);
void orc_rns_decompose(const orc_rns_base *b, const uint64_t *value, uint64_t *residues);
void orc_rns_decompose_multiple(const orc_rns_base *b, const uint64_t *values,
                                uint64_t *multi_residues, size_t count);
void orc_rns_wrapping_decompose_small(const orc_rns_base *b, const uint64_t *small,
                                      uint64_t *multi_residues, size_t count,
                                      uint64_t small_modulus);

/* ---- fast base conversion (primus_rns/src/converter.rs) */
typedef struct orc_base_converter {
    const orc_rns_base *ibase, *obase;
    uint64_t *matrix; /* [Lout][Lin] */
} orc_base_converter;
orc_base_converter *orc_base_converter_new(const orc_rns_base *ibase, const orc_rns_base *obase);
void orc_base_converter_delete(orc_base_converter *c);
void orc_fast_convert_array(const orc_base_converter *c, const uint64_t *in, uint64_t *out,
                            size_t n);

/* ---- gadget decomposition (primus_decompose/src/big_integer) */
typedef struct orc_gadget_basis {
    uint32_t W, L;
    uint32_t log_basis;
    uint32_t decompose_length;
    uint32_t drop_bits;
    int has_init_carry;
    uint32_t init_carry_index;
    uint64_t init_carry_mask;
    uint64_t carry_mask;
    uint64_t basis, basis_minus_one;
    int has_split;
    uint64_t *split;           /* [W] */
    uint64_t *next_pow2_sub_q; /* [W] */
    uint64_t *modulus;         /* [W] */
    uint64_t *scalars;         /* [d][W] */
    uint64_t *scalar_residues; /* [d][L] */
    uint32_t *mask_index;      /* [d] */
    uint64_t *mask0, *mask1;   /* [d] */
    uint32_t *mask_shr, *mask_shl; /* [d] */
} orc_gadget_basis;
orc_gadget_basis *orc_gadget_basis_new(const orc_rns_base *base, uint32_t log_basis,
                                       int32_t reverse_length);
void orc_gadget_basis_delete(orc_gadget_basis *g);
void orc_gadget_basis_info(const orc_gadget_basis *g, uint32_t *decompose_length,
                           uint32_t *drop_bits, uint64_t *scalar_residues);
/* init_value_carry_slice_inplace */
void orc_gadget_init_carry(const orc_gadget_basis *g, uint64_t *values, uint8_t *carries,
                           size_t count);
/* one unsigned_decompose_slice_inplace for digit `level` */
void orc_gadget_unsigned_digit(const orc_gadget_basis *g, uint32_t level, const uint64_t *values,
                               uint64_t *digits, uint8_t *carries, size_t count);
/* all digits: values [count][W] untouched; digits out [d][count] (unsigned digits in [0,B)) */
void orc_gadget_decompose_all(const orc_gadget_basis *g, const uint64_t *values, uint64_t *digits,
                              size_t count);

/* single-word basis (primus_decompose/src/primitive) */
typedef struct orc_approx_basis {
    int has_modulus;
    uint64_t modulus;
    int modulus_is_pow2;
    uint64_t basis, basis_minus_one, modulus_minus_basis;
    uint32_t decompose_length, value_bits, log_basis, drop_bits;
    int has_init_carry;
    uint64_t init_carry_mask, carry_mask;
    int has_split;
    uint64_t split, next_pow2_sub_q;
    uint64_t *scalars;
    uint64_t *mask;
    uint32_t *shr;
} orc_approx_basis;
orc_approx_basis *orc_approx_basis_new(int has_modulus, uint64_t modulus, uint32_t log_basis,
                                       int32_t reverse_length);
void orc_approx_basis_delete(orc_approx_basis *b);
void orc_approx_basis_info(const orc_approx_basis *b, uint32_t *decompose_length,
                           uint32_t *drop_bits, uint32_t *value_bits, uint64_t *scalars);
/* init_value_carry then every signed digit: digits[d] (decompose: carry -> q - B + t or 0) */
void orc_approx_decompose(const orc_approx_basis *b, uint64_t value, uint64_t *digits);

/* ---- GLev MAC / external product / key switch (primus_lattice, primus_fhe_core)
 * k = GLWE dimension; a GLWE is (k+1) DCRT polys [k+1][L][N]; a GLev is d GLWEs;
 * a GGSW is (k+1) GLevs.  Tables are the L per-limb NTT tables.              */
typedef struct orc_lattice_ctx {
    orc_ntt_table **tables;
    uint32_t L;
    size_t n;
    const orc_rns_base *base;
    const orc_gadget_basis *basis;
} orc_lattice_ctx;
/* acc (NTT domain, [k+1][L][N]) += GLev (x) crt_poly (coefficient form [L][N]) */
void orc_glev_mac_crt_poly(const orc_lattice_ctx *c, uint32_t k, uint64_t *acc,
                           const uint64_t *glev, const uint64_t *crt_poly);
/* acc += GLev (x) BigUint poly ([N][W]) */
void orc_glev_mac_big_uint_poly(const orc_lattice_ctx *c, uint32_t k, uint64_t *acc,
                                const uint64_t *glev, const uint64_t *big_poly);
/* result (NTT domain) = GLWE (coefficient form) (x) GGSW */
void orc_external_product(const orc_lattice_ctx *c, uint32_t k, const uint64_t *glwe_in,
                          const uint64_t *ggsw, uint64_t *glwe_out);
void orc_external_product_batch(const orc_lattice_ctx *c, uint32_t k, const uint64_t *glwe_in,
                                const uint64_t *ggsw, uint64_t *glwe_out, size_t batch,
                                int threads);
/* key switch: key = k_in GLevs (each d x (k_out+1) x L x N); c_in coefficient form
 * [(k_in+1)][L][N]; c_out NTT domain [(k_out+1)][L][N] */
void orc_key_switch(const orc_lattice_ctx *c, uint32_t k_in, uint32_t k_out, const uint64_t *key,
                    const uint64_t *c_in, uint64_t *c_out);

/* ---- GLWE encryption / decryption used to build inputs and check results */
void orc_sample_ternary(uint64_t seed, uint64_t stream, const uint64_t *moduli, uint32_t L,
                        size_t n, uint64_t *out);
void orc_sample_gaussian(uint64_t seed, uint64_t stream, double sigma, const uint64_t *moduli,
                         uint32_t L, size_t n, uint64_t *out);
/* secret-key GLWE encryption of msg (coefficient form, [L][N]) scaled by delta_res [L]:
 * b = e + delta*msg + sum a_i s_i (all in NTT domain); sk_ntt [k][L][N] */
void orc_glwe_encrypt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt,
                      const uint64_t *msg, const uint64_t *delta_res, uint64_t seed,
                      double sigma, uint64_t *ct);
/* GGSW of the monomial coeff*X^degree under sk (secret-key form of
 * encrypt_monomial_ggsw, primus_fhe_core/src/public_key/glwe.rs:202-263) */
void orc_ggsw_encrypt_monomial(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt,
                               const uint64_t *coeff_res, size_t degree, uint64_t seed,
                               double sigma, uint64_t *ggsw);
/* GLev of s_in_i under sk_out (key switching key rows, key_switch.rs:27-73) */
void orc_ksk_generate(const orc_lattice_ctx *c, uint32_t k_in, uint32_t k_out,
                      const uint64_t *sk_in_coeff, const uint64_t *sk_out_ntt, uint64_t seed,
                      double sigma, uint64_t *key);
/* BFV decryption through fast base conversion (secret_key/glwe.rs:782-837) */
void orc_glwe_decrypt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt,
                      const uint64_t *ct, uint64_t t, uint64_t gamma, uint64_t *msg);
/* delta = round(Q/t) mod each q_i (parameter/glwe.rs:332-338) */
void orc_bfv_delta(const orc_rns_base *base, uint64_t t, uint64_t *delta_res);

/* ---- hybrid RNS key switch with special primes (no reference counterpart:
 * the reference's key switch is the BigUint gadget form above).  Definition:
 * moduli = Q (L primes) then P (K special primes); digit groups D_g are the
 * consecutive Q limbs [g*alpha, min(L, (g+1)*alpha)).  For each input a_i
 * (coefficient form over Q) and group g, ModUp fast-converts a_i's D_g residues
 * to every other limb of QP (fast_convert_array semantics), keeping D_g's own
 * residues; the extended poly is NTT'd limb by limb and multiply-accumulated
 * with key row [i][g] ([k_in][dnum][k_out+1][L+K][N], NTT domain; the row
 * encrypts P * (Q/Q_g) * ((Q/Q_g)^-1 mod Q_g) * s_in_i under s_out over QP).
 * ModDown of each accumulated poly: inverse NTT of its P limbs, fast
 * conversion P -> Q, NTT, then (acc_Q - conv) * P^-1 mod q_l.  The output is
 * c_out = -ModDown(sum) + (0, .., NTT(b)) over Q in the NTT domain, as the
 * BigUint key switch (key_switch.rs:96-127). */
typedef struct orc_hybrid_ks orc_hybrid_ks;
orc_hybrid_ks *orc_hybrid_ks_new(uint32_t log_n, const uint64_t *moduli, uint32_t L, uint32_t K,
                                 uint32_t alpha);
void orc_hybrid_ks_delete(orc_hybrid_ks *h);
uint32_t orc_hybrid_ks_dnum(const orc_hybrid_ks *h);
/* the key-row message factor of group g, as residues over QP ([L+K]) */
void orc_hybrid_ks_factor(const orc_hybrid_ks *h, uint32_t g, uint64_t *fac);
void orc_hybrid_key_switch(const orc_hybrid_ks *h, uint32_t k_in, uint32_t k_out, const uint64_t *key,
                           const uint64_t *c_in, uint64_t *c_out);

/* ---- NTT-domain automorphism x -> x^degree (primus_fhe_core/src/automorphism/glwe/dcrt.rs) */
/* generate_ntt_permutation (:43-63): out[d] = in[perm[d]] in bit-reversed storage */
void orc_ntt_auto_perm(uint32_t log_n, uint64_t degree, uint32_t *perm);
/* DcrtGlweAutoKey::automorphism_inplace (:269-331): ct_in, ct_out [k+1][L][N] NTT
 * domain; key = k GLevs [k][d][k+1][L][N] (GLev of sigma(s_i) under s) */
void orc_glwe_automorphism(const orc_lattice_ctx *c, uint32_t k, uint64_t degree, const uint64_t *key,
                           const uint64_t *ct_in, uint64_t *ct_out);
/* Field trace by log2(N) automorphisms: DcrtGlweTraceKey::trace_inplace
 * (primus_fhe_core/src/trace/glwe/dcrt.rs:84-108; degrees N+1, N/2+1, .., 3)
 * or, with reverse != 0, DcrtGlweRevTraceKey::trace_inplace (trace/glwe/rev.rs:79-115;
 * degrees 3, 5, .., N+1, each step halving first).  keys: log2(N) automorphism
 * keys in the order applied, each [k][d][k+1][L][N]. */
void orc_glwe_trace(const orc_lattice_ctx *c, uint32_t k, const uint64_t *keys, int reverse,
                    const uint64_t *ct_in, uint64_t *ct_out);
/* Coefficient expansion: DcrtGlweExpandCoeffKey::expand_partial_coefficients_inplace
 * (primus_fhe_core/src/expand_coeff/glwe/dcrt.rs:235-287).  keys as for the
 * forward trace (degrees N+1, N/2+1, ..; the first log2(count) are used);
 * out: [count][k+1][L][N]. */
void orc_glwe_expand(const orc_lattice_ctx *c, uint32_t k, const uint64_t *keys, size_t count,
                     const uint64_t *ct_in, uint64_t *out);

/* ---- encryption with the device-reproducible sampler (CDT Gaussian) ----
 * Discrete Gaussian over [-B, B], B = ceil(24 sigma) (the reference's bound,
 * primus_distr/src/common.rs:282): cdt[m] = floor(2^63 * P(|e| <= m)) for
 * m = 0..B (cdt[B] = 2^63); u = hash64(seed, stream, x, 0): |e| = the least m
 * with (u >> 1) < cdt[m], negative when m > 0 and u & 1.  Returns B + 1. */
uint32_t orc_cdt_table(double sigma, uint64_t *cdt, uint32_t cap);
int64_t orc_cdt_sample(const uint64_t *cdt, uint32_t entries, uint64_t seed, uint64_t stream, uint64_t x);
/* secret-key GLWE encryption (DcrtGlweSecretKey::encrypt_inplace, secret_key/glwe.rs:386-424)
 * of ciphertext `index` of a batch: a_i limb l uniform with stream
 * stream0 + (index k + i) L + l; e with stream stream0 + 2^32 + index;
 * b = NTT(e + scale_l msg) + sum a_i s_i (msg coefficient form [L][N] or NULL) */
void orc_glwe_encrypt_cdt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *sk_ntt, const uint64_t *msg,
                          const uint64_t *scale, double sigma, uint64_t seed, uint64_t stream0, uint64_t index,
                          uint64_t *ct);
/* public-key encryption (DcrtGlwePublicKey::encrypt, primus_fhe_core/src/public_key/glwe.rs:74-126)
 * of ciphertext `index`: v ternary (stream stream0 + 2^33 + index), e_c CDT
 * Gaussian (stream stream0 + 2^32 + index (k+1) + c), ct_c = NTT(e_c) + v pk_c,
 * the body with scale_l * msg added before its NTT.  pk: [k+1][L][N] NTT domain
 * (a secret-key encryption of zero, DcrtGlwePublicKey::new :33-71). */
void orc_glwe_pk_encrypt_cdt(const orc_lattice_ctx *c, uint32_t k, const uint64_t *pk, const uint64_t *msg,
                             const uint64_t *scale, double sigma, uint64_t seed, uint64_t stream0, uint64_t index,
                             uint64_t *ct);
/* DcrtGlwePublicKey::encrypt_monomial_ggsw_inplace (:214-263): GGSW [k+1][d][k+1][L][N]
 * of coeff * X^degree; row r = i d + j uses index r of the samplers above. */
void orc_ggsw_pk_encrypt_monomial(const orc_lattice_ctx *c, uint32_t k, const uint64_t *pk,
                                  const uint64_t *coeff_res, size_t degree, double sigma, uint64_t seed,
                                  uint64_t stream0, uint64_t *ggsw);

/* ---- HEXL-style AVX-512 IFMA52 transforms (hexl_ifma.c): the reference's fastest
 * CPU path, timed as the CPU baseline (q < 2^50, n >= 16, host with avx512ifma) */
typedef struct orc_hexl_table orc_hexl_table;
int orc_hexl_available(void);
orc_hexl_table *orc_hexl_table_new(const orc_ntt_table *t); /* NULL if q >= 2^50 or n < 16 */
void orc_hexl_table_delete(orc_hexl_table *h);
void orc_hexl_forward(const orc_hexl_table *h, uint64_t *a); /* canonical in and out */
void orc_hexl_inverse(const orc_hexl_table *h, uint64_t *a); /* [0, 2q) in, canonical out */
void orc_hexl_precon52(const uint64_t *y, uint64_t *yp, size_t n, uint64_t q);
void orc_hexl_polymul_roundtrip(orc_hexl_table *const *tables, uint32_t L, uint64_t *a, const uint64_t *plain,
                                const uint64_t *plain_p, size_t polys, int threads);

#ifdef __cplusplus
}
#endif
#endif
