/*
 * primus_gpu.h -- C ABI of libprimus_gpu.so, the B200 (sm_100a) backend for
 * the primus lattice-arithmetic path.
 *
 * The reference (serendipity-crypto/primus) is a Rust workspace with no FFI
 * layer: its boundary is a set of traits and inherent methods.  Each entry
 * point below names the reference item it replaces (crate/src/file.rs:line).
 * A Rust `primus_gpu` crate binds these symbols with `extern "C"` and
 * implements `NttTable` / `DcrtTable` on top of them.
 *
 * Conventions
 *  - Every function returns an int status (PG_OK == 0); none aborts.  The
 *    text of the last error on the calling thread is pg_last_error().
 *  - Handles are library owned; data buffers are caller owned.
 *  - `d_*` pointers are device pointers, `h_*` pointers host pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *  - Values are uint64_t.  A DCRT/CRT polynomial is limb-major [L][N]; a
 *    batch of P polynomials is [P][L][N].  BigUint values are little-endian
 *    limbs, coefficient-major [count][W].
 *  - Canonical outputs are in [0, q).  Lazy forward outputs are in [0, 4q)
 *    and equal the reference's lazy values bit for bit.
 *  - Calls on distinct streams with disjoint buffers may run concurrently;
 *    handles are immutable after creation and may be shared across threads.
 */
#ifndef PRIMUS_GPU_H
#define PRIMUS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum {
    PG_OK = 0,
    PG_ERR_INVALID_ARGUMENT = 1,
    PG_ERR_NO_PRIMITIVE_ROOT = 2,   /* NttError::NoPrimitiveRoot  (primus_ntt/src/error.rs:10-16) */
    PG_ERR_DEGREE_TOO_LARGE = 3,    /* NttError::DegreeTooLarge   (primus_ntt/src/error.rs:26-33) */
    PG_ERR_NOT_COPRIME = 4,         /* RNSError::CoPrimeError     (primus_rns/src/error.rs) */
    PG_ERR_UNSUPPORTED = 5,         /* a size this build does not run */
    PG_ERR_OUT_OF_MEMORY = 6,
    PG_ERR_CUDA = 7,
    PG_ERR_TIMEOUT = 8,             /* a bounded device wait ran out */
    PG_ERR_REJECTED = 9             /* admission control refused a request */
};

const char *pg_status_string(int status);
/* message of the last failing call on this thread ("" if none) */
const char *pg_last_error(void);
/* library version string and the compiled device architecture */
const char *pg_version(void);

/* ------------------------------------------------------- device utilities
 * Thin wrappers so that hosts without a CUDA runtime binding (the Rust crate,
 * ctypes) can manage buffers and streams. */
int pg_device_count(int *count);
int pg_set_device(int device);
int pg_malloc(void **d_ptr, size_t bytes);
int pg_free(void *d_ptr);
int pg_host_alloc(void **h_ptr, size_t bytes); /* page-locked */
int pg_host_free(void *h_ptr);
int pg_memcpy_h2d(void *d_dst, const void *h_src, size_t bytes, void *stream);
int pg_memcpy_d2h(void *h_dst, const void *d_src, size_t bytes, void *stream);
/* Wire / disk format of every container (GLWE, GLev, GGSW, keys, DCRT polys):
 * the little-endian u64 words back to back, the reference's bytemuck cast
 * (primus_lattice/src/macros/mod.rs:39-97 from_bytes_assign / to_bytes_inplace).
 * A byte count other than 8 x words is refused (the reference panics).  On
 * little-endian hosts the bytes are the words' memory image, so these are
 * checked synchronous copies into / out of a device buffer. */
int pg_from_bytes(uint64_t *d_dst, size_t words, const uint8_t *h_bytes, size_t nbytes);
int pg_to_bytes(const uint64_t *d_src, size_t words, uint8_t *h_bytes, size_t nbytes);
int pg_memcpy_d2d(void *d_dst, const void *d_src, size_t bytes, void *stream);
int pg_memset(void *d_ptr, int value, size_t bytes, void *stream);
int pg_stream_create(void **stream);
int pg_stream_destroy(void *stream);
int pg_stream_synchronize(void *stream);
int pg_device_synchronize(void);
/* CUDA-event timing on a stream */
int pg_event_create(void **event);
int pg_event_destroy(void *event);
int pg_event_record(void *event, void *stream);
int pg_event_elapsed_ms(void *start, void *stop, float *ms);
/* number of kernels this library has launched in this process */
uint64_t pg_launch_count(void);
/* Scratch that entry points allocate for themselves (when the caller passes no
 * workspace) comes from a per-device pool that keeps freed memory for reuse.
 * Trim the current device's pool to at most keep_bytes of unused memory.
 * No reference counterpart: the reference allocates scratch on the heap. */
int pg_scratch_trim(size_t keep_bytes);

/* --------------------------------------------------------- number theory
 * Host helpers used to pick NTT-friendly primes the way the workloads do. */
/* largest prime p < bound with p = 1 mod m (descending search, deterministic
 * Miller-Rabin); 0 if none */
uint64_t pg_prev_prime_congruent(uint64_t bound, uint64_t m);
/* `count` descending primes below bound, each = 1 mod m */
int pg_ntt_primes(uint64_t bound, uint64_t m, uint32_t count, uint64_t *h_out);
/* minimal primitive 2^log_degree-th root of unity mod q
 * (PrimitiveRoot::try_minimal_primitive_root, primus_ntt/src/root.rs:89-111) */
int pg_minimal_primitive_root(uint32_t log_degree, uint64_t q, uint64_t *root);

/* ------------------------------------------------------------- NTT tables
 * One table holds L primes of one ring degree N = 2^log_n; L = 1 is the
 * single-prime NttTable (primus_ntt/src/ntt/mod.rs:20-117), L > 1 the
 * DcrtTable (primus_ntt/src/dcrt/mod.rs:17-129).  Twiddles (value + Shoup
 * quotient), N^-1 and the monomial tables live in device memory until
 * destroy.  Replaces UintNttTable::new (primitive.rs:113-185) and
 * UintCrtNttTable::new (dcrt/primitive.rs:24-45). */
typedef struct pg_ntt_table pg_ntt_table;

int pg_ntt_table_create(uint32_t log_n, const uint64_t *h_moduli, uint32_t moduli_count,
                        pg_ntt_table **out);
int pg_ntt_table_destroy(pg_ntt_table *table);
/* A table over limbs [first, first + count) of `table` that shares its device
 * arrays (DcrtTable::ntt_tables / iter, primus_ntt/src/dcrt/mod.rs: the
 * per-prime tables of a DCRT table; count = 1 gives one prime's NttTable).
 * The view keeps the parent's schedule setting and starts with default shapes;
 * destroy it with pg_ntt_table_destroy before its parent. */
int pg_ntt_table_view(const pg_ntt_table *table, uint32_t first, uint32_t count, pg_ntt_table **out);
/* NTT kernel shapes.  Each ring degree has a default shape (rows per CTA,
 * elements per thread, cluster size) and, for N = 2^10 .. 2^16, alternatives
 * that compute identical values at different speed.  pg_ntt_autotune times
 * every shape of the table's degree on `polys` seeded polys of its moduli (at
 * most 1 GiB) for the canonical forward, the inverse and the fused round trip,
 * and keeps the fastest of each in the table.  The alternatives run on the fast
 * schedules only (integer shapes: canonical forward with every modulus below
 * 2^58, inverse and round trip below 2^50; FP64 shapes: every modulus below 2^50
 * and the FP64 schedule enabled); the lazy forward always runs the default shape.  It allocates its own buffers and synchronizes; call it before
 * the table is shared between threads or streams.  No reference counterpart
 * (the reference's CPU transforms have one shape). */
typedef struct pg_ntt_tuning {
    int32_t variant[3]; /* chosen shape per mode: forward, inverse, round trip */
    float us[3];        /* its time per launch over `rows` rows */
    float default_us[3];/* the default shape's time, for comparison */
    uint64_t rows;
} pg_ntt_tuning;
enum { PG_NTT_MODE_FORWARD = 0, PG_NTT_MODE_INVERSE = 1, PG_NTT_MODE_ROUND_TRIP = 2 };
int pg_ntt_autotune(pg_ntt_table *table, size_t polys, pg_ntt_tuning *out);
/* Built-in ceilings on the current device (no reference counterpart): a
 * streaming copy of 512 MiB (read + write bytes per second, GB/s) and the
 * register-only rate of the forward butterfly on the fast integer schedule and
 * on the FP64 schedule (G butterflies/s, q just below 2^50).  Allocates 1 GiB
 * and synchronizes the device; a measurement call, not for a serving path. */
typedef struct pg_calibration {
    double hbm_copy_gbs;
    double int_butterflies_gps;
    double fp64_butterflies_gps;
} pg_calibration;
int pg_calibrate(pg_calibration *out);
int pg_ntt_variant_count(uint32_t log_n);
const char *pg_ntt_variant_name(uint32_t log_n, int variant); /* NULL if out of range */
int pg_ntt_set_variant(pg_ntt_table *table, int mode, int variant);
/* FP64 butterfly schedule on (enable = 1, the default when every modulus is
 * below 2^50) or off (0: every transform of this table runs on the integer
 * pipe only).  Both schedules return the same canonical residues: the FP64 one
 * carries residues as doubles holding integers below 2^53, each operation's
 * result exact (quotient estimates are corrected exactly, as Shoup's are).
 * No reference counterpart.  Returns PG_ERR_UNSUPPORTED when enabling it on a
 * table with a modulus at or above 2^50.  Resets the autotuned shapes; like
 * pg_ntt_autotune, call it before the table is shared between threads or streams. */
int pg_ntt_set_fp64(pg_ntt_table *table, int enable);
int pg_ntt_fp64_enabled(const pg_ntt_table *table);
/* poly_length(), moduli_count(), crt_poly_length() */
int pg_ntt_table_info(const pg_ntt_table *table, uint32_t *log_n, uint32_t *moduli_count,
                      size_t *poly_length, size_t *crt_poly_length);
/* host copies of limb `limb`'s tables: root, inv_root, inv_n and the
 * bit-reversed root_powers / scrambled inv_root_powers (values and Shoup
 * quotients, N each); any output may be NULL */
int pg_ntt_table_export(const pg_ntt_table *table, uint32_t limb, uint64_t *root,
                        uint64_t *inv_root, uint64_t *inv_n, uint64_t *h_root_powers,
                        uint64_t *h_root_powers_q, uint64_t *h_inv_root_powers,
                        uint64_t *h_inv_root_powers_q);
/* the same tables computed on the host only, without a device (for checks) */
int pg_ntt_host_tables(uint32_t log_n, uint64_t q, uint64_t *root, uint64_t *inv_root,
                       uint64_t *inv_n, uint64_t *h_root_powers, uint64_t *h_root_powers_q,
                       uint64_t *h_inv_root_powers, uint64_t *h_inv_root_powers_q);

/* Forward NTT of `polys` DCRT polynomials in place ([polys][L][N]), natural
 * order in ([0,4q)), bit-reversed order out: [0,4q) if lazy else [0,q).
 * Replaces NttTable::lazy_transform_slice / transform_slice
 * (primitive.rs:211-244) and DcrtTable::{lazy_,}transform_slice
 * (dcrt/primitive.rs:96-115). */
int pg_ntt_forward(const pg_ntt_table *table, uint64_t *d_data, size_t polys, int lazy,
                   void *stream);
/* Inverse NTT in place, bit-reversed in ([0,2q)), natural out ([0,q)).
 * Replaces {lazy_,}inverse_transform_slice (primitive.rs:246-296,
 * dcrt/primitive.rs:117-141). */
int pg_ntt_inverse(const pg_ntt_table *table, uint64_t *d_data, size_t polys, int lazy,
                   void *stream);
/* Host-slice forms with the reference's exact call semantics (copy in,
 * transform, copy out, synchronous).  Large slices run as a pipeline of
 * chunks on three streams, so copies in, transforms and copies out overlap
 * when the host memory is pinned (pg_host_alloc). */
int pg_ntt_forward_host(const pg_ntt_table *table, uint64_t *h_data, size_t polys, int lazy);
int pg_ntt_inverse_host(const pg_ntt_table *table, uint64_t *h_data, size_t polys, int lazy);
/* NTT of coeff*X^degree into every limb (coeff < every q), of X^degree and of
 * -X^degree; any degree (exponents mod 2N, X^N = -1).  Replaces transform_monomial / transform_coeff_one_monomial /
 * transform_coeff_minus_one_monomial (primitive.rs:298-397, dcrt/mod.rs:100-128). */
int pg_ntt_monomial(const pg_ntt_table *table, uint64_t coeff, size_t degree, uint64_t *d_out,
                    void *stream);
int pg_ntt_coeff_one_monomial(const pg_ntt_table *table, size_t degree, uint64_t *d_out,
                              void *stream);
int pg_ntt_coeff_minus_one_monomial(const pg_ntt_table *table, size_t degree, uint64_t *d_out,
                                    void *stream);

/* ---------------------------------------------------- pointwise DCRT ops
 * Element-wise over [polys][L][N] with limb l reduced mod moduli[l]; canonical
 * inputs and outputs.  `rhs_polys` is polys or 1 (one rhs broadcast to every
 * poly).  Replace DcrtPolynomial / ArrayBase ops in primus_poly. */
/* x *= y        (DcrtPolynomial::mul_assign, primus_poly/src/dcrt/mul.rs:97-110) */
int pg_dcrt_mul(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *d_y, size_t polys,
                size_t rhs_polys, void *stream);
/* x += y * z    (DcrtPolynomial::add_mul_assign, primus_poly/src/dcrt/mod.rs:94-114) */
int pg_dcrt_add_mul(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *d_y,
                    const uint64_t *d_z, size_t polys, size_t rhs_polys, void *stream);
/* x += y, x -= y, x = -x (primus_poly/src/dcrt/{add,sub,neg}.rs) */
int pg_dcrt_add(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *d_y, size_t polys,
                size_t rhs_polys, void *stream);
int pg_dcrt_sub(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *d_y, size_t polys,
                size_t rhs_polys, void *stream);
int pg_dcrt_neg(const pg_ntt_table *table, uint64_t *d_x, size_t polys, void *stream);
/* x *= scalar[l] per limb (DcrtPolynomial::mul_scalar_assign, dcrt/mul.rs:27-34) */
int pg_dcrt_mul_scalar(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *h_scalars,
                       size_t polys, void *stream);
/* x += y * scalar[l] (DcrtPolynomial::add_mul_scalar_assign, dcrt/mul.rs:37-58) */
int pg_dcrt_add_mul_scalar(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *d_y,
                           const uint64_t *h_scalars, size_t polys, void *stream);
/* (a, b) = (a + s, (a - s) * w) with w a per-element Shoup factor
 * polynomial (values d_w, quotients d_wq from pg_dcrt_shoup_prepare), one
 * [L][N] w shared by every poly
 * (DcrtPolynomial::butterfly_mul_factor_inplace, dcrt/mul.rs:119-155) */
int pg_dcrt_butterfly_mul_factor(const pg_ntt_table *table, uint64_t *d_a, const uint64_t *d_s,
                                 const uint64_t *d_w, const uint64_t *d_wq, uint64_t *d_b,
                                 size_t polys, void *stream);
/* Shoup quotients floor(v*2^64/q_l) of a [rhs_polys][L][N] operand, so that
 * products against it take the one-mulhi Shoup path (ShoupFactor::new,
 * primus_factor/src/shoup_factor/mod.rs:44-55) */
int pg_dcrt_shoup_prepare(const pg_ntt_table *table, const uint64_t *d_values,
                          uint64_t *d_quotients, size_t polys, void *stream);
/* x *= (w, w') with Shoup-prepared rhs (DcrtPolynomial::mul_factor_assign
 * element-wise form) */
int pg_dcrt_mul_prepared(const pg_ntt_table *table, uint64_t *d_x, const uint64_t *d_w,
                         const uint64_t *d_wq, size_t polys, size_t rhs_polys, void *stream);

/* ------------------------------------------------- fused polynomial multiply
 * For every row of [polys][L][N]: forward NTT, multiply by the NTT-domain
 * plaintext (one [L][N] operand with its Shoup quotients from
 * pg_dcrt_shoup_prepare), inverse NTT -- one launch, one HBM read and one
 * write per row.  Output equals transform_slice -> DcrtPolynomial::mul_assign
 * -> inverse_transform_slice (the reference's three calls) bit for bit. */
int pg_dcrt_polymul_ntt_plain(const pg_ntt_table *table, uint64_t *d_data,
                              const uint64_t *d_plain, const uint64_t *d_plain_q, size_t polys,
                              void *stream);
/* The same on a host slice [polys][L][N] in place (the plaintext stays resident
 * on the device): the reference's three calls on &mut [u64], through the
 * pipelined host path of pg_ntt_forward_host.  Synchronous; the pipeline runs
 * after the work already on `stream` and `stream` is ordered after it (NULL: no
 * ordering with other streams). */
int pg_dcrt_polymul_ntt_plain_host(const pg_ntt_table *table, uint64_t *h_data,
                                   const uint64_t *d_plain, const uint64_t *d_plain_q, size_t polys,
                                   void *stream);

/* ------------------------------------------------------------- RNS base
 * RNSBase (primus_rns/src/base.rs:24-90): moduli, Q = prod q_i as a BigUint of
 * W little-endian limbs, punctured products Q/q_i and their inverses mod q_i.
 * Fails with PG_ERR_NOT_COPRIME like RNSBase::new. */
typedef struct pg_rns_base pg_rns_base;

int pg_rns_base_create(const uint64_t *h_moduli, uint32_t moduli_count, pg_rns_base **out);
int pg_rns_base_destroy(pg_rns_base *base);
/* moduli_count(), big_uint_value_len() (= W); h_product receives W limbs if non-NULL */
int pg_rns_base_info(const pg_rns_base *base, uint32_t *moduli_count, uint32_t *big_uint_len,
                     uint64_t *h_product);
/* CRT composition of `count` values: residues [L][count] -> BigUint [count][W]
 * in [0, Q) (compose_multiple_values_inplace, base.rs:422-449) */
int pg_rns_compose(const pg_rns_base *base, const uint64_t *d_residues, uint64_t *d_values,
                   size_t count, void *stream);
/* BigUint [count][W] -> residues [L][count] (decompose_big_uint_values_inplace,
 * base.rs:285-309) */
int pg_rns_decompose(const pg_rns_base *base, const uint64_t *d_values, uint64_t *d_residues,
                     size_t count, void *stream);
/* signed lift of small values in [0, small_modulus) into every residue
 * (wrapping_decompose_small_values_inplace, base.rs:201-231) */
int pg_rns_wrapping_decompose_small(const pg_rns_base *base, const uint64_t *d_small,
                                    uint64_t *d_residues, size_t count, uint64_t small_modulus,
                                    void *stream);
/* dest[l][x] = dest[l][x] + factor[l] * lift_l(small[x]) mod q_l, the lift as above
 * (add_wrapping_decompose_small_values_scaled, base.rs:238-283: the same values as
 * the lift followed by add_mul_factor, without the lifted copy).  h_factor: [L]
 * host scalars below their moduli; dest: [L][count] canonical. */
int pg_rns_add_wrapping_decompose_small_scaled(const pg_rns_base *base, const uint64_t *d_small,
                                               uint64_t *d_dest, size_t count, uint64_t small_modulus,
                                               const uint64_t *h_factor, void *stream);

/* ------------------------------------------------------ fast base conversion
 * BaseConverter (primus_rns/src/converter.rs:12-47); fast_convert_array
 * (:147-175): y_j = sum_i [x_i * (Q/q_i)^-1]_{q_i} * (Q/q_i mod p_j) mod p_j,
 * no correction, input [L_in][n] -> output [L_out][n]. */
typedef struct pg_base_converter pg_base_converter;

int pg_base_converter_create(const pg_rns_base *ibase, const pg_rns_base *obase,
                             pg_base_converter **out);
int pg_base_converter_destroy(pg_base_converter *conv);
int pg_fast_convert_array(const pg_base_converter *conv, const uint64_t *d_in, uint64_t *d_out,
                          size_t n, void *stream);

/* ----------------------------------------------------- gadget decomposition
 * BigUintApproxSignedBasis (primus_decompose/src/big_integer/basis.rs:34-193)
 * over the product of an RNS base; reverse_length < 0 means None. */
typedef struct pg_gadget_basis pg_gadget_basis;

int pg_gadget_basis_create(const pg_rns_base *base, uint32_t log_basis, int32_t reverse_length,
                           pg_gadget_basis **out);
int pg_gadget_basis_destroy(pg_gadget_basis *basis);
/* decompose_length(), drop_bits(), and the gadget scalars' residues [d][L] */
int pg_gadget_basis_info(const pg_gadget_basis *basis, uint32_t *decompose_length,
                         uint32_t *drop_bits, uint64_t *h_scalar_residues);
/* every unsigned digit of `count` BigUint values [count][W] -> [d][count],
 * digits in [0, B): init_value_carry_slice (basis.rs:307-342) then
 * unsigned_decompose_slice_inplace per level (common.rs:184-200) */
int pg_gadget_decompose(const pg_gadget_basis *basis, const uint64_t *d_values,
                        uint64_t *d_digits, size_t count, void *stream);
/* the same digits lifted into the RNS base: [d][L][count]
 * (wrapping_decompose_small_values_inplace applied per level) */
int pg_gadget_decompose_lift(const pg_gadget_basis *basis, const uint64_t *d_values,
                             uint64_t *d_residues, size_t count, void *stream);

/* --------------------------------------------- GLev MAC, external product, key switch
 * Layouts: GLWE = (k+1) DCRT polys [a_1..a_k, b] (primus_lattice/src/glwe/dcrt.rs:19-27);
 * GLev = d GLWEs (glev/dcrt.rs:16-24); GGSW = (k+1) GLevs (ggsw/dcrt.rs:10-21).
 * Key and GGSW operands are in the NTT domain; outputs are canonical NTT-domain
 * residues.  The table's moduli must equal the basis's RNS base.  Scratch:
 * pass d_workspace of at least *_workspace_size() bytes, or NULL to let the
 * call take stream-ordered scratch from the library's pool (pg_scratch_trim). */
/* batch GLWE (CRT/coefficient form, [batch][k+1][L][N]) x one GGSW -> GLWE
 * (NTT domain, [batch][k+1][L][N]); CrtGlwe::mul_dcrt_ggsw_inplace
 * (primus_lattice/src/glwe/crt.rs:202-229) */
size_t pg_ext_product_workspace_size(const pg_ntt_table *table, const pg_gadget_basis *basis,
                                     uint32_t k, size_t batch);
int pg_ext_product(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                   const uint64_t *d_glwe_in, const uint64_t *d_ggsw, uint64_t *d_glwe_out,
                   size_t batch, void *d_workspace, size_t workspace_bytes, void *stream);
/* The external product followed by inverse_transform_slice of every output
 * poly (primus_ntt/src/ntt/primitive.rs:246-296): the GLWE comes back in
 * coefficient form, the shape of a blind-rotation accumulator step.  For k = 1,
 * one prime, single-word gadget values, N = 2^10..2^12 and batches of at least
 * 64 ciphertexts the whole step (decompose -> NTT -> MAC -> INTT) is one kernel;
 * pg_ext_product uses the same kernel without the inverse for those shapes.
 * Workspace as pg_ext_product. */
int pg_ext_product_coeff(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                         const uint64_t *d_glwe_in, const uint64_t *d_ggsw, uint64_t *d_glwe_out,
                         size_t batch, void *d_workspace, size_t workspace_bytes, void *stream);
/* acc ([k+1][L][N], NTT domain) += GLev x poly, the poly as CRT residues [L][N]
 * (add_dcrt_glev_mul_crt_poly_assign, glwe/dcrt.rs:170-247) or as BigUints
 * [N][W] (add_dcrt_glev_mul_big_uint_poly_assign, glwe/dcrt.rs:249-325) */
int pg_glev_mac_crt_poly(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                         uint64_t *d_acc, const uint64_t *d_glev, const uint64_t *d_crt_poly,
                         void *d_workspace, size_t workspace_bytes, void *stream);
int pg_glev_mac_big_uint_poly(const pg_ntt_table *table, const pg_gadget_basis *basis,
                              uint32_t k, uint64_t *d_acc, const uint64_t *d_glev,
                              const uint64_t *d_big_poly, void *d_workspace,
                              size_t workspace_bytes, void *stream);
/* key switch s_in -> s_out of a batch: key [k_in][d][k_out+1][L][N] (NTT),
 * c_in [batch][k_in+1][L][N] (coefficient form), c_out [batch][k_out+1][L][N]
 * (NTT domain); CrtGlweKeySwitchingKey::key_swithching_inplace
 * (primus_fhe_core/src/key_switch.rs:79-128) */
size_t pg_key_switch_workspace_size(const pg_ntt_table *table, const pg_gadget_basis *basis,
                                    uint32_t k_in, uint32_t k_out, size_t batch);
int pg_key_switch(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k_in,
                  uint32_t k_out, const uint64_t *d_key, const uint64_t *d_c_in,
                  uint64_t *d_c_out, size_t batch, void *d_workspace, size_t workspace_bytes,
                  void *stream);
/* GLWE automorphism X -> X^degree (degree odd) in the NTT domain:
 * DcrtGlweAutoKey::automorphism_inplace (primus_fhe_core/src/automorphism/glwe/dcrt.rs:269-331).
 * Every poly of each ciphertext is permuted in the NTT domain
 * (generate_ntt_permutation, :43-63), the k masks are inverse-transformed and
 * key-switched with the automorphism key, the permuted body is added:
 * c_out = -(sum_i key_i (x) sigma(a_i)) + (0, .., sigma(b)).  c_in, c_out:
 * [batch][k+1][L][N] NTT domain (must not overlap); key: k GLevs
 * [k][d][k+1][L][N] (GLev of sigma(s_i) under s, NTT domain). */
size_t pg_glwe_automorphism_workspace_size(const pg_ntt_table *table, const pg_gadget_basis *basis,
                                           uint32_t k, size_t batch);
int pg_glwe_automorphism(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                         uint64_t degree, const uint64_t *d_key, const uint64_t *d_c_in, uint64_t *d_c_out,
                         size_t batch, void *d_workspace, size_t workspace_bytes, void *stream);
/* Field trace: DcrtGlweTraceKey::trace_inplace
 * (primus_fhe_core/src/trace/glwe/dcrt.rs:84-108): c_out = c_in, then
 * c_out += sigma_d(c_out) for d = N+1, N/2+1, .., 3 (log2 N automorphisms).
 * With reverse != 0, DcrtGlweRevTraceKey::trace_inplace (trace/glwe/rev.rs:79-115):
 * d = 3, 5, .., N+1, c_out *= 2^-1 mod q_l before each automorphism.  keys:
 * log2(N) automorphism keys in the order applied, each [k][d][k+1][L][N];
 * c_in, c_out: [batch][k+1][L][N] NTT domain, the same buffer or disjoint. */
size_t pg_glwe_trace_workspace_size(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                                    size_t batch);
int pg_glwe_trace(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k, const uint64_t *d_keys,
                  int reverse, const uint64_t *d_c_in, uint64_t *d_c_out, size_t batch, void *d_workspace,
                  size_t workspace_bytes, void *stream);
/* Coefficient expansion: DcrtGlweExpandCoeffKey::expand_partial_coefficients_inplace
 * (primus_fhe_core/src/expand_coeff/glwe/dcrt.rs:235-287; count = N is
 * expand_coefficients_inplace).  count: a power of two <= N; keys as for the
 * forward trace (degrees N+1, N/2+1, ..; the first log2(count) are read);
 * c_in: one ciphertext [k+1][L][N]; out: [count][k+1][L][N] (c_in may be out's
 * first slot).  For an input encrypting m, output j encrypts
 * sum_i m[j + count*i] X^(count*i) (m[j] alone when count = N). */
size_t pg_glwe_expand_workspace_size(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                                     size_t count);
int pg_glwe_expand_coefficients(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                                const uint64_t *d_keys, size_t count, const uint64_t *d_c_in, uint64_t *d_out,
                                void *d_workspace, size_t workspace_bytes, void *stream);
/* BFV-style GLWE decryption through fast base conversion:
 * DcrtGlweSecretKey::decrypt_inplace (primus_fhe_core/src/secret_key/glwe.rs:782-837).
 * phase = b - sum a_i s_i (NTT domain), inverse NTT, x [t gamma]_q, fast
 * conversion to {t, gamma} (converter.rs:147-175), x -Q^-1, gamma correction.
 * The decryptor holds the per-limb constants for one table, plaintext modulus t
 * and correction modulus gamma (t < gamma < 2^62, pairwise coprime with the
 * moduli: PG_ERR_NOT_COPRIME otherwise).  sk: [k][L][N] NTT domain; ct:
 * [batch][k+1][L][N] NTT domain; msg out: [batch][N] values in [0, t). */
typedef struct pg_bfv_decryptor pg_bfv_decryptor;
int pg_bfv_decryptor_create(const pg_ntt_table *table, uint64_t plain_modulus, uint64_t gamma,
                            pg_bfv_decryptor **out);
int pg_bfv_decryptor_destroy(pg_bfv_decryptor *decryptor);
size_t pg_bfv_decrypt_workspace_size(const pg_bfv_decryptor *decryptor, size_t batch);
int pg_bfv_decrypt(const pg_bfv_decryptor *decryptor, uint32_t k, const uint64_t *d_sk_ntt,
                   const uint64_t *d_ct, uint64_t *d_msg, size_t batch, void *d_workspace,
                   size_t workspace_bytes, void *stream);

/* Secret-key GLWE encryption on the device: DcrtGlweSecretKey::encrypt_inplace
 * (primus_fhe_core/src/secret_key/glwe.rs:386-424); with a gadget factor as
 * `scale` the rows of a GLev / key-switching key (:683-708).  Samplers are pure
 * functions of (seed, stream, index), identical in the oracle:
 *   mask a_i limb l of ciphertext j: uniform below q_l, stream stream0 + (j k + i) L + l
 *   noise of ciphertext j: discrete Gaussian (sigma, bound ceil(24 sigma)) by a
 *   cumulative table, stream stream0 + 2^32 + j
 *   b = NTT(e + scale_l * msg) + sum_i a_i s_i
 * sk: [k][L][N] NTT domain; msg: [batch][L][N] residues in coefficient form, or
 * NULL for encryptions of zero; h_scale: [L] host values below each q_l (e.g.
 * Delta = round(Q/t) mod q_l); ct out: [batch][k+1][L][N] NTT domain. */
typedef struct pg_glwe_encryptor pg_glwe_encryptor;
int pg_glwe_encryptor_create(const pg_ntt_table *table, double sigma, pg_glwe_encryptor **out);
int pg_glwe_encryptor_destroy(pg_glwe_encryptor *encryptor);
int pg_glwe_encrypt(const pg_glwe_encryptor *encryptor, uint32_t k, const uint64_t *d_sk_ntt,
                    const uint64_t *d_msg, const uint64_t *h_scale, uint64_t seed, uint64_t stream0,
                    uint64_t *d_ct, size_t batch, void *stream);
/* Public-key encryption (primus_fhe_core/src/public_key/glwe.rs).  A public key
 * [k+1][L][N] (NTT domain) is a secret-key encryption of zero
 * (DcrtGlwePublicKey::new, :33-71): pg_glwe_encrypt with d_msg = NULL.
 * pg_glwe_pk_encrypt: DcrtGlwePublicKey::encrypt (:74-126) of `batch`
 * ciphertexts, ct_c = NTT(e_c) + NTT(v) pk_c with scale_l * msg added to the
 * body's noise before its NTT; samplers, for ciphertext j:
 *   v   ternary: bits 2(x mod 16) of hash(seed, stream0 + 2^33 + j, x / 16):
 *       0,1 -> 0, 2 -> 1, 3 -> -1
 *   e_c discrete Gaussian (as pg_glwe_encrypt), stream stream0 + 2^32 + j (k+1) + c
 * pg_ggsw_pk_encrypt_monomial: DcrtGlwePublicKey::encrypt_monomial_ggsw_inplace
 * (:214-263), GGSW [k+1][d][k+1][L][N] of coeff * X^degree (degree < N): row
 * r = i d + j is ciphertext r of the samplers above, with coeff_l * g_{j,l}
 * added at coefficient `degree` of component i (:128-193). */
int pg_glwe_pk_encrypt(const pg_glwe_encryptor *encryptor, uint32_t k, const uint64_t *d_pk,
                       const uint64_t *d_msg, const uint64_t *h_scale, uint64_t seed, uint64_t stream0,
                       uint64_t *d_ct, size_t batch, void *stream);
int pg_ggsw_pk_encrypt_monomial(const pg_glwe_encryptor *encryptor, const pg_gadget_basis *basis, uint32_t k,
                                const uint64_t *d_pk, const uint64_t *h_coeff_residues, size_t degree,
                                uint64_t seed, uint64_t stream0, uint64_t *d_ggsw, void *stream);

/* pg_ext_product for callers that cannot allocate device memory when they
 * call (hosts holding only device pointers owned by another runtime, serving
 * processes that reserve HBM at start-up and forbid later allocations).  No
 * counterpart in the reference: it exists for this library's C callers.
 * Shapes the fused external-product kernel takes (k = 1, one prime,
 * single-word gadget values, N = 2^10..2^12, batch >= 64, 16-byte aligned
 * key and output) need no scratch and run there, up to 2^31 - 1 ciphertexts
 * per call.  Every other shape keeps its scratch in a fixed 32 MiB device
 * array inside the library, held by every GPU that loads it until the process
 * exits; a batch needing more is refused before any launch with
 * PG_ERR_UNSUPPORTED and a message giving the largest batch of that shape.
 * The first call on each device looks up the array's device address, so make
 * that first call before any stream capture.  No scratch word needs to start
 * at zero, but every call shares the array: calls whose work overlaps on the
 * GPU (other streams, other threads) race, so serialise them. */
int pg_ext_product_noalloc(const pg_ntt_table *table, const pg_gadget_basis *basis, uint32_t k,
                           const uint64_t *d_glwe_in, const uint64_t *d_ggsw,
                           uint64_t *d_glwe_out, size_t batch, void *stream);

/* Hybrid RNS key switch with K special primes and digit groups of `alpha`
 * consecutive Q limbs (dnum = ceil(L / alpha) groups).  No reference
 * counterpart: the reference's key switch is the BigUint gadget form
 * (pg_key_switch).  The table holds L + K primes, Q first then P.
 *   for each mask a_i and group g: ModUp (a_i's D_g residues kept, every other
 *   QP limb by fast base conversion), forward NTT, acc[c] += ext (.) key[i][g][c];
 *   ModDown: inverse NTT of acc's P limbs, fast conversion P -> Q, forward NTT,
 *   (acc_Q - conv) * P^-1;  c_out = -ModDown(acc) + (0, .., NTT(b)).
 * key: [k_in][dnum][k_out+1][L+K][N] NTT domain, row [i][g] encrypting
 * [P]_{q_l} * s_in_i on the limbs of D_g (0 elsewhere) under s_out over QP.
 * c_in: [batch][k_in+1][L][N] coefficient form; c_out: [batch][k_out+1][L][N]
 * NTT domain, canonical.  alpha <= 8, K <= 8. */
typedef struct pg_hybrid_ks pg_hybrid_ks;
int pg_hybrid_ks_create(const pg_ntt_table *table, uint32_t L, uint32_t K, uint32_t alpha,
                        pg_hybrid_ks **out);
int pg_hybrid_ks_destroy(pg_hybrid_ks *ks);
uint32_t pg_hybrid_ks_dnum(const pg_hybrid_ks *ks);
size_t pg_hybrid_ks_workspace_size(const pg_hybrid_ks *ks, uint32_t k_in, uint32_t k_out, size_t batch);
int pg_key_switch_hybrid(const pg_hybrid_ks *ks, uint32_t k_in, uint32_t k_out, const uint64_t *d_key,
                         const uint64_t *d_c_in, uint64_t *d_c_out, size_t batch, void *d_workspace,
                         size_t workspace_bytes, void *stream);

/* ----------------------------------------------- uneven batches of products
 * A job multiplies two coefficient-form DCRT polys of its own ring degree:
 * a <- a * b (negacyclic), b <- NTT(b), using the first moduli_count primes of
 * the batch's table for that degree -- per limb the reference's
 * transform_slice x2, mul_assign, inverse_transform_slice
 * (primus_ntt/src/ntt/primitive.rs:234-296, primus_poly/src/dcrt/mul.rs:97-110).
 * One run launches, per ring degree present, a forward NTT over every a- and
 * b-row and a fused multiply + inverse NTT over every a-row (for N <= 2^12 with
 * every modulus below 2^50, one launch doing both per row), the degrees on
 * parallel streams.  With use_graph the first run of a job shape is captured
 * into a CUDA graph and later runs of the same shape replay it. */
typedef struct pg_polymul_job {
    uint64_t *d_a;          /* [moduli_count][N], result */
    uint64_t *d_b;          /* [moduli_count][N], left in the NTT domain; both are transformed
                               in place, so no buffer may overlap another of the same run
                               (overlapping a and b of one job are refused) */
    uint32_t log_n;
    uint32_t moduli_count;
} pg_polymul_job;
typedef struct pg_polymul_batch pg_polymul_batch;

/* tables: one per ring degree (distinct log_n), each with enough primes */
int pg_polymul_batch_create(const pg_ntt_table *const *tables, uint32_t table_count,
                            pg_polymul_batch **out);
int pg_polymul_batch_destroy(pg_polymul_batch *batch);
/* make room for `rows` row descriptors (a job of L limbs takes 3L) so that later
 * calls up to that size allocate nothing; the batch starts with 4096 */
int pg_polymul_batch_reserve(pg_polymul_batch *batch, size_t rows);
int pg_polymul_batch_run(pg_polymul_batch *batch, const pg_polymul_job *h_jobs, size_t count,
                         int use_graph, void *stream);

/* ------------------------------------------------------- request server
 * Continuous batching of mixed requests on one GPU (no reference counterpart:
 * the reference is a library of synchronous calls).  Clients keep keys and
 * ciphertexts resident in device memory and submit single requests; a worker
 * thread forms batches of one kind and shape whenever one of its slots (a
 * stream plus an equal share of memory_budget_bytes of scratch) is free, taking
 * as many pending requests as fit the slot's scratch (admission by memory), so
 * requests that arrive while others run join the next batch and batches on
 * different slots overlap.  A completion thread polls each batch's event and
 * then marks its requests done.  Results are identical to running each request
 * alone. */
enum { PG_REQ_POLYMUL = 1, PG_REQ_EXT_PRODUCT = 2, PG_REQ_KEY_SWITCH = 3 };

typedef struct pg_request {
    int kind;
    uint32_t key;            /* ext product / key switch: id from pg_server_register_key */
    uint64_t *d_a;           /* polymul: a <- a * b, b <- NTT(b) (pg_polymul_job) */
    uint64_t *d_b;
    uint32_t log_n;
    uint32_t moduli_count;
    const uint64_t *d_in;    /* ext product / key switch: one ciphertext in ... */
    uint64_t *d_out;         /* ... and its result (NTT domain) */
} pg_request;

typedef struct pg_server_config {
    size_t memory_budget_bytes; /* scratch shared by the slots */
    uint32_t slots;             /* concurrent batches (streams), 1..64 */
    uint32_t max_batch;         /* requests per batch */
    uint32_t max_queue;         /* pending requests before submit rejects (0: 2^20) */
} pg_server_config;

typedef struct pg_server_stats {
    uint64_t submitted, completed, rejected, batches;
    double mean_batch, p50_us, p99_us, max_us; /* latency = submit -> completion */
    double enqueue_mean_us, enqueue_max_us;    /* host time to put one batch on its stream */
} pg_server_stats_t;

typedef struct pg_server pg_server;

/* polymul_tables: one per ring degree polymul requests may use */
int pg_server_create(const pg_server_config *config, const pg_ntt_table *const *polymul_tables,
                     uint32_t table_count, pg_server **out);
/* stops the worker; drain first so that no request is left pending */
int pg_server_destroy(pg_server *server);
/* a GGSW (kind PG_REQ_EXT_PRODUCT, k_out ignored) or key-switching key
 * (PG_REQ_KEY_SWITCH) resident on the device; the layouts of pg_ext_product /
 * pg_key_switch */
int pg_server_register_key(pg_server *server, int kind, const pg_ntt_table *table,
                           const pg_gadget_basis *basis, uint32_t k_in, uint32_t k_out,
                           const uint64_t *d_key, uint32_t *key_id);
/* register a hybrid key switch key (pg_key_switch_hybrid layout) for
 * PG_REQ_KEY_SWITCH requests; the context and key stay owned by the caller */
int pg_server_register_hybrid_key(pg_server *server, const pg_hybrid_ks *ks, uint32_t k_in, uint32_t k_out,
                                  const uint64_t *d_key, uint32_t *key_id);
/* queue one request; PG_ERR_REJECTED when the queue is full or the request
 * cannot fit one slot's scratch, PG_ERR_INVALID_ARGUMENT when malformed */
int pg_server_submit(pg_server *server, const pg_request *request, uint64_t *ticket);
/* wait for a request (timeout_us < 0: no limit); PG_ERR_TIMEOUT if not done */
int pg_server_wait(pg_server *server, uint64_t ticket, int64_t timeout_us, double *latency_us);
/* wait until nothing is pending or running */
int pg_server_drain(pg_server *server, int64_t timeout_us);
int pg_server_stats(pg_server *server, pg_server_stats_t *out, int reset);
/* load replay: submit requests[i] at arrival_us[i] microseconds after the call
 * (from the calling thread), wait for all; latency_us[i] = completion time minus
 * scheduled arrival (-1 when rejected) */
int pg_server_replay(pg_server *server, const pg_request *requests, const double *arrival_us,
                     size_t count, double *latency_us);

/* ------------------------------------------------------- seeded inputs
 * Device-side fill with the counter-based generator (uniform below q_l per
 * limb; stream id = stream0 + poly*L + limb). */
int pg_fill_uniform(const pg_ntt_table *table, uint64_t *d_out, size_t polys, uint64_t seed,
                    uint64_t stream0, void *stream);
/* host form of the same generator: out[i] for i < n, uniform below q */
int pg_fill_uniform_host(uint64_t seed, uint64_t stream_id, uint64_t q, size_t n,
                         uint64_t *h_out);

#ifdef __cplusplus
}
#endif
#endif /* PRIMUS_GPU_H */
