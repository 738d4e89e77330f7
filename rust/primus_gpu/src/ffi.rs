//! Raw bindings to `libprimus_gpu.so`, one declaration per entry point of
//! `include/primus_gpu.h` (same names, same argument order).  Pointers named
//! `d_*` in the header are device pointers, `h_*` host pointers; `stream` is
//! a `cudaStream_t` (null = the legacy default stream).  Every function
//! returns a status (`PG_OK` = 0) except the size, count and string queries.
#![allow(non_camel_case_types, clippy::too_many_arguments)]

use std::ffi::{c_char, c_void};

pub const PG_OK: i32 = 0;
pub const PG_ERR_INVALID_ARGUMENT: i32 = 1;
pub const PG_ERR_NO_PRIMITIVE_ROOT: i32 = 2;
pub const PG_ERR_DEGREE_TOO_LARGE: i32 = 3;
pub const PG_ERR_NOT_COPRIME: i32 = 4;
pub const PG_ERR_UNSUPPORTED: i32 = 5;
pub const PG_ERR_OUT_OF_MEMORY: i32 = 6;
pub const PG_ERR_CUDA: i32 = 7;
pub const PG_ERR_TIMEOUT: i32 = 8;
pub const PG_ERR_REJECTED: i32 = 9;

pub const PG_NTT_MODE_FORWARD: i32 = 0;
pub const PG_NTT_MODE_INVERSE: i32 = 1;
pub const PG_NTT_MODE_ROUND_TRIP: i32 = 2;

pub const PG_REQ_POLYMUL: i32 = 1;
pub const PG_REQ_EXT_PRODUCT: i32 = 2;
pub const PG_REQ_KEY_SWITCH: i32 = 3;

macro_rules! opaque {
    ($($name:ident),*) => { $( #[repr(C)] pub struct $name { _private: [u8; 0] } )* };
}
opaque!(PgNttTable, PgRnsBase, PgBaseConverter, PgGadgetBasis, PgBfvDecryptor, PgGlweEncryptor, PgHybridKs,
        PgPolymulBatch, PgServer);

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PgNttTuning {
    pub variant: [i32; 3],
    pub us: [f32; 3],
    pub default_us: [f32; 3],
    pub rows: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PgCalibration {
    pub hbm_copy_gbs: f64,
    pub int_butterflies_gps: f64,
    pub fp64_butterflies_gps: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct PgPolymulJob {
    pub d_a: *mut u64,
    pub d_b: *mut u64,
    pub log_n: u32,
    pub moduli_count: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct PgRequest {
    pub kind: i32,
    pub key: u32,
    pub d_a: *mut u64,
    pub d_b: *mut u64,
    pub log_n: u32,
    pub moduli_count: u32,
    pub d_in: *const u64,
    pub d_out: *mut u64,
}

impl Default for PgRequest {
    fn default() -> Self {
        Self {
            kind: 0,
            key: 0,
            d_a: std::ptr::null_mut(),
            d_b: std::ptr::null_mut(),
            log_n: 0,
            moduli_count: 0,
            d_in: std::ptr::null(),
            d_out: std::ptr::null_mut(),
        }
    }
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PgServerConfig {
    pub memory_budget_bytes: usize,
    pub slots: u32,
    pub max_batch: u32,
    pub max_queue: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct PgServerStats {
    pub submitted: u64,
    pub completed: u64,
    pub rejected: u64,
    pub batches: u64,
    pub mean_batch: f64,
    pub p50_us: f64,
    pub p99_us: f64,
    pub max_us: f64,
    pub enqueue_mean_us: f64,
    pub enqueue_max_us: f64,
}

#[link(name = "primus_gpu")]
unsafe extern "C" {
    pub fn pg_status_string(status: i32) -> *const c_char;
    pub fn pg_last_error() -> *const c_char;
    pub fn pg_version() -> *const c_char;
    pub fn pg_device_count(count: *mut i32) -> i32;
    pub fn pg_set_device(device: i32) -> i32;
    pub fn pg_malloc(d_ptr: *mut *mut c_void, bytes: usize) -> i32;
    pub fn pg_free(d_ptr: *mut c_void) -> i32;
    pub fn pg_host_alloc(h_ptr: *mut *mut c_void, bytes: usize) -> i32;
    pub fn pg_host_free(h_ptr: *mut c_void) -> i32;
    pub fn pg_memcpy_h2d(d_dst: *mut c_void, h_src: *const c_void, bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_memcpy_d2h(h_dst: *mut c_void, d_src: *const c_void, bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_from_bytes(d_dst: *mut u64, words: usize, h_bytes: *const u8, nbytes: usize) -> i32;
    pub fn pg_to_bytes(d_src: *const u64, words: usize, h_bytes: *mut u8, nbytes: usize) -> i32;
    pub fn pg_memcpy_d2d(d_dst: *mut c_void, d_src: *const c_void, bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_memset(d_ptr: *mut c_void, value: i32, bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_stream_create(stream: *mut *mut c_void) -> i32;
    pub fn pg_stream_destroy(stream: *mut c_void) -> i32;
    pub fn pg_stream_synchronize(stream: *mut c_void) -> i32;
    pub fn pg_device_synchronize() -> i32;
    pub fn pg_event_create(event: *mut *mut c_void) -> i32;
    pub fn pg_event_destroy(event: *mut c_void) -> i32;
    pub fn pg_event_record(event: *mut c_void, stream: *mut c_void) -> i32;
    pub fn pg_event_elapsed_ms(start: *mut c_void, stop: *mut c_void, ms: *mut f32) -> i32;
    pub fn pg_launch_count() -> u64;
    pub fn pg_scratch_trim(keep_bytes: usize) -> i32;
    pub fn pg_prev_prime_congruent(bound: u64, m: u64) -> u64;
    pub fn pg_ntt_primes(bound: u64, m: u64, count: u32, h_out: *mut u64) -> i32;
    pub fn pg_minimal_primitive_root(log_degree: u32, q: u64, root: *mut u64) -> i32;
    pub fn pg_ntt_table_create(log_n: u32, h_moduli: *const u64, moduli_count: u32, out_: *mut *mut PgNttTable) -> i32;
    pub fn pg_ntt_table_destroy(table: *mut PgNttTable) -> i32;
    pub fn pg_ntt_table_view(table: *const PgNttTable, first: u32, count: u32, out_: *mut *mut PgNttTable) -> i32;
    pub fn pg_ntt_autotune(table: *mut PgNttTable, polys: usize, out_: *mut PgNttTuning) -> i32;
    pub fn pg_calibrate(out_: *mut PgCalibration) -> i32;
    pub fn pg_ntt_variant_count(log_n: u32) -> i32;
    pub fn pg_ntt_variant_name(log_n: u32, variant: i32) -> *const c_char;
    pub fn pg_ntt_set_variant(table: *mut PgNttTable, mode: i32, variant: i32) -> i32;
    pub fn pg_ntt_set_fp64(table: *mut PgNttTable, enable: i32) -> i32;
    pub fn pg_ntt_fp64_enabled(table: *const PgNttTable) -> i32;
    pub fn pg_ntt_table_info(table: *const PgNttTable, log_n: *mut u32, moduli_count: *mut u32, poly_length: *mut usize, crt_poly_length: *mut usize) -> i32;
    pub fn pg_ntt_table_export(table: *const PgNttTable, limb: u32, root: *mut u64, inv_root: *mut u64, inv_n: *mut u64, h_root_powers: *mut u64, h_root_powers_q: *mut u64, h_inv_root_powers: *mut u64, h_inv_root_powers_q: *mut u64) -> i32;
    pub fn pg_ntt_host_tables(log_n: u32, q: u64, root: *mut u64, inv_root: *mut u64, inv_n: *mut u64, h_root_powers: *mut u64, h_root_powers_q: *mut u64, h_inv_root_powers: *mut u64, h_inv_root_powers_q: *mut u64) -> i32;
    pub fn pg_ntt_forward(table: *const PgNttTable, d_data: *mut u64, polys: usize, lazy: i32, stream: *mut c_void) -> i32;
    pub fn pg_ntt_inverse(table: *const PgNttTable, d_data: *mut u64, polys: usize, lazy: i32, stream: *mut c_void) -> i32;
    pub fn pg_ntt_forward_host(table: *const PgNttTable, h_data: *mut u64, polys: usize, lazy: i32) -> i32;
    pub fn pg_ntt_inverse_host(table: *const PgNttTable, h_data: *mut u64, polys: usize, lazy: i32) -> i32;
    pub fn pg_ntt_monomial(table: *const PgNttTable, coeff: u64, degree: usize, d_out: *mut u64, stream: *mut c_void) -> i32;
    pub fn pg_ntt_coeff_one_monomial(table: *const PgNttTable, degree: usize, d_out: *mut u64, stream: *mut c_void) -> i32;
    pub fn pg_ntt_coeff_minus_one_monomial(table: *const PgNttTable, degree: usize, d_out: *mut u64, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_mul(table: *const PgNttTable, d_x: *mut u64, d_y: *const u64, polys: usize, rhs_polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_add_mul(table: *const PgNttTable, d_x: *mut u64, d_y: *const u64, d_z: *const u64, polys: usize, rhs_polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_add(table: *const PgNttTable, d_x: *mut u64, d_y: *const u64, polys: usize, rhs_polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_sub(table: *const PgNttTable, d_x: *mut u64, d_y: *const u64, polys: usize, rhs_polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_neg(table: *const PgNttTable, d_x: *mut u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_mul_scalar(table: *const PgNttTable, d_x: *mut u64, h_scalars: *const u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_add_mul_scalar(table: *const PgNttTable, d_x: *mut u64, d_y: *const u64, h_scalars: *const u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_butterfly_mul_factor(table: *const PgNttTable, d_a: *mut u64, d_s: *const u64, d_w: *const u64, d_wq: *const u64, d_b: *mut u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_shoup_prepare(table: *const PgNttTable, d_values: *const u64, d_quotients: *mut u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_mul_prepared(table: *const PgNttTable, d_x: *mut u64, d_w: *const u64, d_wq: *const u64, polys: usize, rhs_polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_polymul_ntt_plain(table: *const PgNttTable, d_data: *mut u64, d_plain: *const u64, d_plain_q: *const u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_dcrt_polymul_ntt_plain_host(table: *const PgNttTable, h_data: *mut u64, d_plain: *const u64, d_plain_q: *const u64, polys: usize, stream: *mut c_void) -> i32;
    pub fn pg_rns_base_create(h_moduli: *const u64, moduli_count: u32, out_: *mut *mut PgRnsBase) -> i32;
    pub fn pg_rns_base_destroy(base: *mut PgRnsBase) -> i32;
    pub fn pg_rns_base_info(base: *const PgRnsBase, moduli_count: *mut u32, big_uint_len: *mut u32, h_product: *mut u64) -> i32;
    pub fn pg_rns_compose(base: *const PgRnsBase, d_residues: *const u64, d_values: *mut u64, count: usize, stream: *mut c_void) -> i32;
    pub fn pg_rns_decompose(base: *const PgRnsBase, d_values: *const u64, d_residues: *mut u64, count: usize, stream: *mut c_void) -> i32;
    pub fn pg_rns_wrapping_decompose_small(base: *const PgRnsBase, d_small: *const u64, d_residues: *mut u64, count: usize, small_modulus: u64, stream: *mut c_void) -> i32;
    pub fn pg_rns_add_wrapping_decompose_small_scaled(base: *const PgRnsBase, d_small: *const u64, d_dest: *mut u64, count: usize, small_modulus: u64, h_factor: *const u64, stream: *mut c_void) -> i32;
    pub fn pg_base_converter_create(ibase: *const PgRnsBase, obase: *const PgRnsBase, out_: *mut *mut PgBaseConverter) -> i32;
    pub fn pg_base_converter_destroy(conv: *mut PgBaseConverter) -> i32;
    pub fn pg_fast_convert_array(conv: *const PgBaseConverter, d_in: *const u64, d_out: *mut u64, n: usize, stream: *mut c_void) -> i32;
    pub fn pg_gadget_basis_create(base: *const PgRnsBase, log_basis: u32, reverse_length: i32, out_: *mut *mut PgGadgetBasis) -> i32;
    pub fn pg_gadget_basis_destroy(basis: *mut PgGadgetBasis) -> i32;
    pub fn pg_gadget_basis_info(basis: *const PgGadgetBasis, decompose_length: *mut u32, drop_bits: *mut u32, h_scalar_residues: *mut u64) -> i32;
    pub fn pg_gadget_decompose(basis: *const PgGadgetBasis, d_values: *const u64, d_digits: *mut u64, count: usize, stream: *mut c_void) -> i32;
    pub fn pg_gadget_decompose_lift(basis: *const PgGadgetBasis, d_values: *const u64, d_residues: *mut u64, count: usize, stream: *mut c_void) -> i32;
    pub fn pg_ext_product_workspace_size(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, batch: usize) -> usize;
    pub fn pg_ext_product(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_glwe_in: *const u64, d_ggsw: *const u64, d_glwe_out: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_ext_product_coeff(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_glwe_in: *const u64, d_ggsw: *const u64, d_glwe_out: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_glev_mac_crt_poly(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_acc: *mut u64, d_glev: *const u64, d_crt_poly: *const u64, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_glev_mac_big_uint_poly(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_acc: *mut u64, d_glev: *const u64, d_big_poly: *const u64, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_key_switch_workspace_size(table: *const PgNttTable, basis: *const PgGadgetBasis, k_in: u32, k_out: u32, batch: usize) -> usize;
    pub fn pg_key_switch(table: *const PgNttTable, basis: *const PgGadgetBasis, k_in: u32, k_out: u32, d_key: *const u64, d_c_in: *const u64, d_c_out: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_glwe_automorphism_workspace_size(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, batch: usize) -> usize;
    pub fn pg_glwe_automorphism(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, degree: u64, d_key: *const u64, d_c_in: *const u64, d_c_out: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_glwe_trace_workspace_size(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, batch: usize) -> usize;
    pub fn pg_glwe_trace(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_keys: *const u64, reverse: i32, d_c_in: *const u64, d_c_out: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_glwe_expand_workspace_size(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, count: usize) -> usize;
    pub fn pg_glwe_expand_coefficients(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_keys: *const u64, count: usize, d_c_in: *const u64, d_out: *mut u64, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_bfv_decryptor_create(table: *const PgNttTable, plain_modulus: u64, gamma: u64, out_: *mut *mut PgBfvDecryptor) -> i32;
    pub fn pg_bfv_decryptor_destroy(decryptor: *mut PgBfvDecryptor) -> i32;
    pub fn pg_bfv_decrypt_workspace_size(decryptor: *const PgBfvDecryptor, batch: usize) -> usize;
    pub fn pg_bfv_decrypt(decryptor: *const PgBfvDecryptor, k: u32, d_sk_ntt: *const u64, d_ct: *const u64, d_msg: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_glwe_encryptor_create(table: *const PgNttTable, sigma: f64, out_: *mut *mut PgGlweEncryptor) -> i32;
    pub fn pg_glwe_encryptor_destroy(encryptor: *mut PgGlweEncryptor) -> i32;
    pub fn pg_glwe_encrypt(encryptor: *const PgGlweEncryptor, k: u32, d_sk_ntt: *const u64, d_msg: *const u64, h_scale: *const u64, seed: u64, stream0: u64, d_ct: *mut u64, batch: usize, stream: *mut c_void) -> i32;
    pub fn pg_glwe_pk_encrypt(encryptor: *const PgGlweEncryptor, k: u32, d_pk: *const u64, d_msg: *const u64, h_scale: *const u64, seed: u64, stream0: u64, d_ct: *mut u64, batch: usize, stream: *mut c_void) -> i32;
    pub fn pg_ggsw_pk_encrypt_monomial(encryptor: *const PgGlweEncryptor, basis: *const PgGadgetBasis, k: u32, d_pk: *const u64, h_coeff_residues: *const u64, degree: usize, seed: u64, stream0: u64, d_ggsw: *mut u64, stream: *mut c_void) -> i32;
    pub fn pg_ext_product_noalloc(table: *const PgNttTable, basis: *const PgGadgetBasis, k: u32, d_glwe_in: *const u64, d_ggsw: *const u64, d_glwe_out: *mut u64, batch: usize, stream: *mut c_void) -> i32;
    pub fn pg_hybrid_ks_create(table: *const PgNttTable, L: u32, K: u32, alpha: u32, out_: *mut *mut PgHybridKs) -> i32;
    pub fn pg_hybrid_ks_destroy(ks: *mut PgHybridKs) -> i32;
    pub fn pg_hybrid_ks_dnum(ks: *const PgHybridKs) -> u32;
    pub fn pg_hybrid_ks_workspace_size(ks: *const PgHybridKs, k_in: u32, k_out: u32, batch: usize) -> usize;
    pub fn pg_key_switch_hybrid(ks: *const PgHybridKs, k_in: u32, k_out: u32, d_key: *const u64, d_c_in: *const u64, d_c_out: *mut u64, batch: usize, d_workspace: *mut c_void, workspace_bytes: usize, stream: *mut c_void) -> i32;
    pub fn pg_polymul_batch_create(tables: *const *const PgNttTable, table_count: u32, out_: *mut *mut PgPolymulBatch) -> i32;
    pub fn pg_polymul_batch_destroy(batch: *mut PgPolymulBatch) -> i32;
    pub fn pg_polymul_batch_reserve(batch: *mut PgPolymulBatch, rows: usize) -> i32;
    pub fn pg_polymul_batch_run(batch: *mut PgPolymulBatch, h_jobs: *const PgPolymulJob, count: usize, use_graph: i32, stream: *mut c_void) -> i32;
    pub fn pg_server_create(config: *const PgServerConfig, polymul_tables: *const *const PgNttTable, table_count: u32, out_: *mut *mut PgServer) -> i32;
    pub fn pg_server_destroy(server: *mut PgServer) -> i32;
    pub fn pg_server_register_key(server: *mut PgServer, kind: i32, table: *const PgNttTable, basis: *const PgGadgetBasis, k_in: u32, k_out: u32, d_key: *const u64, key_id: *mut u32) -> i32;
    pub fn pg_server_register_hybrid_key(server: *mut PgServer, ks: *const PgHybridKs, k_in: u32, k_out: u32, d_key: *const u64, key_id: *mut u32) -> i32;
    pub fn pg_server_submit(server: *mut PgServer, request: *const PgRequest, ticket: *mut u64) -> i32;
    pub fn pg_server_wait(server: *mut PgServer, ticket: u64, timeout_us: i64, latency_us: *mut f64) -> i32;
    pub fn pg_server_drain(server: *mut PgServer, timeout_us: i64) -> i32;
    pub fn pg_server_stats(server: *mut PgServer, out_: *mut PgServerStats, reset: i32) -> i32;
    pub fn pg_server_replay(server: *mut PgServer, requests: *const PgRequest, arrival_us: *const f64, count: usize, latency_us: *mut f64) -> i32;
    pub fn pg_fill_uniform(table: *const PgNttTable, d_out: *mut u64, polys: usize, seed: u64, stream0: u64, stream: *mut c_void) -> i32;
    pub fn pg_fill_uniform_host(seed: u64, stream_id: u64, q: u64, n: usize, h_out: *mut u64) -> i32;
}
