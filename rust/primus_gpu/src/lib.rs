//! `primus_gpu`: the B200 backend of primus' lattice-arithmetic path as a
//! drop-in for the `NttTable` / `DcrtTable` traits of `primus_ntt`
//! (`primus_ntt/src/ntt/mod.rs:20-117`, `primus_ntt/src/dcrt/mod.rs:17-129`).
//!
//! The tables live on the GPU (`pg_ntt_table_create`: twiddles resident in
//! HBM); the trait's slice methods take host slices, so each call copies the
//! slice in, runs the transform and copies it back (`pg_ntt_forward_host` /
//! `pg_ntt_inverse_host`).  Callers that keep their data on the device use the
//! batched entry points through [`DeviceBuffer`] and the inherent methods
//! below, which is where the GPU pays off.
//!
//! Errors: only construction fails, as in the reference (`NttError`); a failing
//! transform panics with the library's message, as the reference's
//! `assert!`s do on misuse.
//!
//! Status of this crate: not compiled here (the image that built the library
//! has no Rust toolchain).  It is meant to sit in the primus workspace as a
//! member beside `primus_ntt` (see `Cargo.toml`).
#![allow(clippy::missing_safety_doc)]

pub mod ffi;

use std::ffi::{CStr, c_void};
use std::ptr;

use primus_integer::{DataMut, RawData};
use primus_ntt::{DcrtTable, NttError, NttTable};
use primus_poly::{CrtPolynomial, DcrtPolynomial, NttPolynomial, Polynomial};
use primus_reduce::{FieldContext, Modulus};

/// The library's message for the last failed call on this thread.
pub fn last_error() -> String {
    unsafe { CStr::from_ptr(ffi::pg_last_error()) }.to_string_lossy().into_owned()
}

fn check(status: i32, what: &str) {
    if status != ffi::PG_OK {
        panic!("primus_gpu: {what}: {}", last_error());
    }
}

/// Status codes of `pg_ntt_table_create` as the reference's `NttError`
/// (`primus_ntt/src/error.rs:7-35`).
fn ntt_error(status: i32, log_n: u32, modulus: u64) -> NttError<u64> {
    match status {
        ffi::PG_ERR_NO_PRIMITIVE_ROOT => NttError::NoPrimitiveRoot { degree: 2u64 << log_n, modulus },
        ffi::PG_ERR_DEGREE_TOO_LARGE => NttError::DegreeTooLarge { degree: 1usize << log_n, modulus },
        _ => NttError::NttTableErr,
    }
}

/// A device array of `u64` owned by this process (freed on drop).
pub struct DeviceBuffer {
    ptr: *mut u64,
    len: usize,
}

unsafe impl Send for DeviceBuffer {}
unsafe impl Sync for DeviceBuffer {}

impl DeviceBuffer {
    pub fn new(len: usize) -> Self {
        let mut p: *mut c_void = ptr::null_mut();
        check(unsafe { ffi::pg_malloc(&mut p, len * 8) }, "pg_malloc");
        Self { ptr: p as *mut u64, len }
    }

    pub fn from_slice(h: &[u64]) -> Self {
        let b = Self::new(h.len());
        b.upload(h);
        b
    }

    pub fn upload(&self, h: &[u64]) {
        assert!(h.len() <= self.len);
        check(unsafe { ffi::pg_memcpy_h2d(self.ptr as *mut c_void, h.as_ptr() as *const c_void, h.len() * 8,
                                           ptr::null_mut()) }, "pg_memcpy_h2d");
        check(unsafe { ffi::pg_stream_synchronize(ptr::null_mut()) }, "pg_stream_synchronize");
    }

    pub fn download(&self, h: &mut [u64]) {
        assert!(h.len() <= self.len);
        check(unsafe { ffi::pg_memcpy_d2h(h.as_mut_ptr() as *mut c_void, self.ptr as *const c_void, h.len() * 8,
                                           ptr::null_mut()) }, "pg_memcpy_d2h");
        check(unsafe { ffi::pg_stream_synchronize(ptr::null_mut()) }, "pg_stream_synchronize");
    }

    pub fn as_ptr(&self) -> *const u64 {
        self.ptr
    }

    pub fn as_mut_ptr(&self) -> *mut u64 {
        self.ptr
    }

    pub fn len(&self) -> usize {
        self.len
    }

    pub fn is_empty(&self) -> bool {
        self.len == 0
    }
}

impl Drop for DeviceBuffer {
    fn drop(&mut self) {
        unsafe { ffi::pg_free(self.ptr as *mut c_void) };
    }
}

/// One prime's NTT table on the GPU: `UintNttTable` semantics
/// (`primus_ntt/src/ntt/primitive.rs`), minimal primitive root, bit-reversed
/// outputs, bit-exact lazy values.
pub struct GpuNttTable {
    raw: *mut ffi::PgNttTable,
    n: usize,
}

// tables are immutable after creation; calls on distinct buffers may run concurrently
unsafe impl Send for GpuNttTable {}
unsafe impl Sync for GpuNttTable {}

impl GpuNttTable {
    pub fn raw(&self) -> *const ffi::PgNttTable {
        self.raw
    }

    fn monomial_into(&self, values: &mut [u64], f: impl FnOnce(*mut u64) -> i32, what: &str) {
        assert_eq!(values.len(), self.n);
        let out = DeviceBuffer::new(self.n);
        check(f(out.as_mut_ptr()), what);
        out.download(values);
    }
}

impl Drop for GpuNttTable {
    fn drop(&mut self) {
        unsafe { ffi::pg_ntt_table_destroy(self.raw) };
    }
}

impl NttTable for GpuNttTable {
    type ValueT = u64;

    fn new<M>(log_n: u32, modulus: M) -> Result<Self, NttError<u64>>
    where
        M: FieldContext<u64>,
    {
        let q = modulus.value_unchecked();
        let mut raw = ptr::null_mut();
        match unsafe { ffi::pg_ntt_table_create(log_n, &q, 1, &mut raw) } {
            ffi::PG_OK => Ok(Self { raw, n: 1usize << log_n }),
            st => Err(ntt_error(st, log_n, q)),
        }
    }

    fn poly_length(&self) -> usize {
        self.n
    }

    fn transform_inplace<S: RawData<Elem = u64> + DataMut>(&self, mut poly: Polynomial<S>) -> NttPolynomial<S> {
        self.transform_slice(poly.0.as_mut_slice());
        NttPolynomial::new(poly.0)
    }

    fn inverse_transform_inplace<S: RawData<Elem = u64> + DataMut>(&self, mut values: NttPolynomial<S>) -> Polynomial<S> {
        self.inverse_transform_slice(values.0.as_mut_slice());
        Polynomial::new(values.0)
    }

    fn lazy_transform_slice(&self, poly: &mut [u64]) {
        assert_eq!(poly.len() % self.n, 0);
        check(unsafe { ffi::pg_ntt_forward_host(self.raw, poly.as_mut_ptr(), poly.len() / self.n, 1) },
              "lazy_transform_slice");
    }

    fn transform_slice(&self, poly: &mut [u64]) {
        assert_eq!(poly.len() % self.n, 0);
        check(unsafe { ffi::pg_ntt_forward_host(self.raw, poly.as_mut_ptr(), poly.len() / self.n, 0) },
              "transform_slice");
    }

    fn lazy_inverse_transform_slice(&self, values: &mut [u64]) {
        assert_eq!(values.len() % self.n, 0);
        check(unsafe { ffi::pg_ntt_inverse_host(self.raw, values.as_mut_ptr(), values.len() / self.n, 1) },
              "lazy_inverse_transform_slice");
    }

    fn inverse_transform_slice(&self, values: &mut [u64]) {
        assert_eq!(values.len() % self.n, 0);
        check(unsafe { ffi::pg_ntt_inverse_host(self.raw, values.as_mut_ptr(), values.len() / self.n, 0) },
              "inverse_transform_slice");
    }

    fn transform_monomial(&self, coeff: u64, degree: usize, values: &mut [u64]) {
        self.monomial_into(values, |d| unsafe { ffi::pg_ntt_monomial(self.raw, coeff, degree, d, ptr::null_mut()) },
                           "transform_monomial");
    }

    fn transform_coeff_one_monomial(&self, degree: usize, values: &mut [u64]) {
        self.monomial_into(values,
                           |d| unsafe { ffi::pg_ntt_coeff_one_monomial(self.raw, degree, d, ptr::null_mut()) },
                           "transform_coeff_one_monomial");
    }

    fn transform_coeff_minus_one_monomial(&self, degree: usize, values: &mut [u64]) {
        self.monomial_into(values,
                           |d| unsafe { ffi::pg_ntt_coeff_minus_one_monomial(self.raw, degree, d, ptr::null_mut()) },
                           "transform_coeff_minus_one_monomial");
    }
}

/// L primes' tables on the GPU (`UintCrtNttTable`, `primus_ntt/src/dcrt/primitive.rs`):
/// every transform is one launch over all L rows of every poly of the slice.
/// `ntt_tables()` / `iter()` are per-prime views over the same device arrays
/// (`pg_ntt_table_view`), owned by this table.
pub struct GpuDcrtTable {
    raw: *mut ffi::PgNttTable,
    views: Vec<GpuNttTable>,
    n: usize,
    moduli_count: usize,
}

unsafe impl Send for GpuDcrtTable {}
unsafe impl Sync for GpuDcrtTable {}

impl GpuDcrtTable {
    pub fn raw(&self) -> *const ffi::PgNttTable {
        self.raw
    }

    /// Times every kernel shape of this degree on `polys` seeded polys and keeps
    /// the fastest per mode in the table (`pg_ntt_autotune`).
    pub fn autotune(&mut self, polys: usize) -> ffi::PgNttTuning {
        let mut t = ffi::PgNttTuning::default();
        check(unsafe { ffi::pg_ntt_autotune(self.raw, polys, &mut t) }, "pg_ntt_autotune");
        t
    }

    /// Batched forward transform of `polys` polys resident on the device.
    pub fn forward_device(&self, data: &DeviceBuffer, polys: usize, lazy: bool, stream: *mut c_void) {
        assert!(polys * self.n * self.moduli_count <= data.len());
        check(unsafe { ffi::pg_ntt_forward(self.raw, data.as_mut_ptr(), polys, lazy as i32, stream) }, "pg_ntt_forward");
    }

    /// Batched inverse transform of `polys` polys resident on the device.
    pub fn inverse_device(&self, data: &DeviceBuffer, polys: usize, lazy: bool, stream: *mut c_void) {
        assert!(polys * self.n * self.moduli_count <= data.len());
        check(unsafe { ffi::pg_ntt_inverse(self.raw, data.as_mut_ptr(), polys, lazy as i32, stream) }, "pg_ntt_inverse");
    }

    /// Forward transform, product with an NTT-domain plaintext (Shoup-prepared
    /// quotients in `plain_q`) and inverse transform of `polys` polys in one
    /// launch (`pg_dcrt_polymul_ntt_plain`).
    pub fn polymul_ntt_plain(&self, data: &DeviceBuffer, plain: &DeviceBuffer, plain_q: &DeviceBuffer, polys: usize,
                             stream: *mut c_void) {
        check(unsafe {
            ffi::pg_dcrt_polymul_ntt_plain(self.raw, data.as_mut_ptr(), plain.as_ptr(), plain_q.as_ptr(), polys, stream)
        }, "pg_dcrt_polymul_ntt_plain");
    }
}

impl Drop for GpuDcrtTable {
    fn drop(&mut self) {
        // the views go first: they share the parent's device arrays
        self.views.clear();
        unsafe { ffi::pg_ntt_table_destroy(self.raw) };
    }
}

impl DcrtTable for GpuDcrtTable {
    type ValueT = u64;
    type NttTables = GpuNttTable;

    fn new<M>(log_n: u32, moduli: &[M]) -> Result<Self, NttError<u64>>
    where
        M: FieldContext<u64>,
    {
        let qs: Vec<u64> = moduli.iter().map(|m| m.value_unchecked()).collect();
        let mut raw = ptr::null_mut();
        let st = unsafe { ffi::pg_ntt_table_create(log_n, qs.as_ptr(), qs.len() as u32, &mut raw) };
        if st != ffi::PG_OK {
            // the first modulus without a root names the error, as the reference's per-modulus loop does
            let bad = qs.iter().copied().find(|&q| {
                let mut r = 0u64;
                unsafe { ffi::pg_minimal_primitive_root(log_n + 1, q, &mut r) != ffi::PG_OK }
            });
            return Err(ntt_error(st, log_n, bad.unwrap_or(qs.first().copied().unwrap_or(0))));
        }
        let mut views = Vec::with_capacity(qs.len());
        for i in 0..qs.len() as u32 {
            let mut v = ptr::null_mut();
            check(unsafe { ffi::pg_ntt_table_view(raw, i, 1, &mut v) }, "pg_ntt_table_view");
            views.push(GpuNttTable { raw: v, n: 1usize << log_n });
        }
        Ok(Self { raw, views, n: 1usize << log_n, moduli_count: qs.len() })
    }

    fn ntt_tables(&self) -> &[GpuNttTable] {
        &self.views
    }

    fn iter(&self) -> std::slice::Iter<'_, GpuNttTable> {
        self.views.iter()
    }

    fn poly_length(&self) -> usize {
        self.n
    }

    fn moduli_count(&self) -> usize {
        self.moduli_count
    }

    fn crt_poly_length(&self) -> usize {
        self.n * self.moduli_count
    }

    fn transform_inplace<S: RawData<Elem = u64> + DataMut>(&self, mut crt_poly: CrtPolynomial<S>) -> DcrtPolynomial<S> {
        self.transform_slice(crt_poly.0.as_mut_slice());
        DcrtPolynomial::new(crt_poly.0)
    }

    fn inverse_transform_inplace<S: RawData<Elem = u64> + DataMut>(&self, mut dcrt_poly: DcrtPolynomial<S>) -> CrtPolynomial<S> {
        self.inverse_transform_slice(dcrt_poly.0.as_mut_slice());
        CrtPolynomial::new(dcrt_poly.0)
    }

    fn lazy_transform_slice(&self, poly: &mut [u64]) {
        let polys = poly.len() / self.crt_poly_length();
        assert_eq!(polys * self.crt_poly_length(), poly.len());
        check(unsafe { ffi::pg_ntt_forward_host(self.raw, poly.as_mut_ptr(), polys, 1) }, "lazy_transform_slice");
    }

    fn transform_slice(&self, poly: &mut [u64]) {
        let polys = poly.len() / self.crt_poly_length();
        assert_eq!(polys * self.crt_poly_length(), poly.len());
        check(unsafe { ffi::pg_ntt_forward_host(self.raw, poly.as_mut_ptr(), polys, 0) }, "transform_slice");
    }

    fn lazy_inverse_transform_slice(&self, poly: &mut [u64]) {
        let polys = poly.len() / self.crt_poly_length();
        assert_eq!(polys * self.crt_poly_length(), poly.len());
        check(unsafe { ffi::pg_ntt_inverse_host(self.raw, poly.as_mut_ptr(), polys, 1) },
              "lazy_inverse_transform_slice");
    }

    fn inverse_transform_slice(&self, poly: &mut [u64]) {
        let polys = poly.len() / self.crt_poly_length();
        assert_eq!(polys * self.crt_poly_length(), poly.len());
        check(unsafe { ffi::pg_ntt_inverse_host(self.raw, poly.as_mut_ptr(), polys, 0) }, "inverse_transform_slice");
    }

    // one launch for all limbs instead of the trait's per-limb default
    fn transform_monomial(&self, coeff: u64, degree: usize, values: &mut [u64]) {
        assert_eq!(values.len(), self.crt_poly_length());
        let out = DeviceBuffer::new(values.len());
        check(unsafe { ffi::pg_ntt_monomial(self.raw, coeff, degree, out.as_mut_ptr(), ptr::null_mut()) },
              "transform_monomial");
        out.download(values);
    }

    fn transform_coeff_one_monomial(&self, degree: usize, values: &mut [u64]) {
        assert_eq!(values.len(), self.crt_poly_length());
        let out = DeviceBuffer::new(values.len());
        check(unsafe { ffi::pg_ntt_coeff_one_monomial(self.raw, degree, out.as_mut_ptr(), ptr::null_mut()) },
              "transform_coeff_one_monomial");
        out.download(values);
    }

    fn transform_coeff_minus_one_monomial(&self, degree: usize, values: &mut [u64]) {
        assert_eq!(values.len(), self.crt_poly_length());
        let out = DeviceBuffer::new(values.len());
        check(unsafe { ffi::pg_ntt_coeff_minus_one_monomial(self.raw, degree, out.as_mut_ptr(), ptr::null_mut()) },
              "transform_coeff_minus_one_monomial");
        out.download(values);
    }
}

/// RNS base of a table's moduli (`RNSBase`, `primus_rns/src/base.rs`).
pub struct GpuRnsBase {
    raw: *mut ffi::PgRnsBase,
}

unsafe impl Send for GpuRnsBase {}
unsafe impl Sync for GpuRnsBase {}

impl GpuRnsBase {
    /// `RNSBase::new`: `PG_ERR_NOT_COPRIME` is the reference's `RNSError::CoPrimeError`.
    pub fn new(moduli: &[u64]) -> Result<Self, i32> {
        let mut raw = ptr::null_mut();
        match unsafe { ffi::pg_rns_base_create(moduli.as_ptr(), moduli.len() as u32, &mut raw) } {
            ffi::PG_OK => Ok(Self { raw }),
            st => Err(st),
        }
    }

    pub fn raw(&self) -> *const ffi::PgRnsBase {
        self.raw
    }
}

impl Drop for GpuRnsBase {
    fn drop(&mut self) {
        unsafe { ffi::pg_rns_base_destroy(self.raw) };
    }
}

/// Approximate signed gadget basis (`BigUintApproxSignedBasis::new`,
/// `primus_decompose/src/big_integer/basis.rs:34-193`).
pub struct GpuGadgetBasis {
    raw: *mut ffi::PgGadgetBasis,
}

unsafe impl Send for GpuGadgetBasis {}
unsafe impl Sync for GpuGadgetBasis {}

impl GpuGadgetBasis {
    /// `reverse_length`: `None` for the full length floor(bits(Q) / log_basis).
    pub fn new(base: &GpuRnsBase, log_basis: u32, reverse_length: Option<u32>) -> Result<Self, i32> {
        let mut raw = ptr::null_mut();
        let rl = reverse_length.map(|r| r as i32).unwrap_or(-1);
        match unsafe { ffi::pg_gadget_basis_create(base.raw, log_basis, rl, &mut raw) } {
            ffi::PG_OK => Ok(Self { raw }),
            st => Err(st),
        }
    }

    pub fn raw(&self) -> *const ffi::PgGadgetBasis {
        self.raw
    }
}

impl Drop for GpuGadgetBasis {
    fn drop(&mut self) {
        unsafe { ffi::pg_gadget_basis_destroy(self.raw) };
    }
}

/// `CrtGlwe::mul_dcrt_ggsw_inplace` (`primus_lattice/src/glwe/crt.rs:202-229`)
/// for a batch of `batch` GLWE ciphertexts `[batch][k+1][L][N]` (coefficient
/// form) against one GGSW `[k+1][d][k+1][L][N]` (NTT domain); outputs in the
/// NTT domain.  Scratch comes from the library's pool.
pub fn ext_product(table: &GpuDcrtTable, basis: &GpuGadgetBasis, k: u32, glwe_in: &DeviceBuffer, ggsw: &DeviceBuffer,
                   glwe_out: &DeviceBuffer, batch: usize, stream: *mut c_void) {
    check(unsafe {
        ffi::pg_ext_product(table.raw, basis.raw, k, glwe_in.as_ptr(), ggsw.as_ptr(), glwe_out.as_mut_ptr(), batch,
                            ptr::null_mut(), 0, stream)
    }, "pg_ext_product");
}

/// `CrtGlweKeySwitchingKey::key_swithching_inplace` (`primus_fhe_core/src/key_switch.rs:79-128`)
/// for a batch: key `[k_in][d][k_out+1][L][N]`, inputs `[batch][k_in+1][L][N]`
/// (coefficient form), outputs `[batch][k_out+1][L][N]` (NTT domain).
pub fn key_switch(table: &GpuDcrtTable, basis: &GpuGadgetBasis, k_in: u32, k_out: u32, key: &DeviceBuffer,
                  c_in: &DeviceBuffer, c_out: &DeviceBuffer, batch: usize, stream: *mut c_void) {
    check(unsafe {
        ffi::pg_key_switch(table.raw, basis.raw, k_in, k_out, key.as_ptr(), c_in.as_ptr(), c_out.as_mut_ptr(), batch,
                           ptr::null_mut(), 0, stream)
    }, "pg_key_switch");
}
