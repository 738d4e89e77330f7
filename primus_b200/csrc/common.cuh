// Device-side modular arithmetic shared by every kernel of libprimus_gpu.
//
// All arithmetic is exact unsigned 64/128-bit integer math.  The Shoup lazy
// multiply is the reference's ShoupFactor::lazy_factor_mul_modulo
// (primus_factor/src/shoup_factor/mod.rs:108-113): w*b - q*hi64(w'*b), which
// lands in [0, 2q) for any 64-bit b.  Because the same formula is evaluated on
// the same operands, lazy intermediate values match the CPU path bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define PG_DEV __device__ __forceinline__
#define PG_HD __host__ __device__ __forceinline__

namespace pg {

// hi 64 bits of a 64x64 product
PG_DEV uint64_t mulhi64(uint64_t a, uint64_t b) { return __umul64hi(a, b); }

// Shoup lazy multiply: result in [0, 2q).  Hand-scheduled in 32-bit pieces:
// hw = hi64(w' * b) with one carry chain, then w*b - q*hw mod 2^64 computed as
// w*b + (2^64 - q)*hw with wide multiply-adds (no separate 64-bit subtract).
// nq = 2^64 - q is passed in precomputed.
PG_DEV uint64_t shoup_lazy_nq(uint64_t w, uint64_t wq, uint64_t b, uint64_t nq) {
    uint64_t r;
    asm("{\n\t"
        ".reg .u32 a0, a1, b0, b1, t, m0, m1, s0, s1, c2, w0, w1, n0, n1, h0, h1, r0, r1;\n\t"
        ".reg .u64 m, hw, acc, tz;\n\t"
        "mov.b64 {a0, a1}, %2;\n\t"
        "mov.b64 {b0, b1}, %3;\n\t"
        "mul.hi.u32 t, a0, b0;\n\t"
        "cvt.u64.u32 tz, t;\n\t"
        "mad.wide.u32 m, a0, b1, tz;\n\t"
        "mov.b64 {m0, m1}, m;\n\t"
        "mad.lo.cc.u32 s0, a1, b0, m0;\n\t"
        "madc.hi.cc.u32 s1, a1, b0, m1;\n\t"
        "addc.u32 c2, 0, 0;\n\t"
        "mov.b64 m, {s1, c2};\n\t"
        "mad.wide.u32 hw, a1, b1, m;\n\t"
        "mov.b64 {h0, h1}, hw;\n\t"
        "mov.b64 {w0, w1}, %1;\n\t"
        "mov.b64 {n0, n1}, %4;\n\t"
        "mul.wide.u32 acc, w0, b0;\n\t"
        "mad.wide.u32 acc, n0, h0, acc;\n\t"
        "mov.b64 {r0, r1}, acc;\n\t"
        "mad.lo.u32 r1, w0, b1, r1;\n\t"
        "mad.lo.u32 r1, w1, b0, r1;\n\t"
        "mad.lo.u32 r1, n0, h1, r1;\n\t"
        "mad.lo.u32 r1, n1, h0, r1;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "}"
        : "=l"(r)
        : "l"(w), "l"(wq), "l"(b), "l"(nq));
    return r;
}

// The same product with the quotient estimate formed without the high word of
// the low 32x32 partial product (one multiply fewer): the estimate is the exact
// Shoup quotient or one less, so the result lies in [0, 3q).  Used only inside
// transforms whose outputs are reduced to canonical values at the end.
PG_DEV uint64_t shoup_lazy3_nq(uint64_t w, uint64_t wq, uint64_t b, uint64_t nq) {
    uint64_t r;
    asm("{\n\t"
        ".reg .u32 a0, a1, b0, b1, m0, m1, s0, s1, c2, w0, w1, n0, n1, h0, h1, r0, r1;\n\t"
        ".reg .u64 m, hw, acc;\n\t"
        "mov.b64 {a0, a1}, %2;\n\t"
        "mov.b64 {b0, b1}, %3;\n\t"
        "mul.wide.u32 m, a0, b1;\n\t"
        "mov.b64 {m0, m1}, m;\n\t"
        "mad.lo.cc.u32 s0, a1, b0, m0;\n\t"
        "madc.hi.cc.u32 s1, a1, b0, m1;\n\t"
        "addc.u32 c2, 0, 0;\n\t"
        "mov.b64 m, {s1, c2};\n\t"
        "mad.wide.u32 hw, a1, b1, m;\n\t"
        "mov.b64 {h0, h1}, hw;\n\t"
        "mov.b64 {w0, w1}, %1;\n\t"
        "mov.b64 {n0, n1}, %4;\n\t"
        "mul.wide.u32 acc, w0, b0;\n\t"
        "mad.wide.u32 acc, n0, h0, acc;\n\t"
        "mov.b64 {r0, r1}, acc;\n\t"
        "mad.lo.u32 r1, w0, b1, r1;\n\t"
        "mad.lo.u32 r1, w1, b0, r1;\n\t"
        "mad.lo.u32 r1, n0, h1, r1;\n\t"
        "mad.lo.u32 r1, n1, h0, r1;\n\t"
        "mov.b64 %0, {r0, r1};\n\t"
        "}"
        : "=l"(r)
        : "l"(w), "l"(wq), "l"(b), "l"(nq));
    return r;
}

PG_DEV uint64_t shoup_lazy(uint64_t w, uint64_t wq, uint64_t b, uint64_t q) { return shoup_lazy_nq(w, wq, b, 0 - q); }

// Shoup full multiply: result in [0, q)
PG_DEV uint64_t shoup_mul(uint64_t w, uint64_t wq, uint64_t b, uint64_t q) {
    uint64_t t = shoup_lazy(w, wq, b, q);
    return t >= q ? t - q : t;
}

PG_DEV uint64_t reduce_once(uint64_t v, uint64_t m) { return v >= m ? v - m : v; }

// Loads through explicitly global addresses.  A generic pointer may point into
// shared memory, so a generic load that follows a store to shared memory in
// program order cannot be issued before that store: a loop that stages global
// values through shared memory would wait one full memory latency per element.
// ld_stream (ld.global.cg, cached in L2 only) reads data the kernel streams
// once; ld_table (ld.global.nc, the read-only path) reads tables no kernel
// writes while it runs.
PG_DEV uint64_t ld_stream(const uint64_t* p) { return __ldcg((const unsigned long long*)p); }
PG_DEV uint64_t ld_table(const uint64_t* p) { return __ldg((const unsigned long long*)p); }
// ld.global.ca: cached in L1 too, for per-thread runs of consecutive words
PG_DEV uint64_t ld_cached(const uint64_t* p) { return __ldca((const unsigned long long*)p); }

// UintModulus::reduce_add (primus_modulus/src/unsigned_integer/ops.rs:34-41)
PG_DEV uint64_t add_mod(uint64_t a, uint64_t b, uint64_t m) {
    uint64_t s = a + b;
    return s >= m ? s - m : s;
}

// UintModulus::reduce_sub (ops.rs:81-87)
PG_DEV uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t m) { return b > a ? a - b + m : a - b; }

// UintModulus::reduce_neg (ops.rs:105-111)
PG_DEV uint64_t neg_mod(uint64_t a, uint64_t m) { return a == 0 ? 0 : m - a; }

// Exact (a*b + c) mod q for q < 2^62 via Barrett with ratio = floor(2^128/q)
// (BarrettModulus, primus_modulus/src/barrett/ops.rs:41-76, 342-355).  The
// output is canonical, so it equals the CPU path's value for any exact method.
struct Barrett {
    uint64_t q, r0, r1;  // ratio = r1*2^64 + r0
    // floor(2^(n+62) / q) with n = bitlen(q) when 2 <= n <= 62, else 0: the
    // factor of the shifted-operand Barrett reduction (barrett_mul)
    uint64_t mu;
};

PG_DEV uint64_t barrett_reduce_2limb(uint64_t lo, uint64_t hi, const Barrett& m) {
    uint64_t ah = mulhi64(lo, m.r0);
    // b = lo*r1 + ah (128-bit)
    uint64_t b0 = lo * m.r1;
    uint64_t b1 = mulhi64(lo, m.r1);
    b0 += ah;
    b1 += (b0 < ah);
    // c = hi*r0 (128-bit)
    uint64_t c0 = hi * m.r0;
    uint64_t c1 = mulhi64(hi, m.r0);
    uint64_t s = b0 + c0;
    uint64_t carry = s < b0;
    uint64_t qq = hi * m.r1 + b1 + c1 + carry;
    uint64_t r = lo - qq * m.q;
    // lazy result is in [0, 3q) at worst for q < 2^62; two conditional subtracts
    r = r >= m.q ? r - m.q : r;
    return r >= m.q ? r - m.q : r;
}

// x mod q for x = hi*2^64 + lo < 2^(n+62), n = bitlen(q) <= 62 (m.mu != 0).
// Barrett's reduction on the operand shifted right by n-2 bits (Barrett 1986;
// the pre-shifted form of Harvey's modular-multiplication analysis):
// c = x >> (n-2) < 2^64 and est = floor(c * mu / 2^64) never exceeds x/q and
// falls short of it by less than 2.5 (x - c*2^(n-2) < 2^(n-2) <= q/2 and
// c*(2^(n+62)/q - mu)/2^64 < 1), so x - est*q lies in [0, 3q), below 2^64,
// and two conditional subtractions make it canonical.  Four 64-bit
// multiplies per product instead of the nine of the 128-bit ratio form.
PG_DEV uint64_t barrett_reduce_shifted(uint64_t lo, uint64_t hi, const Barrett& m) {
    const uint32_t s = 62 - __clzll(m.q);  // n - 2, in [0, 60]
    const uint64_t c = (lo >> s) | ((hi << 1) << (63 - s));
    const uint64_t est = mulhi64(c, m.mu);
    uint64_t r = lo - est * m.q;
    r = r >= m.q ? r - m.q : r;
    return r >= m.q ? r - m.q : r;
}

// any 128-bit x mod q: the shifted form (four multiplies) when x < 2^(n+62),
// which holds for sums of up to 2^(62-n) products of residues, else the
// 128-bit ratio form; the same canonical residue either way
PG_DEV uint64_t barrett_reduce_128(uint64_t lo, uint64_t hi, const Barrett& m) {
    if (m.mu && (hi >> (62 - __clzll(m.q))) == 0) return barrett_reduce_shifted(lo, hi, m);
    return barrett_reduce_2limb(lo, hi, m);
}

PG_DEV uint64_t barrett_mul(uint64_t a, uint64_t b, const Barrett& m) {
    const uint64_t lo = a * b, hi = mulhi64(a, b);
    return m.mu ? barrett_reduce_shifted(lo, hi, m) : barrett_reduce_2limb(lo, hi, m);
}

PG_DEV uint64_t barrett_mul_add(uint64_t a, uint64_t b, uint64_t c, const Barrett& m) {
    uint64_t lo = a * b;
    uint64_t hi = mulhi64(a, b);
    lo += c;
    hi += (lo < c);
    return m.mu ? barrett_reduce_shifted(lo, hi, m) : barrett_reduce_2limb(lo, hi, m);
}

// Counter-based seeded generator (identical to the host generator): a 64-bit
// hash of (seed, stream, index, attempt); uniform values below q by rejection
// on the top bitlen(q-1) bits.
PG_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

PG_HD uint64_t hash64(uint64_t seed, uint64_t stream, uint64_t index, uint64_t attempt) {
    uint64_t h = mix64(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull);
    h = mix64(h ^ (stream * 0xD1B54A32D192ED03ull));
    h = mix64(h ^ (index * 0xA0761D6478BD642Full) ^ (attempt * 0xE7037ED1A0B428DBull));
    return h;
}

PG_DEV uint64_t uniform_at(uint64_t seed, uint64_t stream, uint64_t index, uint64_t q) {
    if (q <= 1) return 0;
    int bits = 64 - __clzll(q - 1);
    // rejection accepts with probability > 1/2; 64 attempts bound the loop
    for (uint64_t attempt = 0; attempt < 64; ++attempt) {
        uint64_t v = hash64(seed, stream, index, attempt) >> (64 - bits);
        if (v < q) return v;
    }
    return 0;
}

}  // namespace pg
