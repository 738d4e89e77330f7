// Shared NTT kernel templates (forward / inverse / fused round trip) and their
// launchers, included by ntt.cu (default dispatch) and ntt_variants.cu (the
// alternative shapes the autotuner times).
//
// Negacyclic NTT / INTT kernels for sm_100a.
//
// Semantics: the reference's UintNttTable (primus_ntt/src/ntt/primitive.rs).
//   forward  (lazy_transform_slice :211-232): for gap = N/2 .. 1, chunk c of
//            size 2*gap uses root_powers[2^s + c] (s = stage); Harvey
//            butterfly u = x mod 2q; v = w*y (Shoup lazy); x = u+v; y = u+2q-v.
//   inverse  (lazy_inverse_transform_slice :246-286): for gap = 1 .. N/4,
//            GS butterfly with inv_root_powers read sequentially; the last
//            stage (gap N/2) is fused with the N^-1 scaling.
// Every butterfly is evaluated with the reference's formula on the same
// operands and stages run in the reference's order, so lazy outputs match the
// CPU values bit for bit.  Only the assignment of butterflies to threads
// differs.
//
// Layout and schedule (B200):
//   * N <= 2^13: one CTA owns one row (or several small rows) in shared memory.
//     Each thread holds E = 2^LOG_E elements in registers and runs LOG_E stages
//     per round; rounds exchange through padded shared memory (index i is
//     stored at i + i/16, which keeps 64-bit accesses within two-way bank
//     conflicts for every round).
//   * N = 2^14 .. 2^16: a thread-block cluster of C = N / M CTAs owns one row
//     (512 KiB at N = 2^16) in distributed shared memory, each CTA a block of
//     M = 2^LOG_M elements (4096 by default).  Forward: each thread takes one
//     column {gt + j N/E} (coalesced HBM reads), runs the first LOG_E stages in
//     registers and scatters the results to the CTAs owning the blocks
//     (st.shared::cluster); the remaining stages run as local rounds.  Inverse
//     mirrors this.  A row is read from and written to HBM exactly once, also
//     for the fused fwd -> x plain -> inv round trip.
#pragma once

#include <cooperative_groups.h>

#include "internal.hpp"

namespace cg = cooperative_groups;

namespace pg {

PG_DEV int padi(int i) { return i + (i >> 4); }

// a signed gadget digit (stored as digit < basis) lifted mod q:
// RNSBase::wrapping_decompose_small_values_inplace (primus_rns/src/base.rs:201-231);
// half = 2 for basis 2 (both digits stay), else (basis + 1) / 2
PG_DEV uint64_t lift_digit(uint64_t v, uint64_t q, uint64_t basis, uint64_t half) {
    return v < half ? v : v + (q - basis);
}
__host__ __device__ constexpr int padded(int m) { return m + (m >> 4); }

template <int V>
struct IC {
    static constexpr int value = V;
};

// compile-time loop: f(IC<B>), f(IC<B+1>), ..., f(IC<E_-1>); every index is a
// constant, so register arrays indexed by it stay in registers
template <int B, int E_, typename F>
PG_DEV void static_for(F&& f) {
    if constexpr (B < E_) {
        f(IC<B>{});
        static_for<B + 1, E_>(f);
    }
}

// Harvey forward butterfly; x, y in [0, 4q) -> [0, 4q).  nq = 2^64 - q.
PG_DEV void fwd_bfly(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q2, uint64_t nq) {
    uint64_t u = x >= q2 ? x - q2 : x;
    uint64_t v = shoup_lazy_nq(w.x, w.y, y, nq);
    x = u + v;
    y = u + q2 - v;
}

// Forward butterfly without the u = x mod 2q step.  Used only where the
// canonical result is returned (transform_slice, the fused round trip): the
// bound grows by 2q per stage, so after log2(N) <= 16 stages from [0, 4q) the
// values stay below 52q < 2^64 for q < 2^58 (v below 3q from the one-multiply-
// shorter Shoup estimate, so the bound grows by 3q per stage from 4q), and the
// final canonical reduction yields the same residues as the Harvey schedule.
PG_DEV void fwd_bfly_fast(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q2, uint64_t nq) {
    const uint64_t q3 = q2 + (q2 >> 1);
    uint64_t u = x;
    uint64_t v = shoup_lazy3_nq(w.x, w.y, y, nq);
    x = u + v;
    y = u + q3 - v;
}

// Gentleman-Sande inverse butterfly; x, y in [0, 2q) -> [0, 2q)
PG_DEV void inv_bfly(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q2, uint64_t nq) {
    uint64_t u = x, v = y;
    uint64_t s = u + v;
    x = s >= q2 ? s - q2 : s;
    y = shoup_lazy_nq(w.x, w.y, u + q2 - v, nq);
}

// Inverse butterfly without the x reduction, for inputs below `bnd` (a power-of-two
// multiple of 2q known at compile time): x = u + v (< 2 bnd), y = w (u + bnd - v)
// in [0, 3q) (one-multiply-shorter Shoup estimate; 3q is below the next stage's
// bound 2 bnd >= 4q).  Used only where the result is canonical (the inverse
// always is) and every q < 2^50, so that the unreduced sums stay below 2^64
// (see inv_round).
PG_DEV void inv_bfly_fast(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t bnd, uint64_t nq) {
    uint64_t u = x, v = y;
    x = u + v;
    y = shoup_lazy3_nq(w.x, w.y, u + bnd - v, nq);
}

// Last inverse stage fused with N^-1: x = N^-1 (u+v), y = (w N^-1)(u+bnd-v),
// canonical; inputs below bnd (2q on the exact schedule)
PG_DEV void inv_last_bfly(uint64_t& x, uint64_t& y, const ulonglong2 s, const ulonglong2 sr, uint64_t q,
                          uint64_t nq, uint64_t bnd) {
    uint64_t u = x, v = y;
    uint64_t a = shoup_lazy_nq(s.x, s.y, u + v, nq);
    uint64_t b = shoup_lazy_nq(sr.x, sr.y, u + bnd - v, nq);
    x = a >= q ? a - q : a;
    y = b >= q ? b - q : b;
}

// Stage around which the unreduced inverse schedule reduces its values once: the
// round that contains this stage first reduces its elements to [0, q).  Before
// it values stay below 2^9 q; after it below 2^12 q (< 2^62 for q < 2^50).
constexpr int kFastInvReduceStage = 8;

// any 64-bit v -> v mod q, using floor(2^64/q) (the high word of the Barrett ratio)
PG_DEV uint64_t reduce_full(uint64_t v, uint64_t q, uint64_t inv64, uint64_t nq) {
    uint64_t r = v + nq * mulhi64(inv64, v);
    return r >= q ? r - q : r;
}

PG_DEV uint64_t canon4(uint64_t v, uint64_t q, uint64_t q2) {
    v = v >= q2 ? v - q2 : v;
    return v >= q ? v - q : v;
}

// ---------------------------------------------------------------------------
// FP64 schedule (kSchedFp64, every q < 2^50).  The B200 FP64 pipe issues as
// many operations per clock as the integer multiply pipe and is idle in the
// integer schedules, and a double holds every integer below 2^53 exactly, so
// residues travel as doubles holding signed integers and every operation
// below is exact (each result is an integer of magnitude below 2^53, which
// round-to-nearest reproduces).  Register and shared-memory words keep the
// double's bit pattern.  Twiddle tables hold wq = w / q correctly rounded
// (wq < 1 because w < q), 8 bytes per twiddle; tw_fp recovers w from it.
//
// fmulmod(y, w, wq, q) = w y mod q in (-0.75 q, 0.75 q) for |y| < 2^51:
//   t  = fma(y, wq, 1.5*2^52) rounds y*wq to the nearest integer (|y wq| < 2^51
//        keeps t in [2^52, 2^53), where doubles are the integers), qt = t - 1.5*2^52;
//        |qt - y w/q| <= 1/2 + |y| 2^-53 < 3/4.
//   ph = fl(qt q), pl = qt q - ph exactly (the error of a product, by fma);
//        |qt| < 2^51 so |ph| < 2^101 and |pl| <= 2^47.
//   r  = fma(w, y, -ph) = (w y - qt q) + pl exactly: |w y - qt q| < 0.75 q and
//        |pl| <= 2^47, so the exact value is an integer below 2^53.
//   r - pl = w y - qt q, exact.
// freduce(x, q, qinv) = x - rint(x qinv) q in [-q/2 - 1, q/2 + 1] for |x| < 2^53.
// ---------------------------------------------------------------------------
constexpr double kMagic52 = 6755399441055744.0;  // 1.5 * 2^52
constexpr double kTwo52 = 4503599627370496.0;    // 2^52

PG_DEV double as_f(uint64_t b) { return __longlong_as_double((long long)b); }
PG_DEV uint64_t as_u(double d) { return (uint64_t)__double_as_longlong(d); }
// exact conversions of integers in [0, 2^52)
PG_DEV double u52_to_f(uint64_t v) { return __dsub_rn(as_f(v | 0x4330000000000000ull), kTwo52); }
PG_DEV uint64_t f_to_u52(double d) { return as_u(__dadd_rn(d, kTwo52)) & 0xFFFFFFFFFFFFFull; }

PG_DEV double fmulmod(double y, double w, double wq, double q) {
    const double qt = __dsub_rn(__fma_rn(y, wq, kMagic52), kMagic52);
    const double ph = __dmul_rn(qt, q);
    const double pl = __fma_rn(qt, q, -ph);
    const double r = __fma_rn(w, y, -ph);
    return __dsub_rn(r, pl);
}

PG_DEV double freduce(double x, double q, double qinv) {
    const double qt = __dsub_rn(__fma_rn(x, qinv, kMagic52), kMagic52);
    return __fma_rn(-qt, q, x);
}

// x in (-q, q) -> [0, q)
PG_DEV double fcanon(double x, double q) { return x < 0.0 ? __dadd_rn(x, q) : x; }

// table entry wq = w / q (correctly rounded) -> (w, wq) as double bit patterns.
// |wq - w/q| <= 2^-53 so |wq q - w| <= q 2^-53 < 1/8 for q < 2^50: rounding
// wq q to the nearest integer (by the 1.5 * 2^52 constant) gives w exactly.
PG_DEV ulonglong2 tw_fp(double wq, double q) {
    const double w = __dsub_rn(__fma_rn(wq, q, kMagic52), kMagic52);
    return make_ulonglong2(as_u(w), as_u(wq));
}

// Cooley-Tukey forward butterfly: (u + w y, u - w y).  RU reduces u first.
// Inputs below 2q + 2 in magnitude; with u reduced at least every other stage
// (the stages of even bit index p) the outputs stay below 2q + 2: a reducing
// stage gives at most q/2 + 1 + 0.75 q, the next one adds at most 0.75 q.
template <bool RU>
PG_DEV void fwd_bfly_fp(uint64_t& x, uint64_t& y, const ulonglong2 w, double q, double qinv) {
    double u = as_f(x);
    if constexpr (RU) u = freduce(u, q, qinv);
    const double v = fmulmod(as_f(y), as_f(w.x), as_f(w.y), q);
    x = as_u(__dadd_rn(u, v));
    y = as_u(__dsub_rn(u, v));
}

// Gentleman-Sande inverse butterfly: (reduce(u + v), w (u - v)); inputs below
// q in magnitude (u - v below 2q < 2^51), outputs below 0.75 q.
PG_DEV void inv_bfly_fp(uint64_t& x, uint64_t& y, const ulonglong2 w, double q, double qinv) {
    const double u = as_f(x), v = as_f(y);
    x = as_u(freduce(__dadd_rn(u, v), q, qinv));
    y = as_u(fmulmod(__dsub_rn(u, v), as_f(w.x), as_f(w.y), q));
}

// Two Gentleman-Sande stages at once on (x0, x1, x2, x3) (stage p pairs (x0, x1)
// with wa and (x2, x3) with wb, stage p+1 pairs the results (0, 2) and (1, 3)
// with wc), inputs below q in magnitude: the stage-p sums (< 2q) are not
// reduced; the stage-(p+1) sums and the difference s01 - s23 (< 4q) are, so
// every product's input stays below 2^51 and the outputs below 0.75 q.
// 41 FP64 operations for four butterflies instead of 44.
PG_DEV void inv_bfly4_fp(uint64_t& x0, uint64_t& x1, uint64_t& x2, uint64_t& x3, const ulonglong2 wa,
                         const ulonglong2 wb, const ulonglong2 wc, double q, double qinv) {
    const double a0 = as_f(x0), a1 = as_f(x1), a2 = as_f(x2), a3 = as_f(x3);
    const double s01 = __dadd_rn(a0, a1), s23 = __dadd_rn(a2, a3);
    const double d01 = fmulmod(__dsub_rn(a0, a1), as_f(wa.x), as_f(wa.y), q);
    const double d23 = fmulmod(__dsub_rn(a2, a3), as_f(wb.x), as_f(wb.y), q);
    x0 = as_u(freduce(__dadd_rn(s01, s23), q, qinv));
    x2 = as_u(fmulmod(freduce(__dsub_rn(s01, s23), q, qinv), as_f(wc.x), as_f(wc.y), q));
    x1 = as_u(freduce(__dadd_rn(d01, d23), q, qinv));
    x3 = as_u(fmulmod(__dsub_rn(d01, d23), as_f(wc.x), as_f(wc.y), q));
}

// last inverse stage fused with N^-1; writes canonical integers (not doubles)
PG_DEV void inv_last_bfly_fp(uint64_t& x, uint64_t& y, const ulonglong2 s, const ulonglong2 sr, double q) {
    const double u = as_f(x), v = as_f(y);
    x = f_to_u52(fcanon(fmulmod(__dadd_rn(u, v), as_f(s.x), as_f(s.y), q), q));
    y = f_to_u52(fcanon(fmulmod(__dsub_rn(u, v), as_f(sr.x), as_f(sr.y), q), q));
}

// insert LOG_E zero bits at bit position g into t
template <int LOG_E>
PG_DEV uint32_t group_base(uint32_t t, int g) {
    uint32_t lo = t & ((1u << g) - 1u);
    return ((t >> g) << (g + LOG_E)) | lo;
}

// two consecutive twiddles (value, quotient, value, quotient) with one 256-bit
// load; p must be 32-byte aligned (callers guarantee an even index)
PG_DEV void ldg_tw2(const ulonglong2* p, ulonglong2& a, ulonglong2& b) {
    uint64_t a0, a1, b0, b1;
    asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a0), "=l"(a1), "=l"(b0), "=l"(b1) : "l"(p));
    a = make_ulonglong2(a0, a1);
    b = make_ulonglong2(b0, b1);
}

// FP64 tables: 2 (16-byte aligned) or 4 (32-byte aligned) consecutive quotients
PG_DEV void ldg_f2(const double* p, double& a, double& b) {
    asm("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "l"(p));
}
PG_DEV void ldg_f4(const double* p, double (&w)[4]) {
    uint64_t b0, b1, b2, b3;
    asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(b0), "=l"(b1), "=l"(b2), "=l"(b3) : "l"(p));
    w[0] = as_f(b0);
    w[1] = as_f(b1);
    w[2] = as_f(b2);
    w[3] = as_f(b3);
}

// One forward round over register group x (x[jj] is local index base + (jj << G)
// of a 2^LOG_M block).  Stage bits P_HI down to P_LO; stage bit p is block stage
// sp = LOG_M-1-p and uses tw[(tw_base << sp) + (i >> (p+1))], tw_base = C + rank
// for a cluster block (1 for a whole row).  When a stage needs two or more
// twiddles their first index is a multiple of their count, so they are fetched
// in 32-byte pieces (two integer or four FP64 twiddles).
// K: 0 = exact schedule, 1 = fast integer schedule, 2 = FP64 schedule (then q2
// and nq carry the bit patterns of q and 1/q as doubles and tw is the FP64
// quotient table, TW = double)
template <int LOG_M, int LOG_E, int G, int P_HI, int P_LO, int K, typename TW>
PG_DEV void fwd_round(uint64_t (&x)[1 << LOG_E], uint32_t base, uint32_t tw_base, const TW* __restrict__ tw,
                      uint64_t q2, uint64_t nq) {
    constexpr int E = 1 << LOG_E;
    static_for<0, P_HI - P_LO + 1>([&](auto it) {
        constexpr int p = P_HI - decltype(it)::value;
        constexpr int r = p - G;
        constexpr int half = 1 << r;
        constexpr int sp = LOG_M - 1 - p;
        constexpr int nk = E >> (r + 1);
        const TW* row = tw + (tw_base << sp) + (base >> (p + 1));
        auto bfly_k = [&](auto kk, const ulonglong2 w) {
            constexpr int k = decltype(kk)::value;
            static_for<0, half>([&](auto ll) {
                constexpr int jj = (k << (r + 1)) | decltype(ll)::value;
                if constexpr (K == 2)
                    fwd_bfly_fp<(p & 1) == 0>(x[jj], x[jj + half], w, as_f(q2), as_f(nq));
                else if constexpr (K == 1)
                    fwd_bfly_fast(x[jj], x[jj + half], w, q2, nq);
                else
                    fwd_bfly(x[jj], x[jj + half], w, q2, nq);
            });
        };
        if constexpr (K == 2) {
            const double q = as_f(q2);
            if constexpr (nk == 1) {
                bfly_k(IC<0>{}, tw_fp(__ldg(row), q));
            } else if constexpr (nk == 2) {
                double w0, w1;
                ldg_f2(row, w0, w1);
                bfly_k(IC<0>{}, tw_fp(w0, q));
                bfly_k(IC<1>{}, tw_fp(w1, q));
            } else {
                static_for<0, nk / 4>([&](auto kp) {
                    constexpr int k = 4 * decltype(kp)::value;
                    double w[4];
                    ldg_f4(row + k, w);
                    bfly_k(IC<k>{}, tw_fp(w[0], q));
                    bfly_k(IC<k + 1>{}, tw_fp(w[1], q));
                    bfly_k(IC<k + 2>{}, tw_fp(w[2], q));
                    bfly_k(IC<k + 3>{}, tw_fp(w[3], q));
                });
            }
        } else if constexpr (nk == 1) {
            bfly_k(IC<0>{}, __ldg(row));
        } else {
            static_for<0, nk / 2>([&](auto kp) {
                constexpr int k = 2 * decltype(kp)::value;
                ulonglong2 w0, w1;
                ldg_tw2(row + k, w0, w1);
                bfly_k(IC<k>{}, w0);
                bfly_k(IC<k + 1>{}, w1);
            });
        }
    });
}

// One inverse round, stage bits P_LO up to P_HI (gap 2^p).  The element at
// local index i of CTA rank `rank` has row index rank*M + i; stage p uses the
// inverse powers at N - (N >> p) + ((rank*M + i) >> (p+1)) of the device table,
// which stores inv_root_powers[j + 1] at j (so paired loads are aligned).  The
// last stage of the transform (p == LOG_N-1) is the N^-1-scaled one.
//
// FASTI (every q < 2^50, inputs below 2q): no per-butterfly reduction of x.
// Rounds before the one containing stage kFastInvReduceStage see inputs below
// 2^p * 2q at stage p; that round first reduces its elements to [0, q) (inv64 =
// floor(2^64/q)) and sees inputs below 2^(p - P_LO) * 2q; later rounds count
// from the earliest start that round can have, kFastInvReduceStage - LOG_E + 1
// (a bound at least as large as the true one).  Outputs are canonical either
// way, so the values equal the exact Harvey schedule's.
//
// KI: 0 = exact, 1 = the unreduced integer schedule above (FASTI), 2 = FP64
// schedule (q and nq carry the bit patterns of q and 1/q as doubles, the
// tables are the FP64 ones; the last stage writes canonical integers).
// The FP64 schedule's inverse stages P .. P_HI of a round: pairs of stages in
// radix 4 (inv_bfly4_fp), a lone stage and the N^-1-scaled last stage in radix
// 2.  Twiddle indexing as in inv_round.
template <int LOG_N, int LOG_M, int LOG_E, int G, int P, int P_HI>
PG_DEV void inv_stages_fp(uint64_t (&x)[1 << LOG_E], uint32_t base, uint32_t rank, const double* __restrict__ itw,
                          const ulonglong2* sptr, const ulonglong2* srptr, double q, double qinv) {
    if constexpr (P <= P_HI) {
        constexpr int E = 1 << LOG_E;
        constexpr uint32_t N = 1u << LOG_N;
        constexpr int r = P - G;
        constexpr int h = 1 << r;
        if constexpr (P == LOG_N - 1) {
            const ulonglong2 s = *sptr, sr = *srptr;
            static_for<0, E>([&](auto jt) {
                constexpr int jj = decltype(jt)::value;
                if constexpr (!(jj & h)) inv_last_bfly_fp(x[jj], x[jj + h], s, sr, q);
            });
        } else if constexpr (P + 1 <= P_HI && P + 1 < LOG_N - 1) {
            // the first twiddle of each stage-P pair of groups sits at an even index
            const double* row0 = itw + (N - (N >> P)) + (((rank << LOG_M) + base) >> (P + 1));
            const double* row1 = itw + (N - (N >> (P + 1))) + (((rank << LOG_M) + base) >> (P + 2));
            constexpr int n4 = E >> (r + 2);  // radix-4 groups of this stage pair
            auto bfly4_k = [&](auto kk, const ulonglong2 wa, const ulonglong2 wb, const ulonglong2 wc) {
                constexpr int k2 = decltype(kk)::value;
                static_for<0, h>([&](auto ll) {
                    constexpr int j0 = (k2 << (r + 2)) | decltype(ll)::value;
                    inv_bfly4_fp(x[j0], x[j0 + h], x[j0 + 2 * h], x[j0 + 3 * h], wa, wb, wc, q, qinv);
                });
            };
            if constexpr (n4 == 1) {
                double qa, qb;
                ldg_f2(row0, qa, qb);
                bfly4_k(IC<0>{}, tw_fp(qa, q), tw_fp(qb, q), tw_fp(__ldg(row1), q));
            } else {
                // with two or more groups the stage-P indices start at a multiple
                // of 4 and the stage-(P+1) ones at a multiple of 2
                static_for<0, n4 / 2>([&](auto kp) {
                    constexpr int k2 = 2 * decltype(kp)::value;
                    double wq[4], c0, c1;
                    ldg_f4(row0 + 2 * k2, wq);
                    ldg_f2(row1 + k2, c0, c1);
                    bfly4_k(IC<k2>{}, tw_fp(wq[0], q), tw_fp(wq[1], q), tw_fp(c0, q));
                    bfly4_k(IC<k2 + 1>{}, tw_fp(wq[2], q), tw_fp(wq[3], q), tw_fp(c1, q));
                });
            }
            inv_stages_fp<LOG_N, LOG_M, LOG_E, G, P + 2, P_HI>(x, base, rank, itw, sptr, srptr, q, qinv);
        } else {
            const double* row = itw + (N - (N >> P)) + (((rank << LOG_M) + base) >> (P + 1));
            static_for<0, (E >> (r + 1))>([&](auto kk) {
                constexpr int k = decltype(kk)::value;
                const ulonglong2 w = tw_fp(__ldg(row + k), q);
                static_for<0, h>([&](auto ll) {
                    constexpr int jj = (k << (r + 1)) | decltype(ll)::value;
                    inv_bfly_fp(x[jj], x[jj + h], w, q, qinv);
                });
            });
            inv_stages_fp<LOG_N, LOG_M, LOG_E, G, P + 1, P_HI>(x, base, rank, itw, sptr, srptr, q, qinv);
        }
    }
}

template <int LOG_N, int LOG_M, int LOG_E, int G, int P_LO, int P_HI, int KI = 0, typename TW = ulonglong2>
PG_DEV void inv_round(uint64_t (&x)[1 << LOG_E], uint32_t base, uint32_t rank, const TW* __restrict__ itw,
                      const ulonglong2* sptr, const ulonglong2* srptr, uint64_t q, uint64_t nq,
                      uint64_t inv64 = 0) {
    constexpr bool FASTI = KI == 1, FP = KI == 2;
    const uint64_t q2 = 2 * q;
    constexpr int E = 1 << LOG_E;
    constexpr uint32_t N = 1u << LOG_N;
    constexpr bool RED = FASTI && P_LO <= kFastInvReduceStage && kFastInvReduceStage <= P_HI;
    constexpr bool AFTER = FASTI && P_LO > kFastInvReduceStage;
    constexpr int BASE = RED ? P_LO : (AFTER ? kFastInvReduceStage - LOG_E + 1 : 0);
    if constexpr (RED) {
#pragma unroll
        for (int jj = 0; jj < E; ++jj) x[jj] = reduce_full(x[jj], q, inv64, nq);
    }
    if constexpr (FP) {
        inv_stages_fp<LOG_N, LOG_M, LOG_E, G, P_LO, P_HI>(x, base, rank, itw, sptr, srptr, as_f(q), as_f(nq));
    } else {
    static_for<0, P_HI - P_LO + 1>([&](auto it) {
        constexpr int p = P_LO + decltype(it)::value;
        constexpr int r = p - G;
        constexpr int half = 1 << r;
        constexpr int nk = E >> (r + 1);
        // bound of this stage's inputs
        const uint64_t bnd = FASTI ? (q2 << (p - BASE)) : q2;
        if constexpr (p == LOG_N - 1) {
            const ulonglong2 s = *sptr, sr = *srptr;
            static_for<0, E>([&](auto jt) {
                constexpr int jj = decltype(jt)::value;
                if constexpr (!(jj & half)) {
                    if constexpr (FP)
                        inv_last_bfly_fp(x[jj], x[jj + half], s, sr, as_f(q));
                    else
                        inv_last_bfly(x[jj], x[jj + half], s, sr, q, nq, bnd);
                }
            });
        } else {
            const ulonglong2* row = itw + (N - (N >> p)) + (((rank << LOG_M) + base) >> (p + 1));
            auto bfly_k = [&](auto kk, const ulonglong2 w) {
                constexpr int k = decltype(kk)::value;
                static_for<0, half>([&](auto ll) {
                    constexpr int jj = (k << (r + 1)) | decltype(ll)::value;
                    if constexpr (FP)
                        inv_bfly_fp(x[jj], x[jj + half], w, as_f(q), as_f(nq));
                    else if constexpr (FASTI)
                        inv_bfly_fast(x[jj], x[jj + half], w, bnd, nq);
                    else
                        inv_bfly(x[jj], x[jj + half], w, q2, nq);
                });
            };
            if constexpr (nk == 1) {
                bfly_k(IC<0>{}, __ldg(row));
            } else {
                static_for<0, nk / 2>([&](auto kp) {
                    constexpr int k = 2 * decltype(kp)::value;
                    ulonglong2 w0, w1;
                    ldg_tw2(row + k, w0, w1);
                    bfly_k(IC<k>{}, w0);
                    bfly_k(IC<k + 1>{}, w1);
                });
            }
        }
    });
    }
}

template <int LOG_E, int G>
PG_DEV void load_smem(uint64_t (&x)[1 << LOG_E], const uint64_t* sm, uint32_t base) {
    // base and jj << G have disjoint bits, so padi(base | off) = padi(base) + padi(off)
    const uint64_t* p = sm + padi(base);
#pragma unroll
    for (int jj = 0; jj < (1 << LOG_E); ++jj) x[jj] = p[padi(jj << G)];
}

template <int LOG_E, int G>
PG_DEV void store_smem(const uint64_t (&x)[1 << LOG_E], uint64_t* sm, uint32_t base) {
    uint64_t* p = sm + padi(base);
#pragma unroll
    for (int jj = 0; jj < (1 << LOG_E); ++jj) p[padi(jj << G)] = x[jj];
}

// Barrier between two rounds whose E-element groups sit at bit G1 and G2 of
// the element index (group_base inserts the group's LOG_E bits at G into the
// thread index).  A warp's threads fix thread-index bits 5 .. LOG_T-1; each of
// them lands at the same element bit in both rounds unless it lies in
// [min(G1, G2), max(G1, G2)).  When none does, every warp stores and then
// loads the same set of elements (and last read those locations itself), so a
// warp barrier orders the exchange; otherwise the whole CTA synchronises.
// With 32 or fewer threads per row every exchange stays inside one warp.
template <int LOG_T, int G1, int G2>
PG_DEV void exchange_sync() {
    constexpr int lo = G1 < G2 ? G1 : G2, hi = G1 < G2 ? G2 : G1;
    constexpr bool warp_local = LOG_T <= 5 || hi <= 5 || lo >= LOG_T;
    if constexpr (warp_local)
        __syncwarp();
    else
        __syncthreads();
}

// Forward rounds over the low TOP bits of a block (the bits above TOP were
// processed earlier): round R covers bits [P_LO, P_HI], its group spans
// [P_LO, P_LO + LOG_E).
template <int TOP, int LOG_E, int R>
struct FwdRounds {
    static constexpr int P_HI = TOP - 1 - R * LOG_E;
    static constexpr int P_LO = (P_HI - LOG_E + 1) > 0 ? (P_HI - LOG_E + 1) : 0;
    static constexpr int G = P_LO;
    static constexpr bool LAST = (P_LO == 0);
    static constexpr int COUNT = (TOP + LOG_E - 1) / LOG_E;
};

// Runs forward rounds R..last; x holds round R-1's group on entry (stored to
// smem first).  On exit x holds the last round's group (G = 0: E contiguous
// elements at tid*E).
template <int LOG_M, int TOP, int LOG_E, int R, int FAST, typename TW>
PG_DEV void fwd_rest(uint64_t (&x)[1 << LOG_E], uint64_t* sm, uint32_t tid, uint32_t tw_base,
                     const TW* __restrict__ tw, uint64_t q2, uint64_t nq) {
    if constexpr (R < FwdRounds<TOP, LOG_E, 0>::COUNT) {
        using Cur = FwdRounds<TOP, LOG_E, R>;
        using Prev = FwdRounds<TOP, LOG_E, R - 1>;
        store_smem<LOG_E, Prev::G>(x, sm, group_base<LOG_E>(tid, Prev::G));
        exchange_sync<LOG_M - LOG_E, Prev::G, Cur::G>();
        const uint32_t base = group_base<LOG_E>(tid, Cur::G);
        load_smem<LOG_E, Cur::G>(x, sm, base);
        fwd_round<LOG_M, LOG_E, Cur::G, Cur::P_HI, Cur::P_LO, FAST>(x, base, tw_base, tw, q2, nq);
        fwd_rest<LOG_M, TOP, LOG_E, R + 1, FAST>(x, sm, tid, tw_base, tw, q2, nq);
    }
}

template <int TOP, int LOG_E, int R>
struct InvRounds {
    static constexpr int P_LO = R * LOG_E;
    static constexpr int P_HI = (P_LO + LOG_E - 1) < (TOP - 1) ? (P_LO + LOG_E - 1) : (TOP - 1);
    static constexpr int G = P_LO < (TOP - LOG_E) ? P_LO : (TOP - LOG_E);
    static constexpr bool LAST = (P_HI == TOP - 1);
    static constexpr int COUNT = (TOP + LOG_E - 1) / LOG_E;
};

// Runs inverse rounds R .. R_END-1; x holds round R-1's group on entry
// (R >= 1) and is stored to smem first.  On exit x holds round R_END-1's group.
template <int LOG_N, int LOG_M, int TOP, int LOG_E, int R, int R_END, int FASTI = 0, typename TW = ulonglong2>
PG_DEV void inv_range(uint64_t (&x)[1 << LOG_E], uint64_t* sm, uint32_t tid, uint32_t rank,
                      const TW* __restrict__ itw, const ulonglong2* sptr, const ulonglong2* srptr, uint64_t q,
                      uint64_t nq, uint64_t inv64 = 0) {
    if constexpr (R < R_END) {
        using Cur = InvRounds<TOP, LOG_E, R>;
        using Prev = InvRounds<TOP, LOG_E, R - 1>;
        store_smem<LOG_E, Prev::G>(x, sm, group_base<LOG_E>(tid, Prev::G));
        exchange_sync<LOG_M - LOG_E, Prev::G, Cur::G>();
        const uint32_t base = group_base<LOG_E>(tid, Cur::G);
        load_smem<LOG_E, Cur::G>(x, sm, base);
        inv_round<LOG_N, LOG_M, LOG_E, Cur::G, Cur::P_LO, Cur::P_HI, FASTI>(x, base, rank, itw, sptr, srptr, q, nq,
                                                                           inv64);
        inv_range<LOG_N, LOG_M, TOP, LOG_E, R + 1, R_END, FASTI>(x, sm, tid, rank, itw, sptr, srptr, q, nq, inv64);
    }
}

// Butterfly schedules (template parameter S of the kernels).  All return the same
// canonical values; the faster ones need headroom below 2^64 (or 2^53):
//   kSchedExact    the reference's Harvey / Gentleman-Sande schedule (lazy outputs)
//   kSchedFastFwd  forward without the u = x mod 2q step: every q < 2^58
//   kSchedFastBoth also the inverse without the x reduction: every q < 2^50
//   kSchedFp64     both directions on the FP64 pipe (fwd_bfly_fp / inv_bfly_fp):
//                  every q < 2^50, canonical (non-lazy) forward outputs
constexpr int kSchedExact = 0, kSchedFastFwd = 1, kSchedFastBoth = 2, kSchedFp64 = 3;

// twiddle tables of a schedule: (w, w') pairs, or the FP64 quotient tables
template <bool FP>
PG_DEV auto fwd_table(const NttArgs& a) {
    if constexpr (FP) return a.fwd_fp; else return a.fwd;
}
template <bool FP>
PG_DEV auto inv_table(const NttArgs& a) {
    if constexpr (FP) return a.inv_fp; else return a.inv;
}

// per-row constants of the FP64 schedule: q and 1/q (correctly rounded)
struct FpMod {
    double q, qinv;
};

PG_DEV FpMod fp_mod(uint64_t qi) {
    FpMod m;
    m.q = u52_to_f(qi);
    m.qinv = __drcp_rn(m.q);
    return m;
}

// ============================================================================
// Single-CTA kernel: ROWS rows of N = 2^LOG_N per CTA, T = N/E threads per row.
// FAST selects the forward schedule without per-butterfly reduction of u (only
// when the caller needs canonical or multiplied outputs and every q < 2^58).
// ============================================================================
template <int LOG_N, int LOG_E, int ROWS, int MODE, int S>
__global__ void __launch_bounds__((1 << (LOG_N - LOG_E)) * ROWS) ntt_block_kernel(NttArgs a) {
    constexpr int N = 1 << LOG_N, E = 1 << LOG_E, T = N / E;
    constexpr bool FP = S == kSchedFp64;
    constexpr int KF = FP ? 2 : (S >= 1 ? 1 : 0), KI = FP ? 2 : (S >= 2 ? 1 : 0);  // round kinds
    constexpr bool FAST = KF == 1, FASTI = KI == 1;
    extern __shared__ uint64_t smem_block[];
    const uint32_t tid = threadIdx.x;
    // launch order is limb-major (all polys of limb 0, then limb 1, ...) so that
    // concurrently running CTAs share one prime's twiddles in L2
    const uint64_t u = (uint64_t)blockIdx.x * ROWS + threadIdx.y;
    const bool active = u < a.rows;
    const uint64_t polys = a.desc ? 1 : a.rows / a.L;  // descriptor rows need no [P][L] shape
    uint32_t limb = active ? (uint32_t)(u / polys) : 0;
    const uint64_t row = active ? (u % polys) * a.L + limb : 0;
    uint64_t* sm = smem_block + threadIdx.y * padded(N);
    uint64_t* g = a.data + row * N;
    uint64_t* mulp = nullptr;  // descriptor multiplicand (the pair form's b row)
    if (a.desc) {  // descriptor-driven rows (ragged batches)
        const RowDesc d = a.desc[active ? u : 0];
        g = d.data;
        limb = d.limb;
        mulp = d.mul;
    }
    const uint64_t q = a.moduli[limb], q2 = q << 1, nq = 0 - q;
    const FpMod fm = fp_mod(FP ? q : 3);
    // the rounds' modulus words: (2q, -q) on the integer schedules, (q, 1/q) as doubles on FP64
    const uint64_t mA = FP ? as_u(fm.q) : q2, mB = FP ? as_u(fm.qinv) : nq;
    uint64_t x[E];
    uint64_t xb[E];  // (pair form) NTT(b), canonical: elements tid*E .. tid*E+E-1

    if constexpr (MODE == MODE_PAIR) {
        static_assert(FP, "the pair form runs on the FP64 schedule");
        // b <- NTT(b): the forward of the multiplicand row, kept in registers for
        // the product and stored back in place (coalesced, through smem)
        const auto* tw = fwd_table<FP>(a) + (size_t)limb * N;
        using R0 = FwdRounds<LOG_N, LOG_E, 0>;
        uint64_t* bp = mulp;  // every pair descriptor carries its b row
#pragma unroll
        for (int jj = 0; jj < E; ++jj) {
            x[jj] = active ? bp[tid + jj * T] : 0;
            x[jj] = as_u(freduce(u52_to_f(x[jj]), fm.q, fm.qinv));  // inputs < 4q < 2^52
        }
        fwd_round<LOG_N, LOG_E, R0::G, R0::P_HI, R0::P_LO, KF>(x, tid, 1, tw, mA, mB);
        fwd_rest<LOG_N, LOG_N, LOG_E, 1, KF>(x, sm, tid, 1, tw, mA, mB);
#pragma unroll
        for (int jj = 0; jj < E; ++jj) xb[jj] = f_to_u52(fcanon(freduce(as_f(x[jj]), fm.q, fm.qinv), fm.q));
        __syncthreads();
        store_smem<LOG_E, 0>(xb, sm, tid * E);
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k = 0; k < E; ++k) bp[tid + k * T] = sm[padi(tid + k * T)];
        }
        __syncthreads();  // every read of the exchange buffer is done before a's rounds
    }

    if constexpr (MODE == MODE_FWD || MODE == MODE_RT || MODE == MODE_PAIR) {
        const auto* tw = fwd_table<FP>(a) + (size_t)limb * N;
        using R0 = FwdRounds<LOG_N, LOG_E, 0>;
        // round 0 reads the row straight from HBM: x[jj] = row[tid + jj*T] (or the
        // lifted gadget digits of the row's digit row)
        const uint64_t* src = a.lift_src ? a.lift_src + (row / a.L) * N : g;
#pragma unroll
        for (int jj = 0; jj < E; ++jj) {
            x[jj] = active ? src[tid + jj * T] : 0;
            if (a.lift_src) x[jj] = lift_digit(x[jj], q, a.lift_basis, a.lift_half);
            if constexpr (FP) x[jj] = as_u(freduce(u52_to_f(x[jj]), fm.q, fm.qinv));  // inputs < 4q < 2^52
        }
        fwd_round<LOG_N, LOG_E, R0::G, R0::P_HI, R0::P_LO, KF>(x, tid, 1, tw, mA, mB);
        fwd_rest<LOG_N, LOG_N, LOG_E, 1, KF>(x, sm, tid, 1, tw, mA, mB);
        // x = E contiguous outputs at tid*E
        if constexpr (MODE == MODE_FWD) {
            if constexpr (FP) {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = f_to_u52(fcanon(freduce(as_f(x[jj]), fm.q, fm.qinv), fm.q));
            } else if constexpr (FAST) {
                const uint64_t inv64 = a.bar[limb].r1;
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = reduce_full(x[jj], q, inv64, nq);
            } else if (!a.lazy) {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = canon4(x[jj], q, q2);
            }
            __syncthreads();
            store_smem<LOG_E, 0>(x, sm, tid * E);
            __syncthreads();
            if (active) {
#pragma unroll
                for (int k = 0; k < E; ++k) g[tid + k * T] = sm[padi(tid + k * T)];
            }
        } else if constexpr (MODE == MODE_PAIR) {
            // x * NTT(b): w canonical, wq = w * (1/q) within 2^-52 relative of w/q, so the
            // product of |x| < 2q + 2 lands in [-q, q] (a valid inverse input)
#pragma unroll
            for (int jj = 0; jj < E; ++jj) {
                const double w = u52_to_f(xb[jj]);
                x[jj] = as_u(fmulmod(as_f(x[jj]), w, __dmul_rn(w, fm.qinv), fm.q));
            }
        } else {
            // pointwise product with the NTT-domain plaintext (Shoup-prepared);
            // the lazy product in [0, 2q) is a valid inverse input
            const uint64_t* pv = a.plain + (size_t)limb * N + tid * E;
            const uint64_t* pq = a.plain_q + (size_t)limb * N + tid * E;
            if constexpr (FP) {
                // w = plaintext (canonical), wq = w * (1/q): within 2^-52 relative of w/q, so the
                // product of |x| < 2q + 2 lands in [-q, q] (a valid inverse input)
#pragma unroll
                for (int jj = 0; jj < E; ++jj) {
                    const double w = u52_to_f(__ldg(pv + jj));
                    x[jj] = as_u(fmulmod(as_f(x[jj]), w, __dmul_rn(w, fm.qinv), fm.q));
                }
            } else {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = shoup_lazy_nq(__ldg(pv + jj), __ldg(pq + jj), x[jj], nq);
            }
        }
    }
    // ---------------- inverse
    if constexpr (MODE != MODE_FWD) {
        const auto* itw = inv_table<FP>(a) + (size_t)limb * N;
        const ulonglong2* sptr = (FP ? a.inv_n_fp : a.inv_n) + limb;
        const ulonglong2* srptr = (FP ? a.inv_last_fp : a.inv_last) + limb;
        const uint64_t iA = FP ? as_u(fm.q) : q, iB = FP ? as_u(fm.qinv) : nq;
        using I0 = InvRounds<LOG_N, LOG_E, 0>;
        if constexpr (MODE == MODE_INV) {
            // stage the bit-reversed row through smem (coalesced), then round 0;
            // every global load is issued before the first shared-memory store
#pragma unroll
            for (int k = 0; k < E; ++k) x[k] = active ? ld_stream(g + tid + k * T) : 0;
            // descriptor rows may carry an NTT-domain multiplicand (canonical inputs)
            if (mulp && active) {
                const Barrett bar = a.bar[limb];
#pragma unroll
                for (int k = 0; k < E; ++k) x[k] = barrett_mul(x[k], ld_stream(mulp + tid + k * T), bar);
            }
#pragma unroll
            for (int k = 0; k < E; ++k) {
                uint64_t v = x[k];
                if constexpr (FP) v = as_u(freduce(u52_to_f(v), fm.q, fm.qinv));  // inputs < 2q < 2^52
                sm[padi(tid + k * T)] = v;
            }
            __syncthreads();
            load_smem<LOG_E, I0::G>(x, sm, group_base<LOG_E>(tid, I0::G));
        } else {
            // round trip: the forward's last group (tid*E .. tid*E+E-1) is the
            // inverse's first group (I0::G == 0), so it stays in registers
            static_assert(I0::G == 0, "round trip needs the first inverse group to be contiguous");
        }
        const uint64_t inv64 = FASTI ? a.bar[limb].r1 : 0;
        inv_round<LOG_N, LOG_N, LOG_E, I0::G, I0::P_LO, I0::P_HI, KI>(x, group_base<LOG_E>(tid, I0::G), 0, itw, sptr,
                                                                      srptr, iA, iB, inv64);
        inv_range<LOG_N, LOG_N, LOG_N, LOG_E, 1, I0::COUNT, KI>(x, sm, tid, 0, itw, sptr, srptr, iA, iB, inv64);
        // last group: elements tid + jj*T, coalesced store
        using Last = InvRounds<LOG_N, LOG_E, I0::COUNT - 1>;
        static_assert(Last::G == LOG_N - LOG_E, "last inverse group");
        if (active) {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) g[tid + jj * T] = x[jj];
        }
    }
}

// ============================================================================
// Cluster kernel: a row of N = 2^LOG_N is owned by C = 2^(LOG_N - LOG_M) CTAs.
//   cross phase: thread gt = rank*T + tid owns the column {gt + jj*N/E} (the
//     top LOG_E index bits vary), i.e. the first LOG_E forward stages (last
//     LOG_E inverse stages); coalesced HBM access.
//   local phase: CTA rank owns block [rank*M, (rank+1)*M) in shared memory and
//     runs the remaining stages in rounds of LOG_E.
// The two phases exchange through distributed shared memory
// (st.shared::cluster) between cluster barriers.
// ============================================================================
PG_DEV void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory"); }
PG_DEV void cluster_arrive_release() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
PG_DEV void cluster_wait_acquire() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }

PG_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// st.shared::cluster of one u64 into CTA `rank`'s shared memory at the same offset
PG_DEV void st_cluster(uint32_t local_addr, uint32_t rank, uint64_t v) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(remote) : "r"(local_addr), "r"(rank));
    asm volatile("st.shared::cluster.u64 [%0], %1;\n" ::"r"(remote), "l"(v) : "memory");
}

// CTAs per SM the register budget is sized for: the whole 64K-entry register
// file is shared by MINB CTAs of T threads, i.e. 65536 / (MINB * T) registers
// per thread (64 for the shapes below), so independent CTAs overlap each
// other's barrier and exchange phases.
__host__ __device__ constexpr int cluster_min_blocks(int threads) { return 1024 / threads; }

// One row of the cluster kernel: row u of the launch (see ntt_cluster_kernel).
// Where a forward transform of the cluster kernel takes its inputs and puts its
// canonical outputs.  RowIO: the launch's rows (or, with NttArgs::lift_src, the
// lifted gadget digits).  A policy with kLoad supplies the E inputs of a thread's
// column itself, as values below 4q:
//   template <int E> void load(p, limb, q, i0, stride, x[E])   x[jj] = input i0 + jj * stride
// and one with kStore takes the canonical outputs of a thread's column of a
// forward or inverse transform instead of the row store:
//   template <int E, class V> void store(p, limb, q, i0, stride, V value)
// output i0 + k * stride being value(k) for k < E (the policy may issue its own
// loads for all E outputs before it reads the values), where p is the row's
// poly index (row = p * L + limb).  Fused producers and
// consumers (the key switch's base conversions) use them to skip a pass
// through HBM; the transform itself is unchanged.
struct RowIO {
    static constexpr bool kLoad = false, kStore = false;
};

template <int LOG_N, int LOG_M, int LOG_E, int MODE, int S, class IO = RowIO>
PG_DEV void cluster_row(const NttArgs& a, uint64_t* sm, const uint64_t u, const IO& io = IO{}) {
    constexpr bool FP = S == kSchedFp64;
    constexpr int KF = FP ? 2 : (S >= 1 ? 1 : 0), KI = FP ? 2 : (S >= 2 ? 1 : 0);  // round kinds
    constexpr bool FAST = KF == 1, FASTI = KI == 1;
    constexpr int LOG_C = LOG_N - LOG_M;
    constexpr int N = 1 << LOG_N, M = 1 << LOG_M, E = 1 << LOG_E, LOG_T = LOG_M - LOG_E, T = 1 << LOG_T;
    constexpr int LOG_K = LOG_E - LOG_C;  // top block bits handled by the cross phase
    constexpr int K = 1 << LOG_K;
    constexpr int TOP = LOG_M - LOG_K;    // block bits handled by the local rounds
    constexpr int GX = LOG_N - LOG_E;     // cross group stride bit (N/E)
    static_assert(LOG_K >= 0 && TOP >= LOG_E, "shape");
    const uint32_t tid = threadIdx.x;
    const uint32_t rank = blockIdx.x & ((1 << LOG_C) - 1);
    // rows run limb-major so that concurrently running clusters share one
    // prime's twiddles in L2
    const uint64_t polys = a.desc ? 1 : a.rows / a.L;  // descriptor rows need no [P][L] shape
    uint32_t limb = (uint32_t)(u / polys);
    const uint64_t row = (u % polys) * a.L + limb;
    uint64_t* g = a.data + row * N;
    const uint64_t* mulp = nullptr;
    if (a.desc) {  // descriptor-driven rows (ragged batches)
        const RowDesc d = a.desc[u];
        g = d.data;
        limb = d.limb;
        mulp = d.mul;
    }
    const uint64_t q = a.moduli[limb], nq = 0 - q;
    const FpMod fm = fp_mod(FP ? q : 3);
    const uint32_t gt = (rank << LOG_T) + tid;  // cross group (column) of this thread
    uint64_t x[E];

    if constexpr (MODE == MODE_FWD || MODE == MODE_RT) {
        const uint64_t q2 = q << 1;
        // the rounds' modulus words: (2q, -q) on the integer schedules, (q, 1/q) as doubles on FP64
        const uint64_t mA = FP ? as_u(fm.q) : q2, mB = FP ? as_u(fm.qinv) : nq;
        const auto* tw = fwd_table<FP>(a) + (size_t)limb * N;
        // matched by the wait before the first remote store; relaxed is enough
        // because this CTA has not touched shared memory yet
        cluster_arrive_relaxed();
        if constexpr (IO::kLoad) {
            static_assert(MODE == MODE_FWD, "a loading policy feeds forward transforms");
            io.template load<E>(row / a.L, limb, q, gt, 1u << GX, x);
        } else {
            const uint64_t* src = a.lift_src ? a.lift_src + (row / a.L) * N : g;  // digits to lift, or the row
#pragma unroll
            for (int jj = 0; jj < E; ++jj) {
                x[jj] = src[gt + (jj << GX)];
                if (a.lift_src) x[jj] = lift_digit(x[jj], q, a.lift_basis, a.lift_half);
            }
        }
        if constexpr (FP) {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) x[jj] = as_u(freduce(u52_to_f(x[jj]), fm.q, fm.qinv));  // inputs < 4q < 2^52
        }
        fwd_round<LOG_N, LOG_E, GX, LOG_N - 1, GX, KF>(x, gt, 1, tw, mA, mB);
        cluster_wait_acquire();  // every CTA of the cluster is running
        // element gt + jj*N/E lives in block jj >> LOG_K at local index gt + (jj & (K-1)) * N/E
        const uint32_t la = smem_u32(sm + padi(gt));
#pragma unroll
        for (int jj = 0; jj < E; ++jj)
            st_cluster(la + 8 * padi((jj & (K - 1)) << GX), (uint32_t)(jj >> LOG_K), x[jj]);
        cluster_arrive_release();
        cluster_wait_acquire();
        // local rounds over the low TOP block bits
        using R0 = FwdRounds<TOP, LOG_E, 0>;
        load_smem<LOG_E, R0::G>(x, sm, group_base<LOG_E>(tid, R0::G));
        fwd_round<LOG_M, LOG_E, R0::G, R0::P_HI, R0::P_LO, KF>(x, group_base<LOG_E>(tid, R0::G), (1u << LOG_C) + rank,
                                                               tw, mA, mB);
        fwd_rest<LOG_M, TOP, LOG_E, 1, KF>(x, sm, tid, (1u << LOG_C) + rank, tw, mA, mB);
        if constexpr (MODE == MODE_FWD) {
            if constexpr (FP) {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = f_to_u52(fcanon(freduce(as_f(x[jj]), fm.q, fm.qinv), fm.q));
            } else if constexpr (FAST) {
                const uint64_t inv64 = a.bar[limb].r1;
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = reduce_full(x[jj], q, inv64, nq);
            } else if (!a.lazy) {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = canon4(x[jj], q, q2);
            }
            __syncthreads();
            store_smem<LOG_E, 0>(x, sm, tid * E);
            __syncthreads();
            if constexpr (IO::kStore) {
                io.template store<E>(row / a.L, limb, q, rank * M + tid, T,
                                     [&](int k) { return sm[padi(tid + k * T)]; });
            } else {
                uint64_t* gb = g + rank * M;
#pragma unroll
                for (int k = 0; k < E; ++k) gb[tid + k * T] = sm[padi(tid + k * T)];
            }
        } else {
            const uint64_t* pv = a.plain + (size_t)limb * N + rank * M + tid * E;
            const uint64_t* pq = a.plain_q + (size_t)limb * N + rank * M + tid * E;
            if constexpr (FP) {
                // as in the block kernel: products in [-q, q]
#pragma unroll
                for (int jj = 0; jj < E; ++jj) {
                    const double w = u52_to_f(__ldg(pv + jj));
                    x[jj] = as_u(fmulmod(as_f(x[jj]), w, __dmul_rn(w, fm.qinv), fm.q));
                }
            } else {
#pragma unroll
                for (int jj = 0; jj < E; ++jj) x[jj] = shoup_lazy_nq(__ldg(pv + jj), __ldg(pq + jj), x[jj], nq);
            }
        }
    }
    // ---------------- inverse
    if constexpr (MODE != MODE_FWD) {
        const auto* itw = inv_table<FP>(a) + (size_t)limb * N;
        const uint64_t iA = FP ? as_u(fm.q) : q, iB = FP ? as_u(fm.qinv) : nq;
        using I0 = InvRounds<TOP, LOG_E, 0>;
        using ILast = InvRounds<TOP, LOG_E, I0::COUNT - 1>;
        static_assert(I0::COUNT >= 2, "cluster path needs two local rounds");
        if constexpr (MODE == MODE_INV) {
            // every global load is issued before the first shared-memory store
            const uint64_t* gb = g + rank * M;
#pragma unroll
            for (int k = 0; k < E; ++k) x[k] = ld_stream(gb + tid + k * T);
            // descriptor rows may carry an NTT-domain multiplicand (canonical inputs)
            if (mulp) {
                const Barrett bar = a.bar[limb];
#pragma unroll
                for (int k = 0; k < E; ++k) x[k] = barrett_mul(x[k], ld_stream(mulp + rank * M + tid + k * T), bar);
            }
#pragma unroll
            for (int k = 0; k < E; ++k) {
                uint64_t v = x[k];
                if constexpr (FP) v = as_u(freduce(u52_to_f(v), fm.q, fm.qinv));  // inputs < 2q < 2^52
                sm[padi(tid + k * T)] = v;
            }
            __syncthreads();
            load_smem<LOG_E, I0::G>(x, sm, group_base<LOG_E>(tid, I0::G));
        }
        const uint64_t inv64 = FASTI ? a.bar[limb].r1 : 0;
        inv_round<LOG_N, LOG_M, LOG_E, I0::G, I0::P_LO, I0::P_HI, KI>(x, group_base<LOG_E>(tid, I0::G), rank, itw,
                                                                      nullptr, nullptr, iA, iB, inv64);
        inv_range<LOG_N, LOG_M, TOP, LOG_E, 1, I0::COUNT - 1, KI>(x, sm, tid, rank, itw, nullptr, nullptr, iA, iB,
                                                                  inv64);
        {
            // last local round: its smem loads precede the cluster arrive, so no
            // CTA overwrites a block that another CTA is still reading
            using Prev = InvRounds<TOP, LOG_E, I0::COUNT - 2>;
            store_smem<LOG_E, Prev::G>(x, sm, group_base<LOG_E>(tid, Prev::G));
            exchange_sync<LOG_T, Prev::G, ILast::G>();
            const uint32_t base = group_base<LOG_E>(tid, ILast::G);
            load_smem<LOG_E, ILast::G>(x, sm, base);
            // release: these shared-memory reads must be performed before any
            // other CTA, released by this barrier, overwrites the block
            cluster_arrive_release();
            inv_round<LOG_N, LOG_M, LOG_E, ILast::G, ILast::P_LO, ILast::P_HI, KI>(x, base, rank, itw, nullptr,
                                                                                   nullptr, iA, iB, inv64);
            cluster_wait_acquire();
            // element at row index i = rank*M + base + (jj << G) belongs to cross
            // group c = i mod N/E (CTA c >> LOG_T, thread c mod T) as element i >> GX:
            // it goes to slot (i >> GX) * T + (c mod T) of that CTA's buffer
            const uint32_t i0 = (rank << LOG_M) + base;
#pragma unroll
            for (int jj = 0; jj < E; ++jj) {
                const uint32_t i = i0 + ((uint32_t)jj << ILast::G);
                const uint32_t c = i & ((1u << GX) - 1);
                st_cluster(smem_u32(sm + padi(((i >> GX) << LOG_T) + (c & (T - 1)))), c >> LOG_T, x[jj]);
            }
            cluster_arrive_release();
            cluster_wait_acquire();
        }
        // cross inverse stages (the last LOG_E, including the N^-1-scaled one)
#pragma unroll
        for (int jj = 0; jj < E; ++jj) x[jj] = sm[padi((jj << LOG_T) + tid)];
        inv_round<LOG_N, LOG_N, LOG_E, GX, GX, LOG_N - 1, KI>(x, gt, 0, itw, (FP ? a.inv_n_fp : a.inv_n) + limb,
                                                              (FP ? a.inv_last_fp : a.inv_last) + limb, iA, iB, inv64);
        if constexpr (IO::kStore) {
            static_assert(MODE == MODE_INV, "a storing policy takes forward or inverse outputs");
            io.template store<E>(row / a.L, limb, q, gt, 1u << GX, [&](int jj) { return x[jj]; });
        } else {
#pragma unroll
            for (int jj = 0; jj < E; ++jj) g[gt + (jj << GX)] = x[jj];
        }
    }
}

// The cluster kernel: a grid of rows * C CTAs, one row per cluster of C CTAs.
template <int LOG_N, int LOG_M, int LOG_E, int MODE, int S, class IO = RowIO>
__global__ void __launch_bounds__(1 << (LOG_M - LOG_E), cluster_min_blocks(1 << (LOG_M - LOG_E)))
    ntt_cluster_kernel(NttArgs a, IO io) {
    extern __shared__ uint64_t smem_cl[];
    cluster_row<LOG_N, LOG_M, LOG_E, MODE, S, IO>(a, smem_cl, blockIdx.x >> (LOG_N - LOG_M), io);
}

}  // namespace pg

namespace pg {

inline bool fast_fwd_ok(const NttArgs& a) { return a.max_modulus < (1ull << 58); }
inline bool fast_inv_ok(const NttArgs& a) { return a.max_modulus < (1ull << 50); }

template <int LOG_N, int LOG_E, int ROWS, int MODE, int S>
static int launch_block(const NttArgs& a, cudaStream_t st) {
    constexpr int T = 1 << (LOG_N - LOG_E);
    constexpr size_t smem = (size_t)ROWS * padded(1 << LOG_N) * sizeof(uint64_t);
    auto kern = ntt_block_kernel<LOG_N, LOG_E, ROWS, MODE, S>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return cuda_status(attr, "ntt_block_kernel: shared memory attribute");
    dim3 block(T, ROWS);
    dim3 grid((unsigned)((a.rows + ROWS - 1) / ROWS));
    kern<<<grid, block, smem, st>>>(a);
    count_launch();
    PG_LAUNCH_CHECK("ntt_block_kernel launch");
    return PG_OK;
}

// Cluster placement: the load-balancing policy (the hardware may put several
// CTAs of one cluster on an SM) by default; spread = true asks for the spread
// policy (each CTA of a cluster on its own SM).  Measured at N = 2^16, L = 24,
// 128 polys: forward 1,761 -> 1,638 us, inverse 2,023 -> 1,923 us, round trip
// unchanged; at N = 2^15 2-3% on every mode.
template <int LOG_N, int LOG_M, int LOG_E, int MODE, int S, class IO = RowIO>
static int launch_cluster(const NttArgs& a, cudaStream_t st, bool spread = false, const IO& io = IO{}) {
    constexpr int C = 1 << (LOG_N - LOG_M), T = 1 << (LOG_M - LOG_E);
    constexpr size_t smem = (size_t)padded(1 << LOG_M) * sizeof(uint64_t);
    auto kern = ntt_cluster_kernel<LOG_N, LOG_M, LOG_E, MODE, S, IO>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return cuda_status(attr, "ntt_cluster_kernel: shared memory attribute");
    if (a.rows * C > 0x7fffffffull) return set_error(PG_ERR_UNSUPPORTED, "too many rows for one launch");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.rows * C));
    cfg.blockDim = dim3(T);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeClusterSchedulingPolicyPreference;
    at[1].val.clusterSchedulingPolicyPreference =
        spread ? cudaClusterSchedulingPolicySpread : cudaClusterSchedulingPolicyLoadBalancing;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    if constexpr (C > 8) {
        static const cudaError_t np = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (np != cudaSuccess) return cuda_status(np, "ntt_cluster_kernel: non-portable cluster size");
    }
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a, io);
    count_launch();
    if (e != cudaSuccess) return cuda_status(e, "ntt_cluster_kernel launch");
    return PG_OK;
}

}  // namespace pg
