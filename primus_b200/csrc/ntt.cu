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
//   * N = 2^14 .. 2^16: a thread-block cluster of C = N / 2^13 CTAs owns one
//     row (512 KiB at N = 2^16) in distributed shared memory.  Forward: the
//     first log2(C) stages pair elements 2^13 apart, so each CTA takes a slab
//     of columns {l + 2^13 j}, runs those stages in registers and scatters the
//     results to the owning CTA's shared memory (st.shared::cluster); the
//     remaining 13 stages are local.  Inverse mirrors this.  A row is read from
//     and written to HBM exactly once, also for the fused fwd -> x plain -> inv
//     round trip.
#include <cooperative_groups.h>

#include "internal.hpp"

namespace cg = cooperative_groups;

namespace pg {

PG_DEV int padi(int i) { return i + (i >> 4); }
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
// values stay below 36q < 2^64 for q < 2^58, and the final canonical
// reduction yields the same residues as the Harvey schedule.
PG_DEV void fwd_bfly_fast(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q2, uint64_t nq) {
    uint64_t u = x;
    uint64_t v = shoup_lazy_nq(w.x, w.y, y, nq);
    x = u + v;
    y = u + q2 - v;
}

// Gentleman-Sande inverse butterfly; x, y in [0, 2q) -> [0, 2q)
PG_DEV void inv_bfly(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q2, uint64_t nq) {
    uint64_t u = x, v = y;
    uint64_t s = u + v;
    x = s >= q2 ? s - q2 : s;
    y = shoup_lazy_nq(w.x, w.y, u + q2 - v, nq);
}

// Last inverse stage fused with N^-1: x = N^-1 (u+v), y = (w N^-1)(u+2q-v), canonical
PG_DEV void inv_last_bfly(uint64_t& x, uint64_t& y, const ulonglong2 s, const ulonglong2 sr, uint64_t q,
                          uint64_t nq) {
    uint64_t u = x, v = y;
    uint64_t a = shoup_lazy_nq(s.x, s.y, u + v, nq);
    uint64_t b = shoup_lazy_nq(sr.x, sr.y, u + 2 * q - v, nq);
    x = a >= q ? a - q : a;
    y = b >= q ? b - q : b;
}

// any 64-bit v -> v mod q, using floor(2^64/q) (the high word of the Barrett ratio)
PG_DEV uint64_t reduce_full(uint64_t v, uint64_t q, uint64_t inv64, uint64_t nq) {
    uint64_t r = v + nq * mulhi64(inv64, v);
    return r >= q ? r - q : r;
}

PG_DEV uint64_t canon4(uint64_t v, uint64_t q, uint64_t q2) {
    v = v >= q2 ? v - q2 : v;
    return v >= q ? v - q : v;
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

// One forward round over register group x (x[jj] is local index base + (jj << G)
// of a 2^LOG_M block).  Stage bits P_HI down to P_LO; stage bit p is block stage
// sp = LOG_M-1-p and uses tw[(tw_base << sp) + (i >> (p+1))], tw_base = C + rank
// for a cluster block (1 for a whole row).  When a stage needs two or more
// twiddles their first index is even, so they are fetched in 32-byte pairs.
template <int LOG_M, int LOG_E, int G, int P_HI, int P_LO, bool FAST>
PG_DEV void fwd_round(uint64_t (&x)[1 << LOG_E], uint32_t base, uint32_t tw_base, const ulonglong2* __restrict__ tw,
                      uint64_t q2, uint64_t nq) {
    constexpr int E = 1 << LOG_E;
    static_for<0, P_HI - P_LO + 1>([&](auto it) {
        constexpr int p = P_HI - decltype(it)::value;
        constexpr int r = p - G;
        constexpr int half = 1 << r;
        constexpr int sp = LOG_M - 1 - p;
        constexpr int nk = E >> (r + 1);
        const ulonglong2* row = tw + (tw_base << sp) + (base >> (p + 1));
        auto bfly_k = [&](auto kk, const ulonglong2 w) {
            constexpr int k = decltype(kk)::value;
            static_for<0, half>([&](auto ll) {
                constexpr int jj = (k << (r + 1)) | decltype(ll)::value;
                if constexpr (FAST)
                    fwd_bfly_fast(x[jj], x[jj + half], w, q2, nq);
                else
                    fwd_bfly(x[jj], x[jj + half], w, q2, nq);
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
    });
}

// One inverse round, stage bits P_LO up to P_HI (gap 2^p).  The element at
// local index i of CTA rank `rank` has row index rank*M + i; stage p uses the
// inverse powers at N - (N >> p) + ((rank*M + i) >> (p+1)) of the device table,
// which stores inv_root_powers[j + 1] at j (so paired loads are aligned).  The
// last stage of the transform (p == LOG_N-1) is the N^-1-scaled one.
template <int LOG_N, int LOG_M, int LOG_E, int G, int P_LO, int P_HI>
PG_DEV void inv_round(uint64_t (&x)[1 << LOG_E], uint32_t base, uint32_t rank, const ulonglong2* __restrict__ itw,
                      const ulonglong2* sptr, const ulonglong2* srptr, uint64_t q, uint64_t nq) {
    const uint64_t q2 = 2 * q;
    constexpr int E = 1 << LOG_E;
    constexpr uint32_t N = 1u << LOG_N;
    static_for<0, P_HI - P_LO + 1>([&](auto it) {
        constexpr int p = P_LO + decltype(it)::value;
        constexpr int r = p - G;
        constexpr int half = 1 << r;
        constexpr int nk = E >> (r + 1);
        if constexpr (p == LOG_N - 1) {
            const ulonglong2 s = *sptr, sr = *srptr;
            static_for<0, E>([&](auto jt) {
                constexpr int jj = decltype(jt)::value;
                if constexpr (!(jj & half)) inv_last_bfly(x[jj], x[jj + half], s, sr, q, nq);
            });
        } else {
            const ulonglong2* row = itw + (N - (N >> p)) + (((rank << LOG_M) + base) >> (p + 1));
            auto bfly_k = [&](auto kk, const ulonglong2 w) {
                constexpr int k = decltype(kk)::value;
                static_for<0, half>([&](auto ll) {
                    constexpr int jj = (k << (r + 1)) | decltype(ll)::value;
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
template <int LOG_M, int TOP, int LOG_E, int R, bool FAST>
PG_DEV void fwd_rest(uint64_t (&x)[1 << LOG_E], uint64_t* sm, uint32_t tid, uint32_t tw_base,
                     const ulonglong2* __restrict__ tw, uint64_t q2, uint64_t nq) {
    if constexpr (R < FwdRounds<TOP, LOG_E, 0>::COUNT) {
        using Cur = FwdRounds<TOP, LOG_E, R>;
        using Prev = FwdRounds<TOP, LOG_E, R - 1>;
        store_smem<LOG_E, Prev::G>(x, sm, group_base<LOG_E>(tid, Prev::G));
        __syncthreads();
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
template <int LOG_N, int LOG_M, int TOP, int LOG_E, int R, int R_END>
PG_DEV void inv_range(uint64_t (&x)[1 << LOG_E], uint64_t* sm, uint32_t tid, uint32_t rank,
                      const ulonglong2* __restrict__ itw, const ulonglong2* sptr, const ulonglong2* srptr, uint64_t q,
                      uint64_t nq) {
    if constexpr (R < R_END) {
        using Cur = InvRounds<TOP, LOG_E, R>;
        using Prev = InvRounds<TOP, LOG_E, R - 1>;
        store_smem<LOG_E, Prev::G>(x, sm, group_base<LOG_E>(tid, Prev::G));
        __syncthreads();
        const uint32_t base = group_base<LOG_E>(tid, Cur::G);
        load_smem<LOG_E, Cur::G>(x, sm, base);
        inv_round<LOG_N, LOG_M, LOG_E, Cur::G, Cur::P_LO, Cur::P_HI>(x, base, rank, itw, sptr, srptr, q, nq);
        inv_range<LOG_N, LOG_M, TOP, LOG_E, R + 1, R_END>(x, sm, tid, rank, itw, sptr, srptr, q, nq);
    }
}

// ============================================================================
// Single-CTA kernel: ROWS rows of N = 2^LOG_N per CTA, T = N/E threads per row.
// FAST selects the forward schedule without per-butterfly reduction of u (only
// when the caller needs canonical or multiplied outputs and every q < 2^58).
// ============================================================================
template <int LOG_N, int LOG_E, int ROWS, int MODE, bool FAST>
__global__ void __launch_bounds__((1 << (LOG_N - LOG_E)) * ROWS) ntt_block_kernel(NttArgs a) {
    constexpr int N = 1 << LOG_N, E = 1 << LOG_E, T = N / E;
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
    const uint64_t* mulp = nullptr;
    if (a.desc) {  // descriptor-driven rows (ragged batches)
        const RowDesc d = a.desc[active ? u : 0];
        g = d.data;
        limb = d.limb;
        mulp = d.mul;
    }
    const uint64_t q = a.moduli[limb], q2 = q << 1, nq = 0 - q;
    uint64_t x[E];

    if constexpr (MODE == MODE_FWD || MODE == MODE_RT) {
        const ulonglong2* tw = a.fwd + (size_t)limb * N;
        using R0 = FwdRounds<LOG_N, LOG_E, 0>;
        // round 0 reads the row straight from HBM: x[jj] = row[tid + jj*T]
#pragma unroll
        for (int jj = 0; jj < E; ++jj) x[jj] = active ? g[tid + jj * T] : 0;
        fwd_round<LOG_N, LOG_E, R0::G, R0::P_HI, R0::P_LO, FAST>(x, tid, 1, tw, q2, nq);
        fwd_rest<LOG_N, LOG_N, LOG_E, 1, FAST>(x, sm, tid, 1, tw, q2, nq);
        // x = E contiguous outputs at tid*E
        if constexpr (MODE == MODE_FWD) {
            if constexpr (FAST) {
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
        } else {
            // pointwise product with the NTT-domain plaintext (Shoup-prepared);
            // the lazy product in [0, 2q) is a valid inverse input
            const uint64_t* pv = a.plain + (size_t)limb * N + tid * E;
            const uint64_t* pq = a.plain_q + (size_t)limb * N + tid * E;
#pragma unroll
            for (int jj = 0; jj < E; ++jj) x[jj] = shoup_lazy_nq(__ldg(pv + jj), __ldg(pq + jj), x[jj], nq);
        }
    }
    // ---------------- inverse
    if constexpr (MODE != MODE_FWD) {
        const ulonglong2* itw = a.inv + (size_t)limb * N;
        const ulonglong2* sptr = a.inv_n + limb;
        const ulonglong2* srptr = a.inv_last + limb;
        using I0 = InvRounds<LOG_N, LOG_E, 0>;
        if constexpr (MODE == MODE_INV) {
            // stage the bit-reversed row through smem (coalesced), then round 0
#pragma unroll
            for (int k = 0; k < E; ++k) {
                uint64_t v = active ? g[tid + k * T] : 0;
                // descriptor rows may carry an NTT-domain multiplicand (canonical inputs)
                if (mulp && active) v = barrett_mul(v, mulp[tid + k * T], a.bar[limb]);
                sm[padi(tid + k * T)] = v;
            }
            __syncthreads();
            load_smem<LOG_E, I0::G>(x, sm, group_base<LOG_E>(tid, I0::G));
        } else {
            // round trip: the forward's last group (tid*E .. tid*E+E-1) is the
            // inverse's first group (I0::G == 0), so it stays in registers
            static_assert(I0::G == 0, "round trip needs the first inverse group to be contiguous");
        }
        inv_round<LOG_N, LOG_N, LOG_E, I0::G, I0::P_LO, I0::P_HI>(x, group_base<LOG_E>(tid, I0::G), 0, itw, sptr, srptr,
                                                                  q, nq);
        inv_range<LOG_N, LOG_N, LOG_N, LOG_E, 1, I0::COUNT>(x, sm, tid, 0, itw, sptr, srptr, q, nq);
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

template <int LOG_N, int LOG_M, int LOG_E, int MODE, bool FAST>
__global__ void __launch_bounds__(1 << (LOG_M - LOG_E), cluster_min_blocks(1 << (LOG_M - LOG_E)))
    ntt_cluster_kernel(NttArgs a) {
    constexpr int LOG_C = LOG_N - LOG_M;
    constexpr int N = 1 << LOG_N, M = 1 << LOG_M, E = 1 << LOG_E, LOG_T = LOG_M - LOG_E, T = 1 << LOG_T;
    constexpr int LOG_K = LOG_E - LOG_C;  // top block bits handled by the cross phase
    constexpr int K = 1 << LOG_K;
    constexpr int TOP = LOG_M - LOG_K;    // block bits handled by the local rounds
    constexpr int GX = LOG_N - LOG_E;     // cross group stride bit (N/E)
    static_assert(LOG_K >= 0 && TOP >= LOG_E, "shape");
    extern __shared__ uint64_t smem_cl[];
    uint64_t* sm = smem_cl;
    const uint32_t tid = threadIdx.x;
    const uint32_t rank = blockIdx.x & ((1 << LOG_C) - 1);
    // grid is exactly rows * C; clusters run limb-major so that concurrently
    // running clusters share one prime's twiddles in L2
    const uint64_t u = blockIdx.x >> LOG_C;
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
    const uint32_t gt = (rank << LOG_T) + tid;  // cross group (column) of this thread
    uint64_t x[E];

    if constexpr (MODE == MODE_FWD || MODE == MODE_RT) {
        const uint64_t q2 = q << 1;
        const ulonglong2* tw = a.fwd + (size_t)limb * N;
        // matched by the wait before the first remote store; relaxed is enough
        // because this CTA has not touched shared memory yet
        cluster_arrive_relaxed();
#pragma unroll
        for (int jj = 0; jj < E; ++jj) x[jj] = g[gt + (jj << GX)];
        fwd_round<LOG_N, LOG_E, GX, LOG_N - 1, GX, FAST>(x, gt, 1, tw, q2, nq);
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
        fwd_round<LOG_M, LOG_E, R0::G, R0::P_HI, R0::P_LO, FAST>(x, group_base<LOG_E>(tid, R0::G), (1u << LOG_C) + rank,
                                                                 tw, q2, nq);
        fwd_rest<LOG_M, TOP, LOG_E, 1, FAST>(x, sm, tid, (1u << LOG_C) + rank, tw, q2, nq);
        if constexpr (MODE == MODE_FWD) {
            if constexpr (FAST) {
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
            uint64_t* gb = g + rank * M;
#pragma unroll
            for (int k = 0; k < E; ++k) gb[tid + k * T] = sm[padi(tid + k * T)];
        } else {
            const uint64_t* pv = a.plain + (size_t)limb * N + rank * M + tid * E;
            const uint64_t* pq = a.plain_q + (size_t)limb * N + rank * M + tid * E;
#pragma unroll
            for (int jj = 0; jj < E; ++jj) x[jj] = shoup_lazy_nq(__ldg(pv + jj), __ldg(pq + jj), x[jj], nq);
        }
    }
    // ---------------- inverse
    if constexpr (MODE != MODE_FWD) {
        const ulonglong2* itw = a.inv + (size_t)limb * N;
        using I0 = InvRounds<TOP, LOG_E, 0>;
        using ILast = InvRounds<TOP, LOG_E, I0::COUNT - 1>;
        static_assert(I0::COUNT >= 2, "cluster path needs two local rounds");
        if constexpr (MODE == MODE_INV) {
            uint64_t* gb = g + rank * M;
#pragma unroll
            for (int k = 0; k < E; ++k) {
                uint64_t v = gb[tid + k * T];
                // descriptor rows may carry an NTT-domain multiplicand (canonical inputs)
                if (mulp) v = barrett_mul(v, mulp[rank * M + tid + k * T], a.bar[limb]);
                sm[padi(tid + k * T)] = v;
            }
            __syncthreads();
            load_smem<LOG_E, I0::G>(x, sm, group_base<LOG_E>(tid, I0::G));
        }
        inv_round<LOG_N, LOG_M, LOG_E, I0::G, I0::P_LO, I0::P_HI>(x, group_base<LOG_E>(tid, I0::G), rank, itw, nullptr,
                                                                  nullptr, q, nq);
        inv_range<LOG_N, LOG_M, TOP, LOG_E, 1, I0::COUNT - 1>(x, sm, tid, rank, itw, nullptr, nullptr, q, nq);
        {
            // last local round: its smem loads precede the cluster arrive, so no
            // CTA overwrites a block that another CTA is still reading
            using Prev = InvRounds<TOP, LOG_E, I0::COUNT - 2>;
            store_smem<LOG_E, Prev::G>(x, sm, group_base<LOG_E>(tid, Prev::G));
            __syncthreads();
            const uint32_t base = group_base<LOG_E>(tid, ILast::G);
            load_smem<LOG_E, ILast::G>(x, sm, base);
            // release: these shared-memory reads must be performed before any
            // other CTA, released by this barrier, overwrites the block
            cluster_arrive_release();
            inv_round<LOG_N, LOG_M, LOG_E, ILast::G, ILast::P_LO, ILast::P_HI>(x, base, rank, itw, nullptr, nullptr, q,
                                                                               nq);
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
        inv_round<LOG_N, LOG_N, LOG_E, GX, GX, LOG_N - 1>(x, gt, 0, itw, a.inv_n + limb, a.inv_last + limb, q, nq);
#pragma unroll
        for (int jj = 0; jj < E; ++jj) g[gt + (jj << GX)] = x[jj];
    }
}

}  // namespace pg

namespace pg {

// ============================================================================
// Fused external product (GLWE x GGSW, k = 1, one prime, single-word values):
// CrtGlwe::mul_dcrt_ggsw_inplace (primus_lattice/src/glwe/crt.rs:202-229) and,
// for OUT_COEFF, inverse_transform_slice of both output polys.  One CTA per
// ciphertext.  For each input poly i the CTA decomposes its coefficients into
// d gadget digits (digits of one poly kept in shared memory), then for each
// digit j lifts the digit row to residues mod q, runs the forward NTT in
// shared memory and multiply-accumulates the NTT-domain row against the
// GGSW rows key[i][j][c] into 128-bit register accumulators, one per output
// element.  Outputs are canonical residues (NTT domain, or coefficient form
// after the in-kernel inverse NTT): the same residues as the reference's
// per-digit sequence, since every step is exact arithmetic mod q.
// ============================================================================
struct ExtFusedArgs {
    const uint64_t* in;   // [B][2][N] coefficient form
    const uint64_t* key;  // [2][d][2][N] NTT domain
    uint64_t* out;        // [B][2][N]
    const ulonglong2* fwd;
    const ulonglong2* inv;
    const ulonglong2* inv_n;
    const ulonglong2* inv_last;
    Barrett bar;
    GadgetWord gw;
    uint64_t B;
    int out_coeff;
};

// d digits of one word v (init_value_carry_slice_inplace, basis.rs:307-331, and
// unsigned_decompose, common.rs:150-160, with W = 1), written to dst[j * N]
template <typename DT, int N>
PG_DEV void decompose_word(uint64_t v, const GadgetWord& g, DT* dst) {
    if (g.has_split && v >= g.split) v += g.npq;
    uint64_t carry = g.has_init ? ((v & g.init_mask) != 0) : 0;
    for (uint32_t j = 0; j < g.d; ++j) {
        const DigitMask m = g.masks[j];
        // limb 1 is the zero guard limb: only limb 0 contributes bits
        uint64_t temp = m.index == 0 ? (v & m.mask0) >> m.shr : 0;
        temp += carry;
        carry = (temp & g.carry_mask) != 0;
        dst[(size_t)j * N] = (DT)(temp & g.bm1);
    }
}

template <int LOG_N, int LOG_E, typename DT, bool FAST>
__global__ void __launch_bounds__(1 << (LOG_N - LOG_E)) ext_fused_kernel(ExtFusedArgs a) {
    constexpr int N = 1 << LOG_N, E = 1 << LOG_E, T = N / E, KP = 2;
    extern __shared__ uint64_t smem_ext[];
    // shared memory: NTT exchange buffer | 128-bit accumulators [KP][E][T] | digits [d][N]
    uint64_t* sm = smem_ext;
    ulonglong2* acc = reinterpret_cast<ulonglong2*>(smem_ext + padded(N));
    DT* dg = reinterpret_cast<DT*>(acc + KP * N);
    const uint32_t tid = threadIdx.x;
    const uint64_t b = blockIdx.x;
    const Barrett bar = a.bar;
    const uint64_t q = bar.q, q2 = q << 1, nq = 0 - q;
    const uint32_t d = a.gw.d;
    const uint64_t basis = a.gw.basis, half = (basis + 1) / 2, lift = q - basis;
    using R0 = FwdRounds<LOG_N, LOG_E, 0>;
    static_assert(R0::G == LOG_N - LOG_E, "first forward group is the column tid + jj*T");
    // each thread owns accumulator entries (c, e, tid): no other thread touches them
#pragma unroll
    for (int ce = 0; ce < KP * E; ++ce) acc[ce * T + tid] = make_ulonglong2(0, 0);
    uint32_t terms = 0;
    for (int i = 0; i < KP; ++i) {
        // this thread's coefficients tid + jj*T; it alone reads their digits back
        const uint64_t* src = a.in + (b * KP + i) * N;
#pragma unroll
        for (int jj = 0; jj < E; ++jj) decompose_word<DT, N>(src[tid + jj * T], a.gw, dg + tid + jj * T);
        for (uint32_t j = 0; j < d; ++j) {
            uint64_t x[E];
#pragma unroll
            for (int jj = 0; jj < E; ++jj) {
                const uint64_t v = dg[(size_t)j * N + tid + jj * T];
                x[jj] = (basis == 2 || v < half) ? v : lift + v;  // wrapping_decompose_small_values
            }
            fwd_round<LOG_N, LOG_E, R0::G, R0::P_HI, R0::P_LO, FAST>(x, tid, 1, a.fwd, q2, nq);
            __syncthreads();  // the previous row's last shared-memory reads are done
            fwd_rest<LOG_N, LOG_N, LOG_E, 1, FAST>(x, sm, tid, 1, a.fwd, q2, nq);
            if constexpr (!FAST) {
#pragma unroll
                for (int e = 0; e < E; ++e) x[e] = canon4(x[e], q, q2);
            }
            // x = NTT-domain elements tid*E .. tid*E+E-1 of digit row (i, j); products
            // are below 2^122, so 8 of them plus a folded value stay below 2^128
            const bool fold = terms == 8;
            terms = fold ? 1 : terms + 1;
            const uint64_t* kp = a.key + ((size_t)(i * d + j) * KP) * N + tid * E;
#pragma unroll
            for (int c = 0; c < KP; ++c)
#pragma unroll
                for (int e = 0; e < E; e += 2) {
                    ulonglong2 w;
                    asm("ld.global.nc.v2.u64 {%0, %1}, [%2];" : "=l"(w.x), "=l"(w.y) : "l"(kp + c * N + e));
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        ulonglong2 s = acc[(c * E + e + h) * T + tid];
                        if (fold) {
                            s.x = barrett_reduce_2limb(s.x, s.y, bar);
                            s.y = 0;
                        }
                        const uint64_t kv = h ? w.y : w.x;
                        const uint64_t pl = kv * x[e + h], ph = mulhi64(kv, x[e + h]);
                        s.x += pl;
                        s.y += ph + (s.x < pl);
                        acc[(c * E + e + h) * T + tid] = s;
                    }
                }
        }
    }
    uint64_t* out = a.out + b * KP * N;
    if (!a.out_coeff) {
#pragma unroll
        for (int c = 0; c < KP; ++c)
#pragma unroll
            for (int e = 0; e < E; e += 2) {
                const ulonglong2 s0 = acc[(c * E + e) * T + tid], s1 = acc[(c * E + e + 1) * T + tid];
                const uint64_t r0 = barrett_reduce_2limb(s0.x, s0.y, bar);
                const uint64_t r1 = barrett_reduce_2limb(s1.x, s1.y, bar);
                asm volatile("st.global.v2.u64 [%0], {%1, %2};" ::"l"(out + c * N + tid * E + e), "l"(r0), "l"(r1)
                             : "memory");
            }
        return;
    }
    // coefficient form: inverse NTT of each output poly; the first inverse group
    // is the contiguous tid*E .. tid*E+E-1, so the accumulators feed it directly
    using I0 = InvRounds<LOG_N, LOG_E, 0>;
    static_assert(I0::G == 0, "first inverse group is contiguous");
#pragma unroll 1
    for (int c = 0; c < KP; ++c) {
        uint64_t x[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const ulonglong2 s = acc[(c * E + e) * T + tid];
            x[e] = barrett_reduce_2limb(s.x, s.y, bar);
        }
        __syncthreads();  // earlier shared-memory reads of the exchange buffer are done
        inv_round<LOG_N, LOG_N, LOG_E, I0::G, I0::P_LO, I0::P_HI>(x, tid * E, 0, a.inv, a.inv_n, a.inv_last, q, nq);
        inv_range<LOG_N, LOG_N, LOG_N, LOG_E, 1, I0::COUNT>(x, sm, tid, 0, a.inv, a.inv_n, a.inv_last, q, nq);
#pragma unroll
        for (int jj = 0; jj < E; ++jj) out[c * N + tid + jj * T] = x[jj];
    }
}

}  // namespace pg

// ============================================================================
// Launch dispatch
// ============================================================================
namespace pg {

template <int LOG_N, int LOG_E, int ROWS, int MODE, bool FAST>
static int launch_block(const NttArgs& a, cudaStream_t st) {
    constexpr int T = 1 << (LOG_N - LOG_E);
    constexpr size_t smem = (size_t)ROWS * padded(1 << LOG_N) * sizeof(uint64_t);
    auto kern = ntt_block_kernel<LOG_N, LOG_E, ROWS, MODE, FAST>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return cuda_status(attr, "ntt_block_kernel: shared memory attribute");
    dim3 block(T, ROWS);
    dim3 grid((unsigned)((a.rows + ROWS - 1) / ROWS));
    kern<<<grid, block, smem, st>>>(a);
    count_launch();
    PG_LAUNCH_CHECK("ntt_block_kernel launch");
    return PG_OK;
}

template <int LOG_N, int LOG_M, int LOG_E, int MODE, bool FAST>
static int launch_cluster(const NttArgs& a, cudaStream_t st) {
    constexpr int C = 1 << (LOG_N - LOG_M), T = 1 << (LOG_M - LOG_E);
    constexpr size_t smem = (size_t)padded(1 << LOG_M) * sizeof(uint64_t);
    auto kern = ntt_cluster_kernel<LOG_N, LOG_M, LOG_E, MODE, FAST>;
    static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return cuda_status(attr, "ntt_cluster_kernel: shared memory attribute");
    if (a.rows * C > 0x7fffffffull) return set_error(PG_ERR_UNSUPPORTED, "too many rows for one launch");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(a.rows * C));
    cfg.blockDim = dim3(T);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if constexpr (C > 8) {
        static const cudaError_t np = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (np != cudaSuccess) return cuda_status(np, "ntt_cluster_kernel: non-portable cluster size");
    }
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a);
    count_launch();
    if (e != cudaSuccess) return cuda_status(e, "ntt_cluster_kernel launch");
    return PG_OK;
}

// block size (2^PG_NTT_LOG_M elements) each CTA of a cluster owns
#ifndef PG_NTT_LOG_M
#define PG_NTT_LOG_M 12
#endif

template <int MODE, bool FAST>
static int launch_mode(const NttArgs& a, uint32_t log_n, cudaStream_t st) {
    switch (log_n) {
        case 1: return launch_block<1, 1, 128, MODE, FAST>(a, st);
        case 2: return launch_block<2, 2, 128, MODE, FAST>(a, st);
        case 3: return launch_block<3, 3, 128, MODE, FAST>(a, st);
        case 4: return launch_block<4, 3, 64, MODE, FAST>(a, st);
        case 5: return launch_block<5, 3, 32, MODE, FAST>(a, st);
        case 6: return launch_block<6, 3, 16, MODE, FAST>(a, st);
        case 7: return launch_block<7, 3, 8, MODE, FAST>(a, st);
        case 8: return launch_block<8, 3, 4, MODE, FAST>(a, st);
        case 9: return launch_block<9, 3, 2, MODE, FAST>(a, st);
        case 10: return launch_block<10, 3, 1, MODE, FAST>(a, st);
        case 11: return launch_block<11, 3, 1, MODE, FAST>(a, st);
        case 12: return launch_block<12, 4, 1, MODE, FAST>(a, st);
        case 13: return launch_block<13, 4, 1, MODE, FAST>(a, st);
        case 14: return launch_cluster<14, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        case 15: return launch_cluster<15, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        case 16: return launch_cluster<16, PG_NTT_LOG_M, 4, MODE, FAST>(a, st);
        default: return set_error(PG_ERR_UNSUPPORTED, "this build runs NTTs for log_n in [1, 16]");
    }
}

// fast schedule: every modulus below 2^58 so 36q < 2^64 (see fwd_bfly_fast)
static bool fast_ok(const NttArgs& a) { return a.max_modulus < (1ull << 58); }


// the opt-in maximum of dynamic shared memory per CTA on sm_100 (227 KiB)
constexpr size_t kExtFusedMaxSmem = 227 * 1024;

template <int LOG_N, int LOG_E, typename DT, bool FAST>
static int launch_ext_fused_t(const ExtFusedArgs& a, size_t smem, cudaStream_t st) {
    constexpr int T = 1 << (LOG_N - LOG_E);
    auto kern = ext_fused_kernel<LOG_N, LOG_E, DT, FAST>;
    // shared memory grows with the digit count; raise the limit to the largest allowed once
    static const cudaError_t attr =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kExtFusedMaxSmem);
    if (attr != cudaSuccess) return cuda_status(attr, "ext_fused_kernel: shared memory attribute");
    kern<<<(unsigned)a.B, T, smem, st>>>(a);
    count_launch();
    PG_LAUNCH_CHECK("ext_fused_kernel launch");
    return PG_OK;
}

template <typename DT, bool FAST>
static int launch_ext_fused_n(const ExtFusedArgs& a, uint32_t log_n, size_t smem, cudaStream_t st) {
    switch (log_n) {
        case 10: return launch_ext_fused_t<10, 3, DT, FAST>(a, smem, st);
        case 11: return launch_ext_fused_t<11, 3, DT, FAST>(a, smem, st);
        case 12: return launch_ext_fused_t<12, 3, DT, FAST>(a, smem, st);
        default: return set_error(PG_ERR_UNSUPPORTED, "fused external product: log_n outside 10..12");
    }
}

static size_t ext_fused_smem(const pg_ntt_table* t, const GadgetWord& gw) {
    const size_t dt = gw.log_basis <= 16 ? 2 : 8;
    return (size_t)padded((int)t->n) * 8 + 2 * t->n * 16 + (size_t)gw.d * t->n * dt;
}

bool ext_fused_eligible(const pg_ntt_table* t, const GadgetWord& gw, uint32_t k) {
    if (k != 1 || t->L != 1 || t->log_n < 10 || t->log_n > 12) return false;
    if (gw.basis < 2 || gw.basis > t->moduli[0] || gw.d == 0) return false;
    return ext_fused_smem(t, gw) <= kExtFusedMaxSmem;
}

int launch_ext_fused(const pg_ntt_table* t, const GadgetWord& gw, const uint64_t* in, const uint64_t* key,
                     uint64_t* out, size_t batch, bool out_coeff, cudaStream_t st) {
    if (batch == 0) return PG_OK;
    if (batch > 0x7fffffffull) return set_error(PG_ERR_UNSUPPORTED, "too many ciphertexts for one launch");
    ExtFusedArgs a{};
    a.in = in;
    a.key = key;
    a.out = out;
    a.fwd = t->d_fwd;
    a.inv = t->d_inv;
    a.inv_n = t->d_inv_n;
    a.inv_last = t->d_inv_last;
    a.bar = h_barrett(t->moduli[0]);
    a.gw = gw;
    a.B = batch;
    a.out_coeff = out_coeff ? 1 : 0;
    const size_t smem = ext_fused_smem(t, gw);
    const bool fast = t->moduli[0] < (1ull << 58);
    if (gw.log_basis <= 16)
        return fast ? launch_ext_fused_n<uint16_t, true>(a, t->log_n, smem, st)
                    : launch_ext_fused_n<uint16_t, false>(a, t->log_n, smem, st);
    return fast ? launch_ext_fused_n<uint64_t, true>(a, t->log_n, smem, st)
                : launch_ext_fused_n<uint64_t, false>(a, t->log_n, smem, st);
}

int launch_ntt(const NttArgs& a, uint32_t log_n, int mode, cudaStream_t st) {
    if (a.rows == 0) return PG_OK;
    switch (mode) {
        case MODE_FWD:
            if (!a.lazy && fast_ok(a)) return launch_mode<MODE_FWD, true>(a, log_n, st);
            return launch_mode<MODE_FWD, false>(a, log_n, st);
        case MODE_INV: return launch_mode<MODE_INV, false>(a, log_n, st);
        case MODE_RT:
            if (fast_ok(a)) return launch_mode<MODE_RT, true>(a, log_n, st);
            return launch_mode<MODE_RT, false>(a, log_n, st);
    }
    return set_error(PG_ERR_INVALID_ARGUMENT, "bad NTT mode");
}

// ---------------------------------------------------------------- monomials
// transform_monomial (primus_ntt/src/ntt/primitive.rs:298-349): out[i] =
// coeff * psi^((2 rev(i) + 1) * degree mod 2N); kind 0 = general coeff,
// 1 = X^degree, 2 = -X^degree (index XOR N selects -psi^k).
__global__ void monomial_kernel(uint64_t* out, const ulonglong2* __restrict__ ordinal, const uint64_t* __restrict__ moduli,
                                uint32_t log_n, uint32_t L, uint64_t coeff, uint64_t degree, int kind) {
    const size_t n = (size_t)1 << log_n;
    const size_t total = n * L;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
        const uint32_t l = (uint32_t)(idx >> log_n);
        const uint32_t i = (uint32_t)(idx & (n - 1));
        const uint64_t q = moduli[l];
        uint64_t v;
        if (kind == 0 && coeff == 0) {
            v = 0;
        } else if (degree == 0) {
            v = kind == 0 ? coeff : (kind == 1 ? 1 : q - 1);
        } else {
            const uint32_t rev = __brev(i) >> (32 - log_n);
            size_t e = ((2 * (size_t)rev + 1) * degree) & (2 * n - 1);
            const ulonglong2* o = ordinal + (size_t)l * 2 * n;
            if (kind == 2 || (kind == 0 && coeff == q - 1)) {
                v = o[e ^ n].x;
            } else if (kind == 1 || coeff == 1) {
                v = o[e].x;
            } else {
                v = shoup_mul(o[e].x, o[e].y, coeff, q);
            }
        }
        out[idx] = v;
    }
}

static int launch_monomial(const pg_ntt_table* t, uint64_t coeff, size_t degree, uint64_t* d_out, int kind,
                           cudaStream_t st) {
    if (!t || !d_out) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL table or output");
    if (degree >= t->n) return set_error(PG_ERR_INVALID_ARGUMENT, "degree must be below N");
    const size_t total = t->n * t->L;
    const unsigned threads = 256;
    const unsigned blocks = (unsigned)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    monomial_kernel<<<blocks, threads, 0, st>>>(d_out, t->d_ordinal, t->d_moduli, t->log_n, t->L, coeff, degree, kind);
    count_launch();
    PG_LAUNCH_CHECK("monomial_kernel launch");
    return PG_OK;
}

static int check_table_data(const pg_ntt_table* t, const void* d, size_t polys) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (!d && polys) return set_error(PG_ERR_INVALID_ARGUMENT, "data is NULL");
    if (t->log_n > 16) return set_error(PG_ERR_UNSUPPORTED, "this build runs NTTs for log_n in [1, 16]");
    return PG_OK;
}

static int host_roundtrip(const pg_ntt_table* t, uint64_t* h, size_t polys, int lazy, int mode) {
    int rc = check_table_data(t, h, polys);
    if (rc) return rc;
    if (polys == 0) return PG_OK;
    const size_t bytes = polys * t->L * t->n * sizeof(uint64_t);
    uint64_t* d = nullptr;
    PG_CUDA(cudaMalloc(&d, bytes));
    cudaError_t e = cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_status(e, "host transform: copy in");
    }
    rc = launch_ntt(make_args(t, d, polys * t->L, lazy), t->log_n, mode, 0);
    if (rc == PG_OK) {
        e = cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_status(e, "host transform: copy out");
    }
    cudaFree(d);
    return rc;
}

}  // namespace pg

using namespace pg;

extern "C" {

int pg_ntt_forward(const pg_ntt_table* t, uint64_t* d_data, size_t polys, int lazy, void* stream) {
    int rc = check_table_data(t, d_data, polys);
    if (rc) return rc;
    return launch_ntt(make_args(t, d_data, polys * t->L, lazy), t->log_n, MODE_FWD, (cudaStream_t)stream);
}

int pg_ntt_inverse(const pg_ntt_table* t, uint64_t* d_data, size_t polys, int lazy, void* stream) {
    int rc = check_table_data(t, d_data, polys);
    if (rc) return rc;
    return launch_ntt(make_args(t, d_data, polys * t->L, lazy), t->log_n, MODE_INV, (cudaStream_t)stream);
}

int pg_ntt_forward_host(const pg_ntt_table* t, uint64_t* h_data, size_t polys, int lazy) {
    return host_roundtrip(t, h_data, polys, lazy, MODE_FWD);
}

int pg_ntt_inverse_host(const pg_ntt_table* t, uint64_t* h_data, size_t polys, int lazy) {
    return host_roundtrip(t, h_data, polys, lazy, MODE_INV);
}

int pg_ntt_monomial(const pg_ntt_table* t, uint64_t coeff, size_t degree, uint64_t* d_out, void* stream) {
    return launch_monomial(t, coeff, degree, d_out, 0, (cudaStream_t)stream);
}

int pg_ntt_coeff_one_monomial(const pg_ntt_table* t, size_t degree, uint64_t* d_out, void* stream) {
    return launch_monomial(t, 1, degree, d_out, 1, (cudaStream_t)stream);
}

int pg_ntt_coeff_minus_one_monomial(const pg_ntt_table* t, size_t degree, uint64_t* d_out, void* stream) {
    return launch_monomial(t, 1, degree, d_out, 2, (cudaStream_t)stream);
}

int pg_dcrt_polymul_ntt_plain(const pg_ntt_table* t, uint64_t* d_data, const uint64_t* d_plain,
                              const uint64_t* d_plain_q, size_t polys, void* stream) {
    int rc = check_table_data(t, d_data, polys);
    if (rc) return rc;
    if (!d_plain || !d_plain_q) return set_error(PG_ERR_INVALID_ARGUMENT, "plaintext is NULL");
    NttArgs a = make_args(t, d_data, polys * t->L, 0);
    a.plain = d_plain;
    a.plain_q = d_plain_q;
    return launch_ntt(a, t->log_n, MODE_RT, (cudaStream_t)stream);
}

}  // extern "C"
