// Host side of libprimus_gpu: status handling, device utilities, number theory
// and NTT table construction.
//
// Table construction restates UintNttTable::new (primus_ntt/src/ntt/primitive.rs:113-185)
// with try_minimal_primitive_root (primus_ntt/src/root.rs:89-111) so that the
// device twiddles -- and therefore every output -- equal the reference's.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "internal.hpp"

namespace pg {

static thread_local std::string t_last_error;
std::atomic<uint64_t> g_launches{0};

int set_error(int status, const std::string& msg) {
    t_last_error = msg;
    return status;
}

void clear_error() { t_last_error.clear(); }

int cuda_status(cudaError_t err, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
    if (err == cudaErrorMemoryAllocation) return set_error(PG_ERR_OUT_OF_MEMORY, m);
    return set_error(PG_ERR_CUDA, m);
}

uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = h_mulmod(r, a, q);
        a = h_mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

uint64_t h_invmod(uint64_t a, uint64_t q) {
    __int128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr != 0) {
        __int128 quo = r / nr, tmp;
        tmp = t - quo * nt;
        t = nt;
        nt = tmp;
        tmp = r - quo * nr;
        r = nr;
        nr = tmp;
    }
    if (r != 1) return 0;
    if (t < 0) t += q;
    return (uint64_t)t;
}

bool h_is_prime(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t p : small) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    // witnesses that make Miller-Rabin deterministic for every 64-bit n
    static const uint64_t bases[] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    for (uint64_t b : bases) {
        uint64_t a = b % n;
        if (a == 0) continue;
        uint64_t x = h_powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (int r = 1; r < s; ++r) {
            x = h_mulmod(x, x, n);
            if (x == n - 1) {
                composite = false;
                break;
            }
        }
        if (composite) return false;
    }
    return true;
}

Barrett h_barrett(uint64_t q) {
    // ratio = floor(2^128 / q) (BarrettModulus::new_unchecked, primus_modulus/src/barrett/mod.rs:66-73)
    u128 rem = ((u128)1) % q;
    uint64_t r1 = (uint64_t)((rem << 64) / q);
    rem = (rem << 64) % q;
    uint64_t r0 = (uint64_t)((rem << 64) / q);
    Barrett b;
    b.q = q;
    b.r0 = r0;
    b.r1 = r1;
    // shifted-operand Barrett factor floor(2^(n+62) / q), n = bitlen(q)
    const int n = 64 - __builtin_clzll(q | 1);
    b.mu = (n >= 2 && n <= 62) ? (uint64_t)((((u128)1) << (n + 62)) / q) : 0;
    return b;
}

static uint32_t bit_reverse(uint32_t x, uint32_t bits) {
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

// try_minimal_primitive_root (root.rs:89-111): the smallest primitive
// 2^log_degree-th root of unity.  The reference starts from a random primitive
// root and minimises over all odd powers; starting from the first r = 2, 3, ...
// whose power is primitive reaches the same minimum.
static int minimal_root(uint32_t log_degree, uint64_t q, uint64_t& out) {
    if (log_degree == 0 || log_degree >= 63 || q < 3)
        return set_error(PG_ERR_INVALID_ARGUMENT, "minimal_root: bad degree or modulus");
    uint64_t degree = 1ull << log_degree;
    uint64_t quotient = (q - 1) >> log_degree;
    if (quotient * degree != q - 1) {
        char buf[160];
        snprintf(buf, sizeof buf, "There is no primitive root with the degree %llu and the modulus %llu!",
                 (unsigned long long)degree, (unsigned long long)q);
        return set_error(PG_ERR_NO_PRIMITIVE_ROOT, buf);
    }
    uint64_t w = 0;
    bool found = false;
    for (uint64_t r = 2; r < q && r < 1000000; ++r) {
        w = h_powmod(r, quotient, q);
        uint64_t x = w;
        for (uint32_t i = 0; i + 1 < log_degree; ++i) x = h_mulmod(x, x, q);
        if (w != 0 && x == q - 1) {
            found = true;
            break;
        }
    }
    if (!found) return set_error(PG_ERR_NO_PRIMITIVE_ROOT, "no primitive root found (modulus not prime?)");
    uint64_t best = w, g2 = h_mulmod(w, w, q), cur = w;
    uint64_t g2q = h_shoup_quotient(g2, q);
    for (uint64_t i = 0; i < degree; ++i) {
        if (cur < best) best = cur;
        cur = h_shoup_mul(g2, g2q, cur, q);
    }
    out = best;
    return PG_OK;
}

int build_host_table(uint32_t log_n, uint64_t q, HostNttTable& t) {
    if (log_n == 0 || log_n > 24) return set_error(PG_ERR_INVALID_ARGUMENT, "log_n must be in [1, 24]");
    if (q < 3 || (q >> 62) != 0) return set_error(PG_ERR_INVALID_ARGUMENT, "modulus must be in [3, 2^62)");
    uint64_t root;
    int rc = minimal_root(log_n + 1, q, root);
    if (rc) return rc;
    const size_t n = (size_t)1 << log_n;
    if ((uint64_t)n >= q) {
        char buf[128];
        snprintf(buf, sizeof buf, "degree should less than modulus: %zu >= %llu", n, (unsigned long long)q);
        return set_error(PG_ERR_DEGREE_TOO_LARGE, buf);
    }
    t.q = q;
    t.log_n = log_n;
    t.root = root;
    try {
        t.ordinal.assign(2 * n, 0);
        t.ordinal_q.assign(2 * n, 0);
        t.root_powers.assign(n, 0);
        t.root_powers_q.assign(n, 0);
        t.inv_root_powers.assign(n, 0);
        t.inv_root_powers_q.assign(n, 0);
    } catch (const std::bad_alloc&) {
        return set_error(PG_ERR_OUT_OF_MEMORY, "host table allocation failed");
    }
    // ordinal_root_powers psi^0 .. psi^(2N-1) (primitive.rs:130-137)
    const uint64_t rq = h_shoup_quotient(root, q);
    t.ordinal[0] = 1;
    t.ordinal[1] = root;
    uint64_t p = root;
    for (size_t i = 2; i < 2 * n; ++i) {
        p = h_shoup_mul(root, rq, p, q);
        t.ordinal[i] = p;
    }
    for (size_t i = 0; i < 2 * n; ++i) t.ordinal_q[i] = h_shoup_quotient(t.ordinal[i], q);
    t.inv_root = t.ordinal[2 * n - 1];
    // root_powers[rev(i)] = psi^i (:139-149)
    for (size_t i = 0; i < n; ++i) {
        uint32_t r = bit_reverse((uint32_t)i, log_n);
        t.root_powers[r] = t.ordinal[i];
        t.root_powers_q[r] = t.ordinal_q[i];
    }
    // inv_root_powers[rev(i) + 1] = psi^-(i+1), slot 0 = 1 (:151-159)
    t.inv_root_powers[0] = 1;
    t.inv_root_powers_q[0] = h_shoup_quotient(1, q);
    for (size_t i = 0; i + 1 < n; ++i) {
        uint32_t r = bit_reverse((uint32_t)i, log_n);
        t.inv_root_powers[r + 1] = t.ordinal[2 * n - 1 - i];
        t.inv_root_powers_q[r + 1] = t.ordinal_q[2 * n - 1 - i];
    }
    t.inv_n = h_invmod((uint64_t)n, q);
    t.inv_n_q = h_shoup_quotient(t.inv_n, q);
    return PG_OK;
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

// the device's scratch pool, created on first use (NULL if creation failed)
cudaMemPool_t scratch_pool(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = scratch_pool(dev);
    if (!pool) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

cudaError_t scratch_free(void* p, cudaStream_t st) { return cudaFreeAsync(p, st); }

}  // namespace pg

using namespace pg;

// ======================================================================= C ABI
extern "C" {

const char* pg_status_string(int status) {
    switch (status) {
        case PG_OK: return "ok";
        case PG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PG_ERR_NO_PRIMITIVE_ROOT: return "no primitive root";
        case PG_ERR_DEGREE_TOO_LARGE: return "degree too large";
        case PG_ERR_NOT_COPRIME: return "moduli are not co-prime";
        case PG_ERR_UNSUPPORTED: return "unsupported size";
        case PG_ERR_OUT_OF_MEMORY: return "out of memory";
        case PG_ERR_CUDA: return "CUDA error";
        case PG_ERR_TIMEOUT: return "device wait timed out";
        case PG_ERR_REJECTED: return "request rejected";
        default: return "unknown status";
    }
}

const char* pg_last_error(void) { return t_last_error.c_str(); }

const char* pg_version(void) { return "primus_b200 0.1 (sm_100a)"; }

uint64_t pg_launch_count(void) { return g_launches.load(); }

int pg_scratch_trim(size_t keep_bytes) {
    int dev = 0;
    PG_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool = scratch_pool(dev);
    if (!pool) return set_error(PG_ERR_CUDA, "scratch pool unavailable");
    PG_CUDA(cudaMemPoolTrimTo(pool, keep_bytes));
    return PG_OK;
}

int pg_device_count(int* count) {
    if (!count) return set_error(PG_ERR_INVALID_ARGUMENT, "count is NULL");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return cuda_status(e, "cudaGetDeviceCount");
    }
    *count = c;
    return PG_OK;
}

int pg_set_device(int device) {
    PG_CUDA(cudaSetDevice(device));
    return PG_OK;
}

int pg_malloc(void** d_ptr, size_t bytes) {
    if (!d_ptr) return set_error(PG_ERR_INVALID_ARGUMENT, "d_ptr is NULL");
    *d_ptr = nullptr;
    if (bytes == 0) return PG_OK;
    PG_CUDA(cudaMalloc(d_ptr, bytes));
    return PG_OK;
}

int pg_free(void* d_ptr) {
    if (d_ptr) PG_CUDA(cudaFree(d_ptr));
    return PG_OK;
}

int pg_host_alloc(void** h_ptr, size_t bytes) {
    if (!h_ptr) return set_error(PG_ERR_INVALID_ARGUMENT, "h_ptr is NULL");
    *h_ptr = nullptr;
    if (bytes == 0) return PG_OK;
    PG_CUDA(cudaMallocHost(h_ptr, bytes));
    return PG_OK;
}

int pg_host_free(void* h_ptr) {
    if (h_ptr) PG_CUDA(cudaFreeHost(h_ptr));
    return PG_OK;
}

int pg_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, void* stream) {
    if (bytes == 0) return PG_OK;
    PG_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream));
    return PG_OK;
}

int pg_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, void* stream) {
    if (bytes == 0) return PG_OK;
    PG_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    return PG_OK;
}

int pg_from_bytes(uint64_t* d_dst, size_t words, const uint8_t* h_bytes, size_t nbytes) {
    if (nbytes != words * sizeof(uint64_t))
        return set_error(PG_ERR_INVALID_ARGUMENT, "byte count is not 8 x the destination's word count");
    if (nbytes == 0) return PG_OK;
    if (!d_dst || !h_bytes) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    PG_CUDA(cudaMemcpy(d_dst, h_bytes, nbytes, cudaMemcpyHostToDevice));
    return PG_OK;
}

int pg_to_bytes(const uint64_t* d_src, size_t words, uint8_t* h_bytes, size_t nbytes) {
    if (nbytes != words * sizeof(uint64_t))
        return set_error(PG_ERR_INVALID_ARGUMENT, "byte count is not 8 x the source's word count");
    if (nbytes == 0) return PG_OK;
    if (!d_src || !h_bytes) return set_error(PG_ERR_INVALID_ARGUMENT, "NULL buffer");
    PG_CUDA(cudaMemcpy(h_bytes, d_src, nbytes, cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_memcpy_d2d(void* d_dst, const void* d_src, size_t bytes, void* stream) {
    if (bytes == 0) return PG_OK;
    PG_CUDA(cudaMemcpyAsync(d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return PG_OK;
}

int pg_memset(void* d_ptr, int value, size_t bytes, void* stream) {
    if (bytes == 0) return PG_OK;
    PG_CUDA(cudaMemsetAsync(d_ptr, value, bytes, (cudaStream_t)stream));
    return PG_OK;
}

int pg_stream_create(void** stream) {
    if (!stream) return set_error(PG_ERR_INVALID_ARGUMENT, "stream is NULL");
    cudaStream_t s;
    PG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = (void*)s;
    return PG_OK;
}

int pg_stream_destroy(void* stream) {
    if (stream) PG_CUDA(cudaStreamDestroy((cudaStream_t)stream));
    return PG_OK;
}

int pg_stream_synchronize(void* stream) {
    PG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return PG_OK;
}

int pg_device_synchronize(void) {
    PG_CUDA(cudaDeviceSynchronize());
    return PG_OK;
}

int pg_event_create(void** event) {
    if (!event) return set_error(PG_ERR_INVALID_ARGUMENT, "event is NULL");
    cudaEvent_t e;
    PG_CUDA(cudaEventCreate(&e));
    *event = (void*)e;
    return PG_OK;
}

int pg_event_destroy(void* event) {
    if (event) PG_CUDA(cudaEventDestroy((cudaEvent_t)event));
    return PG_OK;
}

int pg_event_record(void* event, void* stream) {
    PG_CUDA(cudaEventRecord((cudaEvent_t)event, (cudaStream_t)stream));
    return PG_OK;
}

int pg_event_elapsed_ms(void* start, void* stop, float* ms) {
    if (!ms) return set_error(PG_ERR_INVALID_ARGUMENT, "ms is NULL");
    PG_CUDA(cudaEventSynchronize((cudaEvent_t)stop));
    PG_CUDA(cudaEventElapsedTime(ms, (cudaEvent_t)start, (cudaEvent_t)stop));
    return PG_OK;
}

uint64_t pg_prev_prime_congruent(uint64_t bound, uint64_t m) {
    if (bound < 3 || m == 0) return 0;
    uint64_t v = ((bound - 2) / m) * m + 1;
    for (;;) {
        if (v < 2) return 0;
        if (h_is_prime(v)) return v;
        if (v < m + 1) return 0;
        v -= m;
    }
}

int pg_ntt_primes(uint64_t bound, uint64_t m, uint32_t count, uint64_t* h_out) {
    if (!h_out && count) return set_error(PG_ERR_INVALID_ARGUMENT, "h_out is NULL");
    uint64_t b = bound;
    for (uint32_t i = 0; i < count; ++i) {
        uint64_t p = pg_prev_prime_congruent(b, m);
        if (!p) return set_error(PG_ERR_INVALID_ARGUMENT, "not enough primes below the bound");
        h_out[i] = p;
        b = p;
    }
    return PG_OK;
}

int pg_minimal_primitive_root(uint32_t log_degree, uint64_t q, uint64_t* root) {
    if (!root) return set_error(PG_ERR_INVALID_ARGUMENT, "root is NULL");
    return minimal_root(log_degree, q, *root);
}

int pg_ntt_host_tables(uint32_t log_n, uint64_t q, uint64_t* root, uint64_t* inv_root, uint64_t* inv_n,
                       uint64_t* h_root_powers, uint64_t* h_root_powers_q, uint64_t* h_inv_root_powers,
                       uint64_t* h_inv_root_powers_q) {
    HostNttTable t;
    int rc = build_host_table(log_n, q, t);
    if (rc) return rc;
    size_t n = (size_t)1 << log_n;
    if (root) *root = t.root;
    if (inv_root) *inv_root = t.inv_root;
    if (inv_n) *inv_n = t.inv_n;
    if (h_root_powers) memcpy(h_root_powers, t.root_powers.data(), n * 8);
    if (h_root_powers_q) memcpy(h_root_powers_q, t.root_powers_q.data(), n * 8);
    if (h_inv_root_powers) memcpy(h_inv_root_powers, t.inv_root_powers.data(), n * 8);
    if (h_inv_root_powers_q) memcpy(h_inv_root_powers_q, t.inv_root_powers_q.data(), n * 8);
    return PG_OK;
}

static void free_table(pg_ntt_table* t) {
    if (!t) return;
    if (t->view) {
        delete t;
        return;
    }
    cudaFree(t->d_moduli);
    cudaFree(t->d_fwd);
    cudaFree(t->d_inv);
    cudaFree(t->d_ordinal);
    cudaFree(t->d_inv_n);
    cudaFree(t->d_inv_last);
    cudaFree(t->d_barrett);
    cudaFree(t->d_fwd_fp);
    cudaFree(t->d_inv_fp);
    cudaFree(t->d_inv_n_fp);
    cudaFree(t->d_inv_last_fp);
    delete t;
}

int pg_ntt_table_create(uint32_t log_n, const uint64_t* h_moduli, uint32_t moduli_count, pg_ntt_table** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!h_moduli || moduli_count == 0) return set_error(PG_ERR_INVALID_ARGUMENT, "need at least one modulus");
    pg_ntt_table* t = new (std::nothrow) pg_ntt_table();
    if (!t) return set_error(PG_ERR_OUT_OF_MEMORY, "table allocation failed");
    t->log_n = log_n;
    t->L = moduli_count;
    t->n = (size_t)1 << log_n;
    t->moduli.assign(h_moduli, h_moduli + moduli_count);
    t->host.resize(moduli_count);
    for (uint32_t l = 0; l < moduli_count; ++l) {
        int rc = build_host_table(log_n, h_moduli[l], t->host[l]);
        if (rc) {
            free_table(t);
            return rc;
        }
    }
    const size_t n = t->n, L = moduli_count;
    std::vector<ulonglong2> fwd(L * n), inv(L * n), ord(L * 2 * n), invn(L), invlast(L);
    std::vector<Barrett> bar(L);
    for (size_t l = 0; l < L; ++l) {
        const HostNttTable& h = t->host[l];
        for (size_t i = 0; i < n; ++i) {
            fwd[l * n + i] = make_ulonglong2(h.root_powers[i], h.root_powers_q[i]);
            // device slot j holds inv_root_powers[j + 1] so that pairs used by one
            // stage start at an even index (32-byte aligned)
            inv[l * n + i] = i + 1 < n ? make_ulonglong2(h.inv_root_powers[i + 1], h.inv_root_powers_q[i + 1])
                                       : make_ulonglong2(0, 0);
        }
        for (size_t i = 0; i < 2 * n; ++i) ord[l * 2 * n + i] = make_ulonglong2(h.ordinal[i], h.ordinal_q[i]);
        invn[l] = make_ulonglong2(h.inv_n, h.inv_n_q);
        // scaled_r = inv_root_powers[N-1] * N^-1 (primitive.rs:272-277)
        uint64_t sr = h_shoup_mul(h.inv_root_powers[n - 1], h.inv_root_powers_q[n - 1], h.inv_n, h.q);
        invlast[l] = make_ulonglong2(sr, h_shoup_quotient(sr, h.q));
        bar[l] = h_barrett(h.q);
    }
    cudaError_t e = cudaGetDevice(&t->device);
    if (e == cudaSuccess) e = cudaMalloc(&t->d_moduli, L * 8);
    if (e == cudaSuccess) e = cudaMalloc(&t->d_fwd, L * n * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMalloc(&t->d_inv, L * n * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMalloc(&t->d_ordinal, L * 2 * n * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMalloc(&t->d_inv_n, L * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMalloc(&t->d_inv_last, L * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMalloc(&t->d_barrett, L * sizeof(Barrett));
    if (e == cudaSuccess) e = cudaMemcpy(t->d_moduli, h_moduli, L * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->d_fwd, fwd.data(), L * n * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->d_inv, inv.data(), L * n * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(t->d_ordinal, ord.data(), L * 2 * n * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->d_inv_n, invn.data(), L * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(t->d_inv_last, invlast.data(), L * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->d_barrett, bar.data(), L * sizeof(Barrett), cudaMemcpyHostToDevice);
    // FP64-schedule copies: w / q correctly rounded (forward and inverse tables; the
    // kernels recover w = rint(wq q)), (w, w / q) pairs for the two N^-1 factors
    uint64_t maxq = 0;
    for (uint64_t m : t->moduli) maxq = m > maxq ? m : maxq;
    if (e == cudaSuccess && maxq < (1ull << 50)) {
        auto fp = [](const ulonglong2& v, uint64_t q) {
            const double w = (double)v.x;
            const double wq = w / (double)q;
            uint64_t a, b;
            std::memcpy(&a, &w, 8);
            std::memcpy(&b, &wq, 8);
            return make_ulonglong2(a, b);
        };
        std::vector<double> ffwd(L * n), finv(L * n);
        std::vector<ulonglong2> finvn(L), finvlast(L);
        for (size_t l = 0; l < L; ++l) {
            const uint64_t q = t->moduli[l];
            for (size_t i = 0; i < n; ++i) {
                ffwd[l * n + i] = (double)fwd[l * n + i].x / (double)q;
                finv[l * n + i] = (double)inv[l * n + i].x / (double)q;
            }
            finvn[l] = fp(invn[l], q);
            finvlast[l] = fp(invlast[l], q);
        }
        e = cudaMalloc(&t->d_fwd_fp, L * n * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&t->d_inv_fp, L * n * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&t->d_inv_n_fp, L * sizeof(ulonglong2));
        if (e == cudaSuccess) e = cudaMalloc(&t->d_inv_last_fp, L * sizeof(ulonglong2));
        if (e == cudaSuccess)
            e = cudaMemcpy(t->d_fwd_fp, ffwd.data(), L * n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(t->d_inv_fp, finv.data(), L * n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(t->d_inv_n_fp, finvn.data(), L * sizeof(ulonglong2), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(t->d_inv_last_fp, finvlast.data(), L * sizeof(ulonglong2), cudaMemcpyHostToDevice);
        t->fp64 = e == cudaSuccess;
    }
    if (e != cudaSuccess) {
        free_table(t);
        return cuda_status(e, "pg_ntt_table_create: device upload");
    }
    *out = t;
    return PG_OK;
}

int pg_ntt_set_fp64(pg_ntt_table* t, int enable) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (enable && !t->d_fwd_fp)
        return set_error(PG_ERR_UNSUPPORTED, "the FP64 schedule needs every modulus below 2^50");
    t->fp64 = enable ? 1 : 0;
    for (int m = 0; m < 3; ++m) t->variant[m] = 0;  // tuned shapes belong to the previous schedule
    return PG_OK;
}

int pg_ntt_fp64_enabled(const pg_ntt_table* t) { return t && t->fp64 ? 1 : 0; }

int pg_ntt_table_view(const pg_ntt_table* t, uint32_t first, uint32_t count, pg_ntt_table** out) {
    if (!out) return set_error(PG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (count == 0 || first >= t->L || count > t->L - first)
        return set_error(PG_ERR_INVALID_ARGUMENT, "limb range outside the table");
    pg_ntt_table* v = new (std::nothrow) pg_ntt_table();
    if (!v) return set_error(PG_ERR_OUT_OF_MEMORY, "table allocation failed");
    const size_t n = t->n;
    v->view = true;
    v->log_n = t->log_n;
    v->L = count;
    v->n = n;
    v->device = t->device;
    v->moduli.assign(t->moduli.begin() + first, t->moduli.begin() + first + count);
    v->host.assign(t->host.begin() + first, t->host.begin() + first + count);
    v->d_moduli = t->d_moduli + first;
    v->d_fwd = t->d_fwd + first * n;
    v->d_inv = t->d_inv + first * n;
    v->d_ordinal = t->d_ordinal + first * 2 * n;
    v->d_inv_n = t->d_inv_n + first;
    v->d_inv_last = t->d_inv_last + first;
    v->d_barrett = t->d_barrett + first;
    if (t->d_fwd_fp) {
        v->d_fwd_fp = t->d_fwd_fp + first * n;
        v->d_inv_fp = t->d_inv_fp + first * n;
        v->d_inv_n_fp = t->d_inv_n_fp + first;
        v->d_inv_last_fp = t->d_inv_last_fp + first;
    }
    v->fp64 = t->fp64;
    *out = v;
    return PG_OK;
}

int pg_ntt_table_destroy(pg_ntt_table* table) {
    free_table(table);
    return PG_OK;
}

int pg_ntt_table_info(const pg_ntt_table* t, uint32_t* log_n, uint32_t* moduli_count, size_t* poly_length,
                      size_t* crt_poly_length) {
    if (!t) return set_error(PG_ERR_INVALID_ARGUMENT, "table is NULL");
    if (log_n) *log_n = t->log_n;
    if (moduli_count) *moduli_count = t->L;
    if (poly_length) *poly_length = t->n;
    if (crt_poly_length) *crt_poly_length = t->n * t->L;
    return PG_OK;
}

int pg_ntt_table_export(const pg_ntt_table* t, uint32_t limb, uint64_t* root, uint64_t* inv_root, uint64_t* inv_n,
                        uint64_t* h_root_powers, uint64_t* h_root_powers_q, uint64_t* h_inv_root_powers,
                        uint64_t* h_inv_root_powers_q) {
    if (!t || limb >= t->L) return set_error(PG_ERR_INVALID_ARGUMENT, "bad table or limb");
    const HostNttTable& h = t->host[limb];
    size_t n = t->n;
    if (root) *root = h.root;
    if (inv_root) *inv_root = h.inv_root;
    if (inv_n) *inv_n = h.inv_n;
    if (h_root_powers) memcpy(h_root_powers, h.root_powers.data(), n * 8);
    if (h_root_powers_q) memcpy(h_root_powers_q, h.root_powers_q.data(), n * 8);
    if (h_inv_root_powers) memcpy(h_inv_root_powers, h.inv_root_powers.data(), n * 8);
    if (h_inv_root_powers_q) memcpy(h_inv_root_powers_q, h.inv_root_powers_q.data(), n * 8);
    return PG_OK;
}

int pg_fill_uniform_host(uint64_t seed, uint64_t stream_id, uint64_t q, size_t n, uint64_t* h_out) {
    if (!h_out && n) return set_error(PG_ERR_INVALID_ARGUMENT, "h_out is NULL");
    for (size_t i = 0; i < n; ++i) {
        uint64_t v = 0;
        if (q > 1) {
            int bits = 64 - __builtin_clzll(q - 1);
            for (uint64_t attempt = 0; attempt < 64; ++attempt) {
                uint64_t h = pg::hash64(seed, stream_id, i, attempt) >> (64 - bits);
                if (h < q) {
                    v = h;
                    break;
                }
            }
        }
        h_out[i] = v;
    }
    return PG_OK;
}

}  // extern "C"
