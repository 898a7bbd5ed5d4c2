// qs_api.cu — the C ABI (include/qsketch_c.h): sketch construction, host-side table
// preparation (seeds, hash masks, prime sizing) and the stream-ordered launch sequence.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <functional>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/qsketch_c.h"
#include "qs_kernels.h"

using namespace qsb;

namespace {

thread_local std::string g_err;

qs_status fail(qs_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

qs_status cuda_fail(cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(QS_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    }
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return fail(QS_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return fail(QS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(expr, what)                                     \
    do {                                                   \
        cudaError_t _e = (expr);                           \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)
#define CKB(expr, what)                                          \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return bail(cuda_fail(_e, what)); \
    } while (0)

// lib/qsketch.cu:50-115
const uint64_t kPrimes[] = {402653171, 268435399, 201326557, 134217689, 100663291, 67108859, 50331599, 33554393,
                            25165813,  16777213,  12582893,  8388593,   6291449,   4194301,  3145721,  2097143,
                            1572853,   1048573,   786431,    524287,    393209,    262139,   196597,   131071,
                            98299,     65521,     49139,     32749,     24571,     16381,    12281,    8191,
                            6143,      4093,      3067,      2039,      1531,      1021,     761,      509,
                            383,       251,       191,       127,       89,        61,       47,       31,
                            23,        13,        11,        7,         5,         3,        2};

// Allocation-failure injection (qs_test_fail_allocations): the allocation after this many
// more fails as if the device were out of memory; -1 = off.
std::atomic<int32_t> g_fail_alloc_after{-1};

// Autotuner table: the fastest pass-1 setting per size class floor(log2(n_low)).
std::mutex g_tune_mu;
std::map<int, qs_tune_config> g_tune;

int size_class(uint64_t n_low) { return n_low ? 63 - __builtin_clzll(n_low) : 0; }

bool tune_lookup(uint64_t n_low, qs_tune_config* out) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(size_class(n_low));
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}

}  // namespace

namespace qsb {
void set_last_error(const char* text) { g_err = text; }
}  // namespace qsb

struct qs_sketch {
    qs_params p{};
    int device = 0;
    uint32_t kind = 0;
    uint64_t max_batch = 0;
    uint64_t fresh = 0;       // keys inserted since create / clear (drives the chunk-size ramp)
    uint64_t ramp_first = 0;  // first chunk of the ramp, 0 = no ramp
    int agg = 1;
    std::vector<uint32_t> seeds;
    std::vector<uint32_t> masks;  // mask words
    std::vector<void*> allocs;
    MswsDev D{};
    MswsLaunch L{};
    CmDev C{};
    int cm_grid = 0;
    // host-buffer pipeline
    cudaStream_t io[2] = {nullptr, nullptr};
    cudaEvent_t done = nullptr;
    uint32_t* stage_keys[2] = {nullptr, nullptr};
    uint32_t* stage_out[2] = {nullptr, nullptr};
    uint64_t stage_n = 0;
    std::mutex mu;
    // launch accounting and optional per-launch event timing (qs_set_profiling)
    uint64_t launches[3] = {0, 0, 0};  // insert pass, repair, query
    bool prof = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[3];
    size_t ev_used[3] = {0, 0, 0};

    cudaError_t prof_begin(int k, cudaStream_t st) {
        ++launches[k];
        if (!prof) return cudaSuccess;
        if (ev_used[k] == ev[k].size()) {
            cudaEvent_t a, b;
            cudaError_t e = cudaEventCreate(&a);
            if (e == cudaSuccess) e = cudaEventCreate(&b);
            if (e != cudaSuccess) return e;
            ev[k].push_back({a, b});
        }
        return cudaEventRecord(ev[k][ev_used[k]].first, st);
    }
    cudaError_t prof_end(int k, cudaStream_t st) {
        if (!prof) return cudaSuccess;
        return cudaEventRecord(ev[k][ev_used[k]++].second, st);
    }

    template <class T>
    cudaError_t alloc(T** ptr, size_t count) {
        void* v = nullptr;
        const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
        if (g_fail_alloc_after.load() >= 0 && g_fail_alloc_after.fetch_sub(1) == 0) {
            g_fail_alloc_after.store(-1);
            return cudaErrorMemoryAllocation;  // injected (qs_test_fail_allocations)
        }
        cudaError_t e = cudaMalloc(&v, bytes);
        if (e != cudaSuccess) return e;
        allocs.push_back(v);
        e = cudaMemset(v, 0, bytes);
        *ptr = static_cast<T*>(v);
        return e;
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// generate_hashmask (lib/hashmask.cu:32-83): per mask, draw uniform_int_distribution(0,
// m_bits - padding - 1) until `ones` distinct bits are set (lib/hashmask.cu:5-20).
void gen_hashmask(uint32_t rng_seed, size_t n, size_t m_bits, size_t ones, size_t padding, uint8_t* out) {
    const size_t mb = (m_bits + 7) / 8;
    std::memset(out, 0, n * mb);
    std::minstd_rand0 eng(rng_seed);  // std::default_random_engine of libstdc++
    std::uniform_int_distribution<uint32_t> dis(0, (uint32_t)(m_bits - padding - 1));
    for (size_t i = 0; i < n; ++i) {
        uint8_t* m = out + i * mb;
        size_t j = 0;
        while (j < ones) {
            const uint32_t id = dis(eng);
            const uint8_t bit = (uint8_t)(1u << (id % 8));
            if (!(m[id / 8] & bit)) {
                m[id / 8] |= bit;
                ++j;
            }
        }
    }
}

// CPU_Tools::random(.., 1, UINT_MAX) (include/tool/tool.h:206-220).
void draw_seeds(uint32_t rng_seed, size_t count, uint32_t* out) {
    std::minstd_rand0 eng(rng_seed);
    std::uniform_int_distribution<uint32_t> dis(1u, std::numeric_limits<uint32_t>::max());
    for (size_t i = 0; i < count; ++i) out[i] = dis(eng);
}

qs_status check_status_word(qs_sketch* sk) {
    Ctl c;
    if (!sk->D.ctl) return QS_OK;
    cudaError_t e = cudaMemcpy(&c, sk->D.ctl, sizeof c, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "read status");
    if (c.status & ST_TIMEOUT) return fail(QS_ERR_TIMEOUT, "a bounded device wait timed out");
    if (c.status & ST_CAPACITY) return fail(QS_ERR_CAPACITY, "flagged-bucket list overflow");
    if (c.status & ST_POOL_FULL)
        return fail(QS_ERR_POOL_FULL, "high-level bucket pool exhausted (%llu keys dropped)",
                    (unsigned long long)c.dropped);
    return QS_OK;
}

qs_status ctl_reset(qs_sketch* sk, cudaStream_t st) {
    static const Ctl init = [] {
        Ctl c;
        std::memset(&c, 0, sizeof c);
        c.next_id = FIRST_ID;
        return c;
    }();
    CK(cudaMemcpyAsync(sk->D.ctl, &init, sizeof init, cudaMemcpyHostToDevice, st), "reset control block");
    return QS_OK;
}

qs_status setup_io(qs_sketch* sk) {
    if (sk->io[0]) return QS_OK;
    sk->stage_n = std::min<uint64_t>(sk->max_batch, 1ull << 22);
    for (int i = 0; i < 2; ++i) {
        CK(cudaStreamCreateWithFlags(&sk->io[i], cudaStreamNonBlocking), "io stream");
        CK(sk->alloc(&sk->stage_keys[i], sk->stage_n), "staging keys");
        CK(sk->alloc(&sk->stage_out[i], sk->stage_n), "staging counts");
    }
    CK(cudaEventCreateWithFlags(&sk->done, cudaEventDisableTiming), "io event");
    return QS_OK;
}

// skip: optional bitmap over the keys (bit set = the key is not for this sketch); chunk
// offsets are multiples of max_batch, itself a multiple of 32.
// table (learned split, optional): pass 1 looks keys up in this exact table itself, counts the
// hits there and marks them in `skipbuf` (max_batch / 32 words, cleared per chunk here) for the
// replay.
qs_status insert_device(qs_sketch* sk, const uint32_t* d_keys, size_t n, cudaStream_t st,
                        const uint32_t* skip = nullptr, const TableDev* table = nullptr, uint32_t* skipbuf = nullptr) {
    if (sk->kind == QS_KIND_MSWS) {
        for (size_t off = 0; off < n;) {
            uint64_t c = std::min<uint64_t>(sk->max_batch, n - off);
            // after a create or clear the chunks grow geometrically from ramp_first keys, so
            // the buckets of heavy keys link in a small first chunk (sizes stay multiples of 32)
            if (sk->ramp_first && sk->fresh < sk->max_batch)
                c = std::min<uint64_t>(c, std::max<uint64_t>(sk->ramp_first, sk->fresh));
            off += c;
            sk->fresh += c;
            const uint64_t start = off - c;
            MswsDev D = sk->D;
            D.skip = skip ? skip + start / 32 : nullptr;
            MswsDev D1 = D;
            if (table) {
                CK(cudaMemsetAsync(skipbuf, 0, (c + 31) / 32 * 4, st), "skip bits");
                D1.tbl_keys = table->keys;
                D1.tbl_counts = table->counts;
                D1.tbl_slots = table->slots;
                D1.skip_out = skipbuf;
                D.skip = skipbuf;  // the replay leaves the table's keys out
            }
            CK(sk->prof_begin(0, st), "profile");
            CK(msws_insert_pass(d_keys + start, c, D1, sk->L, sk->agg, st), "msws insert");
            CK(sk->prof_end(0, st), "profile");
            CK(sk->prof_begin(1, st), "profile");
            CK(msws_repair(d_keys + start, c, D, sk->L, st), "msws repair");
            CK(sk->prof_end(1, st), "profile");
        }
    } else {
        CK(sk->prof_begin(0, st), "profile");
        CK(cm_insert(d_keys, n, sk->C, sk->agg ? 1 : 0, sk->cm_grid, st), "cm insert");
        CK(sk->prof_end(0, st), "profile");
    }
    return QS_OK;
}

qs_status query_device(qs_sketch* sk, const uint32_t* d_keys, size_t n, uint32_t* d_out, cudaStream_t st) {
    CK(sk->prof_begin(2, st), "profile");
    if (sk->kind == QS_KIND_MSWS)
        CK(msws_query(d_keys, n, d_out, sk->D, sk->L, st), "msws query");
    else
        CK(cm_query(d_keys, n, d_out, sk->C, sk->cm_grid, st), "cm query");
    CK(sk->prof_end(2, st), "profile");
    return QS_OK;
}

}  // namespace

extern "C" {

uint32_t qs_abi_version(void) { return QS_ABI_VERSION; }

const char* qs_status_string(qs_status s) {
    switch (s) {
        case QS_OK: return "ok";
        case QS_ERR_INVALID_ARG: return "invalid argument";
        case QS_ERR_OOM: return "out of device memory";
        case QS_ERR_CUDA: return "CUDA error";
        case QS_ERR_POOL_FULL: return "high-level pool exhausted";
        case QS_ERR_TIMEOUT: return "device wait timed out";
        case QS_ERR_NO_DEVICE: return "no usable CUDA device";
        case QS_ERR_CAPACITY: return "size limit exceeded";
    }
    return "unknown status";
}

const char* qs_last_error_string(void) { return g_err.c_str(); }

void qs_params_default(qs_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->kind = QS_KIND_MSWS;
    p->m_low = 8;
    p->m_high = 32;
    p->n_high = 1024;            // src/main.cu:390-391
    p->seed_sz = 1;              // lib/default.cu:52
    p->hash_mask_table_sz = 1021;  // lib/default.cu:54
    p->hash_mask_ones = 3;       // lib/default.cu:53
    p->seed_rng = 1;
    p->mask_rng = 1;
    p->device = -1;
}

uint64_t qs_find_greatest_prime(uint64_t upper_bound) {
    for (uint64_t x : kPrimes)
        if (x <= upper_bound) return x;
    return 0;
}

uint64_t qs_number_of_buckets(uint64_t insert_keys, uint64_t m, double factor, uint32_t ones) {
    if (m == 0 || factor <= 0) return 0;
    const uint64_t row = (uint64_t)(((double)(uint64_t)((double)insert_keys / factor)) * ones) / m;
    return qs_find_greatest_prime(row);
}

qs_status qs_generate_hashmask(uint32_t rng_seed, size_t n, size_t m_bits, size_t ones, size_t padding, uint8_t* out) {
    if (!out || m_bits == 0 || m_bits <= padding || ones == 0 || ones > m_bits - padding)
        return fail(QS_ERR_INVALID_ARG, "generate_hashmask: bad sizes");
    gen_hashmask(rng_seed, n, m_bits, ones, padding, out);
    return QS_OK;
}

qs_status qs_draw_seeds(uint32_t rng_seed, size_t count, uint32_t* out) {
    if (!out && count) return fail(QS_ERR_INVALID_ARG, "draw_seeds: null output");
    draw_seeds(rng_seed, count, out);
    return QS_OK;
}

qs_status qs_create(const qs_params* params, qs_sketch** out) {
    if (!params || !out) return fail(QS_ERR_INVALID_ARG, "qs_create: null argument");
    *out = nullptr;
    const qs_params& p = *params;
    if (p.kind != QS_KIND_MSWS && p.kind != QS_KIND_PLAIN_CM && p.kind != QS_KIND_BUCKET)
        return fail(QS_ERR_INVALID_ARG, "unknown kind %u", p.kind);
    if (p.seed_sz != 1) return fail(QS_ERR_INVALID_ARG, "seed_sz must be 1 (lib/default.cu:52)");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return cuda_fail(e == cudaSuccess ? cudaErrorNoDevice : e, "cudaGetDeviceCount");
    int dev = p.device;
    if (dev < 0) cudaGetDevice(&dev);
    if (dev >= ndev) return fail(QS_ERR_INVALID_ARG, "device %d out of range", dev);
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (major != 10 || minor != 0)
        return fail(QS_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a only", dev, major, minor);
    DeviceGuard guard(dev);

    qs_sketch* sk = new qs_sketch();
    sk->p = p;
    sk->device = dev;
    sk->kind = p.kind;
    sk->max_batch = p.max_batch ? p.max_batch : (1ull << 22);
    if (p.first_chunk & 31) {
        delete sk;
        return fail(QS_ERR_INVALID_ARG, "first_chunk must be a multiple of 32");
    }
    sk->ramp_first = (p.flags & QS_FLAG_NO_CHUNK_RAMP) ? 0 : (p.first_chunk ? p.first_chunk : (1ull << 18));
    if (sk->max_batch > (1ull << 26) || (sk->max_batch & 31)) {
        delete sk;
        return fail(QS_ERR_INVALID_ARG, "max_batch must be a multiple of 32 and at most 2^26");
    }
    // aggregate: 1 none, 2 warp, 3 warp + block, 0 = default (3)
    if (p.aggregate > 3) {
        delete sk;
        return fail(QS_ERR_INVALID_ARG, "aggregate out of [0, 3]");
    }
    sk->agg = p.aggregate == 0 ? 2 : (int)p.aggregate - 1;
    auto bail = [&](qs_status s) {
        qs_destroy(sk);
        return s;
    };

    if (p.kind == QS_KIND_MSWS) {
        if (p.m_low != 8) return bail(fail(QS_ERR_INVALID_ARG, "m_low must be 8 (32 B low buckets)"));
        if (p.m_high != 32) return bail(fail(QS_ERR_INVALID_ARG, "m_high must be 32"));
        uint64_t n_low = p.n_low ? p.n_low : qs_find_greatest_prime(p.low_bytes / 32);
        if (n_low == 0 || n_low > 0xffffffffull) return bail(fail(QS_ERR_INVALID_ARG, "n_low out of range"));
        if (p.n_high < 2 || p.n_high > (1ull << 30)) return bail(fail(QS_ERR_INVALID_ARG, "n_high out of [2, 2^30]"));
        const uint32_t H = p.hash_mask_table_sz;
        if (H == 0 || H > 16384) return bail(fail(QS_ERR_INVALID_ARG, "hash_mask_table_sz out of [1, 16384]"));
        // insert knobs: explicit, else the autotuner's entry for this size class, else defaults
        qs_tune_config tc{};
        const bool tuned = p.lanes_per_key == 0 && p.aggregate == 0 && p.route == 0 && p.ctas_per_sm == 0 &&
                           p.keys_per_tile == 0 && tune_lookup(n_low, &tc);
        const uint32_t tile = tuned && tc.keys_per_tile ? tc.keys_per_tile : (p.keys_per_tile ? p.keys_per_tile : 2048u);
        if (tile != 256 && tile != 512 && tile != 1024 && tile != 2048)
            return bail(fail(QS_ERR_INVALID_ARG, "keys_per_tile must be 0, 256, 512, 1024 or 2048"));
        // default 4 lanes per key (measured fastest on every workload here)
        const uint32_t route = tuned ? tc.route : (p.route ? p.route : 1u);
        const uint32_t lpk = tuned ? tc.lanes_per_key : (p.lanes_per_key ? p.lanes_per_key : 4u);
        if (lpk != 1 && lpk != 2 && lpk != 4 && lpk != 8 && lpk != 16 && lpk != 32)
            return bail(fail(QS_ERR_INVALID_ARG, "lanes_per_key must be 0, 1, 2, 4, 8, 16 or 32"));
        if (route > 3) return bail(fail(QS_ERR_INVALID_ARG, "route out of [0, 3]"));
        if (route == 2 && lpk > 8) return bail(fail(QS_ERR_INVALID_ARG, "route 2 needs at most 8 lanes per key"));
        if (p.ctas_per_sm > 64) return bail(fail(QS_ERR_INVALID_ARG, "ctas_per_sm out of [0, 64]"));
        if (tuned) {
            sk->agg = (int)tc.aggregate - 1;
            if (!p.max_batch && tc.max_batch) sk->max_batch = tc.max_batch;
            if (!p.first_chunk && !(p.flags & QS_FLAG_NO_CHUNK_RAMP)) sk->ramp_first = tc.first_chunk;
        }
        std::vector<uint8_t> bytes((size_t)H * 4);
        if (p.mask_table) {
            std::memcpy(bytes.data(), p.mask_table, bytes.size());
        } else {
            if (p.hash_mask_ones == 0 || p.hash_mask_ones > (uint32_t)LOW_COUNTERS)
                return bail(fail(QS_ERR_INVALID_ARG, "hash_mask_ones out of [1, 28]"));
            gen_hashmask(p.mask_rng, H, 32, p.hash_mask_ones, 4, bytes.data());  // device_sketch_v3.h:559
        }
        sk->masks.resize(H);
        for (uint32_t i = 0; i < H; ++i) {
            uint32_t w = (uint32_t)bytes[4 * i] | ((uint32_t)bytes[4 * i + 1] << 8) | ((uint32_t)bytes[4 * i + 2] << 16) |
                         ((uint32_t)bytes[4 * i + 3] << 24);
            if (w == 0 || (w >> LOW_COUNTERS)) return bail(fail(QS_ERR_INVALID_ARG, "mask %u selects no counter or a bit above 27", i));
            sk->masks[i] = w;
        }
        sk->seeds.resize(1);
        if (p.seeds)
            sk->seeds[0] = p.seeds[0];
        else if (p.hash_seed)
            sk->seeds[0] = p.hash_seed;
        else
            draw_seeds(p.seed_rng, 1, sk->seeds.data());

        MswsDev& D = sk->D;
        D.n_low = n_low;
        D.n_high = p.n_high;
        D.fm_low = make_fastmod((uint32_t)n_low);
        D.fm_mask = make_fastmod(H);
        D.seed = sk->seeds[0];
        D.n_masks = H;
        D.compat_v3 = (p.flags & QS_FLAG_COMPAT_V3) ? 1u : 0u;
        D.route = route == 3 ? 0u : route;  // 0 in the kernel = adaptive per tile
        const uint64_t B = sk->max_batch;
        const uint64_t cap = std::min<uint64_t>(n_low, B);
        D.flag_cap = (uint32_t)cap;
        D.max_tiles = (uint32_t)((B + REPAIR_TILE - 1) / REPAIR_TILE);
        D.long_cap = (uint32_t)std::min<uint64_t>(cap, 1ull << 16);  // slots with grid-computed totals
        uint32_t* masks_d = nullptr;
        CKB(sk->alloc(&D.low, n_low * LOW_WORDS), "alloc low table");
        CKB(sk->alloc(&D.high, p.n_high * HIGH_WORDS), "alloc high table");
        CKB(sk->alloc(&masks_d, H), "alloc masks");
        D.masks = masks_d;
        CKB(sk->alloc(&D.ctl, 1), "alloc control");
        CKB(sk->alloc(&D.flag_list, cap), "alloc flag list");
        CKB(sk->alloc(&D.tile_counts, D.max_tiles), "alloc tile counts");
        CKB(sk->alloc(&D.rec[0], B), "alloc records");
        CKB(sk->alloc(&D.rec[1], B), "alloc records");
        CKB(sk->alloc(&D.hist, (uint64_t)256 * D.max_tiles + 256), "alloc histograms");  // + digit totals
        CKB(sk->alloc(&D.seg_beg, cap), "alloc segments");
        CKB(sk->alloc(&D.totals, (uint64_t)D.long_cap * LOW_COUNTERS), "alloc totals");
        CKB(sk->alloc(&D.rpos[0], B), "alloc record positions");
        CKB(sk->alloc(&D.rpos[1], B), "alloc record positions");
        CKB(sk->alloc(&D.sw, cap), "alloc link order");
        CKB(sk->alloc(&D.sw_base, cap), "alloc link order");
        CKB(sk->alloc(&D.sw_bits, (B + 31) / 32), "alloc link order");
        CKB(sk->alloc(&D.sw_cnt, (B + SW_BLOCK - 1) / SW_BLOCK), "alloc link order");
        CKB(cudaMemcpy(masks_d, sk->masks.data(), (size_t)H * 4, cudaMemcpyHostToDevice), "upload masks");
        qs_status s = ctl_reset(sk, 0);
        if (s != QS_OK) return bail(s);
        CKB(cudaStreamSynchronize(0), "create sync");
        e = msws_configure(dev, H, &sk->L);
        if (e != cudaSuccess) return bail(cuda_fail(e, "configure kernels"));
        sk->L.lanes_per_key = (int)lpk;
        sk->L.tile_keys = (int)tile;
        sk->L.ctas_per_sm = tuned ? (int)tc.ctas_per_sm : (int)p.ctas_per_sm;
    } else if (p.kind == QS_KIND_BUCKET) {
        // the reference's warp (m = 32) and sub-warp (m = 8, 16) sketches: n buckets of m u32
        // counters, masks of m bits with `ones` set (generate_hashmask(H, m), padding 0;
        // device_sketch_v1.h:254-274)
        const uint32_t m = p.m_low;
        if (m != 8 && m != 16 && m != 32) return bail(fail(QS_ERR_INVALID_ARG, "bucket sketch: m_low must be 8, 16 or 32"));
        const uint64_t n = p.n_low ? p.n_low : qs_find_greatest_prime(p.low_bytes / (4ull * m));
        if (n == 0 || n > 0xffffffffull) return bail(fail(QS_ERR_INVALID_ARG, "bucket sketch: n out of range"));
        const uint32_t H = p.hash_mask_table_sz;
        if (H == 0 || H > 16384) return bail(fail(QS_ERR_INVALID_ARG, "hash_mask_table_sz out of [1, 16384]"));
        const uint32_t mb = m / 8;  // bytes per mask
        std::vector<uint8_t> bytes((size_t)H * mb);
        if (p.mask_table) {
            std::memcpy(bytes.data(), p.mask_table, bytes.size());
        } else {
            if (p.hash_mask_ones == 0 || p.hash_mask_ones > m)
                return bail(fail(QS_ERR_INVALID_ARG, "hash_mask_ones out of [1, m_low]"));
            gen_hashmask(p.mask_rng, H, m, p.hash_mask_ones, 0, bytes.data());
        }
        sk->masks.resize(H);
        for (uint32_t i = 0; i < H; ++i) {
            uint32_t w = 0;
            for (uint32_t k = 0; k < mb; ++k) w |= (uint32_t)bytes[(size_t)mb * i + k] << (8 * k);
            if (w == 0) return bail(fail(QS_ERR_INVALID_ARG, "mask %u selects no counter", i));
            sk->masks[i] = w;
        }
        sk->seeds.resize(1);
        if (p.seeds)
            sk->seeds[0] = p.seeds[0];
        else if (p.hash_seed)
            sk->seeds[0] = p.hash_seed;
        else
            draw_seeds(p.seed_rng, 1, sk->seeds.data());  // ds.resize(1, _ss), device_sketch_v1.h:267
        CmDev& C = sk->C;
        C.n = n;
        C.fm = make_fastmod((uint32_t)n);
        C.rows = m;
        C.seeds[0] = sk->seeds[0];
        C.n_masks = H;
        C.fm_mask = make_fastmod(H);
        uint32_t* masks_d = nullptr;
        CKB(sk->alloc(&C.table, n * m), "alloc bucket table");
        CKB(sk->alloc(&masks_d, H), "alloc masks");
        CKB(cudaMemcpy(masks_d, sk->masks.data(), (size_t)H * 4, cudaMemcpyHostToDevice), "upload masks");
        C.masks = masks_d;
        CKB(sk->alloc(&sk->D.ctl, 1), "alloc control");  // status word (bounded remove loops)
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        sk->cm_grid = sms * 8;
        CKB(cudaDeviceSynchronize(), "create sync");
    } else {
        const uint32_t rows = p.m_low;
        if (rows == 0 || rows > (uint32_t)MAX_CM_ROWS) return bail(fail(QS_ERR_INVALID_ARG, "cm rows out of [1, 16]"));
        uint64_t n = p.n_low ? p.n_low : qs_find_greatest_prime(p.low_bytes / (4ull * rows));
        if (n == 0 || n > 0xffffffffull) return bail(fail(QS_ERR_INVALID_ARG, "cm n out of range"));
        sk->seeds.resize(rows);
        if (p.seeds)
            std::memcpy(sk->seeds.data(), p.seeds, rows * 4);
        else
            draw_seeds(p.seed_rng, rows, sk->seeds.data());  // ds.resize(_m, _ss), device_sketch_v0.h:130
        CmDev& C = sk->C;
        C.n = n;
        C.fm = make_fastmod((uint32_t)n);
        C.rows = rows;
        for (uint32_t j = 0; j < rows; ++j) C.seeds[j] = sk->seeds[j];
        CKB(sk->alloc(&C.table, n * rows), "alloc cm table");
        CKB(sk->alloc(&sk->D.ctl, 1), "alloc control");  // status word (bounded remove loops)
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        sk->cm_grid = sms * 8;
        CKB(cudaDeviceSynchronize(), "create sync");
    }
    *out = sk;
    return QS_OK;
}

qs_status qs_destroy(qs_sketch* sk) {
    if (!sk) return QS_OK;
    {
        DeviceGuard guard(sk->device);
        for (int i = 0; i < 2; ++i)
            if (sk->io[i]) {
                cudaStreamSynchronize(sk->io[i]);
                cudaStreamDestroy(sk->io[i]);
            }
        if (sk->done) cudaEventDestroy(sk->done);
        for (auto& v : sk->ev)
            for (auto& pr : v) {
                cudaEventDestroy(pr.first);
                cudaEventDestroy(pr.second);
            }
        cudaDeviceSynchronize();
        for (void* v : sk->allocs) cudaFree(v);
    }
    delete sk;
    return QS_OK;
}

qs_status qs_insert(qs_sketch* sk, const uint32_t* d_keys, size_t n, void* stream) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (n == 0) return QS_OK;
    if (!d_keys) return fail(QS_ERR_INVALID_ARG, "null keys");
    if ((reinterpret_cast<uintptr_t>(d_keys) & 3u) != 0) return fail(QS_ERR_INVALID_ARG, "keys not 4-byte aligned");
    DeviceGuard guard(sk->device);
    return insert_device(sk, d_keys, n, static_cast<cudaStream_t>(stream));
}

qs_status qs_remove(qs_sketch* sk, const uint32_t* d_keys, size_t n, void* stream) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (n == 0) return QS_OK;
    if (!d_keys) return fail(QS_ERR_INVALID_ARG, "null keys");
    if ((reinterpret_cast<uintptr_t>(d_keys) & 3u) != 0) return fail(QS_ERR_INVALID_ARG, "keys not 4-byte aligned");
    DeviceGuard guard(sk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (sk->kind == QS_KIND_MSWS)
        CK(msws_remove(d_keys, n, sk->D, sk->L, st), "msws remove");
    else
        CK(cm_remove(d_keys, n, sk->C, sk->cm_grid, sk->D.ctl ? &sk->D.ctl->status : nullptr, st), "cm remove");
    return QS_OK;
}

qs_status qs_query(qs_sketch* sk, const uint32_t* d_keys, size_t n, uint32_t* d_counts, void* stream) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (n == 0) return QS_OK;
    if (!d_keys || !d_counts) return fail(QS_ERR_INVALID_ARG, "null keys or counts");
    if (((reinterpret_cast<uintptr_t>(d_keys) | reinterpret_cast<uintptr_t>(d_counts)) & 3u) != 0)
        return fail(QS_ERR_INVALID_ARG, "keys/counts not 4-byte aligned");
    DeviceGuard guard(sk->device);
    return query_device(sk, d_keys, n, d_counts, static_cast<cudaStream_t>(stream));
}

qs_status qs_insert_host(qs_sketch* sk, const uint32_t* h_keys, size_t n) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (n == 0) return QS_OK;
    if (!h_keys) return fail(QS_ERR_INVALID_ARG, "null keys");
    DeviceGuard guard(sk->device);
    std::lock_guard<std::mutex> lk(sk->mu);
    qs_status s = setup_io(sk);
    if (s != QS_OK) return s;
    // Chunk c copies on io[c % 2] while chunk c-1 is inserted on io[(c-1) % 2]; the inserts
    // stay in array order through the `done` event.
    bool first = true;
    uint64_t c = 0;
    for (size_t off = 0; off < n; off += sk->stage_n, ++c) {
        const int b = (int)(c & 1);
        const uint64_t len = std::min<uint64_t>(sk->stage_n, n - off);
        CK(cudaMemcpyAsync(sk->stage_keys[b], h_keys + off, len * 4, cudaMemcpyHostToDevice, sk->io[b]), "H2D keys");
        if (!first) CK(cudaStreamWaitEvent(sk->io[b], sk->done, 0), "order inserts");
        s = insert_device(sk, sk->stage_keys[b], len, sk->io[b]);
        if (s != QS_OK) return s;
        CK(cudaEventRecord(sk->done, sk->io[b]), "record insert");
        first = false;
    }
    CK(cudaStreamSynchronize(sk->io[0]), "sync io");
    CK(cudaStreamSynchronize(sk->io[1]), "sync io");
    return QS_OK;
}

qs_status qs_query_host(qs_sketch* sk, const uint32_t* h_keys, size_t n, uint32_t* h_counts) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (n == 0) return QS_OK;
    if (!h_keys || !h_counts) return fail(QS_ERR_INVALID_ARG, "null keys or counts");
    DeviceGuard guard(sk->device);
    std::lock_guard<std::mutex> lk(sk->mu);
    qs_status s = setup_io(sk);
    if (s != QS_OK) return s;
    uint64_t c = 0;
    for (size_t off = 0; off < n; off += sk->stage_n, ++c) {
        const int b = (int)(c & 1);
        const uint64_t len = std::min<uint64_t>(sk->stage_n, n - off);
        CK(cudaMemcpyAsync(sk->stage_keys[b], h_keys + off, len * 4, cudaMemcpyHostToDevice, sk->io[b]), "H2D keys");
        s = query_device(sk, sk->stage_keys[b], len, sk->stage_out[b], sk->io[b]);
        if (s != QS_OK) return s;
        CK(cudaMemcpyAsync(h_counts + off, sk->stage_out[b], len * 4, cudaMemcpyDeviceToHost, sk->io[b]), "D2H counts");
    }
    CK(cudaStreamSynchronize(sk->io[0]), "sync io");
    CK(cudaStreamSynchronize(sk->io[1]), "sync io");
    return QS_OK;
}

qs_status qs_clear(qs_sketch* sk, void* stream) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    DeviceGuard guard(sk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (sk->kind == QS_KIND_MSWS) {
        CK(cudaMemsetAsync(sk->D.low, 0, sk->D.n_low * LOW_WORDS * 4, st), "clear low");
        CK(cudaMemsetAsync(sk->D.high, 0, sk->D.n_high * HIGH_WORDS * 4, st), "clear high");
        sk->fresh = 0;
        return ctl_reset(sk, st);
    }
    CK(cudaMemsetAsync(sk->C.table, 0, sk->C.n * sk->C.rows * 4, st), "clear table");
    return QS_OK;
}

qs_status qs_sync(qs_sketch* sk, void* stream) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    DeviceGuard guard(sk->device);
    CK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "stream sync");
    return check_status_word(sk);
}

qs_status qs_get_stats(qs_sketch* sk, qs_stats* out) {
    if (!sk || !out) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(sk->device);
    std::memset(out, 0, sizeof *out);
    if (sk->kind != QS_KIND_MSWS) return QS_OK;
    CK(cudaDeviceSynchronize(), "stats sync");
    Ctl c;
    CK(cudaMemcpy(&c, sk->D.ctl, sizeof c, cudaMemcpyDeviceToHost), "read stats");
    out->status_bits = c.status;
    const uint64_t cap = (uint64_t)START + sk->D.n_high;
    out->next_level_id = (uint32_t)std::min<uint64_t>(c.next_id, cap);
    out->linked_buckets = out->next_level_id - FIRST_ID;
    out->dropped_keys = c.dropped;
    out->repaired_buckets = c.repaired_buckets;
    out->repaired_keys = c.repaired_keys;
    return QS_OK;
}

qs_status qs_set_profiling(qs_sketch* sk, int enable) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    DeviceGuard guard(sk->device);
    CK(cudaDeviceSynchronize(), "profiling sync");
    sk->prof = enable != 0;
    sk->D.prof = enable != 0 ? 1u : 0u;  // the repair's device phase timers
    for (int k = 0; k < 3; ++k) sk->ev_used[k] = 0;
    return QS_OK;
}

qs_status qs_get_profile(qs_sketch* sk, qs_profile* out) {
    if (!sk || !out) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(sk->device);
    CK(cudaDeviceSynchronize(), "profile sync");
    std::memset(out, 0, sizeof *out);
    double ms[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k)
        for (size_t i = 0; i < sk->ev_used[k]; ++i) {
            float t = 0;
            CK(cudaEventElapsedTime(&t, sk->ev[k][i].first, sk->ev[k][i].second), "event time");
            ms[k] += t;
        }
    out->insert_ms = ms[0];
    out->repair_ms = ms[1];
    out->query_ms = ms[2];
    out->insert_timed = sk->ev_used[0];
    out->repair_timed = sk->ev_used[1];
    out->query_timed = sk->ev_used[2];
    out->insert_launches = sk->launches[0];
    out->repair_launches = sk->launches[1];
    out->query_launches = sk->launches[2];
    for (int k = 0; k < 3; ++k) sk->ev_used[k] = 0;
    if (sk->kind == QS_KIND_MSWS) {
        Ctl c;
        CK(cudaMemcpy(&c, sk->D.ctl, sizeof c, cudaMemcpyDeviceToHost), "read repair phases");
        out->repairs_active = c.repairs;
        for (int k = 0; k < 12; ++k) out->repair_phase_ms[k] = (double)c.phase_ns[k] * 1e-6;
        CK(cudaMemset(&sk->D.ctl->repairs, 0, sizeof(Ctl) - offsetof(Ctl, repairs)), "reset repair phases");
    }
    return QS_OK;
}

qs_status qs_reset_status(qs_sketch* sk) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (!sk->D.ctl) return QS_OK;
    DeviceGuard guard(sk->device);
    CK(cudaDeviceSynchronize(), "sync");
    CK(cudaMemset(&sk->D.ctl->status, 0, 4), "reset status");
    return QS_OK;
}

qs_status qs_get_info(qs_sketch* sk, uint64_t* n_low, uint64_t* n_high, uint32_t* m_low, uint32_t* seeds_out,
                      uint8_t* mask_table_out) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    if (sk->kind == QS_KIND_MSWS) {
        if (n_low) *n_low = sk->D.n_low;
        if (n_high) *n_high = sk->D.n_high;
        if (m_low) *m_low = LOW_WORDS;
        if (mask_table_out) std::memcpy(mask_table_out, sk->masks.data(), sk->masks.size() * 4);
    } else {
        if (n_low) *n_low = sk->C.n;
        if (n_high) *n_high = 0;
        if (m_low) *m_low = sk->C.rows;
        if (mask_table_out && sk->kind == QS_KIND_BUCKET)  // H masks of m/8 bytes
            for (size_t i = 0; i < sk->masks.size(); ++i)
                for (uint32_t k = 0; k < sk->C.rows / 8; ++k)
                    mask_table_out[i * (sk->C.rows / 8) + k] = (uint8_t)(sk->masks[i] >> (8 * k));
    }
    if (seeds_out) std::memcpy(seeds_out, sk->seeds.data(), sk->seeds.size() * 4);
    return QS_OK;
}

qs_status qs_get_params(qs_sketch* sk, qs_params* out) {
    if (!sk || !out) return fail(QS_ERR_INVALID_ARG, "qs_get_params: null argument");
    *out = sk->p;
    out->seeds = nullptr;       // the caller's arrays are not kept
    out->mask_table = nullptr;
    out->hash_seed = sk->seeds.empty() ? 0u : sk->seeds[0];
    out->n_low = sk->kind == QS_KIND_MSWS ? sk->D.n_low : sk->C.n;
    out->hash_mask_table_sz = (uint32_t)sk->masks.size();
    out->max_batch = sk->max_batch;
    out->device = sk->device;
    return QS_OK;
}

qs_status qs_get_tables(qs_sketch* sk, uint32_t* h_low, uint32_t* h_high) {
    if (!sk) return fail(QS_ERR_INVALID_ARG, "null sketch");
    DeviceGuard guard(sk->device);
    CK(cudaDeviceSynchronize(), "tables sync");
    if (sk->kind == QS_KIND_MSWS) {
        if (h_low) CK(cudaMemcpy(h_low, sk->D.low, sk->D.n_low * LOW_WORDS * 4, cudaMemcpyDeviceToHost), "copy low");
        if (h_high) CK(cudaMemcpy(h_high, sk->D.high, sk->D.n_high * HIGH_WORDS * 4, cudaMemcpyDeviceToHost), "copy high");
    } else if (h_low) {
        CK(cudaMemcpy(h_low, sk->C.table, sk->C.n * sk->C.rows * 4, cudaMemcpyDeviceToHost), "copy table");
    }
    return QS_OK;
}

// ---- snapshots (the reference declares read_file / write_file, include/qsketch.h:70-71, and
// never defines them) -----------------------------------------------------------------------
// Layout, little-endian: SnapHeader, then the seeds (u32), the mask words (u32), the low table
// and (MSWS) the high pool, then a 64-bit FNV-1a checksum of everything before it.
struct SnapHeader {
    char magic[8];  // "QSKSNAP" + NUL
    uint32_t version, kind;
    uint64_t n_low, n_high;
    uint32_t m_low, m_high, n_seeds, n_masks;
    uint32_t hash_mask_ones, flags, next_level_id, status_bits;
    uint64_t dropped_keys, payload_bytes, reserved[2];
};
static_assert(sizeof(SnapHeader) == 96, "snapshot header layout");
constexpr char SNAP_MAGIC[8] = {'Q', 'S', 'K', 'S', 'N', 'A', 'P', 0};

static uint64_t fnv1a64(const unsigned char* p, uint64_t n, uint64_t h = 0xcbf29ce484222325ull) {
    for (uint64_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
    return h;
}

static uint64_t snap_table_words(const qs_sketch* sk, uint64_t* low_words, uint64_t* high_words) {
    *low_words = sk->kind == QS_KIND_MSWS ? sk->D.n_low * LOW_WORDS : sk->C.n * sk->C.rows;
    *high_words = sk->kind == QS_KIND_MSWS ? sk->D.n_high * HIGH_WORDS : 0;
    return *low_words + *high_words;
}

qs_status qs_snapshot_bytes(qs_sketch* sk, uint64_t* bytes) {
    if (!sk || !bytes) return fail(QS_ERR_INVALID_ARG, "qs_snapshot_bytes: null argument");
    uint64_t lw, hw;
    const uint64_t tw = snap_table_words(sk, &lw, &hw);
    *bytes = sizeof(SnapHeader) + 4 * (sk->seeds.size() + sk->masks.size() + tw) + 8;
    return QS_OK;
}

qs_status qs_snapshot_save(qs_sketch* sk, void* h_buf, uint64_t buf_bytes) {
    uint64_t need = 0;
    qs_status st = qs_snapshot_bytes(sk, &need);
    if (st != QS_OK) return st;
    if (!h_buf || buf_bytes < need) return fail(QS_ERR_INVALID_ARG, "qs_snapshot_save: buffer of %llu bytes needed",
                                                (unsigned long long)need);
    DeviceGuard guard(sk->device);
    CK(cudaDeviceSynchronize(), "snapshot sync");
    SnapHeader h{};
    std::memcpy(h.magic, SNAP_MAGIC, 8);
    h.version = 1;
    h.kind = sk->kind;
    uint64_t lw, hw;
    snap_table_words(sk, &lw, &hw);
    if (sk->kind == QS_KIND_MSWS) {
        Ctl c;
        CK(cudaMemcpy(&c, sk->D.ctl, sizeof c, cudaMemcpyDeviceToHost), "read control block");
        h.n_low = sk->D.n_low;
        h.n_high = sk->D.n_high;
        h.m_low = LOW_WORDS;
        h.m_high = HIGH_WORDS;
        h.next_level_id = c.next_id;
        h.status_bits = c.status;
        h.dropped_keys = c.dropped;
        h.hash_mask_ones = sk->p.hash_mask_ones;
        h.flags = sk->D.compat_v3 ? QS_FLAG_COMPAT_V3 : 0u;
    } else {
        h.n_low = sk->C.n;
        h.m_low = sk->C.rows;
    }
    h.n_seeds = (uint32_t)sk->seeds.size();
    h.n_masks = (uint32_t)sk->masks.size();
    h.payload_bytes = need - sizeof h - 8;
    unsigned char* out = static_cast<unsigned char*>(h_buf);
    std::memcpy(out, &h, sizeof h);
    unsigned char* q = out + sizeof h;
    std::memcpy(q, sk->seeds.data(), 4 * sk->seeds.size());
    q += 4 * sk->seeds.size();
    std::memcpy(q, sk->masks.data(), 4 * sk->masks.size());
    q += 4 * sk->masks.size();
    CK(cudaMemcpy(q, sk->kind == QS_KIND_MSWS ? sk->D.low : sk->C.table, lw * 4, cudaMemcpyDeviceToHost), "copy low");
    q += lw * 4;
    if (hw) CK(cudaMemcpy(q, sk->D.high, hw * 4, cudaMemcpyDeviceToHost), "copy high");
    q += hw * 4;
    const uint64_t sum = fnv1a64(out, (uint64_t)(q - out));
    std::memcpy(q, &sum, 8);
    return QS_OK;
}

qs_status qs_snapshot_load(const void* h_buf, uint64_t bytes, int32_t device, qs_sketch** out) {
    if (!h_buf || !out) return fail(QS_ERR_INVALID_ARG, "qs_snapshot_load: null argument");
    *out = nullptr;
    const unsigned char* in = static_cast<const unsigned char*>(h_buf);
    SnapHeader h;
    if (bytes < sizeof h + 8) return fail(QS_ERR_INVALID_ARG, "snapshot: %llu bytes is too short",
                                          (unsigned long long)bytes);
    std::memcpy(&h, in, sizeof h);
    if (std::memcmp(h.magic, SNAP_MAGIC, 8) != 0 || h.version != 1)
        return fail(QS_ERR_INVALID_ARG, "snapshot: not a version-1 QSketch snapshot");
    const bool msws = h.kind == QS_KIND_MSWS, bucket = h.kind == QS_KIND_BUCKET;
    if ((!msws && !bucket && h.kind != QS_KIND_PLAIN_CM) || (msws && (h.m_low != LOW_WORDS || h.m_high != HIGH_WORDS)) ||
        (bucket && h.m_low != 8 && h.m_low != 16 && h.m_low != 32) || h.n_low == 0 || h.n_seeds == 0 ||
        h.n_seeds > MAX_CM_ROWS || ((msws || bucket) && (h.n_masks == 0 || h.n_masks > 16384)))
        return fail(QS_ERR_INVALID_ARG, "snapshot: inconsistent header");
    const uint64_t lw = h.n_low * h.m_low, hw = msws ? h.n_high * h.m_high : 0;
    const uint64_t payload = 4 * ((uint64_t)h.n_seeds + h.n_masks + lw + hw);
    if (h.payload_bytes != payload || bytes < sizeof h + payload + 8)
        return fail(QS_ERR_INVALID_ARG, "snapshot: size does not match its header");
    uint64_t sum;
    std::memcpy(&sum, in + sizeof h + payload, 8);
    if (fnv1a64(in, sizeof h + payload) != sum) return fail(QS_ERR_INVALID_ARG, "snapshot: checksum mismatch");
    const unsigned char* q = in + sizeof h;
    std::vector<uint32_t> seeds(h.n_seeds), masks(h.n_masks);
    std::memcpy(seeds.data(), q, 4 * seeds.size());
    q += 4 * seeds.size();
    std::memcpy(masks.data(), q, 4 * masks.size());
    q += 4 * masks.size();
    qs_params p;
    qs_params_default(&p);
    p.kind = h.kind;
    p.flags = h.flags & QS_FLAG_COMPAT_V3;
    p.n_low = h.n_low;
    p.m_low = h.m_low;
    p.m_high = msws ? h.m_high : 32;
    p.n_high = msws ? h.n_high : 1024;
    p.hash_mask_table_sz = (msws || bucket) ? h.n_masks : 1021;
    p.hash_mask_ones = msws ? h.hash_mask_ones : 3;
    p.seeds = seeds.data();
    std::vector<uint8_t> mbytes;
    if (bucket) {  // H masks of m/8 bytes
        const uint32_t mb = h.m_low / 8;
        mbytes.resize((size_t)h.n_masks * mb);
        for (size_t i = 0; i < masks.size(); ++i)
            for (uint32_t k = 0; k < mb; ++k) mbytes[i * mb + k] = (uint8_t)(masks[i] >> (8 * k));
    }
    p.mask_table = msws ? reinterpret_cast<const uint8_t*>(masks.data()) : (bucket ? mbytes.data() : nullptr);
    p.device = device;
    qs_sketch* sk = nullptr;
    qs_status st = qs_create(&p, &sk);
    if (st != QS_OK) return st;
    DeviceGuard guard(sk->device);
    cudaError_t e = cudaMemcpy(msws ? sk->D.low : sk->C.table, q, lw * 4, cudaMemcpyHostToDevice);
    q += lw * 4;
    if (e == cudaSuccess && hw) e = cudaMemcpy(sk->D.high, q, hw * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && msws) {
        Ctl c;
        e = cudaMemcpy(&c, sk->D.ctl, sizeof c, cudaMemcpyDeviceToHost);
        c.next_id = h.next_level_id;
        c.status = h.status_bits;
        c.dropped = h.dropped_keys;
        if (e == cudaSuccess) e = cudaMemcpy(sk->D.ctl, &c, sizeof c, cudaMemcpyHostToDevice);
        sk->fresh = sk->max_batch;  // a warm sketch: no chunk ramp
    }
    if (e != cudaSuccess) {
        qs_destroy(sk);
        return cuda_fail(e, "snapshot upload");
    }
    *out = sk;
    return QS_OK;
}

qs_status qs_save(qs_sketch* sk, const char* path) {
    if (!path) return fail(QS_ERR_INVALID_ARG, "qs_save: null path");
    uint64_t n = 0;
    qs_status st = qs_snapshot_bytes(sk, &n);
    if (st != QS_OK) return st;
    std::vector<unsigned char> buf(n);
    st = qs_snapshot_save(sk, buf.data(), n);
    if (st != QS_OK) return st;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(QS_ERR_INVALID_ARG, "qs_save: cannot open %s", path);
    const size_t w = std::fwrite(buf.data(), 1, n, f);
    const int c = std::fclose(f);
    if (w != n || c != 0) return fail(QS_ERR_INVALID_ARG, "qs_save: short write to %s", path);
    return QS_OK;
}

qs_status qs_load(const char* path, int32_t device, qs_sketch** out) {
    if (!path || !out) return fail(QS_ERR_INVALID_ARG, "qs_load: null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(QS_ERR_INVALID_ARG, "qs_load: cannot open %s", path);
    std::vector<unsigned char> buf;
    unsigned char tmp[1 << 16];
    size_t r;
    while ((r = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + r);
    std::fclose(f);
    return qs_snapshot_load(buf.data(), buf.size(), device, out);
}

qs_status qs_gen_keys(uint32_t kind, uint64_t seed, uint64_t n_ranks, double s, uint64_t perm_seed, uint32_t* d_keys,
                      uint32_t* d_ranks, size_t n, void* stream) {
    if (kind > 1 || (!d_keys && n)) return fail(QS_ERR_INVALID_ARG, "gen_keys: bad arguments");
    if (kind == 1 && (n_ranks == 0 || n_ranks > (1ull << 32) || s <= 0))
        return fail(QS_ERR_INVALID_ARG, "gen_keys: zipf needs 0 < n_ranks <= 2^32, s > 0");
    CK(gen_keys(kind, seed, n_ranks, s, perm_seed, d_keys, d_ranks, n, static_cast<cudaStream_t>(stream)), "gen_keys");
    return QS_OK;
}

qs_status qs_gen_class_keys(uint64_t seed, uint32_t n_class, double s_class, double s_suffix, uint64_t perm_seed,
                            uint32_t* d_keys, size_t n, void* stream) {
    if ((!d_keys && n) || n_class == 0 || n_class > 65536 || s_class <= 0 || s_suffix <= 0)
        return fail(QS_ERR_INVALID_ARG, "gen_class_keys: bad arguments");
    CK(gen_class_keys(seed, n_class, s_class, s_suffix, perm_seed, d_keys, n, static_cast<cudaStream_t>(stream)),
       "gen_class_keys");
    return QS_OK;
}

qs_status qs_gen_rank_keys(uint64_t perm_seed, uint64_t first, uint32_t* d_keys, size_t n, void* stream) {
    if (!d_keys && n) return fail(QS_ERR_INVALID_ARG, "gen_rank_keys: null output");
    CK(gen_rank_keys(perm_seed, first, d_keys, n, static_cast<cudaStream_t>(stream)), "gen_rank_keys");
    return QS_OK;
}

qs_status qs_rank_histogram(const uint32_t* d_ranks, size_t n, uint32_t* d_hist, uint64_t n_ranks, void* stream) {
    if ((!d_ranks || !d_hist) && n) return fail(QS_ERR_INVALID_ARG, "rank_histogram: null argument");
    CK(rank_histogram(d_ranks, n, d_hist, n_ranks, static_cast<cudaStream_t>(stream)), "rank_histogram");
    return QS_OK;
}

qs_status qs_error_metrics(const uint32_t* d_est, const uint32_t* d_exact, size_t n, double* mean_rel_err,
                           double* mean_ratio, void* stream) {
    if (!mean_rel_err || !mean_ratio) return fail(QS_ERR_INVALID_ARG, "error_metrics: null output");
    double* acc = nullptr;
    CK(cudaMalloc(&acc, 3 * sizeof(double)), "metrics scratch");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(acc, 0, 3 * sizeof(double), st);
    if (e == cudaSuccess) e = error_metrics(d_est, d_exact, n, acc, st);
    double h[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(acc);
    if (e != cudaSuccess) return cuda_fail(e, "error_metrics");
    *mean_rel_err = h[2] > 0 ? h[0] / h[2] : 0.0;
    *mean_ratio = h[2] > 0 ? h[1] / h[2] : 0.0;
    return QS_OK;
}

qs_status qs_probe(uint32_t kind, uint64_t bytes, uint64_t ops, double* ops_per_s) {
    if (!ops_per_s) return fail(QS_ERR_INVALID_ARG, "probe: null output");
    const cudaError_t e = probe(kind, bytes, ops, ops_per_s);
    if (e == cudaErrorLaunchTimeout && (kind == 6 || kind == 8))
        return fail(QS_ERR_TIMEOUT, "probe: a bounded grid-barrier wait gave up");
    CK(e, "probe");
    return QS_OK;
}

void qs_test_fail_allocations(int32_t after) { g_fail_alloc_after.store(after); }

}  // extern "C"

// =====================================================================================
// Learned heavy-hitter split
// =====================================================================================
struct qs_learned {
    qs_learned_params p{};
    qs_sketch* sk = nullptr;
    int device = 0;
    TableDev T{};
    RouteDev R{};
    MlpDev M{};
    std::vector<void*> allocs;
    uint32_t* warm = nullptr;
    uint64_t warm_seen = 0;
    std::vector<uint32_t> tkeys;    // host mirror of the exact table's keys (changed only by admission)
    uint32_t tfill = 0;             // keys in the exact table
    uint32_t* d_sorted = nullptr;   // admission order upload buffer
    uint32_t* d_cand_est = nullptr; // sketch estimates of the chunk's candidates
    uint32_t admit_cap = 0;
    float* d_loss = nullptr;
    uint8_t* d_labels_tmp = nullptr;
    // training buffers, allocated with the sketch (training runs once, inside an insert):
    // word buffers of the warm-up length W (the distinct-key set 2W) and byte buffers of W
    struct {
        uint32_t *set, *distinct, *cnt, *est, *tmp, *train, *perm, *z2;
        uint8_t *labels, *take, *tlab, *plab;
        uint32_t set_slots;
    } tb{};
    TrainScratch tscratch;
    qs_learned_info info{};
    uint32_t adam_step = 0;
    bool table_full = false;  // (almost) no admission possible: routing skips the classifier

    // Full for routing purposes once fewer than 1/1024 of the slots below max fill are left:
    // classifying a whole chunk to fill the last few slots costs more than they can save.
    bool nearly_full() const { return (uint64_t)(T.max_fill - std::min(tfill, T.max_fill)) * 1024 < T.slots; }

    template <class X>
    cudaError_t alloc(X** ptr, size_t count, int fill = 0) {
        void* v = nullptr;
        const size_t bytes = std::max<size_t>(count * sizeof(X), 256);
        cudaError_t e = cudaMalloc(&v, bytes);
        if (e != cudaSuccess) return e;
        allocs.push_back(v);
        e = cudaMemset(v, fill, bytes);
        *ptr = static_cast<X*>(v);
        return e;
    }
};

namespace {

// Admit `order` (most deserving first) into the exact table: placement on the host mirror,
// then the mirror and the fill are uploaded (stream-ordered, synchronised: the mirror is
// the source of the copy).
qs_status learned_admit(qs_learned* lk, const uint32_t* order, uint32_t count, cudaStream_t st) {
    const uint32_t fill = table_admit_host(lk->tkeys.data(), lk->T.slots, order, count, lk->tfill, lk->T.max_fill);
    if (fill == lk->tfill) return QS_OK;
    lk->tfill = fill;
    CK(cudaMemcpyAsync(lk->T.keys, lk->tkeys.data(), (size_t)lk->T.slots * 4, cudaMemcpyHostToDevice, st),
       "table upload");
    CK(cudaMemcpyAsync(lk->T.fill, &lk->tfill, 4, cudaMemcpyHostToDevice, st), "fill upload");
    CK(cudaStreamSynchronize(st), "admit sync");
    return QS_OK;
}

qs_status mlp_init_params(qs_learned* lk) {
    // He-uniform hidden layers, Glorot-uniform output, zero biases; deterministic in init_seed
    std::vector<float> h(MLP_PARAMS, 0.0f);
    std::mt19937 g(lk->p.init_seed);
    auto fill = [&](size_t off, size_t n, float bound) {
        std::uniform_real_distribution<float> d(-bound, bound);
        for (size_t i = 0; i < n; ++i) h[off + i] = d(g);
    };
    fill(0, MLP_W1_N, std::sqrt(6.0f / 32.0f));
    fill(MLP_W1_N, MLP_W2_N, std::sqrt(6.0f / 128.0f));
    fill(MLP_BF16_PARAMS + 256, 128, std::sqrt(6.0f / 129.0f));
    CK(cudaMemcpy(lk->M.params, h.data(), h.size() * 4, cudaMemcpyHostToDevice), "mlp init");
    CK(mlp_refresh_bf16(lk->M, 0), "mlp bf16");
    CK(cudaMemset(lk->M.adam_m, 0, MLP_PARAMS * 4), "adam m");
    CK(cudaMemset(lk->M.adam_v, 0, MLP_PARAMS * 4), "adam v");
    CK(cudaMemset(lk->M.grads, 0, MLP_PARAMS * 4), "grads");
    CK(cudaDeviceSynchronize(), "mlp init sync");
    lk->adam_step = 0;
    return QS_OK;
}

// One pass of Adam over the examples in order; returns the mean loss of the last batch.
// The classifier kernels latch ST_TIMEOUT in M.status if a tensor-core wait gave up.
qs_status mlp_status(qs_learned* lk) {
    uint32_t v = 0;
    CK(cudaMemcpy(&v, lk->M.status, 4, cudaMemcpyDeviceToHost), "mlp status");
    if (v & ST_TIMEOUT) return fail(QS_ERR_TIMEOUT, "a tensor-core wait of the classifier timed out");
    return QS_OK;
}

qs_status mlp_train_pass(qs_learned* lk, const uint32_t* d_keys, const uint8_t* d_labels, uint64_t n, uint32_t batch,
                         float lr, float pos_weight, double* last_loss, cudaStream_t st) {
    float h_loss = 0.0f;
    for (uint64_t off = 0; off < n; off += batch) {
        const uint64_t b = std::min<uint64_t>(batch, n - off);
        CK(mlp_train_step(d_keys + off, d_labels + off, b, pos_weight, 1.0f / (float)b, lk->M, lk->d_loss,
                          ++lk->adam_step, lr, st),
           "mlp train step");
        if (off + batch >= n) {
            CK(cudaMemcpyAsync(&h_loss, lk->d_loss, 4, cudaMemcpyDeviceToHost, st), "loss");
            CK(cudaStreamSynchronize(st), "train sync");
            h_loss /= (float)b;
        }
    }
    *last_loss = h_loss;
    return mlp_status(lk);
}

qs_status learned_train(qs_learned* lk, cudaStream_t st) {
    const auto t0 = std::chrono::steady_clock::now();
    const uint64_t W = lk->warm_seen;
    // the sketch's training buffers (every one holds W elements; the distinct-key set 2W):
    // after the distinct keys the set holds the ranked keys, after the labels tmp the logits,
    // after the epochs perm the positives' logits and then the admission order
    auto& tb = lk->tb;
    uint32_t *d_set = tb.set, *d_distinct = tb.distinct, *d_cnt = tb.cnt, *d_est = tb.est, *d_tmp = tb.tmp;
    uint32_t *d_train = tb.train, *d_perm_keys = tb.perm;
    uint32_t *d_hkeys = tb.set, *d_hest = tb.set + (W + 16), *d_okeys = tb.perm, *d_oest = tb.z2;
    float *d_logit = reinterpret_cast<float*>(tb.tmp), *d_z1 = reinterpret_cast<float*>(tb.perm),
          *d_z2 = reinterpret_cast<float*>(tb.z2);
    uint8_t *d_labels = tb.labels, *d_take = tb.take, *d_tlab = tb.tlab, *d_plab = tb.plab;
    TrainScratch& S = lk->tscratch;
    auto cleanup = [] {};
#define CKT(expr, what)                                 \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) {                        \
            cleanup();                                  \
            return cuda_fail(_e, what);                 \
        }                                               \
    } while (0)
    CKT(distinct_sorted(lk->warm, (uint32_t)W, d_set, d_distinct, d_cnt, S, st), "distinct");
    uint32_t hc = 0;
    CKT(cudaMemcpyAsync(&hc, d_cnt, 4, cudaMemcpyDeviceToHost, st), "distinct count");
    CKT(cudaStreamSynchronize(st), "distinct sync");
    const uint32_t D = hc;
    const auto t_distinct = std::chrono::steady_clock::now();
    // labels from the sketch's own estimates: heavy = among the top heavy_fraction (ties in)
    qs_status s = query_device(lk->sk, d_distinct, D, d_est, st);
    if (s != QS_OK) {
        cleanup();
        return s;
    }
    const uint32_t k = (uint32_t)std::max<uint64_t>(1, (uint64_t)std::ceil(lk->p.heavy_fraction * (double)D));
    uint32_t thr = 0, npos32 = 0, tn32 = 0;
    if (D) CKT(kth_largest(d_est, D, k, d_tmp, S, &thr, st), "heavy threshold");
    CKT(label_keys(d_est, D, thr, d_labels, d_cnt, st), "labels");
    CKT(cudaMemcpyAsync(&npos32, d_cnt, 4, cudaMemcpyDeviceToHost, st), "positives");
    CKT(cudaStreamSynchronize(st), "labels sync");
    const uint64_t npos = npos32;
    // the training set: every labelled-heavy key and a seeded sample of neg_per_pos light keys
    // per heavy one (a key is in the sample when its hash falls below the sampling rate), in
    // ascending key order
    const uint32_t npp = lk->p.neg_per_pos ? lk->p.neg_per_pos : 16u;
    const double rate = std::min(1.0, (double)npp * (double)npos / (double)std::max<uint64_t>(1, D - npos));
    const uint64_t cut = (uint64_t)(rate * 4294967296.0);
    CKT(training_set(d_distinct, d_labels, D, lk->p.init_seed, cut, d_take, d_train, d_tlab, d_cnt, S, st),
        "training set");
    CKT(cudaMemcpyAsync(&tn32, d_cnt, 4, cudaMemcpyDeviceToHost, st), "training set size");
    CKT(cudaStreamSynchronize(st), "training set sync");
    const uint64_t TN = tn32, nneg = TN - npos;
    const auto t_labels = std::chrono::steady_clock::now();
    const float pw = std::min(lk->p.max_pos_weight, (float)nneg / (float)std::max<uint64_t>(1, npos));
    // epochs over a seeded order of the examples, drawn on the device per epoch
    double loss = 0.0, first = -1.0;
    for (uint32_t ep = 0; ep < lk->p.epochs && s == QS_OK; ++ep) {
        const uint64_t seed = ((uint64_t)lk->p.init_seed << 32) ^ (0x5bd1e995ull * (ep + 1));
        CKT(permute_examples(d_train, d_tlab, (uint32_t)TN, seed, d_perm_keys, d_plab, st), "permute examples");
        s = mlp_train_pass(lk, d_perm_keys, d_plab, TN, lk->p.batch, lk->p.lr, pw, &loss, st);
        if (first < 0) first = loss;
    }
    if (s != QS_OK) {
        cleanup();
        return s;
    }
    const auto t_epochs = std::chrono::steady_clock::now();
    // predictions on the warm-up keys: admit the predicted heavy, most confident first
    CKT(mlp_forward(d_distinct, D, lk->M, d_logit, st), "train forward");
    // eligibility cut: the largest logit threshold that keeps `eligible_recall` of the
    // labelled-heavy warm-up keys (the network filters, the sketch's counts rank)
    float zthr = 0.0f;
    if (npos) {
        const double miss = std::min(1.0, std::max(0.0, 1.0 - (double)lk->p.eligible_recall));
        float zq = 0.0f;
        CKT(positive_logit_quantile(d_logit, d_labels, D, (uint32_t)npos, miss, d_z1, d_z2, d_cnt, S, &zq, st),
            "logit quantile");
        zthr = std::min(0.0f, zq);
    }
    s = mlp_status(lk);
    if (s != QS_OK) {
        cleanup();
        return s;
    }
    lk->R.z_threshold = zthr;
    uint32_t conf[3] = {0, 0, 0}, H = 0;
    CKT(predict_keys(d_logit, d_labels, D, zthr, d_take, d_cnt, st), "predict");
    CKT(cudaMemcpyAsync(conf, d_cnt, 12, cudaMemcpyDeviceToHost, st), "confusion counts");
    // the network decides who may enter the table; the sketch's own counts rank them (only the
    // first max_fill of the order can enter); keys are distinct, so the order is total
    CKT(rank_predicted(d_distinct, d_est, d_take, D, d_hkeys, d_hest, d_okeys, d_oest, d_cnt, S, &H, st), "rank");
    const uint64_t tp = conf[0], fp = conf[1], fn = conf[2];
    const uint32_t take = (uint32_t)std::min<uint64_t>(H, lk->T.max_fill);
    std::vector<uint32_t> order(take);
    if (take) {
        CKT(cudaMemcpyAsync(order.data(), d_okeys, (size_t)take * 4, cudaMemcpyDeviceToHost, st), "order copy");
        CKT(cudaStreamSynchronize(st), "order sync");
        s = learned_admit(lk, order.data(), take, st);
        if (s != QS_OK) {
            cleanup();
            return s;
        }
    }
    lk->table_full = lk->nearly_full();
    cleanup();
#undef CKT
    qs_learned_info& I = lk->info;
    I.trained = 1;
    I.train_examples = TN;
    I.train_positives = npos;
    I.threshold = thr;
    I.pos_weight = pw;
    I.loss_first = (float)first;
    I.loss_last = (float)loss;
    I.train_precision = tp + fp ? (float)tp / (float)(tp + fp) : 0.0f;
    I.train_recall = tp + fn ? (float)tp / (float)(tp + fn) : 0.0f;
    I.logit_threshold = zthr;
    I.epochs = lk->p.epochs;
    I.steps = lk->adam_step;
    const auto t_end = std::chrono::steady_clock::now();
    auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
    };
    I.train_ms = ms(t0, t_end);
    I.train_phase_ms[0] = ms(t0, t_distinct);
    I.train_phase_ms[1] = ms(t_distinct, t_labels);
    I.train_phase_ms[2] = ms(t_labels, t_epochs);
    I.train_phase_ms[3] = ms(t_epochs, t_end);
    return QS_OK;
}

// The warm-up window again, now through the router: the sketch is cleared, admitted keys
// count exactly in the table and are left out of the sketch, every other key is inserted.  The
// heavy keys' warm-up occurrences then never link (and freeze) the buckets they share with
// light keys.  No classification here: admission already used the whole window.
qs_status learned_replay_warmup(qs_learned* lk, cudaStream_t st) {
    const auto t0 = std::chrono::steady_clock::now();
    qs_status s = qs_clear(lk->sk, st);
    if (s != QS_OK) return s;
    CK(cudaMemsetAsync(lk->T.counts, 0, (size_t)lk->T.slots * 4, st), "table counts reset");
    const uint64_t W = lk->warm_seen;
    for (uint64_t off = 0; off < W;) {
        const uint64_t c = std::min<uint64_t>(W - off, lk->sk->max_batch);
        lk->R.collect = 0u;
        CK(route_chunk(lk->warm + off, c, lk->T, lk->R, st), "route warm-up");
        s = insert_device(lk->sk, lk->warm + off, c, st, lk->R.skip);
        if (s != QS_OK) return s;
        off += c;
    }
    lk->info.warmup_replayed = 1;
    CK(cudaStreamSynchronize(st), "replay sync");
    lk->info.train_phase_ms[4] =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return QS_OK;
}

}  // namespace

extern "C" {

qs_status qs_learned_admit_keys(qs_learned* lk, const uint32_t* h_keys, size_t n) {
    if (!lk || (!h_keys && n)) return fail(QS_ERR_INVALID_ARG, "qs_learned_admit_keys: null argument");
    if (lk->warm_seen) return fail(QS_ERR_INVALID_ARG, "qs_learned_admit_keys: call before the first insert");
    DeviceGuard guard(lk->device);
    const uint32_t take = (uint32_t)std::min<uint64_t>(n, lk->T.max_fill);
    qs_status s = take ? learned_admit(lk, h_keys, take, 0) : QS_OK;
    if (s != QS_OK) return s;
    lk->warm_seen = lk->p.warmup_keys;  // no warm-up, no training: route from the first key
    lk->table_full = true;              // and no further admission (the network is untrained)
    lk->info.trained = 0;
    return QS_OK;
}

void qs_learned_params_default(qs_learned_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->budget_bytes = 64ull << 20;
    p->table_slots = 1u << 17;
    p->table_max_fill = 0.75f;
    p->warmup_keys = 1ull << 24;
    p->heavy_fraction = 0.005;
    p->epochs = 4;
    p->batch = 16384;  // 128 tiles of 128 examples: one backward launch, one tile per SM
    p->lr = 4e-3f;
    p->max_pos_weight = 64.0f;
    p->eligible_recall = 0.95f;
    p->seed_rng = 1;
    p->mask_rng = 1;
    p->init_seed = 1;
    p->neg_per_pos = 16;
    p->replay_warmup = 1;
    p->max_batch = 1ull << 22;
    p->device = -1;
}

qs_status qs_learned_create(const qs_learned_params* p, qs_learned** out) {
    if (!p || !out) return fail(QS_ERR_INVALID_ARG, "qs_learned_create: null argument");
    *out = nullptr;
    if (p->table_slots < 64 || (p->table_slots & (p->table_slots - 1)))
        return fail(QS_ERR_INVALID_ARG, "table_slots must be a power of two >= 64");
    if (p->warmup_keys == 0 || p->warmup_keys > (1ull << 30) || p->heavy_fraction <= 0 || p->heavy_fraction >= 1 || p->batch == 0 || p->epochs == 0)
        return fail(QS_ERR_INVALID_ARG, "learned params out of range");
    const uint64_t mlp_bytes = (uint64_t)MLP_BF16_PARAMS * 2 + (uint64_t)(MLP_PARAMS - MLP_BF16_PARAMS) * 4;
    const uint64_t table_bytes = (uint64_t)p->table_slots * 8;
    if (p->budget_bytes < table_bytes + mlp_bytes + (1u << 16))
        return fail(QS_ERR_INVALID_ARG, "budget too small for table + network + sketch");
    const uint64_t sketch_bytes = p->budget_bytes - table_bytes - mlp_bytes;
    qs_params sp;
    qs_params_default(&sp);
    sp.n_low = qs_find_greatest_prime(sketch_bytes * 4 / 5 / 32);
    sp.n_high = (sketch_bytes - sp.n_low * 32) / 128;
    sp.hash_seed = p->hash_seed;
    sp.seed_rng = p->seed_rng;
    sp.mask_rng = p->mask_rng;
    sp.max_batch = p->max_batch ? p->max_batch : (1ull << 22);
    sp.device = p->device;
    qs_learned* lk = new qs_learned();
    lk->p = *p;
    if (!lk->p.max_batch) lk->p.max_batch = sp.max_batch;
    qs_status s = qs_create(&sp, &lk->sk);
    if (s != QS_OK) {
        delete lk;
        return s;
    }
    lk->device = lk->sk->device;
    DeviceGuard guard(lk->device);
    auto bail = [&](qs_status st) {
        qs_learned_destroy(lk);
        return st;
    };
    const uint64_t B = lk->sk->max_batch;
    TableDev& T = lk->T;
    T.slots = p->table_slots;
    T.max_fill = (uint32_t)std::max(1.0f, p->table_max_fill * (float)p->table_slots);
    CKB(lk->alloc(&T.keys, T.slots, 0xff), "table keys");
    lk->tkeys.assign(T.slots, TBL_EMPTY);
    CKB(lk->alloc(&T.counts, T.slots), "table counts");
    CKB(lk->alloc(&T.fill, 1), "table fill");
    RouteDev& R = lk->R;
    R.cand_slots = 1u << 18;
    CKB(lk->alloc(&R.skip, B / 32 + 1), "route skip");
    CKB(lk->alloc(&R.misses, B), "route misses");
    CKB(lk->alloc(&R.n_misses, 1), "route misses count");
    CKB(lk->alloc(&R.cand_keys, R.cand_slots, 0xff), "candidates");
    CKB(lk->alloc(&R.n_cand, 1), "candidate count");
    CKB(lk->alloc(&R.cand_list, R.cand_slots), "candidate list");
    lk->admit_cap = std::max<uint32_t>(T.max_fill, R.cand_slots);
    CKB(lk->alloc(&lk->d_sorted, lk->admit_cap), "admission buffer");
    CKB(lk->alloc(&lk->d_cand_est, lk->admit_cap), "candidate estimates");
    MlpDev& M = lk->M;
    CKB(lk->alloc(&M.params, MLP_PARAMS), "mlp params");
    CKB(lk->alloc(&M.grads, MLP_PARAMS), "mlp grads");
    CKB(lk->alloc(&M.adam_m, MLP_PARAMS), "adam m");
    CKB(lk->alloc(&M.adam_v, MLP_PARAMS), "adam v");
    CKB(lk->alloc(&M.W1, MLP_BF16_PARAMS), "mlp bf16");
    CKB(lk->alloc(&M.partials, (uint64_t)MLP_MAX_TILES * MLP_PARTIAL_STRIDE), "mlp partial gradients");
    CKB(lk->alloc(&M.ploss, MLP_MAX_TILES), "mlp partial losses");
    CKB(lk->alloc(&M.status, 1, 0), "mlp status");
    M.W2 = M.W1 + MLP_W1_N;
    M.b1 = M.params + MLP_BF16_PARAMS;
    M.b2 = M.b1 + 128;
    M.w3 = M.b2 + 128;
    M.b3 = M.w3 + 128;
    M.gW1 = M.grads;
    M.gW2 = M.grads + MLP_W1_N;
    M.gb1 = M.grads + MLP_BF16_PARAMS;
    M.gb2 = M.gb1 + 128;
    M.g3 = M.gb2 + 128;
    M.gb3 = M.g3 + 128;
    CKB(lk->alloc(&lk->d_loss, 4), "loss");
    CKB(lk->alloc(&lk->warm, p->warmup_keys), "warm-up keys");
    {
        auto& tb = lk->tb;
        const uint64_t Wk = p->warmup_keys + 16;
        tb.set_slots = 1;
        while (tb.set_slots < 2 * p->warmup_keys) tb.set_slots <<= 1;
        CKB(lk->alloc(&tb.set, std::max<uint64_t>(tb.set_slots, 2 * Wk)), "train set");
        CKB(lk->alloc(&tb.distinct, Wk), "train distinct");
        CKB(lk->alloc(&tb.cnt, 16), "train counts");
        for (uint32_t** b : {&tb.est, &tb.tmp, &tb.train, &tb.perm, &tb.z2}) CKB(lk->alloc(b, Wk), "train buffer");
        for (uint8_t** b : {&tb.labels, &tb.take, &tb.tlab, &tb.plab}) CKB(lk->alloc(b, Wk), "train buffer");
        cudaError_t e = train_scratch_reserve(lk->tscratch, (uint32_t)p->warmup_keys, tb.set_slots);
        if (e != cudaSuccess) return bail(cuda_fail(e, "train scratch"));
    }
    cudaError_t e = mlp_configure();
    if (e != cudaSuccess) return bail(cuda_fail(e, "mlp configure"));
    s = mlp_init_params(lk);
    if (s != QS_OK) return bail(s);
    qs_learned_info& I = lk->info;
    I.budget_bytes = p->budget_bytes;
    I.sketch_bytes = sp.n_low * 32 + sp.n_high * 128;
    I.table_bytes = table_bytes;
    I.mlp_bytes = mlp_bytes;
    I.n_low = sp.n_low;
    I.n_high = sp.n_high;
    I.table_slots = T.slots;
    I.warmup_keys = p->warmup_keys;
    *out = lk;
    return QS_OK;
}

qs_status qs_learned_destroy(qs_learned* lk) {
    if (!lk) return QS_OK;
    {
        DeviceGuard guard(lk->device);
        cudaDeviceSynchronize();
        for (void* v : lk->allocs) cudaFree(v);
        if (lk->tscratch.p) cudaFree(lk->tscratch.p);
        lk->tscratch.p = nullptr;
        if (lk->sk) qs_destroy(lk->sk);
    }
    delete lk;
    return QS_OK;
}

qs_status qs_learned_insert(qs_learned* lk, const uint32_t* d_keys, size_t n, void* stream) {
    if (!lk) return fail(QS_ERR_INVALID_ARG, "null learned sketch");
    if (n == 0) return QS_OK;
    if (!d_keys || (reinterpret_cast<uintptr_t>(d_keys) & 3u)) return fail(QS_ERR_INVALID_ARG, "bad keys pointer");
    DeviceGuard guard(lk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    size_t off = 0;
    while (off < n) {
        if (lk->warm_seen < lk->p.warmup_keys) {
            const uint64_t take = std::min<uint64_t>(n - off, lk->p.warmup_keys - lk->warm_seen);
            CK(cudaMemcpyAsync(lk->warm + lk->warm_seen, d_keys + off, take * 4, cudaMemcpyDeviceToDevice, st),
               "warm-up copy");
            qs_status s = insert_device(lk->sk, d_keys + off, take, st);
            if (s != QS_OK) return s;
            lk->warm_seen += take;
            off += take;
            if (lk->warm_seen == lk->p.warmup_keys) {
                s = learned_train(lk, st);
                if (s == QS_OK && lk->p.replay_warmup != 2) s = learned_replay_warmup(lk, st);
                if (s != QS_OK) return s;
            }
            continue;
        }
        if (lk->table_full) {
            // nothing more to admit: pass 1 looks the keys up in the exact table itself
            const uint64_t c = n - off;
            qs_status s = insert_device(lk->sk, d_keys + off, c, st, nullptr, &lk->T, lk->R.skip);
            if (s != QS_OK) return s;
            off += c;
            continue;
        }
        // route a chunk: table hits count exactly and are skipped by the sketch insert
        uint64_t c = std::min<uint64_t>(n - off, lk->sk->max_batch);
        CK(cudaMemsetAsync(lk->R.n_misses, 0, 4, st), "misses reset");
        lk->R.collect = 1u;
        CK(route_chunk(d_keys + off, c, lk->T, lk->R, st), "route");
        CK(classify_misses(lk->M, lk->R, c, st), "classify");
        qs_status s = insert_device(lk->sk, d_keys + off, c, st, lk->R.skip);
        if (s != QS_OK) return s;
        uint32_t ncand = 0;
        CK(cudaMemcpyAsync(&ncand, lk->R.n_cand, 4, cudaMemcpyDeviceToHost, st), "candidates");
        CK(cudaStreamSynchronize(st), "candidate sync");
        if (ncand) {
            ncand = std::min(ncand, lk->R.cand_slots);
            // rank the chunk's candidates by the sketch's estimate (ties by key), admit in order
            std::vector<uint32_t> cand(ncand), cest(ncand);
            s = query_device(lk->sk, lk->R.cand_list, ncand, lk->d_cand_est, st);
            if (s != QS_OK) return s;
            CK(cudaMemcpyAsync(cand.data(), lk->R.cand_list, ncand * 4, cudaMemcpyDeviceToHost, st), "candidate copy");
            CK(cudaMemcpyAsync(cest.data(), lk->d_cand_est, ncand * 4, cudaMemcpyDeviceToHost, st), "estimate copy");
            CK(cudaStreamSynchronize(st), "candidate sync");
            std::vector<std::pair<int64_t, uint32_t>> order(ncand);
            for (uint32_t i = 0; i < ncand; ++i) order[i] = {-(int64_t)cest[i], cand[i]};
            std::sort(order.begin(), order.end());
            const uint32_t take = std::min<uint32_t>(ncand, lk->admit_cap);
            for (uint32_t i = 0; i < take; ++i) cand[i] = order[i].second;
            const uint32_t before = lk->tfill;
            s = learned_admit(lk, cand.data(), take, st);
            if (s != QS_OK) return s;
            CK(cudaMemsetAsync(lk->R.cand_keys, 0xff, (size_t)lk->R.cand_slots * 4, st), "candidate reset");
            CK(cudaMemsetAsync(lk->R.n_cand, 0, 4, st), "candidate reset");
            CK(cudaStreamSynchronize(st), "admit sync");
            lk->info.admitted_after_warmup += lk->tfill - before;
            lk->table_full = lk->nearly_full();
        }
        off += c;
    }
    return QS_OK;
}

qs_status qs_learned_query(qs_learned* lk, const uint32_t* d_keys, size_t n, uint32_t* d_counts, void* stream) {
    if (!lk) return fail(QS_ERR_INVALID_ARG, "null learned sketch");
    if (n == 0) return QS_OK;
    if (!d_keys || !d_counts) return fail(QS_ERR_INVALID_ARG, "null keys or counts");
    DeviceGuard guard(lk->device);
    CK(learned_query(d_keys, n, lk->T, lk->sk->D, lk->sk->L, d_counts, static_cast<cudaStream_t>(stream)),
       "learned query");
    return QS_OK;
}

qs_status qs_learned_get_info(qs_learned* lk, qs_learned_info* out) {
    if (!lk || !out) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(lk->device);
    CK(cudaDeviceSynchronize(), "info sync");
    uint32_t fill = 0;
    CK(cudaMemcpy(&fill, lk->T.fill, 4, cudaMemcpyDeviceToHost), "fill");
    *out = lk->info;
    out->table_fill = fill;
    out->warmup_seen = lk->warm_seen;
    return QS_OK;
}

qs_status qs_learned_get_table(qs_learned* lk, uint32_t* h_keys, uint32_t* h_counts, uint32_t* h_seed) {
    if (!lk || !h_keys || !h_counts) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(lk->device);
    CK(cudaDeviceSynchronize(), "table sync");
    CK(cudaMemcpy(h_keys, lk->T.keys, (size_t)lk->T.slots * 4, cudaMemcpyDeviceToHost), "table keys");
    CK(cudaMemcpy(h_counts, lk->T.counts, (size_t)lk->T.slots * 4, cudaMemcpyDeviceToHost), "table counts");
    if (h_seed) *h_seed = lk->sk->D.seed;
    return QS_OK;
}

qs_status qs_mlp_get_params(qs_learned* lk, float* h) {
    if (!lk || !h) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(lk->device);
    CK(cudaDeviceSynchronize(), "sync");
    CK(cudaMemcpy(h, lk->M.params, MLP_PARAMS * 4, cudaMemcpyDeviceToHost), "params copy");
    return QS_OK;
}

qs_status qs_mlp_set_params(qs_learned* lk, const float* h) {
    if (!lk || !h) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(lk->device);
    CK(cudaDeviceSynchronize(), "sync");
    CK(cudaMemcpy(lk->M.params, h, MLP_PARAMS * 4, cudaMemcpyHostToDevice), "params copy");
    CK(mlp_refresh_bf16(lk->M, 0), "bf16");
    CK(cudaMemset(lk->M.adam_m, 0, MLP_PARAMS * 4), "adam m");
    CK(cudaMemset(lk->M.adam_v, 0, MLP_PARAMS * 4), "adam v");
    CK(cudaDeviceSynchronize(), "sync");
    lk->adam_step = 0;
    return QS_OK;
}

qs_status qs_mlp_forward(qs_learned* lk, const uint32_t* d_keys, size_t n, float* d_logits, void* stream) {
    if (!lk || (!d_keys && n) || (!d_logits && n)) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(lk->device);
    CK(mlp_forward(d_keys, n, lk->M, d_logits, static_cast<cudaStream_t>(stream)), "mlp forward");
    return QS_OK;
}

qs_status qs_mlp_grads(qs_learned* lk, const uint32_t* d_keys, const uint8_t* d_labels, size_t n, float pos_weight,
                       float* h_grads, double* loss) {
    if (!lk || !d_keys || !d_labels || !h_grads || !loss || n == 0) return fail(QS_ERR_INVALID_ARG, "bad argument");
    DeviceGuard guard(lk->device);
    CK(cudaDeviceSynchronize(), "sync");
    CK(cudaMemset(lk->M.grads, 0, MLP_PARAMS * 4), "grads reset");
    CK(cudaMemset(lk->d_loss, 0, 4), "loss reset");
    CK(mlp_backward(d_keys, d_labels, n, pos_weight, 1.0f / (float)n, lk->M, lk->d_loss, 0), "mlp backward");
    float l = 0;
    CK(cudaMemcpy(&l, lk->d_loss, 4, cudaMemcpyDeviceToHost), "loss copy");
    CK(cudaMemcpy(h_grads, lk->M.grads, MLP_PARAMS * 4, cudaMemcpyDeviceToHost), "grads copy");
    CK(cudaMemset(lk->M.grads, 0, MLP_PARAMS * 4), "grads reset");
    *loss = (double)l / (double)n;
    return mlp_status(lk);
}

qs_status qs_mlp_train(qs_learned* lk, const uint32_t* d_keys, const uint8_t* d_labels, size_t n, uint32_t epochs,
                       uint32_t batch, float lr, float pos_weight, double* last_loss) {
    if (!lk || !d_keys || !d_labels || !last_loss || n == 0 || batch == 0) return fail(QS_ERR_INVALID_ARG, "bad argument");
    DeviceGuard guard(lk->device);
    for (uint32_t e = 0; e < epochs; ++e) {
        qs_status s = mlp_train_pass(lk, d_keys, d_labels, n, batch, lr, pos_weight, last_loss, 0);
        if (s != QS_OK) return s;
    }
    return QS_OK;
}

}  // extern "C"

// ---- batched uneven streams ----------------------------------------------------------------
// All streams' sketches live in one arena sketch (its low table, pool, masks, control block
// and replay scratch); the batch adds the per-stream descriptors and the work-queue state.
struct qs_batch {
    qs_sketch* sk = nullptr;
    uint32_t S = 0;
    std::vector<uint32_t> seeds;
    BatchDev B{};
    cudaStream_t cap = nullptr;  // capture stream for the graph variants
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        const void* keys = nullptr;
        const void* offs = nullptr;
        const void* out = nullptr;
        uint64_t max_total = 0;
    } g[2];  // 0 insert, 1 query
    int graph_ok = -1;  // -1 not tried, 1 works, 0 capture unsupported here
    uint64_t ramp_first = 0;  // per-stream chunk ramp of eager inserts: first slice, 0 = none
    qs_batch_info info{};
    // Pass 1 runs one launch per run of size classes with the same lanes per key; streams are
    // grouped by size class floor(log2 n_low) (the grouped order lives in B.cls_streams).
    std::vector<uint32_t> grp_class;   // size class of each grouped position
    uint32_t class_lpk[MAX_SIZE_CLASSES] = {};
    struct Run {
        uint32_t k_lo, k_hi;
        int lpk;
    };
    std::vector<Run> runs;
};

namespace {

// `timed`: bracket the launches with the arena sketch's profiling events (not while capturing).
BatchWindow flat_window(uint64_t c0, uint64_t c1) {
    BatchWindow W{};
    W.c0 = c0;
    W.c1 = c1;
    W.flat = 1;
    return W;
}

// Consecutive size classes with the same lanes per key share one pass-1 launch.
void batch_rebuild_runs(qs_batch* b) {
    b->runs.clear();
    for (uint32_t k = 0; k < b->S; ++k) {
        const int lpk = (int)b->class_lpk[b->grp_class[k]];
        if (!b->runs.empty() && b->runs.back().lpk == lpk)
            b->runs.back().k_hi = k + 1;
        else
            b->runs.push_back({k, k + 1, lpk});
    }
}

qs_status batch_insert_seq(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, const BatchWindow& W,
                           bool strict, cudaStream_t st, bool timed = true) {
    qs_sketch* sk = b->sk;
    BatchDev B = b->B;
    B.key_off = d_offsets;
    CK(batch_plan(B, sk->D.ctl, W, strict, st), "batch plan");
    if (timed) CK(sk->prof_begin(0, st), "profile");
    for (size_t r = 0; r < b->runs.size(); ++r)
        CK(batch_insert_pass(d_keys, sk->D, B, sk->L, sk->agg, b->runs[r].lpk, b->runs[r].k_lo, b->runs[r].k_hi,
                             (uint32_t)r, st),
           "batch insert");
    if (timed) CK(sk->prof_end(0, st), "profile");
    if (timed) CK(sk->prof_begin(1, st), "profile");
    CK(batch_repair(d_keys, sk->D, B, sk->L, st), "batch repair");
    if (timed) CK(sk->prof_end(1, st), "profile");
    b->info.launches += 3;
    return QS_OK;
}

qs_status batch_query_seq(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, uint64_t total,
                          uint32_t* d_counts, cudaStream_t st, bool timed = true) {
    qs_sketch* sk = b->sk;
    BatchDev B = b->B;
    B.key_off = d_offsets;
    CK(batch_plan(B, sk->D.ctl, flat_window(0, total), false, st), "batch plan");
    if (timed) CK(sk->prof_begin(2, st), "profile");
    CK(batch_query(d_keys, d_counts, sk->D, B, sk->L, st), "batch query");
    if (timed) CK(sk->prof_end(2, st), "profile");
    b->info.launches += 2;
    return QS_OK;
}

// Record `seq` into graph slot k (unless it is already recorded for these buffers) and launch
// it on `st`.  Returns false when capture does not work here; the caller then runs eagerly.
template <class F>
qs_status batch_graph(qs_batch* b, int k, const void* keys, const void* offs, const void* out, uint64_t max_total,
                      cudaStream_t st, F seq, bool* ran) {
    *ran = false;
    if (b->graph_ok == 0) return QS_OK;
    qs_batch::Graph& g = b->g[k];
    if (!g.exec || g.keys != keys || g.offs != offs || g.out != out || g.max_total != max_total) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        if (!b->cap) CK(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "capture stream");
        const uint64_t launches = b->info.launches;
        cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e, "begin capture");
        const qs_status s = seq(b->cap);
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(b->cap, &graph);
        b->info.launches = launches;
        cudaGraphExec_t exec = nullptr;
        if (s == QS_OK && e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (s != QS_OK || e != cudaSuccess || !exec) {
            cudaGetLastError();  // capture is not supported for this sequence: run eagerly from now on
            b->graph_ok = 0;
            return QS_OK;
        }
        b->graph_ok = 1;
        g.exec = exec;
        g.keys = keys;
        g.offs = offs;
        g.out = out;
        g.max_total = max_total;
    }
    CK(cudaGraphLaunch(g.exec, st), "graph launch");
    ++b->info.graph_launches;
    *ran = true;
    return QS_OK;
}

}  // namespace

extern "C" {

void qs_batch_params_default(qs_batch_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->seed_rng = 1;
    p->mask_rng = 1;
    p->hash_mask_table_sz = 1021;
    p->hash_mask_ones = 3;
    p->max_batch = 1ull << 22;
    p->device = -1;
}

qs_status qs_batch_create(const qs_batch_params* p, qs_batch** out) {
    if (!p || !out) return fail(QS_ERR_INVALID_ARG, "qs_batch_create: null argument");
    *out = nullptr;
    const uint32_t S = p->n_streams;
    if (S == 0 || S > (1u << 20)) return fail(QS_ERR_INVALID_ARG, "n_streams out of [1, 2^20]");
    if (!p->n_low || !p->n_high) return fail(QS_ERR_INVALID_ARG, "n_low and n_high arrays are required");
    uint64_t tl = 0, th = 0;
    for (uint32_t s = 0; s < S; ++s) {
        if (p->n_low[s] == 0 || p->n_high[s] < 2) return fail(QS_ERR_INVALID_ARG, "stream %u: n_low >= 1 and n_high >= 2", s);
        tl += p->n_low[s];
        th += p->n_high[s];
        if (tl > 0xffffffffull || th > (1ull << 30))
            return fail(QS_ERR_INVALID_ARG, "total buckets exceed 2^32 - 1 low or 2^30 high");
    }
    qs_params ap;
    qs_params_default(&ap);
    ap.kind = QS_KIND_MSWS;
    ap.n_low = tl;
    ap.n_high = th;
    ap.hash_seed = 1;  // the arena's own multiplier is not used: every stream has its own
    ap.mask_rng = p->mask_rng;
    ap.hash_mask_table_sz = p->hash_mask_table_sz;
    ap.hash_mask_ones = p->hash_mask_ones;
    ap.mask_table = p->mask_table;
    ap.flags = p->flags;
    ap.max_batch = p->max_batch;
    ap.device = p->device;
    ap.aggregate = p->aggregate;
    ap.route = p->route;
    ap.lanes_per_key = p->lanes_per_key;
    ap.ctas_per_sm = p->ctas_per_sm;
    qs_batch* b = new qs_batch();
    qs_status s = qs_create(&ap, &b->sk);
    if (s != QS_OK) {
        delete b;
        return s;
    }
    b->S = S;
    auto bail = [&](qs_status st) {
        qs_batch_destroy(b);
        return st;
    };
    qs_sketch* sk = b->sk;
    DeviceGuard guard(sk->device);
    b->seeds.resize(S);
    if (p->hash_seeds)
        std::memcpy(b->seeds.data(), p->hash_seeds, (size_t)S * 4);
    else
        draw_seeds(p->seed_rng, S, b->seeds.data());
    std::vector<StreamDesc> desc(S);
    uint64_t lb = 0, hb = 0;
    for (uint32_t i = 0; i < S; ++i) {
        if (b->seeds[i] == 0) return bail(fail(QS_ERR_INVALID_ARG, "stream %u: hash seed 0", i));
        desc[i].fm_low = make_fastmod((uint32_t)p->n_low[i]);
        desc[i].seed = b->seeds[i];
        desc[i].low_base = (uint32_t)lb;
        desc[i].high_base = (uint32_t)hb;
        desc[i].n_high = (uint32_t)p->n_high[i];
        lb += p->n_low[i];
        hb += p->n_high[i];
    }
    BatchDev& B = b->B;
    B.n_streams = S;
    StreamDesc* d_desc = nullptr;
    CKB(sk->alloc(&d_desc, S), "alloc stream descriptors");
    B.desc = d_desc;
    CKB(sk->alloc(&B.lo, S), "alloc windows");
    CKB(sk->alloc(&B.hi, S), "alloc windows");
    CKB(sk->alloc(&B.item_off, (uint64_t)S + 1), "alloc work items");
    CKB(sk->alloc(&B.wpre, (uint64_t)S + 1), "alloc window prefix");
    CKB(sk->alloc(&B.win, 2), "alloc window");
    CKB(sk->alloc(&B.work, MAX_SIZE_CLASSES), "alloc work queues");
    {  // streams grouped by size class (stable), each class's lanes per key
        std::vector<uint32_t> order(S);
        for (uint32_t i = 0; i < S; ++i) order[i] = i;
        auto cls = [&](uint32_t i) { return (uint32_t)size_class(p->n_low[i]); };
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) { return cls(a) < cls(c); });
        b->grp_class.resize(S);
        for (uint32_t k = 0; k < S; ++k) b->grp_class[k] = cls(order[k]);
        uint32_t* d_order = nullptr;
        CKB(sk->alloc(&d_order, S), "alloc grouped streams");
        CKB(cudaMemcpy(d_order, order.data(), (size_t)S * 4, cudaMemcpyHostToDevice), "upload grouped streams");
        B.cls_streams = d_order;
        CKB(sk->alloc(&B.cls_item_off, (uint64_t)S + 1), "alloc grouped work items");
        for (uint32_t c = 0; c < MAX_SIZE_CLASSES; ++c) {
            const uint32_t v = p->class_lanes_per_key ? p->class_lanes_per_key[c] : 0u;
            if (v && v != 1 && v != 2 && v != 4 && v != 8 && v != 16 && v != 32)
                return bail(fail(QS_ERR_INVALID_ARG, "class_lanes_per_key[%u] must be 0, 1, 2, 4, 8, 16 or 32", c));
            if (v > 8 && sk->D.route == 2)
                return bail(fail(QS_ERR_INVALID_ARG, "class_lanes_per_key[%u]: fused routing takes at most 8", c));
            b->class_lpk[c] = v ? v : (uint32_t)sk->L.lanes_per_key;
        }
        batch_rebuild_runs(b);
    }
    CKB(sk->alloc(&B.next_id, S), "alloc allocators");
    CKB(sk->alloc(&B.status, S), "alloc stream status");
    CKB(sk->alloc(&B.first, S), "alloc link ranks");
    CKB(cudaMemcpy(d_desc, desc.data(), (size_t)S * sizeof(StreamDesc), cudaMemcpyHostToDevice), "upload descriptors");
    std::vector<uint32_t> first(S, FIRST_ID);
    CKB(cudaMemcpy(B.next_id, first.data(), (size_t)S * 4, cudaMemcpyHostToDevice), "init allocators");
    if (p->first_chunk & 31) return bail(fail(QS_ERR_INVALID_ARG, "first_chunk must be a multiple of 32"));
    b->ramp_first = (p->flags & QS_FLAG_NO_CHUNK_RAMP) ? 0 : (p->first_chunk ? p->first_chunk : (1ull << 14));
    b->info.n_streams = S;
    b->info.low_buckets = tl;
    b->info.high_buckets = th;
    b->info.table_bytes = tl * 32 + th * 128;
    b->info.max_batch = sk->max_batch;
    *out = b;
    return QS_OK;
}

qs_status qs_batch_destroy(qs_batch* b) {
    if (!b) return QS_OK;
    if (b->sk) {
        DeviceGuard guard(b->sk->device);
        cudaDeviceSynchronize();
        for (auto& g : b->g)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        if (b->cap) cudaStreamDestroy(b->cap);
    }
    qs_destroy(b->sk);
    delete b;
    return QS_OK;
}

static qs_status batch_args(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets) {
    if (!b) return fail(QS_ERR_INVALID_ARG, "null batch");
    if (!d_keys || !d_offsets) return fail(QS_ERR_INVALID_ARG, "null keys or offsets");
    if ((reinterpret_cast<uintptr_t>(d_keys) & 3u) || (reinterpret_cast<uintptr_t>(d_offsets) & 7u))
        return fail(QS_ERR_INVALID_ARG, "keys must be 4-byte and offsets 8-byte aligned");
    return QS_OK;
}

qs_status qs_batch_insert(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, uint64_t total,
                          void* stream) {
    qs_status s = batch_args(b, d_keys, d_offsets);
    if (s != QS_OK || total == 0) return s;
    DeviceGuard guard(b->sk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t mb = b->sk->max_batch;
    const uint32_t S = b->S;
    // Per-stream chunk ramp: rounds over every stream's keys [0, f), [f, 2f), [2f, 4f), ...
    // counted from the stream's start, so the hot buckets of each stream link on its first
    // keys instead of sending most of its keys through the ordered replay.  Each round is cut
    // into windows of at most max_batch keys.  Needs the offsets on the host; when they are
    // not valid (or there is no ramp) the flat windows below run and the plan latches the error.
    std::vector<uint64_t> off;
    if (b->ramp_first) {
        off.resize((size_t)S + 1);
        CK(cudaMemcpyAsync(off.data(), d_offsets, off.size() * 8, cudaMemcpyDeviceToHost, st), "offsets copy");
        CK(cudaStreamSynchronize(st), "offsets sync");
        bool ok = off[0] == 0 && off[S] == total;
        for (uint32_t i = 0; ok && i < S; ++i) ok = off[i + 1] >= off[i];
        if (!ok) off.clear();
    }
    if (off.empty()) {
        for (uint64_t c0 = 0; c0 < total; c0 += mb) {
            s = batch_insert_seq(b, d_keys, d_offsets, flat_window(c0, std::min(total, c0 + mb)), false, st);
            if (s != QS_OK) return s;
        }
        ++b->info.inserts;
        return QS_OK;
    }
    uint64_t longest = 0;
    for (uint32_t i = 0; i < S; ++i) longest = std::max(longest, off[i + 1] - off[i]);
    auto run = [&](uint32_t s_lo, uint32_t s_hi, uint64_t r0, uint64_t r1) -> qs_status {
        BatchWindow W{};
        W.s_lo = s_lo;
        W.s_hi = s_hi;
        W.rel_lo = r0;
        W.rel_hi = r1;
        W.flat = 0;
        return batch_insert_seq(b, d_keys, d_offsets, W, false, st);
    };
    for (uint64_t r0 = 0, r1 = b->ramp_first; r0 < longest; r0 = r1, r1 = std::max(r1 * 2, r1 + 1)) {
        uint64_t acc = 0;
        uint32_t first = 0;
        for (uint32_t i = 0; i <= S; ++i) {
            const uint64_t len = i < S ? off[i + 1] - off[i] : 0;
            const uint64_t part = i < S ? std::min(len, r1) - std::min(len, r0) : 0;
            if (i == S || acc + part > mb) {  // close the window [first, i)
                if (acc) {
                    s = run(first, i, r0, r1);
                    if (s != QS_OK) return s;
                }
                acc = 0;
                first = i;
            }
            if (part > mb) {  // one stream's slice alone exceeds a window: split it
                for (uint64_t a = r0; a < std::min(len, r1); a += mb) {
                    s = run(i, i + 1, a, std::min(std::min(len, r1), a + mb));
                    if (s != QS_OK) return s;
                }
                first = i + 1;
                continue;
            }
            acc += part;
        }
    }
    ++b->info.inserts;
    return QS_OK;
}

qs_status qs_batch_query(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, uint64_t total,
                         uint32_t* d_counts, void* stream) {
    qs_status s = batch_args(b, d_keys, d_offsets);
    if (s != QS_OK || total == 0) return s;
    if (!d_counts) return fail(QS_ERR_INVALID_ARG, "null counts");
    if (total > (uint64_t)0xffffffffu * 2048u) return fail(QS_ERR_CAPACITY, "query batch too large");
    DeviceGuard guard(b->sk->device);
    s = batch_query_seq(b, d_keys, d_offsets, total, d_counts, static_cast<cudaStream_t>(stream));
    if (s == QS_OK) ++b->info.queries;
    return s;
}

qs_status qs_batch_insert_graph(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, uint64_t max_total,
                                void* stream) {
    qs_status s = batch_args(b, d_keys, d_offsets);
    if (s != QS_OK || max_total == 0) return s;
    if (max_total > b->sk->max_batch)
        return fail(QS_ERR_CAPACITY, "insert graph: max_total %llu exceeds max_batch %llu",
                    (unsigned long long)max_total, (unsigned long long)b->sk->max_batch);
    DeviceGuard guard(b->sk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    bool ran = false;
    s = batch_graph(b, 0, d_keys, d_offsets, nullptr, max_total, st,
                    [&](cudaStream_t cs) {
                        return batch_insert_seq(b, d_keys, d_offsets, flat_window(0, max_total), true, cs, false);
                    },
                    &ran);
    if (s == QS_OK && !ran) s = batch_insert_seq(b, d_keys, d_offsets, flat_window(0, max_total), true, st);
    if (s == QS_OK) ++b->info.inserts;
    return s;
}

qs_status qs_batch_query_graph(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, uint64_t max_total,
                               uint32_t* d_counts, void* stream) {
    qs_status s = batch_args(b, d_keys, d_offsets);
    if (s != QS_OK || max_total == 0) return s;
    if (!d_counts) return fail(QS_ERR_INVALID_ARG, "null counts");
    if (max_total > (uint64_t)0xffffffffu * 2048u) return fail(QS_ERR_CAPACITY, "query batch too large");
    DeviceGuard guard(b->sk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    bool ran = false;
    s = batch_graph(b, 1, d_keys, d_offsets, d_counts, max_total, st,
                    [&](cudaStream_t cs) {
                        return batch_query_seq(b, d_keys, d_offsets, max_total, d_counts, cs, false);
                    },
                    &ran);
    if (s == QS_OK && !ran) s = batch_query_seq(b, d_keys, d_offsets, max_total, d_counts, st);
    if (s == QS_OK) ++b->info.queries;
    return s;
}

qs_status qs_batch_autotune(qs_batch* b, const uint32_t* d_keys, const uint64_t* d_offsets, uint64_t total,
                            uint32_t reps, uint32_t* h_class_lpk) {
    if (!b || !d_keys || !d_offsets) return fail(QS_ERR_INVALID_ARG, "qs_batch_autotune: null argument");
    qs_sketch* sk = b->sk;
    DeviceGuard guard(sk->device);
    reps = std::max(1u, reps);
    // each size class's grouped range
    std::vector<std::pair<uint32_t, uint32_t>> range(MAX_SIZE_CLASSES, {0u, 0u});
    for (uint32_t k = 0; k < b->S; ++k) {
        auto& r = range[b->grp_class[k]];
        if (r.first == r.second) r.first = k;
        r.second = k + 1;
    }
    std::vector<double> best(MAX_SIZE_CLASSES, 1e300);
    uint32_t pick[MAX_SIZE_CLASSES] = {};
    cudaEvent_t ev[2 * MAX_SIZE_CLASSES];
    for (auto& e : ev) CK(cudaEventCreate(&e), "tuner events");
    auto destroy = [&] {
        for (auto& e : ev) cudaEventDestroy(e);
    };
    const BatchWindow W = flat_window(0, std::min<uint64_t>(total, sk->max_batch));
    qs_status st = QS_OK;
    for (int lpk : {4, 2, 8, 1, 16, 32}) {
        if (lpk > 8 && sk->D.route == 2) continue;
        std::vector<double> t(MAX_SIZE_CLASSES, 0.0);
        for (uint32_t r = 0; r < reps && st == QS_OK; ++r) {
            st = qs_batch_clear(b, nullptr);
            if (st != QS_OK) break;
            BatchDev B = b->B;
            B.key_off = d_offsets;
            cudaError_t e = batch_plan(B, sk->D.ctl, W, false, 0);
            for (uint32_t c = 0; c < MAX_SIZE_CLASSES && e == cudaSuccess; ++c) {
                if (range[c].first == range[c].second) continue;
                cudaEventRecord(ev[2 * c], 0);
                e = batch_insert_pass(d_keys, sk->D, B, sk->L, sk->agg, lpk, range[c].first, range[c].second, c, 0);
                cudaEventRecord(ev[2 * c + 1], 0);
            }
            if (e == cudaSuccess) e = batch_repair(d_keys, sk->D, B, sk->L, 0);
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            for (uint32_t c = 0; c < MAX_SIZE_CLASSES && e == cudaSuccess; ++c) {
                if (range[c].first == range[c].second) continue;
                float ms = 0;
                e = cudaEventElapsedTime(&ms, ev[2 * c], ev[2 * c + 1]);
                t[c] += ms;
            }
            if (e != cudaSuccess) st = cuda_fail(e, "batch autotune");
        }
        if (st != QS_OK) break;
        for (uint32_t c = 0; c < MAX_SIZE_CLASSES; ++c)
            if (range[c].first != range[c].second && t[c] < best[c]) {
                best[c] = t[c];
                pick[c] = (uint32_t)lpk;
            }
    }
    if (st != QS_OK) {
        destroy();
        return st;
    }
    // Per-class picks split pass 1 into several launches per window; a launch has a fixed cost.
    // So the whole insert call decides: each width for every class, and the per-class picks,
    // timed over the full batch (clear + qs_batch_insert), the fastest kept.
    auto time_insert = [&](double* ms) -> qs_status {
        double tot = 0;
        for (uint32_t r = 0; r < reps; ++r) {
            qs_status q = qs_batch_clear(b, nullptr);
            if (q != QS_OK) return q;
            CK(cudaEventRecord(ev[0], 0), "tuner event");
            q = qs_batch_insert(b, d_keys, d_offsets, total, nullptr);
            if (q != QS_OK) return q;
            CK(cudaEventRecord(ev[1], 0), "tuner event");
            CK(cudaEventSynchronize(ev[1]), "tuner sync");
            float m = 0;
            CK(cudaEventElapsedTime(&m, ev[0], ev[1]), "tuner time");
            tot += m;
        }
        *ms = tot / reps;
        return QS_OK;
    };
    uint32_t best_set[MAX_SIZE_CLASSES];
    double best_ms = 1e300;
    auto try_set = [&](const uint32_t* set) -> qs_status {
        std::memcpy(b->class_lpk, set, sizeof b->class_lpk);
        batch_rebuild_runs(b);
        double ms = 0;
        qs_status q = time_insert(&ms);
        if (q == QS_OK && ms < best_ms) {
            best_ms = ms;
            std::memcpy(best_set, set, sizeof best_set);
        }
        return q;
    };
    for (int lpk : {4, 2, 8, 1, 16, 32}) {
        if ((lpk > 8 && sk->D.route == 2) || st != QS_OK) continue;
        uint32_t set[MAX_SIZE_CLASSES];
        for (auto& x : set) x = (uint32_t)lpk;
        st = try_set(set);
    }
    if (st == QS_OK) {
        uint32_t set[MAX_SIZE_CLASSES];
        for (uint32_t c = 0; c < MAX_SIZE_CLASSES; ++c) set[c] = pick[c] ? pick[c] : best_set[0];
        st = try_set(set);
    }
    destroy();
    if (st != QS_OK) return st;
    std::memcpy(b->class_lpk, best_set, sizeof b->class_lpk);
    batch_rebuild_runs(b);
    if (h_class_lpk)
        for (uint32_t c = 0; c < MAX_SIZE_CLASSES; ++c) h_class_lpk[c] = pick[c] ? best_set[c] : 0u;
    return qs_batch_clear(b, nullptr);
}

qs_status qs_batch_clear(qs_batch* b, void* stream) {
    if (!b) return fail(QS_ERR_INVALID_ARG, "null batch");
    qs_status s = qs_clear(b->sk, stream);
    if (s != QS_OK) return s;
    DeviceGuard guard(b->sk->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<uint32_t> first(b->S, FIRST_ID);
    CK(cudaMemcpyAsync(b->B.next_id, first.data(), (size_t)b->S * 4, cudaMemcpyHostToDevice, st), "reset allocators");
    CK(cudaMemsetAsync(b->B.status, 0, (size_t)b->S * 4, st), "reset stream status");
    // the clear restarts the control block's link generation, which tags these
    CK(cudaMemsetAsync(b->B.first, 0, (size_t)b->S * 8, st), "reset link ranks");
    CK(cudaStreamSynchronize(st), "clear sync");  // the host vector above must outlive the copy
    return QS_OK;
}

qs_status qs_batch_sync(qs_batch* b, void* stream) {
    if (!b) return fail(QS_ERR_INVALID_ARG, "null batch");
    DeviceGuard guard(b->sk->device);
    CK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "stream sync");
    Ctl c;
    CK(cudaMemcpy(&c, b->sk->D.ctl, sizeof c, cudaMemcpyDeviceToHost), "read status");
    if (c.status & ST_BAD_OFFSETS) return fail(QS_ERR_INVALID_ARG, "batch offsets are not non-decreasing from 0");
    if (c.status & ST_TIMEOUT) return fail(QS_ERR_TIMEOUT, "a bounded device wait timed out");
    if (c.status & ST_CAPACITY) return fail(QS_ERR_CAPACITY, "batch larger than its window or flag list");
    std::vector<uint32_t> st(b->S);
    CK(cudaMemcpy(st.data(), b->B.status, (size_t)b->S * 4, cudaMemcpyDeviceToHost), "read stream status");
    uint32_t full = 0;
    for (uint32_t v : st) full += (v & ST_POOL_FULL) ? 1u : 0u;
    if (full)
        return fail(QS_ERR_POOL_FULL, "%u stream(s) ran out of high buckets (%llu keys dropped)", full,
                    (unsigned long long)c.dropped);
    return QS_OK;
}

qs_status qs_batch_stream_status(qs_batch* b, uint32_t* h_status) {
    if (!b || !h_status) return fail(QS_ERR_INVALID_ARG, "null argument");
    DeviceGuard guard(b->sk->device);
    CK(cudaDeviceSynchronize(), "status sync");
    CK(cudaMemcpy(h_status, b->B.status, (size_t)b->S * 4, cudaMemcpyDeviceToHost), "read stream status");
    return QS_OK;
}

qs_status qs_batch_seeds(qs_batch* b, uint32_t* h_seeds) {
    if (!b || !h_seeds) return fail(QS_ERR_INVALID_ARG, "null argument");
    std::memcpy(h_seeds, b->seeds.data(), (size_t)b->S * 4);
    return QS_OK;
}

qs_sketch* qs_batch_arena(qs_batch* b) { return b ? b->sk : nullptr; }

qs_status qs_batch_get_info(qs_batch* b, qs_batch_info* out) {
    if (!b || !out) return fail(QS_ERR_INVALID_ARG, "null argument");
    std::vector<uint32_t> st(b->S);
    qs_status s = qs_batch_stream_status(b, st.data());
    if (s != QS_OK) return s;
    *out = b->info;
    out->graph_capture = b->graph_ok == 0 ? 0u : 1u;
    out->streams_pool_full = 0;
    for (uint32_t v : st) out->streams_pool_full += (v & ST_POOL_FULL) ? 1u : 0u;
    return QS_OK;
}

}  // extern "C"

// ---- autotuner ------------------------------------------------------------------------------

extern "C" {

void qs_autotune_reset(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
}

qs_status qs_autotune_lookup(uint64_t n_low, qs_tune_config* out) {
    if (!out) return fail(QS_ERR_INVALID_ARG, "null output");
    if (!tune_lookup(n_low, out)) return fail(QS_ERR_INVALID_ARG, "no tuned setting for this size class");
    return QS_OK;
}

qs_status qs_autotune(const qs_params* base, const uint32_t* d_keys, size_t n, uint32_t reps, qs_tune_config* best,
                      qs_tune_config* h_all, uint32_t max_all, uint32_t* n_all) {
    if (!base || !d_keys || !best || n == 0) return fail(QS_ERR_INVALID_ARG, "qs_autotune: bad argument");
    if (base->kind != QS_KIND_MSWS) return fail(QS_ERR_INVALID_ARG, "qs_autotune: MSWS sketches only");
    if (reinterpret_cast<uintptr_t>(d_keys) & 3u) return fail(QS_ERR_INVALID_ARG, "keys not 4-byte aligned");
    reps = std::max(1u, reps);
    // chunk sizes worth trying: 2^20 .. 2^26, none far beyond the sample; a caller that inserts
    // in calls of a fixed size passes it as base->max_batch: that size is kept, and the sample
    // is inserted in chunks of it (into a sketch that keeps its state from chunk to chunk)
    std::vector<uint64_t> mbs;
    if (base->max_batch) {
        if ((base->max_batch & 31) || base->max_batch > (1ull << 26))
            return fail(QS_ERR_INVALID_ARG, "qs_autotune: max_batch must be a multiple of 32, at most 2^26");
        mbs.push_back(base->max_batch);
    } else {
        for (uint64_t mb = 1ull << 20; mb <= (1ull << 26); mb <<= 1)
            if (mb <= std::max<uint64_t>(1ull << 20, 2 * (uint64_t)n)) mbs.push_back(mb);
    }
    qs_params p = *base;
    p.lanes_per_key = 8;
    p.aggregate = 3;
    p.route = 1;
    p.ctas_per_sm = 0;
    p.max_batch = mbs.back();
    qs_sketch* sk = nullptr;
    qs_status s = qs_create(&p, &sk);
    if (s != QS_OK) return s;
    DeviceGuard guard(sk->device);
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&](qs_status r) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
        qs_destroy(sk);
        return r;
    };
    cudaError_t ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) return cleanup(cuda_fail(ce, "autotune setup"));
    const uint64_t alloc_mb = sk->max_batch;
    uint32_t timed = 0;
    auto run = [&](qs_tune_config& c) -> qs_status {
        sk->L.lanes_per_key = (int)c.lanes_per_key;
        sk->L.ctas_per_sm = (int)c.ctas_per_sm;
        sk->L.tile_keys = (int)c.keys_per_tile;
        sk->agg = (int)c.aggregate - 1;
        sk->D.route = c.route == 3 ? 0u : c.route;
        sk->max_batch = std::min(c.max_batch, alloc_mb);
        sk->ramp_first = c.first_chunk;
        double tot = 0;
        for (uint32_t r = 0; r <= reps; ++r) {  // the first round warms up
            qs_status q = qs_clear(sk, st);
            if (q != QS_OK) return q;
            CK(cudaEventRecord(e0, st), "autotune event");
            q = insert_device(sk, d_keys, n, st);
            if (q != QS_OK) return q;
            CK(cudaEventRecord(e1, st), "autotune event");
            CK(cudaEventSynchronize(e1), "autotune sync");
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1), "autotune time");
            if (r) tot += ms;
        }
        c.insert_ms = tot / reps;
        if (h_all && timed < max_all) h_all[timed] = c;
        ++timed;
        return QS_OK;
    };
    qs_tune_config cur{8u, 3u, 1u, 0u, base->max_batch ? mbs[0] : std::min<uint64_t>(1ull << 22, mbs.back()), 1ull << 18,
                       2048u, 0u, 0.0};
    s = run(cur);
    if (s != QS_OK) return cleanup(s);
    // a setting replaces the incumbent only when it is at least 1 % faster: differences below
    // that are run-to-run noise, and the search order (smaller chunks first) then decides
    auto consider = [&](qs_tune_config c) -> qs_status {
        qs_status q = run(c);
        if (q == QS_OK && c.insert_ms < 0.99 * cur.insert_ms) cur = c;
        return q;
    };
    for (uint32_t lpk : {4u, 2u, 1u, 16u, 32u}) {
        qs_tune_config c = cur;
        c.lanes_per_key = lpk;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    for (uint32_t tile : {1024u, 512u, 256u}) {  // keys per CTA tile
        qs_tune_config c = cur;
        c.keys_per_tile = tile;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    for (uint32_t agg : {1u, 2u, 3u}) {
        if (agg == cur.aggregate) continue;
        qs_tune_config c = cur;
        c.aggregate = agg;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    for (uint32_t route : {2u, 3u}) {
        if (route == 2 && cur.lanes_per_key > 8) continue;
        qs_tune_config c = cur;
        c.route = route;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    for (uint32_t ctas : {1u, 2u, 3u}) {
        qs_tune_config c = cur;
        c.ctas_per_sm = ctas;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    for (uint64_t mb : mbs) {
        if (mb == cur.max_batch) continue;
        qs_tune_config c = cur;
        c.max_batch = mb;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    for (uint64_t first : {0ull, 1ull << 20}) {
        qs_tune_config c = cur;
        c.first_chunk = first;
        if ((s = consider(c)) != QS_OK) return cleanup(s);
    }
    if (n_all) *n_all = timed;
    *best = cur;
    {
        const uint64_t n_low = sk->D.n_low;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[size_class(n_low)] = cur;
    }
    return cleanup(QS_OK);
}

}  // extern "C"
