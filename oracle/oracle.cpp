// oracle.cpp — TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference QSketch
// insert/query semantics, used by tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg as the checker.  Nothing in the product (qsketch_b200/, include/)
// links or calls this file.
//
// Sequential semantics restated from the reference (bu-hpc/QSketch):
//   hash          include/sketch/device_sketch/device_hash_function.h:6-18
//                 hv = key * seed (mod 2^32), seed_sz = 1 (lib/default.cu:52)
//   bucket/mask   include/sketch/device_sketch/device_sketch_v3.h:39-45
//                 bucket = hv % n_low, mask = table[hv % H]
//   insert        device_sketch_v3.h:88-191 (calculation_s2_insert), 54-85
//                 (insert_high, atomic_malloc); low→high switch when a selected 8-bit
//                 counter exceeds 128 (:160); ids start at NEXT_LEVEL_ID_START+1 = 1025
//                 (device_sketch.h:107-111), high bucket at (id-1024)*32 (:119,:185)
//   query         device_sketch_v3.h:311-408 (calculation_s2_search): min over the
//                 selected low bytes + (linked ? min over the selected high counters : 0)
//   plain CM      device_sketch_v0.h:45-54 (insert), :90-100 (query)
//   masks         lib/hashmask.cu:32-83 (generate_hashmask) on std::default_random_engine
//                 (= std::minstd_rand0 in libstdc++), reseeded here with an integer
//   seed draw     device_sketch.h:290 → include/tool/tool.h:206-220
//   primes        lib/qsketch.cu:50-115 (find_greatest_prime)
//   exact counts  include/sketch/host_sketch/host_sketch.h:20-39 (Unordered_Map)
//   error metric  include/analyze/analyze.h:15-41 (Percentage_Functor, average)
//
// Decisions where the reference is racy or unbounded (identical in the GPU path):
//   * the high pool is bounded: a link needs (id - 1024) < n_high; when it is full the
//     bucket becomes SATURATED (word 7 = 2): its keys are dropped and counted, its query
//     is the frozen low minimum.  Ids go out in the array order of the keys that switch
//     buckets, so which buckets saturate is defined by the key order (the GPU path hands
//     them out in the same order).
//   * compat_v3 = 1 reproduces device_sketch_v3.h:187 (the linking key's high increments
//     land on index bit % 8); compat_v3 = 0 uses the bit's own index, as the later
//     device_sketch_v32.h:175 and the paper's Algorithm 4 do.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {
constexpr uint32_t START = 1024;   // lib/default.cu:45
constexpr uint32_t LIMIT = 128;    // device_sketch_v3.h:160
constexpr uint32_t SATURATED = 2;  // reserved value (< START), see header comment
constexpr int W = 8;               // words per low bucket
constexpr int HW = 32;             // counters per high bucket

inline uint32_t low_byte(const uint32_t* w, int i) { return (w[i >> 2] >> (8 * (i & 3))) & 0xffu; }
}  // namespace

extern "C" {

// lib/qsketch.cu:50-115 — the same table of primes near 2^k and 1.5*2^k.
uint64_t or_find_greatest_prime(uint64_t upper_bound) {
    static const uint64_t ps[] = {
        402653171, 268435399, 201326557, 134217689, 100663291, 67108859, 50331599, 33554393,
        25165813,  16777213,  12582893,  8388593,   6291449,   4194301,  3145721,  2097143,
        1572853,   1048573,   786431,    524287,    393209,    262139,   196597,   131071,
        98299,     65521,     49139,     32749,     24571,     16381,    12281,    8191,
        6143,      4093,      3067,      2039,      1531,      1021,     761,      509,
        383,       251,       191,       127,       89,        61,       47,       31,
        23,        13,        11,        7,         5,         3,        2};
    for (uint64_t p : ps)
        if (p <= upper_bound) return p;
    return 0;
}

// lib/hashmask.cu:32-83 with an integer-seeded engine.  Returns 0 on success.
int or_generate_hashmask(uint32_t rng_seed, size_t n, size_t m_bits, size_t ones, size_t padding,
                         uint8_t* out) {
    if (m_bits <= padding || ones > m_bits - padding) return -1;
    const size_t mask_bytes = (m_bits + 7) / 8;
    std::memset(out, 0, n * mask_bytes);
    std::minstd_rand0 eng(rng_seed);
    std::uniform_int_distribution<uint32_t> dis(0, (uint32_t)(m_bits - padding - 1));
    for (size_t i = 0; i < n; ++i) {
        size_t j = 0;
        while (j < ones) {
            uint32_t id = dis(eng);
            uint8_t* m = out + i * mask_bytes;
            uint8_t b = (uint8_t)(1u << (id % 8));
            if ((m[id / 8] & b) == 0) {  // lib/hashmask.cu:5-20 (set)
                m[id / 8] |= b;
                ++j;
            }
        }
    }
    return 0;
}

// include/tool/tool.h:206-220 with min = 1, max = UINT_MAX.
void or_draw_seeds(uint32_t rng_seed, size_t count, uint32_t* out) {
    std::minstd_rand0 eng(rng_seed);
    std::uniform_int_distribution<uint32_t> dis(1u, 0xffffffffu);
    for (size_t i = 0; i < count; ++i) out[i] = dis(eng);
}

// ---------------------------------------------------------------------------------------
// MSWS state.  low: n_low*8 words, high: n_high*32 words, masks: H 32-bit mask words.
typedef struct or_msws {
    uint32_t* low;
    uint64_t n_low;
    uint32_t* high;
    uint64_t n_high;
    const uint32_t* masks;
    uint32_t n_masks;
    uint32_t seed;
    uint32_t next_id;
    int32_t compat_v3;
    uint32_t pool_full;
    uint32_t pad;
    uint64_t dropped;
} or_msws;

static inline void msws_insert_one(or_msws* s, uint32_t key, std::atomic<uint32_t>* shared_next) {
    const uint32_t hv = key * s->seed;
    const uint64_t b = hv % s->n_low;
    const uint32_t mask = s->masks[hv % s->n_masks];
    uint32_t* w = s->low + b * W;
    uint32_t ptr = w[7];
    if (ptr == SATURATED) { ++s->dropped; return; }
    if (ptr > START) {  // device_sketch_v3.h:111-129
        uint32_t* h = s->high + (uint64_t)(ptr - START) * HW;
        for (uint32_t m = mask; m; m &= m - 1) h[__builtin_ctz(m)] += 1;
        return;
    }
    bool over = false;  // device_sketch_v3.h:132-161
    for (uint32_t m = mask; m; m &= m - 1)
        if (low_byte(w, __builtin_ctz(m)) > LIMIT) over = true;
    if (!over) {  // :163-170
        for (uint32_t m = mask; m; m &= m - 1) {
            int i = __builtin_ctz(m);
            w[i >> 2] += 1u << (8 * (i & 3));
        }
        return;
    }
    // :172-190 — allocate (atomic_malloc :69-85) and insert into the new high bucket
    uint32_t id;
    if (shared_next) {
        id = shared_next->fetch_add(1);
        if ((uint64_t)(id - START) >= s->n_high) { w[7] = SATURATED; s->pool_full = 1; ++s->dropped; return; }
    } else {
        if ((uint64_t)(s->next_id - START) >= s->n_high) { w[7] = SATURATED; s->pool_full = 1; ++s->dropped; return; }
        id = s->next_id++;
    }
    w[7] = id;
    uint32_t* h = s->high + (uint64_t)(id - START) * HW;
    for (uint32_t m = mask; m; m &= m - 1) {
        int i = __builtin_ctz(m);
        h[s->compat_v3 ? (i % 8) : i] += 1;
    }
}

void or_msws_insert(or_msws* s, const uint32_t* keys, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) msws_insert_one(s, keys[i], nullptr);
}

// Bucket-partitioned parallel insert, one pass over the keys: T threads each take a
// contiguous block of the keys and count them by partition (bucket % T); after a prefix over
// (partition, block) they scatter their keys into per-partition lists, which keep array
// order; then thread t applies partition t's list.  Per-bucket order is the array order, so
// the tables equal the sequential ones except for the high ids (allocation interleaves
// across threads) and, once the pool runs out, which buckets get one.
void or_msws_insert_mt(or_msws* s, const uint32_t* keys, uint64_t n, int threads) {
    if (threads <= 1 || n < (1u << 16)) { or_msws_insert(s, keys, n); return; }
    const uint32_t T = (uint32_t)threads;
    auto part = [&](uint32_t k) { return (uint32_t)((uint64_t)(uint32_t)(k * s->seed) % s->n_low % T); };
    std::vector<uint64_t> cnt((size_t)T * T, 0);  // [block][partition]
    std::vector<uint32_t> list(n);
    auto block = [&](uint32_t b, uint64_t& lo, uint64_t& hi) { lo = n * b / T; hi = n * (b + 1) / T; };
    {
        std::vector<std::thread> th;
        for (uint32_t b = 0; b < T; ++b)
            th.emplace_back([&, b] {
                uint64_t lo, hi;
                block(b, lo, hi);
                uint64_t* c = &cnt[(size_t)b * T];
                for (uint64_t i = lo; i < hi; ++i) ++c[part(keys[i])];
            });
        for (auto& x : th) x.join();
    }
    std::vector<uint64_t> off((size_t)T * T), pbeg(T + 1, 0);  // off[block][partition]
    uint64_t run = 0;
    for (uint32_t p = 0; p < T; ++p) {
        pbeg[p] = run;
        for (uint32_t b = 0; b < T; ++b) {
            off[(size_t)b * T + p] = run;
            run += cnt[(size_t)b * T + p];
        }
    }
    pbeg[T] = run;
    {
        std::vector<std::thread> th;
        for (uint32_t b = 0; b < T; ++b)
            th.emplace_back([&, b] {
                uint64_t lo, hi;
                block(b, lo, hi);
                uint64_t* o = &off[(size_t)b * T];
                for (uint64_t i = lo; i < hi; ++i) list[o[part(keys[i])]++] = keys[i];
            });
        for (auto& x : th) x.join();
    }
    std::atomic<uint32_t> next(s->next_id);
    std::vector<or_msws> local(T, *s);
    {
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < T; ++t)
            th.emplace_back([&, t] {
                or_msws* ls = &local[t];
                ls->dropped = 0;
                ls->pool_full = 0;
                for (uint64_t i = pbeg[t]; i < pbeg[t + 1]; ++i) msws_insert_one(ls, list[i], &next);
            });
        for (auto& x : th) x.join();
    }
    uint32_t nid = next.load();
    uint64_t cap = START + s->n_high;
    s->next_id = nid > cap ? (uint32_t)cap : nid;
    for (auto& ls : local) { s->dropped += ls.dropped; s->pool_full |= ls.pool_full; }
}

// REMOVE (no code in the reference; the paper defines deletion as insertion with a
// subtraction, doc/main.tex:232): per key in array order, the bucket's level decides where
// the key's selected counters lose one, each floored at 0 — the high counters when the bucket
// is linked, else the low 8-bit counters; a saturated bucket drops the removal (counted).
// Removals never link or unlink a bucket, so within one remove call the result per counter
// is max(0, value - removals) whatever the order.
void or_msws_remove(or_msws* s, const uint32_t* keys, uint64_t n) {
    for (uint64_t k = 0; k < n; ++k) {
        const uint32_t hv = keys[k] * s->seed;
        const uint64_t b = hv % s->n_low;
        const uint32_t mask = s->masks[hv % s->n_masks];
        uint32_t* w = s->low + b * W;
        const uint32_t ptr = w[7];
        if (ptr == SATURATED) { ++s->dropped; continue; }
        if (ptr > START) {
            uint32_t* h = s->high + (uint64_t)(ptr - START) * HW;
            for (uint32_t m = mask; m; m &= m - 1) {
                uint32_t& c = h[__builtin_ctz(m)];
                if (c) --c;
            }
            continue;
        }
        for (uint32_t m = mask; m; m &= m - 1) {
            const int i = __builtin_ctz(m);
            if (low_byte(w, i)) w[i >> 2] -= 1u << (8 * (i & 3));
        }
    }
}

// Count-min REMOVE: each row's counter loses one, floored at 0.
void or_cm_remove(uint32_t* table, uint64_t n, uint32_t m, const uint32_t* seeds, const uint32_t* keys, uint64_t nk) {
    for (uint64_t i = 0; i < nk; ++i)
        for (uint32_t j = 0; j < m; ++j) {
            uint32_t& c = table[j * n + (uint32_t)(keys[i] * seeds[j]) % n];
            if (c) --c;
        }
}

void or_msws_query(const or_msws* s, const uint32_t* keys, uint64_t n, uint32_t* out) {
    for (uint64_t k = 0; k < n; ++k) {
        const uint32_t hv = keys[k] * s->seed;
        const uint64_t b = hv % s->n_low;
        const uint32_t mask = s->masks[hv % s->n_masks];
        const uint32_t* w = s->low + b * W;
        uint32_t lo = 0xffffffffu, hi = 0xffffffffu;
        for (uint32_t m = mask; m; m &= m - 1) lo = std::min(lo, low_byte(w, __builtin_ctz(m)));
        const uint32_t ptr = w[7];
        if (ptr > START) {
            const uint32_t* h = s->high + (uint64_t)(ptr - START) * HW;
            for (uint32_t m = mask; m; m &= m - 1) hi = std::min(hi, h[__builtin_ctz(m)]);
        } else {
            hi = 0;
        }
        out[k] = lo + hi;
    }
}

// ---------------------------------------------------------------------------------------
// Plain count-min (device_sketch_v0.h): rows m, n counters per row, seeds[m].
void or_cm_insert(uint32_t* table, uint64_t n, uint32_t m, const uint32_t* seeds, const uint32_t* keys,
                  uint64_t nk) {
    for (uint64_t i = 0; i < nk; ++i)
        for (uint32_t j = 0; j < m; ++j) table[j * n + (uint32_t)(keys[i] * seeds[j]) % n] += 1;
}

// The same with T threads over contiguous blocks of the keys, relaxed atomic increments (the
// additions commute, so the table equals the sequential one).
void or_cm_insert_mt(uint32_t* table, uint64_t n, uint32_t m, const uint32_t* seeds, const uint32_t* keys,
                     uint64_t nk, int threads) {
    if (threads <= 1) { or_cm_insert(table, n, m, seeds, keys, nk); return; }
    std::vector<std::thread> th;
    for (int b = 0; b < threads; ++b)
        th.emplace_back([=] {
            const uint64_t lo = nk * b / threads, hi = nk * (b + 1) / threads;
            for (uint64_t i = lo; i < hi; ++i)
                for (uint32_t j = 0; j < m; ++j)
                    __atomic_fetch_add(&table[j * n + (uint32_t)(keys[i] * seeds[j]) % n], 1u, __ATOMIC_RELAXED);
        });
    for (auto& x : th) x.join();
}

void or_cm_query(const uint32_t* table, uint64_t n, uint32_t m, const uint32_t* seeds, const uint32_t* keys,
                 uint64_t nk, uint32_t* out) {
    for (uint64_t i = 0; i < nk; ++i) {
        uint32_t c = 0xffffffffu;
        for (uint32_t j = 0; j < m; ++j) c = std::min(c, table[j * n + (uint32_t)(keys[i] * seeds[j]) % n]);
        out[i] = c;
    }
}

// ---------------------------------------------------------------------------------------
// One-level bucket sketch: the reference's warp sketch (device_sketch_v1.h:50-61 insert,
// :135-158 query; m = 32) and sub-warp sketch (device_sketch_v2.h:54-64, :156-185; m < 32).
// n buckets of m u32 counters; key -> hv = key * seed, bucket hv % n, mask word masks[hv % H]
// (bit i selects counter i); insert adds 1 to every selected counter, query is their minimum,
// remove takes 1 from every selected counter, floored at 0.
void or_bucket_insert(uint32_t* table, uint64_t n, uint32_t m, uint32_t seed, const uint32_t* masks, uint32_t H,
                      const uint32_t* keys, uint64_t nk) {
    for (uint64_t i = 0; i < nk; ++i) {
        const uint32_t hv = keys[i] * seed;
        uint32_t* b = table + (hv % n) * m;
        for (uint32_t mm = masks[hv % H]; mm; mm &= mm - 1) b[__builtin_ctz(mm)] += 1;
    }
}

void or_bucket_query(const uint32_t* table, uint64_t n, uint32_t m, uint32_t seed, const uint32_t* masks, uint32_t H,
                     const uint32_t* keys, uint64_t nk, uint32_t* out) {
    for (uint64_t i = 0; i < nk; ++i) {
        const uint32_t hv = keys[i] * seed;
        const uint32_t* b = table + (hv % n) * m;
        uint32_t c = 0xffffffffu;
        for (uint32_t mm = masks[hv % H]; mm; mm &= mm - 1) c = std::min(c, b[__builtin_ctz(mm)]);
        out[i] = c;
    }
}

void or_bucket_remove(uint32_t* table, uint64_t n, uint32_t m, uint32_t seed, const uint32_t* masks, uint32_t H,
                      const uint32_t* keys, uint64_t nk) {
    for (uint64_t i = 0; i < nk; ++i) {
        const uint32_t hv = keys[i] * seed;
        uint32_t* b = table + (hv % n) * m;
        for (uint32_t mm = masks[hv % H]; mm; mm &= mm - 1) {
            uint32_t& c = b[__builtin_ctz(mm)];
            if (c) --c;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Exact counter (host_sketch.h:20-39): counts of `queries` among `keys`.
void or_exact_counts(const uint32_t* keys, uint64_t n, const uint32_t* queries, uint64_t nq, uint32_t* out) {
    std::unordered_map<uint32_t, uint32_t> um;
    um.reserve(nq * 2 + 16);
    for (uint64_t i = 0; i < nq; ++i) um.emplace(queries[i], 0u);
    for (uint64_t i = 0; i < n; ++i) {
        auto it = um.find(keys[i]);
        if (it != um.end()) ++it->second;
    }
    for (uint64_t i = 0; i < nq; ++i) out[i] = um[queries[i]];
}

// Mean |est-exact|/exact and mean est/exact over entries with exact > 0
// (analyze.h:15-41 reports mean(est/exact)*100).
void or_error_metrics(const uint32_t* est, const uint32_t* exact, uint64_t n, double* mean_rel, double* mean_ratio) {
    double r = 0, q = 0;
    uint64_t c = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (!exact[i]) continue;
        double e = est[i], a = exact[i];
        r += (e > a ? e - a : a - e) / a;
        q += e / a;
        ++c;
    }
    *mean_rel = c ? r / c : 0.0;
    *mean_ratio = c ? q / c : 0.0;
}

}  // extern "C"
