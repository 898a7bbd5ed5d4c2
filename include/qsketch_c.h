/*
 * qsketch_c.h — C ABI of the B200-native QSketch insert/query path.
 *
 * The reference exposes its sketches as the C++ abstract class
 *   template<Key_T, Count_T> struct qsketch::Sketch {
 *       virtual int insert(Key_T *keys, size_t n);
 *       virtual int search(Key_T *keys, size_t n, Count_T *counts);
 *       virtual void clear();  virtual ~Sketch(); }
 * (reference include/sketch/sketch.h:5-28) with concrete constructors
 *   Sketch_GPU_Sub_Warp_Level(n_low, m_low, n_high, m_high, seed_sz, n_hash_mask_table)
 *     (include/sketch/device_sketch/device_sketch_v3.h:544-563)
 *   Sketch_GPU_Thread(n, m, seed_sz)
 *     (include/sketch/device_sketch/device_sketch_v0.h:121-131)
 * Key_T = Count_T = unsigned int (reference src/main.cu:3-6).
 *
 * This header is the drop-in boundary: every entry point takes plain pointers and
 * sizes, device pointers where the reference takes device pointers, and a CUDA stream
 * passed as `void *` (0 = legacy default stream).  No C++ or torch types cross it.
 * All calls are stream-ordered and asynchronous; device-side errors (pool exhaustion,
 * bounded-wait timeouts) are latched in a per-sketch status word and reported by
 * qs_sync() / qs_get_stats().  No call aborts the process.
 */
#ifndef QSKETCH_C_H
#define QSKETCH_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QS_ABI_VERSION 2u

/* Status codes.  The reference returns 0 from every call and ignores CUDA errors in
 * release builds (include/qsketch.h:104-105); these replace that. */
typedef enum qs_status {
    QS_OK = 0,
    QS_ERR_INVALID_ARG = 1, /* bad parameter, null handle, unsupported layout */
    QS_ERR_OOM = 2,         /* device allocation failed */
    QS_ERR_CUDA = 3,        /* CUDA runtime error (text via qs_last_error_string) */
    QS_ERR_POOL_FULL = 4,   /* the high-level bucket pool ran out (latched) */
    QS_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up (latched) */
    QS_ERR_NO_DEVICE = 6,   /* no CUDA device / extension compiled for another arch */
    QS_ERR_CAPACITY = 7     /* a call exceeds a documented size limit */
} qs_status;

/* Sketch families on the path. */
typedef enum qs_kind {
    QS_KIND_MSWS = 0,     /* lock-free multi-level sub-warp sketch ("Level"),
                             reference Sketch_GPU_Sub_Warp_Level (device_sketch_v3.h:526) */
    QS_KIND_PLAIN_CM = 1, /* plain count-min ("thread sketch"),
                             reference Sketch_GPU_Thread (device_sketch_v0.h:107) */
    QS_KIND_BUCKET = 2    /* one-level bucket sketch: n_low buckets of m_low (8, 16 or 32) u32
                             counters, a key's mask of m_low bits with hash_mask_ones set
                             selecting its counters in bucket hv % n_low; the reference's warp
                             sketch Sketch_GPU_Warp (device_sketch_v1.h:237, m = 32) and sub-warp
                             sketch Sketch_GPU_Sub_Warp (device_sketch_v2.h:289, m < 32), kept for
                             the ablation against the two-level MSWS */
} qs_kind;

/* Flags. */
#define QS_FLAG_COMPAT_V3 0x1u /* reproduce device_sketch_v3.h:187: the key that links a
                                  bucket adds its high increments at index (bit % 8)
                                  instead of at the bit's own counter */
#define QS_FLAG_NO_CHUNK_RAMP 0x2u /* insert in chunks of max_batch from the first key.  By
                                     default the chunks after a create or clear grow from
                                     first_chunk keys (f, f, 2f, 4f, ... max_batch): the buckets of
                                     heavy keys then link in a small first chunk instead of
                                     sending all their occurrences of a large chunk through the
                                     ordered replay.  Results never depend on the chunking. */

/* Creation parameters.  Zero-initialise and set what you need; qs_params_default()
 * fills the reference defaults (lib/default.cu:39-54). */
typedef struct qs_params {
    uint32_t kind;              /* qs_kind */
    uint32_t flags;             /* QS_FLAG_* */
    /* MSWS: n_low low buckets of m_low u32 words (m_low must be 8: 32 B buckets with
     * 28 packed 8-bit counters + the high-bucket index word), n_high high buckets of
     * m_high u32 counters (m_high must be 32).
     * PLAIN_CM: n_low counters per row, m_low rows (the reference's "m").
     * n_low == 0 derives it from low_bytes with find_greatest_prime(). */
    uint64_t n_low;
    uint64_t low_bytes;
    uint32_t m_low;
    uint32_t m_high;
    uint64_t n_high;
    uint32_t seed_sz;            /* hash seeds per row; must be 1 (lib/default.cu:52) */
    uint32_t hash_mask_table_sz; /* H, masks in the table (lib/default.cu:54: 1021) */
    uint32_t hash_mask_ones;     /* counters per key in a low bucket, the "row count"
                                    (lib/default.cu:53: 3); 1..28 */
    uint32_t hash_seed;          /* MSWS multiplier; 0 = draw it like the reference
                                    (device_sketch.h:290) from seed_rng */
    uint32_t seed_rng;           /* seeds std::minstd_rand0 for hash-seed draws */
    uint32_t mask_rng;           /* seeds std::minstd_rand0 for generate_hashmask */
    const uint32_t *seeds;       /* optional host array of m_low (CM) or 1 (MSWS) seeds;
                                    overrides hash_seed / seed_rng */
    const uint8_t *mask_table;   /* optional host table of H*4 bytes (bits 0..27 only);
                                    overrides mask_rng */
    uint64_t max_batch;          /* keys per internal insert chunk (scratch sizing);
                                    a multiple of 32, at most 2^26; 0 = 1<<22 */
    int32_t device;              /* CUDA device ordinal; -1 = current */
    /* Insert-kernel knobs; none changes any result.  When lanes_per_key, aggregate, route
     * and ctas_per_sm are all 0, qs_create takes them (and max_batch, if 0) from the
     * autotuner's entry for the sketch's size class (qs_autotune), else the defaults
     * 4 / 3 / 1 / 0. */
    uint32_t lanes_per_key;      /* lanes serving one key in pass 1: 1, 2, 4, 8 (one lane
                                    per bucket word, the reference's sub-warp), 16 or 32 */
    uint32_t aggregate;          /* 1 = off, 2 = warp, 3 = warp + block pre-aggregation
                                    of duplicate keys */
    uint32_t route;              /* insert routing between the levels: 1 = load each
                                    bucket's index word first, 2 = read it with the counter
                                    atomic (at most 8 lanes per key), 3 = adaptive per tile */
    uint32_t ctas_per_sm;        /* pass-1 CTAs per SM, 0 = as many as fit */
    uint64_t first_chunk;        /* first chunk of the ramp after a create or clear (multiple
                                    of 32); 0 = 2^18, or the autotuner's choice */
    uint32_t keys_per_tile;      /* pass-1 keys per CTA tile: 256, 512, 1024 or 2048 (0 =
                                    2048, or the autotuner's choice); small chunks spread over
                                    more CTAs with smaller tiles */
} qs_params;

typedef struct qs_sketch qs_sketch;

/* Counters the device keeps per sketch (read after a sync). */
typedef struct qs_stats {
    uint32_t status_bits;     /* bit0 pool full, bit1 timeout */
    uint32_t next_level_id;   /* bump allocator value (starts at 1025) */
    uint64_t linked_buckets;  /* next_level_id - 1025, capped at the pool */
    uint64_t dropped_keys;    /* keys dropped in saturated buckets (pool exhausted) */
    uint64_t repaired_buckets;/* buckets that crossed the 8-bit threshold and were
                                 replayed in stream order, cumulative */
    uint64_t repaired_keys;   /* keys routed through the ordered replay, cumulative */
    uint64_t inserted_keys;   /* keys accepted by qs_insert, cumulative */
} qs_stats;

/* Library / device queries. */
uint32_t qs_abi_version(void);
const char *qs_status_string(qs_status s);
/* Text of the most recent error on this host thread ("" if none). */
const char *qs_last_error_string(void);

/* Fill the reference defaults: MSWS, m_low 8, m_high 32, n_high 1024, seed_sz 1,
 * H 1021, ones 3 (lib/default.cu:39-54, src/main.cu:390-391). */
void qs_params_default(qs_params *p);

/* find_greatest_prime (reference lib/qsketch.cu:50-115): largest prime of the
 * reference's table that is <= upper_bound, 0 if none. */
uint64_t qs_find_greatest_prime(uint64_t upper_bound);

/* Sketch_GPU::number_of_buckets (reference device_sketch.h:371-376):
 * find_greatest_prime(((keys / factor) * ones) / m). */
uint64_t qs_number_of_buckets(uint64_t insert_keys, uint64_t m, double factor,
                              uint32_t hash_mask_ones);

/* generate_hashmask (reference lib/hashmask.cu:32-83) on a std::minstd_rand0 seeded
 * with `rng_seed`: n masks of ceil(m_bits/8) bytes, each with `ones` distinct bits in
 * [0, m_bits - padding).  out must hold n*ceil(m_bits/8) bytes. */
qs_status qs_generate_hashmask(uint32_t rng_seed, size_t n, size_t m_bits, size_t ones,
                               size_t padding, uint8_t *out);

/* The reference's seed draw (device_sketch.h:290 → include/tool/tool.h:206-220):
 * `count` values of uniform_int_distribution<uint>(1, UINT_MAX) on a
 * std::minstd_rand0 seeded with rng_seed. */
qs_status qs_draw_seeds(uint32_t rng_seed, size_t count, uint32_t *out);

/* Construct / destroy.  Replaces the constructors cited above and ~Sketch_GPU
 * (device_sketch.h:387-394).  The handle owns all device memory. */
qs_status qs_create(const qs_params *params, qs_sketch **out);
qs_status qs_destroy(qs_sketch *sk);

/* Sketch::insert (sketch.h:7, device_sketch_v3.h:570-599, device_sketch_v0.h:140-161).
 * d_keys: device pointer to n uint32 keys (any 4-byte alignment).  Results are exactly
 * those of inserting the keys one by one in array order (the sequential semantics of
 * device_sketch_v3.h:88-191), whatever the GPU schedule. */
qs_status qs_insert(qs_sketch *sk, const uint32_t *d_keys, size_t n, void *stream);

/* Sketch::search (sketch.h:8, device_sketch_v3.h:600-632, device_sketch_v0.h:162-189).
 * Writes n uint32 estimates to d_counts (device pointer). */
qs_status qs_query(qs_sketch *sk, const uint32_t *d_keys, size_t n, uint32_t *d_counts,
                   void *stream);

/* REMOVE (no code in the reference; its paper defines deletion as the insertion with a
 * subtraction, doc/main.tex:232).  d_keys: device pointer to n uint32 keys, one occurrence of
 * each taken out.  MSWS: where the key's bucket is linked, its selected high counters lose
 * one, else its selected 8-bit low counters lose one, each floored at 0; a saturated bucket
 * drops the removal (counted in dropped_keys).  Removals never link or unlink a bucket, so
 * the result of a call does not depend on the order of its keys, and a call is ordered after
 * and before the sketch's other calls on the stream.  Count-min: each row's counter loses
 * one, floored at 0.  A removal of a key that was never inserted lowers the estimates of the
 * keys sharing its counters (as in any count-min with deletions); and for MSWS, one whose
 * earlier occurrences were counted in the low level before its bucket linked lowers the high
 * counters instead.  Contended counters are updated by compare-and-swap loops bounded to
 * 2^22 tries (QS_ERR_TIMEOUT if one gives up). */
qs_status qs_remove(qs_sketch *sk, const uint32_t *d_keys, size_t n, void *stream);

/* Host-buffer variants: keys / counts in host memory (pinned or pageable).  The copies
 * run chunked and overlapped with the kernels on internal streams; the call returns
 * when the results are in h_counts (query) or the keys are consumed (insert). */
qs_status qs_insert_host(qs_sketch *sk, const uint32_t *h_keys, size_t n);
qs_status qs_query_host(qs_sketch *sk, const uint32_t *h_keys, size_t n, uint32_t *h_counts);

/* Sketch::clear (sketch.h:14, device_sketch.h:378-381, 115-124): zero the tables and
 * reset the bump allocator to 1025. */
qs_status qs_clear(qs_sketch *sk, void *stream);

/* Synchronise the sketch's work on `stream` and return the latched device status
 * (QS_ERR_POOL_FULL / QS_ERR_TIMEOUT) or QS_OK. */
qs_status qs_sync(qs_sketch *sk, void *stream);
qs_status qs_get_stats(qs_sketch *sk, qs_stats *out);
/* Launch accounting.  Counters are cumulative; times cover the launches issued while
 * profiling was on, measured with CUDA events recorded around each launch on the stream
 * it ran on, and are reset by each qs_get_profile call. */
typedef struct qs_profile {
    double insert_ms;          /* pass-1 insert kernels (MSWS) / insert kernels (CM) */
    double repair_ms;          /* ordered-repair kernels (MSWS) */
    double query_ms;           /* query kernels */
    uint64_t insert_timed, repair_timed, query_timed;
    uint64_t insert_launches, repair_launches, query_launches;
    /* MSWS ordered repair, measured on the device (globaltimer) since the previous
     * qs_get_profile: invocations that found crossed buckets, and, while profiling is on,
     * time per phase —
     * 8 filter build, 0 flag test (and staging of the records), 1 tile scan, 2 record
     * move, radix passes split into 6 tile digit counts, 7 digit scans and 3 scatters,
     * 4 segments and totals, 5 replay, 9 link order (ranks, high buckets written);
     * 10-11 unused.  qs_clear resets them too. */
    uint64_t repairs_active;
    double repair_phase_ms[12];
} qs_profile;
qs_status qs_set_profiling(qs_sketch *sk, int enable);
qs_status qs_get_profile(qs_sketch *sk, qs_profile *out);

/* Clear the latched device status bits. */
qs_status qs_reset_status(qs_sketch *sk);

/* Sizes of the device tables in u32 words (low, high) and the seeds in use. */
qs_status qs_get_info(qs_sketch *sk, uint64_t *n_low, uint64_t *n_high, uint32_t *m_low,
                      uint32_t *seeds_out /* m_low for CM, 1 for MSWS; may be null */,
                      uint8_t *mask_table_out /* H*4 bytes; may be null */);

/* The creation parameters as the sketch holds them (seeds and mask_table come back null;
 * hash_seed is the first seed in use, n_low the bucket count, hash_mask_table_sz the mask
 * count, max_batch and device the values in effect). */
qs_status qs_get_params(qs_sketch *sk, qs_params *out);

/* Copy the device tables to host buffers (debug / oracle comparison):
 * low: n_low*m_low words (MSWS: word 7 of each bucket is the high index),
 * high: n_high*m_high words (null to skip). */
qs_status qs_get_tables(qs_sketch *sk, uint32_t *h_low, uint32_t *h_high);

/* Snapshots: a sketch's whole state — parameters, seeds, mask table, low table, high pool,
 * allocator, latched status and dropped count — as one byte string (version 1: a 96-byte
 * header, the seeds, the mask words, the tables, a 64-bit FNV-1a checksum; little-endian).
 * The reference declares read_file / write_file (include/qsketch.h:70-71) but never defines
 * them; qs_save / qs_load write and read such a snapshot as a file.  A loaded sketch answers
 * every query as the saved one did and continues exactly as it would have; it is created on
 * `device` (-1 = current) with the default insert knobs.  qs_snapshot_load refuses (with
 * QS_ERR_INVALID_ARG, before any device work) a buffer whose header, size or checksum does not
 * hold.  The sketch must not be in use on any stream while it is saved. */
qs_status qs_snapshot_bytes(qs_sketch *sk, uint64_t *bytes);
qs_status qs_snapshot_save(qs_sketch *sk, void *h_buf, uint64_t buf_bytes);
qs_status qs_snapshot_load(const void *h_buf, uint64_t bytes, int32_t device, qs_sketch **out);
qs_status qs_save(qs_sketch *sk, const char *path);
qs_status qs_load(const char *path, int32_t device, qs_sketch **out);

/* Synthetic key streams (bench / tests), written to device memory on `stream`.
 * kind 0: uniform u32 from a seeded xorshift64 stream;
 * kind 1: Zipf(s) over n_ranks ranks (rejection-inversion, Hoermann & Derflinger
 *         1996), rank r mapped to a distinct key by a seeded bijection of u32;
 * d_ranks (may be null) receives the 0-based rank of each key (kind 1 only). */
qs_status qs_gen_keys(uint32_t kind, uint64_t seed, uint64_t n_ranks, double s,
                      uint64_t perm_seed, uint32_t *d_keys, uint32_t *d_ranks, size_t n,
                      void *stream);
/* Structured keys (learned-split workload): key = class << 16 | suffix, the class id is a
 * Zipf(s_class) rank over n_class <= 2^16 classes, the suffix a Zipf(s_suffix) rank over 2^16
 * under the class's own seeded permutation of 16-bit values. */
qs_status qs_gen_class_keys(uint64_t seed, uint32_t n_class, double s_class, double s_suffix, uint64_t perm_seed,
                            uint32_t *d_keys, size_t n, void *stream);
/* The key that qs_gen_keys(kind 1) maps rank r to, for r in [first, first+n). */
qs_status qs_gen_rank_keys(uint64_t perm_seed, uint64_t first, uint32_t *d_keys, size_t n,
                           void *stream);
/* d_hist[r] += occurrences of rank r in d_ranks[0..n) (exact counts for error metrics). */
qs_status qs_rank_histogram(const uint32_t *d_ranks, size_t n, uint32_t *d_hist,
                            uint64_t n_ranks, void *stream);
/* Mean relative error |est-exact|/exact and mean est/exact over n keys (exact > 0),
 * reduced on the device; results written to host doubles. */
qs_status qs_error_metrics(const uint32_t *d_est, const uint32_t *d_exact, size_t n,
                           double *mean_rel_err, double *mean_ratio, void *stream);

/* Roofline probes: time `kind` (0 random sub-warp sector red with 3 words per sector,
 * 1 random 32 B sector load, 2 streaming read, 3 load + returning atomics, 4 returning
 * atomics with the index word, 5 load + red, 7 one red.add.u32 per lane, every lane its own
 * random sector) over a device buffer of `bytes`, returning operations per second (sectors/s,
 * or bytes/s for kind 2); kind 6 times `ops` grid-wide barriers of the ordered replay's form
 * (`bytes` unused) and returns barriers/s. */
qs_status qs_probe(uint32_t kind, uint64_t bytes, uint64_t ops, double *ops_per_s);

/* Failure paths, for tests (no counterpart in the reference):
 * qs_probe kind 8 launches one grid-wide barrier that block 0 never reaches, with every
 * other block's wait bounded by `ops` polls (~128 ns each, at most the ~1 s of the sketch
 * kernels' waits): it returns QS_ERR_TIMEOUT when the waits give up, as they must, and the
 * context stays usable.
 * qs_test_fail_allocations(k) makes the library's (k+1)-th device allocation from now on fail
 * as if the device were out of memory (qs_create then returns QS_ERR_OOM and frees what it
 * had allocated); -1 turns it off.  One failure per call. */
void qs_test_fail_allocations(int32_t after);

/* ---- learned heavy-hitter split (no counterpart in the reference) ------------------------
 * An MLP 32 -> 128 -> 128 -> 1 over the key's bits (BF16 weights, FP32 accumulation on the
 * tensor cores, weighted binary cross-entropy, Adam) decides which keys are heavy.  The
 * first `warmup_keys` keys go to the MSWS sketch alone; then the network is trained on the
 * warm-up window's distinct keys, labelled heavy when the sketch's estimate is in the top
 * `heavy_fraction`, and the warm-up keys it predicts heavy are admitted to an exact
 * open-addressing table (u32 key + u32 count).  Afterwards each key found in the table counts
 * there exactly; every other key goes to the sketch, and keys the network predicts heavy are
 * admitted at the end of their chunk.  The network decides which keys may enter the table;
 * when more are eligible than the table holds (max fill), the sketch's own estimates rank
 * them (ties by key), so admission is deterministic.  A query returns table count + sketch
 * estimate.  Sketch, table and network share
 * `budget_bytes` (sketch low:high = 4:1). */
typedef struct qs_learned_params {
    uint64_t budget_bytes;     /* default 64 MiB */
    uint32_t table_slots;      /* power of two, default 2^17 (1 MiB) */
    float table_max_fill;      /* admission stops at this load factor, default 0.75 */
    uint64_t warmup_keys;      /* default 2^24 */
    double heavy_fraction;     /* default 0.005 */
    uint32_t epochs;           /* default 4 */
    uint32_t batch;            /* training batch, default 16384 */
    float lr;                  /* Adam step, default 4e-3 */
    float max_pos_weight;      /* positive-class weight cap, default 64 */
    float eligible_recall;     /* the logit cut for table eligibility keeps this share of
                                  the labelled-heavy warm-up keys, default 0.95 */
    uint32_t hash_seed;        /* sketch hash multiplier, 0 = draw from seed_rng */
    uint32_t seed_rng, mask_rng, init_seed;
    uint64_t max_batch;        /* keys per routing chunk, default 2^22 */
    int32_t device;
    uint32_t neg_per_pos;      /* training set: every labelled-heavy warm-up key and a seeded
                                  sample of this many light keys per heavy one (0 = 16) */
    uint32_t replay_warmup;    /* 1 (default): after admission the sketch is cleared and the
                                  warm-up window inserted again through the router, so the
                                  admitted keys' warm-up occurrences count in the table and never
                                  link buckets; 2 = keep the warm-up counts in the sketch */
} qs_learned_params;

typedef struct qs_learned qs_learned;

typedef struct qs_learned_info {
    uint64_t budget_bytes, sketch_bytes, table_bytes, mlp_bytes;
    uint64_t n_low, n_high, table_slots, table_fill;
    uint64_t warmup_keys, warmup_seen, train_examples, train_positives, admitted_after_warmup;
    uint32_t threshold, trained, epochs, steps;
    float pos_weight, loss_first, loss_last, train_precision, train_recall, logit_threshold;
    double train_ms;
    uint64_t warmup_replayed;  /* 1 when the warm-up window went through the router again */
    double train_phase_ms[5];  /* distinct warm-up keys; labels and training set; Adam epochs;
                                  classification and admission; replay of the warm-up window */
} qs_learned_info;

#define QS_MLP_PARAMS 20865u /* W1[128x32] | W2[128x128] | b1[128] | b2[128] | w3[128] | b3 */

void qs_learned_params_default(qs_learned_params *p);
/* Diagnostic admission: admit h_keys (host, in the order given, up to the table's max fill)
 * into the exact table and end the warm-up without training, so every later key is routed
 * (table keys count there; no other key is admitted later).
 * With the workload's true heaviest keys this bounds what any classifier could gain with this
 * table; call before the first insert. */
qs_status qs_learned_admit_keys(qs_learned *lk, const uint32_t *h_keys, size_t n);
qs_status qs_learned_create(const qs_learned_params *p, qs_learned **out);
qs_status qs_learned_destroy(qs_learned *lk);
qs_status qs_learned_insert(qs_learned *lk, const uint32_t *d_keys, size_t n, void *stream);
qs_status qs_learned_query(qs_learned *lk, const uint32_t *d_keys, size_t n, uint32_t *d_counts, void *stream);
qs_status qs_learned_get_info(qs_learned *lk, qs_learned_info *out);
/* Debug access (tests, tooling): the exact table's slots (key 0xffffffff = free) and counts,
 * table_slots entries each, and the sketch's hash multiplier (may be null). */
qs_status qs_learned_get_table(qs_learned *lk, uint32_t *h_keys, uint32_t *h_counts, uint32_t *h_seed);
/* The classifier alone (tests and tooling): fp32 parameters in the layout above. */
qs_status qs_mlp_get_params(qs_learned *lk, float *h_params);
qs_status qs_mlp_set_params(qs_learned *lk, const float *h_params);
qs_status qs_mlp_forward(qs_learned *lk, const uint32_t *d_keys, size_t n, float *d_logits, void *stream);
/* Gradient of the weighted BCE (mean over n) at the current parameters; loss = mean loss. */
qs_status qs_mlp_grads(qs_learned *lk, const uint32_t *d_keys, const uint8_t *d_labels, size_t n, float pos_weight,
                       float *h_grads, double *loss);
/* Adam training over (keys, labels) in the given order, batches of `batch`. */
qs_status qs_mlp_train(qs_learned *lk, const uint32_t *d_keys, const uint8_t *d_labels, size_t n, uint32_t epochs,
                       uint32_t batch, float lr, float pos_weight, double *last_loss);

/* ---- autotuner (no counterpart in the reference) -----------------------------------------
 * Times pass-1 knob settings (lanes per key 1-32, keys per CTA tile, aggregation, routing,
 * CTAs per SM, chunk size max_batch, the chunk ramp after a clear; every setting gives
 * identical results) on a scratch sketch built from `base` over the caller's sample keys
 * (device memory, inserted `reps` times after a clear), by a coordinate search from the
 * defaults: lanes per key, then keys per tile, aggregation, routing, CTAs per SM, chunk size,
 * ramp.  A caller that inserts in calls of a fixed size passes it as base->max_batch: the
 * chunk size is then not searched, and the sample is inserted in chunks of that size.  The
 * fastest setting is returned in *best, recorded in a process-wide
 * table for the size class floor(log2(n_low)) of `base`, and used by later qs_create calls
 * of that class whose knobs are all 0.  h_all (may be null) receives up to max_all of the
 * timed settings, *n_all how many were timed. */
typedef struct qs_tune_config {
    uint32_t lanes_per_key, aggregate, route, ctas_per_sm;
    uint64_t max_batch;
    uint64_t first_chunk; /* chunk-size ramp after a clear; 0 = no ramp */
    uint32_t keys_per_tile, pad;
    double insert_ms; /* mean time of one insert of the sample (pass 1 + ordered replay) */
} qs_tune_config;

qs_status qs_autotune(const qs_params *base, const uint32_t *d_keys, size_t n, uint32_t reps, qs_tune_config *best,
                      qs_tune_config *h_all, uint32_t max_all, uint32_t *n_all);
/* The recorded setting for n_low's size class; QS_ERR_INVALID_ARG when there is none. */
qs_status qs_autotune_lookup(uint64_t n_low, qs_tune_config *out);
void qs_autotune_reset(void);

/* ---- batched uneven streams (no counterpart in the reference) ---------------------------
 * One handle owns n_streams independent MSWS sketches (stream s: n_low[s] low buckets,
 * n_high[s] high buckets, hash multiplier seed[s]; one mask table for all) laid out in one
 * table arena.  A call takes the keys of every stream at once as one flat device array and
 * device offsets: stream s is d_keys[d_offsets[s] .. d_offsets[s+1]), offsets non-decreasing
 * from d_offsets[0] = 0 (else QS_ERR_INVALID_ARG at the next sync), empty streams allowed.
 * One persistent launch inserts all streams (tiles of one stream each, taken from a device
 * work queue), followed by the ordered replay; each stream's result is that of inserting its
 * keys alone, in order, into a qs_create'd sketch with the same n_low, n_high, seed and
 * masks.  Long batches run in windows of max_batch keys.  The _graph variants record the
 * whole launch sequence once per (d_keys, d_offsets, d_counts, max_total) in a CUDA graph and
 * replay it; sizes are read on the device, so refill the same buffers and call again.
 * Insert graphs take at most max_total <= max_batch keys (more latches QS_ERR_CAPACITY and
 * the rest is not inserted). */
typedef struct qs_batch_params {
    uint32_t n_streams;           /* 1 .. 2^20 */
    const uint64_t *n_low;        /* host [n_streams], each >= 1; sum < 2^32 */
    const uint64_t *n_high;       /* host [n_streams], each >= 2; sum <= 2^30 */
    const uint32_t *hash_seeds;   /* host [n_streams] or NULL: stream s takes draw s of seed_rng */
    uint32_t seed_rng, mask_rng;
    uint32_t hash_mask_table_sz;  /* default 1021 */
    uint32_t hash_mask_ones;      /* default 3 */
    const uint8_t *mask_table;    /* optional, hash_mask_table_sz*4 bytes */
    uint32_t flags;               /* QS_FLAG_COMPAT_V3 */
    uint32_t aggregate, route;    /* as qs_params */
    uint32_t lanes_per_key, ctas_per_sm; /* as qs_params */
    uint64_t max_batch;           /* keys per window (replay scratch), default 2^22 */
    uint64_t first_chunk;         /* per-stream chunk ramp of qs_batch_insert: rounds over every
                                     stream's keys [0, f), [f, 2f), [2f, 4f), ... (windows of at
                                     most max_batch keys); 0 = 2^14; QS_FLAG_NO_CHUNK_RAMP in
                                     flags: flat windows of max_batch keys */
    int32_t device;
    const uint32_t *class_lanes_per_key; /* optional host [64]: lanes per key of pass 1 for the
                                     streams of size class c = floor(log2 n_low); 0 entries take
                                     lanes_per_key (or its default).  Streams are grouped by size
                                     class and each run of classes with one setting is one pass-1
                                     launch.  qs_batch_autotune sets it from measurements. */
} qs_batch_params;

typedef struct qs_batch qs_batch;

typedef struct qs_batch_info {
    uint64_t n_streams, low_buckets, high_buckets, table_bytes, max_batch;
    uint64_t inserts, queries, graph_launches, launches;
    uint32_t graph_capture;       /* 1: CUDA-graph capture works here; 0: _graph calls run eagerly */
    uint32_t streams_pool_full;   /* streams whose high pool ran out */
} qs_batch_info;

void qs_batch_params_default(qs_batch_params *p);
qs_status qs_batch_create(const qs_batch_params *p, qs_batch **out);
qs_status qs_batch_destroy(qs_batch *b);
/* total = d_offsets[n_streams] as the host knows it (windows are planned from it). */
qs_status qs_batch_insert(qs_batch *b, const uint32_t *d_keys, const uint64_t *d_offsets, uint64_t total,
                          void *stream);
qs_status qs_batch_query(qs_batch *b, const uint32_t *d_keys, const uint64_t *d_offsets, uint64_t total,
                         uint32_t *d_counts, void *stream);
qs_status qs_batch_insert_graph(qs_batch *b, const uint32_t *d_keys, const uint64_t *d_offsets, uint64_t max_total,
                                void *stream);
qs_status qs_batch_query_graph(qs_batch *b, const uint32_t *d_keys, const uint64_t *d_offsets, uint64_t max_total,
                               uint32_t *d_counts, void *stream);
qs_status qs_batch_clear(qs_batch *b, void *stream);
/* The batch autotuner: times pass 1 of each size class's streams with every lanes-per-key
 * setting (1, 2, 4, 8, 16, 32; at most 8 with fused routing) over `reps` inserts of the first
 * window (at most max_batch keys) of the given batch into a cleared sketch and picks each
 * class's fastest; then, because per-class settings split pass 1 into one launch per run of
 * classes, it times the whole qs_batch_insert of the batch with each width for every class and
 * with the per-class picks, and keeps the fastest of those.  No setting changes a result.
 * h_class_lpk (may be null) receives the 64 per-class settings in effect (0 where no stream
 * has that class).  Leaves the sketches cleared. */
qs_status qs_batch_autotune(qs_batch *b, const uint32_t *d_keys, const uint64_t *d_offsets, uint64_t total,
                            uint32_t reps, uint32_t *h_class_lpk);
/* Waits for `stream`; returns the first latched error (any stream's pool running out is
 * QS_ERR_POOL_FULL; qs_batch_stream_status tells which). */
qs_status qs_batch_sync(qs_batch *b, void *stream);
qs_status qs_batch_stream_status(qs_batch *b, uint32_t *h_status /* [n_streams]: bit 0 pool full */);
qs_status qs_batch_seeds(qs_batch *b, uint32_t *h_seeds /* [n_streams] */);
qs_status qs_batch_get_info(qs_batch *b, qs_batch_info *out);
/* The arena sketch behind the batch, for qs_set_profiling / qs_get_profile / qs_get_stats
 * (eager calls are timed per launch: insert = pass 1, repair, query); owned by the batch. */
qs_sketch *qs_batch_arena(qs_batch *b);

/* ---- bucket-sharded sketch across GPUs: routing (no counterpart in the reference) --------
 * A key's whole MSWS state is one low bucket and the high bucket it may link to
 * (device_sketch_v3.h:228, :119, :185), so a sketch shards by bucket: bucket b = hv % n_low
 * (hv = key * hash_seed) belongs to shard floor(b * n_shards / n_low), n_shards contiguous
 * ranges.  qs_shard_partition reorders a device batch by owner shard, stably (each
 * shard's keys keep their array order), writes each shard's key count to d_shard_counts
 * (device, n_shards u32) and, if d_perm is not null, each output key's index in the batch;
 * d_scratch holds qs_shard_scratch_words(n, n_shards) u32.  The parts go to their owners with
 * one all-to-all (qsketch_b200/sharded.py); estimates come back the same way and
 * qs_shard_unpartition puts them at their array positions (d_out[d_perm[i]] = d_in[i]).
 * n_shards <= 32. */
size_t qs_shard_scratch_words(size_t n, uint32_t n_shards);
qs_status qs_shard_partition(const uint32_t *d_keys, size_t n, uint32_t hash_seed, uint64_t n_low,
                             uint32_t n_shards, uint32_t *d_out, uint32_t *d_perm, uint32_t *d_scratch,
                             uint32_t *d_shard_counts, void *stream);
qs_status qs_shard_unpartition(const uint32_t *d_in, const uint32_t *d_perm, size_t n, uint32_t *d_out,
                               void *stream);

/* ---- MSWS insert for callers that cannot allocate device memory ------------------------
 * No counterpart in the reference: its classes allocate their own tables
 * (device_sketch.h:83-114) and the harness allocates key buffers per batch.
 *
 * For code that runs inside an engine owning all device memory (a fixed arena set up at
 * start-up, say) and may not call cudaMalloc/cudaFree while serving — those calls
 * synchronise the device and fragment the arena.  The caller keeps the sketch in its own
 * memory and passes it in: the low table (n_low*8 u32, 32-byte aligned), the high pool
 * (n_high*32 u32), a state block of QS_MSWS_STATE_BYTES (16-byte aligned), and the device mask words
 * (n_masks u32, bits 0..27, e.g. from qs_generate_hashmask).  A new sketch is all three
 * zero-filled.  The call allocates nothing: the ordered replay's scratch is a fixed
 * QS_NOALLOC_SCRATCH_BYTES array inside the library, which every GPU that loads the library
 * holds until the process exits.  Results equal qs_insert's on a sketch with the same
 * seed, masks and tables; query those tables by your own means or copy them into a
 * qs_create'd sketch.
 *
 * Limits: n <= QS_NOALLOC_MAX_KEYS per call and n_low <= QS_NOALLOC_MAX_BUCKETS, else
 * QS_ERR_CAPACITY before anything runs.  The first call on each device looks up the scratch
 * array's device address (with that device current) and configures the kernels; make that
 * first call before any stream capture.  Every call shares the one scratch array and leaves
 * its contents behind (the call clears what must start at zero), so calls that overlap on
 * the GPU — different streams or host threads without ordering between them — race and
 * corrupt each other: order them.  Device status (pool full, timeouts) is latched in the
 * state block's status word (second u32). */
#define QS_NOALLOC_MAX_KEYS (1u << 18)
#define QS_NOALLOC_MAX_BUCKETS (1ull << 26)
#define QS_NOALLOC_SCRATCH_BYTES (16u << 20)
#define QS_MSWS_STATE_BYTES 256u
#define QS_MSWS_STATE_ALIGN 16u /* d_state alignment (it holds 64-bit counters); else
                                   QS_ERR_INVALID_ARG */
qs_status qs_msws_insert_noalloc(uint32_t *d_low, uint64_t n_low, uint32_t *d_high, uint64_t n_high,
                                 void *d_state, const uint32_t *d_masks, uint32_t n_masks,
                                 uint32_t hash_seed, uint32_t flags, const uint32_t *d_keys, size_t n,
                                 void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QSKETCH_C_H */
