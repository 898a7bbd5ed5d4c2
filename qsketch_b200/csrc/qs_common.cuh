// qs_common.cuh — constants, device layout and helpers shared by the sm_100a kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qsb {

// Reference constants (lib/default.cu:39-54, device_sketch_v3.h:160).
constexpr uint32_t START = 1024;       // NEXT_LEVEL_ID_START: ids <= START are reserved
constexpr uint32_t FIRST_ID = START + 1;  // Device_Hash_Table::resize sets 1025 (device_sketch.h:109)
constexpr uint32_t LIMIT = 128;        // a selected 8-bit counter > LIMIT triggers the high level
constexpr uint32_t CROSS = LIMIT + 2;  // a byte reaching 130 under all-adds means order matters
constexpr uint32_t SATURATED = 2;      // word-7 value of a bucket whose link failed (pool full)
constexpr uint32_t FLAG = 0x80000000u; // word-7 bit: bucket crossed during the current chunk
constexpr int LOW_WORDS = 8;           // 32 B low bucket: 7 words of packed counters + index
constexpr int LOW_COUNTERS = 28;       // generate_hashmask(..., 32, 3, 4): bits 0..27
constexpr int HIGH_WORDS = 32;         // 128 B high bucket of u32 counters

// Status bits latched in Ctl::status.
constexpr uint32_t ST_POOL_FULL = 1u;
constexpr uint32_t ST_TIMEOUT = 2u;
constexpr uint32_t ST_CAPACITY = 4u;
constexpr uint32_t ST_BAD_OFFSETS = 8u;  // batched streams: offsets not non-decreasing from 0

// Lemire-Kaser-Kurz direct remainder ("Faster Remainder by Direct Computation", 2019):
// for d < 2^32 and M = ceil(2^64 / d), a % d == mulhi64(M * a mod 2^64, d) for all
// 32-bit a.  Replaces the two run-time `%` of device_sketch_v3.h:42-44 per key.
struct FastMod {
    uint64_t M;
    uint32_t d;
    uint32_t pad;
};

inline FastMod make_fastmod(uint32_t d) {
    FastMod f;
    f.M = (d == 0) ? 0 : (~0ull / d + 1ull);  // d == 1 wraps to 0: a % 1 == 0 below too
    f.d = d;
    f.pad = 0;
    return f;
}

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// a % d as Lemire's direct remainder: low = M * a mod 2^64, a % d = (low * d) >> 64.  With d
// below 2^32 the 128-bit product's high word is (hi * d + mulhi(lo, d)) >> 32 for the 32-bit
// halves hi, lo of low (the fractional part lo * d mod 2^32 cannot carry into it): two
// 32-bit wide multiplies and one high multiply instead of a 64 x 64 product.
__device__ __forceinline__ uint32_t fast_mod(const FastMod& f, uint32_t a) {
    const uint64_t low = f.M * (uint64_t)a;
    const uint32_t lo = (uint32_t)low, hi = (uint32_t)(low >> 32);
    return (uint32_t)(((uint64_t)hi * f.d + __umulhi(lo, f.d)) >> 32);
}

// Per-sketch device control block.
struct Ctl {
    uint32_t next_id;      // bump allocator (atomic_malloc, device_sketch_v3.h:69-85)
    uint32_t status;       // latched ST_* bits
    uint32_t n_flagged;    // buckets flagged in the current chunk
    uint32_t n_records;    // records gathered for the ordered replay
    uint32_t n_long;       // slots whose segment needed a grid-wide count
    uint32_t bar_count;    // blocks that finished the current repair (its last block resets)
    uint32_t link_gen;     // repairs that linked buckets since the create/clear (never reset
                           // otherwise): tags the per-stream link ranks of batched streams
    unsigned long long bar_arrive;  // grid barrier arrivals (a barrier ends at the next multiple
                                    // of the grid size)
    unsigned long long dropped;
    unsigned long long repaired_buckets;
    unsigned long long repaired_keys;
    unsigned long long inserted;
    unsigned long long repairs;        // repair invocations that had flagged buckets
    unsigned long long phase_t;        // globaltimer at the last phase mark
    unsigned long long phase_ns[12];   // accumulated time per repair phase
};

// Everything a MSWS kernel needs, passed by value.
struct MswsDev {
    uint32_t* low;           // n_low * 8 words
    uint32_t* high;          // n_high * 32 words
    const uint32_t* masks;   // n_masks mask words (bit i selects counter i)
    Ctl* ctl;
    uint64_t n_low;
    uint64_t n_high;
    FastMod fm_low;
    FastMod fm_mask;
    uint32_t seed;
    uint32_t n_masks;
    uint32_t compat_v3;
    uint32_t flag_cap;       // capacity of flag_list / per-slot arrays
    // ordered-replay scratch
    uint32_t* flag_list;     // slot -> bucket
    uint32_t* tile_counts;   // per key tile of the chunk
    uint2* rec[2];           // (slot, mask) records, ping-pong for the radix passes
    uint32_t* hist;          // 256 * max record tiles
    uint32_t* seg_beg;       // per slot: first record of its segment
    uint32_t* totals;        // long_cap slots * 28 counts
    uint32_t long_cap;       // slots whose per-counter totals are computed grid-wide
    uint32_t route;          // 0 adaptive, 1 preload, 2 fused (pass-1 routing)
    const uint32_t* skip;    // optional: bit i set = key i of the chunk is not for this sketch
    uint32_t max_tiles;      // tiles of REPAIR_TILE elements in a chunk
    // learned split, pass 1 only: keys found in this exact table count there instead of in
    // the sketch, and pass 1 sets their bits in skip_out (null tbl_keys: no table)
    const uint32_t* tbl_keys;
    uint32_t* tbl_counts;
    uint32_t* skip_out;
    uint32_t tbl_slots;
    uint32_t ins_tile;       // pass-1 keys per tile (0: the stage size)
    uint32_t prof;           // repair phase timers on (qs_set_profiling); off they cost nothing
    // Link order.  One-key-at-a-time insertion hands out high ids in the array order of the
    // keys that switch buckets to the high level; the ordered replay does the same:
    uint32_t* rpos[2];       // per record: its position in array order, carried through the
                             // radix passes beside rec[]
    uint2* sw;               // per slot: the switch key's position (then its rank) or NONE, and
                             // the bucket's keys at or after the switch
    uint32_t* sw_base;       // per slot, batched streams: the stream's allocator before the repair
    uint32_t* sw_bits;       // one bit per record position: a bucket switches there
    uint32_t* sw_cnt;        // switches per SW_BLOCK positions
};
constexpr uint32_t SW_BLOCK = 4096;  // positions per switch count (128 bit words)

// Batched streams: many per-stream MSWS sketches share one low-table arena and one high
// pool arena.  A stream's sketch is the bucket range [low_base, low_base + fm_low.d) of the
// low arena and the id range (high_base + START, high_base + START + n_high) of the pool, so
// a bucket or a high id is one global number and pass 1, the flag machinery and the
// ordered replay work unchanged; only hashing and allocation read the stream's descriptor.
struct StreamDesc {
    FastMod fm_low;      // d = the stream's low bucket count
    uint32_t seed;       // the stream's hash multiplier
    uint32_t low_base;   // first bucket of the stream's sketch in the low arena
    uint32_t high_base;  // global high id = high_base + the stream's own id (from FIRST_ID)
    uint32_t n_high;     // the stream's pool size in buckets (own ids < START + n_high)
};

struct BatchDev {
    const StreamDesc* desc;   // [n_streams]
    const uint64_t* key_off;  // [n_streams + 1] caller's offsets: stream s = keys[off[s], off[s+1])
    uint64_t* lo;             // [n_streams] first flat key of each stream's slice in the window
    uint64_t* hi;             // [n_streams] end of that slice
    uint32_t* item_off;       // [n_streams + 1] prefix of work items (key tiles) per stream
    uint32_t* wpre;           // [n_streams + 1] prefix of the slices' key counts: window key i of
                              // stream s is flat key lo[s] + i - wpre[s]
    uint64_t* win;            // [2] 0 and the window's key count
    uint32_t* work;           // work-queue heads, one per size-class launch of pass 1
    const uint32_t* cls_streams; // [n_streams] the streams grouped by size class (pass-1 launches)
    uint32_t* cls_item_off;   // [n_streams + 1] prefix of work items in the grouped order
    uint32_t* next_id;        // [n_streams] per-stream bump allocators (from FIRST_ID)
    uint32_t* status;         // [n_streams] latched ST_* bits per stream
    unsigned long long* first;// [n_streams] (repair generation << 32) | ~(lowest rank of the
                              // stream's links in that repair): ranks within each stream
    uint32_t n_streams;       // 0: not a batch
    uint32_t pad;
};

// Which keys one batched launch sequence covers: flat mode, the keys [c0, c1) of the caller's
// flat array; else, for the streams [s_lo, s_hi), each stream's keys [rel_lo, rel_hi) counted
// from the stream's start (the per-stream chunk ramp).
struct BatchWindow {
    uint64_t c0, c1;
    uint64_t rel_lo, rel_hi;
    uint32_t s_lo, s_hi;
    uint32_t flat;
    uint32_t pad;
};

// Plain count-min (rows x n counters, one seed per row) or, when `masks` is set, a one-level
// bucket sketch: n buckets of `rows` u32 counters, a key's mask (of rows bits) selecting its
// counters in its bucket hv % n (the reference's warp and sub-warp sketches, v1/v2).
struct CmDev {
    uint32_t* table;  // rows * n
    uint64_t n;
    FastMod fm;
    uint32_t rows;
    uint32_t n_masks;       // bucket sketch: mask count H
    uint32_t seeds[16];
    const uint32_t* masks;  // bucket sketch: H mask words (bit i selects counter i), else null
    FastMod fm_mask;
};

constexpr int REPAIR_TILE = 4096;   // elements per tile in the ordered-replay passes
constexpr int REPAIR_THREADS = 512; // 16 warps x 256 elements
constexpr int MAX_CM_ROWS = 16;
constexpr uint32_t MAX_SIZE_CLASSES = 64;  // floor(log2 n_low) of a batched stream's sketch

// Spread a 4-bit nibble to the low bit of each byte: b0->bit0, b1->bit8, b2->bit16, b3->bit24.
__device__ __forceinline__ uint32_t expand_nibble(uint32_t nib) {
    return (nib * 0x00204081u) & 0x01010101u;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
    return r;
}

}  // namespace qsb
