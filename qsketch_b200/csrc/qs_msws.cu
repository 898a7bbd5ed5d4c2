// qs_msws.cu — MSWS ("Level" QSketch) insert and query kernels for sm_100a.
//
// Reference path: include/sketch/device_sketch/device_sketch_v3.h
//   insert_kernel :194-290, calculation_s2_insert :88-191, insert_high :54-65,
//   atomic_malloc :69-85, search_kernel :411-521, calculation_s2_search :311-408.
//
// Exactness.  The reference applies keys concurrently, so once a bucket's 8-bit counter
// passes 128 its result depends on the schedule.  Here a chunk of keys is applied in two
// steps whose result equals the one-key-at-a-time order of the array:
//   1. k_msws_insert: every key of an unlinked bucket adds its packed 8-bit increments
//      with returning 32-bit atomics (a group of 1-32 lanes per key; 8 lanes, lane w on
//      word w, is the reference's sub-warp).  A bucket's result is independent of order iff no selected
//      counter ends the chunk above 129; a key whose atomic saw old + add >= 130 proves
//      the opposite and flags the bucket (word 7 := FLAG | slot).  Keys of linked buckets
//      add to the high bucket (commutative).
//   2. k_msws_repair (only if something was flagged): gathers the flagged buckets' keys
//      in array order (stable filter + stable LSD radix by slot), restores each bucket's
//      pre-chunk words (u32 addition is a group: pre = final - sum of the packed adds),
//      finds the first key that sees a selected counter > 128, links the bucket there and
//      moves the increments of that key and all later ones to the new high bucket.
#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {

constexpr int INS_THREADS = 256;
constexpr int INS_WARPS = INS_THREADS / 32;
constexpr int INS_TILE = 2048;  // keys per TMA stage (8 KiB)
constexpr int INS_STAGES = 2;      // one tile in flight while one is inserted (a tile takes ~30 us; two
                                   // stages leave the shared memory of five CTAs per SM)
constexpr int INS_MIN_CTAS = 5;  // resident pass-1 CTAs per SM the register budget is cut for: the
                                 // returning atomics are latency bound, so warps in flight pay (4: 17 % slower
                                 // on Zipf 1.1; 6 forces 40 registers and is slower again)
constexpr int AGG_SLOTS = 1024; // per-CTA table merging the linked keys of a tile
// mbarriers of the stages (+ one spare word), padded so the uint4 staging area that follows
// the 4-byte tables stays 16-byte aligned for any stage count
constexpr int INS_BAR_BYTES = (INS_STAGES * 8 + 8 + 15) & ~15;
constexpr int AGG_PROBES = 32;
constexpr uint32_t AGG_EMPTY = 0xffffffffu;
constexpr uint32_t AGG_TBL = 0x80000000u;  // merge-table id tag: the key's exact-table slot

// Aggregation modes (qs_params.aggregate): 1 none, 2 warp (equal keys of a warp merge),
// 3 warp + block (linked keys of a whole tile merge in shared memory, so a heavy hitter
// costs one atomic per high counter per tile instead of one per occurrence).
enum { AGG_NONE = 0, AGG_WARP = 1, AGG_BLOCK = 2 };
// Routing of a tile's keys between the low and the high level:
// ROUTE_PRELOAD loads each bucket's index word first, then sends linked keys to the high
// level (through the tile table) and the others to the packed low atomics;
// ROUTE_FUSED skips the load: lane 7 of each sub-warp adds 0 to the index word in the same
// atomic instruction that adds the low counters, and the rare key that finds its bucket
// linked takes its low increments back (u32 addition is invertible) and counts high.
// A CTA picks the mode of its next tile from the linked share of the last one.
enum { ROUTE_PRELOAD = 0, ROUTE_FUSED = 1 };

struct InsShared {
    uint32_t* keys;   // [INS_STAGES][INS_TILE]
    uint64_t* bar;    // [INS_STAGES]
    uint32_t* akey;   // [AGG_SLOTS]
    uint32_t* acnt;   // [AGG_SLOTS]
    uint32_t* aid;    // [AGG_SLOTS] high id of the key's bucket
    uint4* stage;     // [INS_WARPS][32] per-warp round staging
    uint32_t* masks;  // [n_masks]
    uint32_t* misc;   // [0] keys dropped (saturated buckets), [1] linked keys in this tile,
                      // [2] routing mode of this tile (ROUTE_*)
};

__device__ __forceinline__ InsShared ins_carve(uint8_t* smem, uint32_t n_masks) {
    InsShared S;
    uint8_t* p = smem;
    S.keys = reinterpret_cast<uint32_t*>(p);
    p += INS_STAGES * INS_TILE * 4;
    S.bar = reinterpret_cast<uint64_t*>(p);
    p += INS_BAR_BYTES;
    S.akey = reinterpret_cast<uint32_t*>(p);
    p += AGG_SLOTS * 4;
    S.acnt = reinterpret_cast<uint32_t*>(p);
    p += AGG_SLOTS * 4;
    S.aid = reinterpret_cast<uint32_t*>(p);
    p += AGG_SLOTS * 4;
    S.stage = reinterpret_cast<uint4*>(p);
    p += INS_WARPS * 32 * 16;
    S.misc = reinterpret_cast<uint32_t*>(p);
    p += 16;
    S.masks = reinterpret_cast<uint32_t*>(p);
    (void)n_masks;
    return S;
}

// the carve above: TMA stages 16-byte aligned, mbarriers 8-byte, the uint4 staging 16-byte
static_assert((INS_STAGES * INS_TILE * 4) % 16 == 0, "stage bytes");
static_assert((INS_STAGES * INS_TILE * 4 + INS_BAR_BYTES + 3 * AGG_SLOTS * 4) % 16 == 0, "uint4 staging alignment");

size_t msws_insert_smem(uint32_t n_masks) {
    return (size_t)INS_STAGES * INS_TILE * 4 + INS_BAR_BYTES + 3 * AGG_SLOTS * 4 + INS_WARPS * 32 * 16 + 16 +
           (size_t)n_masks * 4;
}

// ---- pass 1 -------------------------------------------------------------------------------

__device__ __forceinline__ void flag_bucket(const MswsDev& D, uint32_t b) {
    uint32_t* w7 = D.low + (uint64_t)b * LOW_WORDS + 7;
    const uint32_t old = atomicOr(w7, FLAG);
    if (old & FLAG) return;
    const uint32_t slot = atomicAdd(&D.ctl->n_flagged, 1u);
    if (slot < D.flag_cap) {
        D.flag_list[slot] = b;
        atomicExch(w7, FLAG | slot);
    } else {  // cannot happen (a chunk flags at most one bucket per key); no slot to name
        atomicExch(w7, 0xffffffffu);
        atomicOr(&D.ctl->status, ST_CAPACITY);
    }
}

__device__ __forceinline__ bool is_linked(const MswsDev& D, uint32_t w7) {
    return w7 > START && (uint64_t)(w7 - START) < D.n_high;
}

__device__ __forceinline__ bool agg_insert(const InsShared& S, uint32_t key, uint32_t c, uint32_t id) {
    if (key == AGG_EMPTY) return false;
    const uint32_t h = (key * 0x9E3779B1u) >> 22;  // 10 bits
    for (int p = 0; p < AGG_PROBES; ++p) {
        const uint32_t s = (h + p) & (AGG_SLOTS - 1);
        // a key already in the table (the common case for a heavy key) needs no CAS: a slot
        // only goes from empty to a key within a tile
        const uint32_t seen = reinterpret_cast<volatile uint32_t*>(S.akey)[s];
        if (seen == key) {
            atomicAdd(S.acnt + s, c);
            return true;
        }
        if (seen != AGG_EMPTY) continue;
        const uint32_t prev = atomicCAS(S.akey + s, AGG_EMPTY, key);
        if (prev == AGG_EMPTY) {
            S.aid[s] = id;
            atomicAdd(S.acnt + s, c);
            return true;
        }
        if (prev == key) {
            atomicAdd(S.acnt + s, c);
            return true;
        }
    }
    return false;
}

// Does a selected byte (nibble bit k selects byte k) of the pre-add word `old` reach CROSS
// once c is added: byte + c >= CROSS, i.e. byte >= CROSS - c, four bytes at a time.
// Selected bytes all below 64 with c below 64 cannot reach CROSS: a two-operation test
// settles the common case before the four-byte comparison.
__device__ __forceinline__ bool crosses(uint32_t old, uint32_t nib, uint32_t c) {
    if (!nib) return false;
    if (c >= CROSS) return true;
    const uint32_t sel = expand_nibble(nib) * 0xffu;
    if (c < 64u && !(old & sel & 0xC0C0C0C0u)) return false;
    return (__vcmpgeu4(old, (CROSS - c) * 0x01010101u) & sel) != 0u;
}

// One lane, one key (or merged count c of one key) of an unlinked bucket: the selected 8-bit
// counters get c with one returning atomic per word they touch (a mask touches at most
// four words in the unrolled part; more go through the loop), all atomics in flight before
// any result is used.  Returns whether the bucket crosses (flag it).
__device__ __forceinline__ bool low_add(const MswsDev& D, uint32_t b, uint32_t m, uint32_t c) {
    uint32_t* bw = D.low + (uint64_t)b * LOW_WORDS;
    uint32_t mm = m;  // bits 0..27 (checked at creation): words 0..6, never the index word
    uint32_t wv[4], nv[4], old[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t f = __ffs(mm);
        const uint32_t w = f ? (f - 1u) >> 2 : 0u;
        nv[i] = f ? (mm >> (4u * w)) & 0xfu : 0u;
        wv[i] = w;
        mm &= ~(nv[i] << (4u * w));
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) old[i] = nv[i] ? atomicAdd(bw + wv[i], expand_nibble(nv[i]) * c) : 0u;
    bool cross = false;
#pragma unroll
    for (int i = 0; i < 4; ++i) cross |= crosses(old[i], nv[i], c);
    while (mm) {
        const uint32_t w = (uint32_t)(__ffs(mm) - 1) >> 2, nib = (mm >> (4u * w)) & 0xfu;
        mm &= ~(nib << (4u * w));
        cross |= crosses(atomicAdd(bw + w, expand_nibble(nib) * c), nib, c);
    }
    return cross;
}

// One lane: c to the selected high counters of linked bucket `id` (insert_high,
// device_sketch_v3.h:54-65).
__device__ __forceinline__ void high_add(const MswsDev& D, uint32_t id, uint32_t m, uint32_t c) {
    uint32_t* hb = D.high + (uint64_t)(id - START) * HIGH_WORDS;
    uint32_t mm = m;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (mm) {
            atomicAdd(hb + (__ffs(mm) - 1), c);
            mm &= mm - 1;
        }
    }
    for (; mm; mm &= mm - 1) atomicAdd(hb + (__ffs(mm) - 1), c);
}

// Sub-warp rounds over the staged entries of this warp: entry j = (target, mask, count,
// kind).  LPK lanes serve one entry (32/LPK entries per round, LPK rounds for 32 entries);
// lane w of a group owns bucket words w, w+LPK, ... (LPK = 8: one word per lane, the
// reference's sub-warp mapping, device_sketch_v3.h:131-170; LPK = 4, 2, 1: two, four or
// all eight words per lane; LPK = 16, 32: lanes past the eighth idle).  kind 0: low bucket `target`, each owned word
// gets its nibble of 8-bit counters with one returning atomic; kind 1: linked, the owning
// lanes add to the selected high counters of id `target` (insert_high, :54-65, :111-129).
template <int LPK>
__device__ __forceinline__ void staged_rounds(const MswsDev& D, const uint4* st, int nact) {
    static_assert(LPK == 1 || LPK == 2 || LPK == 4 || LPK == 8 || LPK == 16 || LPK == 32, "lanes per key");
    constexpr int KPR = 32 / LPK;                // entries per round
    constexpr int WPL = LPK >= 8 ? 1 : 8 / LPK;  // bucket words per lane
    const int lane = threadIdx.x & 31, sub = lane / LPK, w = lane % LPK;
    uint32_t olds[LPK][WPL];
#pragma unroll
    for (int r = 0; r < LPK; ++r) {
#pragma unroll
        for (int h = 0; h < WPL; ++h) olds[r][h] = 0;
        if (r * KPR >= nact) continue;  // warp-uniform
        const int j = r * KPR + sub;
        if (j >= nact) continue;
        const uint4 e = st[j];
        if (e.w == 0) {
#pragma unroll
            for (int h = 0; h < WPL; ++h) {
                const int ww = w + h * LPK;
                const uint32_t nib = (ww < 7) ? (e.y >> (4 * ww)) & 0xfu : 0u;
                if (nib) olds[r][h] = atomicAdd(D.low + (uint64_t)e.x * LOW_WORDS + ww, expand_nibble(nib) * e.z);
            }
        } else {
            // lane w of the group adds to the selected counters number w, w + LPK, ...
            uint32_t* hb = D.high + (uint64_t)(e.x - START) * HIGH_WORDS;
            uint32_t mm = e.y;
            for (int k = 0; k < w && mm; ++k) mm &= mm - 1;
            while (mm) {
                atomicAdd(hb + (__ffs(mm) - 1), e.z);
                for (int k = 0; k < LPK && mm; ++k) mm &= mm - 1;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < LPK; ++r) {
        if (r * KPR >= nact) continue;  // warp-uniform
        const int j = r * KPR + sub;
        bool cross = false;
        uint4 e = make_uint4(0, 0, 0, 1);
        if (j < nact) e = st[j];
        if (e.w == 0) {
#pragma unroll
            for (int h = 0; h < WPL; ++h) {
                const int ww = w + h * LPK;
                const uint32_t nib = (ww < 7) ? (e.y >> (4 * ww)) & 0xfu : 0u;
                cross |= crosses(olds[r][h], nib, e.z);
            }
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, cross);
        const uint32_t grp = LPK == 32 ? bal : (bal >> (sub * LPK)) & ((1u << (LPK & 31)) - 1u);
        if (w == 0 && grp) flag_bucket(D, e.x);
    }
}

// ROUTE_FUSED rounds (1, 2, 4 or 8 lanes per key): entry j = (bucket, mask, count, key).
// The lane that owns word 7 adds 0 to it in the same instruction that adds the counters, so
// the bucket's index word comes back with the old counter words; a key whose bucket turns
// out linked or saturated takes its low increments back (u32 addition is invertible).
// Returns the linked count.
template <int LPK>
__device__ __forceinline__ uint32_t staged_rounds_fused(const MswsDev& D, const InsShared& S, const uint4* st,
                                                        int nact) {
    static_assert(LPK == 1 || LPK == 2 || LPK == 4 || LPK == 8, "fused rounds: at most 8 lanes per key");
    constexpr int KPR = 32 / LPK, WPL = 8 / LPK;
    constexpr int W7_LANE = 7 % LPK, W7_H = 7 / LPK;  // the owner of word 7 and its slot
    const int lane = threadIdx.x & 31, sub = lane / LPK, w = lane % LPK;
    uint32_t olds[LPK][WPL];
#pragma unroll
    for (int r = 0; r < LPK; ++r) {
#pragma unroll
        for (int h = 0; h < WPL; ++h) olds[r][h] = 0;
        if (r * KPR >= nact) continue;  // warp-uniform
        const int j = r * KPR + sub;
        if (j >= nact) continue;
        const uint4 e = st[j];
#pragma unroll
        for (int h = 0; h < WPL; ++h) {
            const int ww = w + h * LPK;
            const uint32_t nib = (ww < 7) ? (e.y >> (4 * ww)) & 0xfu : 0u;
            if (nib || ww == 7)
                olds[r][h] = atomicAdd(D.low + (uint64_t)e.x * LOW_WORDS + ww, ww == 7 ? 0u : expand_nibble(nib) * e.z);
        }
    }
    uint32_t linked_keys = 0;
#pragma unroll
    for (int r = 0; r < LPK; ++r) {
        if (r * KPR >= nact) continue;  // warp-uniform
        const int j = r * KPR + sub;
        const bool ve = j < nact;
        uint4 e = make_uint4(0, 0, 0, 0);
        if (ve) e = st[j];
        const uint32_t ptr = __shfl_sync(0xffffffffu, olds[r][W7_H], sub * LPK + W7_LANE);
        const bool linked = ve && is_linked(D, ptr);
        const bool sat = ve && ptr == SATURATED;
        bool cross = false;
#pragma unroll
        for (int h = 0; h < WPL; ++h) {
            const int ww = w + h * LPK;
            const uint32_t nib = (ww < 7) ? (e.y >> (4 * ww)) & 0xfu : 0u;
            if ((linked || sat) && nib) atomicAdd(D.low + (uint64_t)e.x * LOW_WORDS + ww, 0u - expand_nibble(nib) * e.z);
            if (ve && !linked && !sat) cross |= crosses(olds[r][h], nib, e.z);
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, cross);
        const uint32_t grp = (bal >> (sub * LPK)) & ((1u << LPK) - 1u);
        if (w == 0) {
            if (grp) flag_bucket(D, e.x);
            if (sat) atomicAdd(S.misc + 0, e.z);
            if (linked) {  // rare in this mode: count high directly
                uint32_t* hb = D.high + (uint64_t)(ptr - START) * HIGH_WORDS;
                for (uint32_t mm = e.y; mm; mm &= mm - 1) atomicAdd(hb + (__ffs(mm) - 1), e.z);
                linked_keys += e.z;
            }
        }
    }
    return linked_keys;
}

// Up to 32 keys held one per lane (valid lanes: lane < cnt), all of one sketch: hash
// multiplier `seed`, `fm_low.d` buckets starting at bucket `base` of the table.
template <int AGG, int LPK>
__device__ __forceinline__ void insert_group(const MswsDev& D, const InsShared& S, uint32_t key, int cnt,
                                             bool use_table, int route, uint64_t idx, uint32_t seed,
                                             const FastMod& fm_low, uint32_t base) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    bool valid = lane < cnt && !(D.skip && ((__ldg(D.skip + (idx >> 5)) >> (idx & 31)) & 1u));
    if (D.tbl_keys) {  // learned split: a key in the exact table counts there, not in the sketch
        const int ts = valid ? table_find(D.tbl_keys, D.tbl_slots, key) : -1;
        const uint32_t hb = __ballot_sync(0xffffffffu, ts >= 0);
        if (hb) {
            // its skip bit (for the replay): two words per warp when the lanes hold
            // consecutive key indices, else one atomic per hit
            const uint64_t i0 = __shfl_sync(0xffffffffu, idx, 0), i31 = __shfl_sync(0xffffffffu, idx, 31);
            if (i31 - i0 == 31) {
                if (lane == 0) {
                    atomicOr(D.skip_out + (i0 >> 5), hb << (i0 & 31));
                    if (i0 & 31) atomicOr(D.skip_out + (i0 >> 5) + 1, hb >> (32 - (i0 & 31)));
                }
            } else if (ts >= 0) {
                atomicOr(D.skip_out + (idx >> 5), 1u << (idx & 31));
            }
            // its count: equal slots of the warp merge, then the tile's through the merge table
            const uint32_t peers = __match_any_sync(0xffffffffu, ts >= 0 ? (uint32_t)ts : 0xffffffffu) & hb;
            if (ts >= 0 && lane == __ffs(peers) - 1) {
                const uint32_t c = __popc(peers);
                if (!(AGG == AGG_BLOCK && use_table && agg_insert(S, key, c, AGG_TBL | (uint32_t)ts)))
                    atomicAdd(D.tbl_counts + ts, c);
            }
            valid = valid && ts < 0;
        }
    }
    const uint32_t hv = key * seed;  // hash_mul_add, device_hash_function.h:6-18
    const uint32_t b = base + fast_mod(fm_low, hv);
    const uint32_t m = S.masks[fast_mod(D.fm_mask, hv)];
    uint32_t c = valid ? 1u : 0u;
    if (AGG != AGG_NONE) {
        const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
        const uint32_t peers = __match_any_sync(0xffffffffu, key) & vmask;
        c = (valid && lane == __ffs(peers) - 1) ? (uint32_t)__popc(peers) : 0u;
    }
    uint4* st = S.stage + wid * 32;
    if (LPK <= 8 && route == ROUTE_FUSED) {  // the fused form exists for up to 8 lanes per key
        const uint32_t am = __ballot_sync(0xffffffffu, c != 0);
        if (c) st[__popc(am & lanemask_lt())] = make_uint4(b, m, c, key);
        __syncwarp();
        const uint32_t lk = __reduce_add_sync(0xffffffffu, staged_rounds_fused<(LPK <= 8 ? LPK : 8)>(D, S, st, __popc(am)));
        if (lane == 0 && lk && D.route == 0) atomicAdd(S.misc + 1, lk);
        __syncwarp();
        return;
    }
    const uint32_t w7 = c ? __ldcg(D.low + (uint64_t)b * LOW_WORDS + 7) : 0u;
    const bool linked = c && is_linked(D, w7);
    const bool sat = c && w7 == SATURATED;
    // the tile's dropped and linked keys: one shared atomic per warp (the linked count only
    // feeds the adaptive routing)
    if (__any_sync(0xffffffffu, sat)) {
        const uint32_t ns = __reduce_add_sync(0xffffffffu, sat ? c : 0u);
        if (lane == 0) atomicAdd(S.misc + 0, ns);
    }
    if (D.route == 0) {
        const uint32_t nl = __reduce_add_sync(0xffffffffu, linked ? c : 0u);
        if (lane == 0 && nl) atomicAdd(S.misc + 1, nl);
    }
    bool direct_high = linked, tabled = false;
    if (AGG == AGG_BLOCK && use_table) {
        if (linked)
            direct_high = !agg_insert(S, key, c, w7);
        else if (c >= 2 && !sat)  // a key repeated within the warp: likely heavy, merge the tile's
            tabled = agg_insert(S, key, c, 0u);
    }
    const bool act = (c && !linked && !sat && !tabled) || direct_high;
    if constexpr (LPK == 1) {  // one lane per key: its own atomics, no staging
        if (direct_high) {
            high_add(D, w7, m, c);
        } else if (act && low_add(D, b, m, c)) {
            flag_bucket(D, b);
        }
        return;
    }
    const uint32_t am = __ballot_sync(0xffffffffu, act);
    if (act) st[__popc(am & lanemask_lt())] = make_uint4(direct_high ? w7 : b, m, c, direct_high ? 1u : 0u);
    __syncwarp();
    staged_rounds<LPK>(D, st, __popc(am));
    __syncwarp();
}

// Merged keys of the tile: per distinct key one add of its count, to the selected high
// counters of a linked bucket (id != 0) or, with crossing detection, to the low bucket (id 0:
// a key repeated within a warp whose bucket is not linked; a count above 255 carries into
// the next byte, but it also crosses, so the bucket is flagged and the replay restores its
// pre-chunk words by subtraction, exact mod 2^32).  The tile's keys are of one sketch:
// multiplier `seed`, `fm_low.d` buckets from bucket `base`.
template <int LPK>
__device__ __forceinline__ void drain_table(const MswsDev& D, const InsShared& S, uint32_t seed,
                                            const FastMod& fm_low, uint32_t base) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint4* st = S.stage + wid * 32;
    for (int s0 = wid * 32; s0 < AGG_SLOTS; s0 += INS_THREADS) {
        const int s = s0 + lane;
        const uint32_t k = S.akey[s];
        bool has = k != AGG_EMPTY;
        uint32_t m = 0, c = 0, id = 0, b = 0;
        if (has) {
            const uint32_t hv = k * seed;
            m = S.masks[fast_mod(D.fm_mask, hv)];
            c = S.acnt[s];
            id = S.aid[s];
            if (id == 0) b = base + fast_mod(fm_low, hv);
            S.akey[s] = AGG_EMPTY;
            S.acnt[s] = 0;
            if (id & AGG_TBL) {  // an exact-table key (learned split): its count goes there
                atomicAdd(D.tbl_counts + (id & ~AGG_TBL), c);
                has = false;
            }
        }
        if constexpr (LPK == 1) {  // one lane per slot
            if (has) {
                if (id) high_add(D, id, m, c);
                else if (low_add(D, b, m, c)) flag_bucket(D, b);
            }
            continue;
        }
        const uint32_t am = __ballot_sync(0xffffffffu, has);
        if (!am) continue;
        if (has) st[__popc(am & lanemask_lt())] = id ? make_uint4(id, m, c, 1u) : make_uint4(b, m, c, 0u);
        __syncwarp();
        staged_rounds<LPK>(D, st, __popc(am));
        __syncwarp();
    }
}

template <int AGG, int LPK>
__global__ void __launch_bounds__(INS_THREADS, INS_MIN_CTAS) k_msws_insert(const uint32_t* __restrict__ keys, uint64_t n,
                                                                MswsDev D) {
    extern __shared__ __align__(128) uint8_t smem[];
    const InsShared S = ins_carve(smem, D.n_masks);
    __shared__ uint32_t s_extra[8];
    __shared__ int s_ok;

    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    griddep_launch_dependents();  // the replay may be scheduled now: it waits for this pass
    // the mask table (written by the host only) is staged while the previous kernel drains
    for (uint32_t i = tid; i < D.n_masks; i += blockDim.x) S.masks[i] = __ldg(D.masks + i);
    for (int i = tid; i < AGG_SLOTS; i += blockDim.x) {
        S.akey[i] = AGG_EMPTY;
        S.acnt[i] = 0;
    }
    griddep_wait();
    if (tid == 0) {
        S.misc[0] = 0;
        S.misc[1] = 0;
        S.misc[2] = D.route == 1 ? ROUTE_PRELOAD
                    : D.route == 2 ? ROUTE_FUSED
                                   : (__ldcg(&D.ctl->next_id) == FIRST_ID ? ROUTE_FUSED : ROUTE_PRELOAD);
    }

    // 16-byte aligned body for the TMA bulk copies; the <= 6 ragged keys go through CTA 0.
    const uintptr_t addr = reinterpret_cast<uintptr_t>(keys);
    const uint64_t head = umin64(n, ((16u - (addr & 15u)) & 15u) >> 2);
    const uint64_t body_n = ((n - head) >> 2) << 2;
    const uint64_t tail = n - head - body_n;
    const uint32_t* body = keys + head;

    if (tid == 0) {
        for (int s = 0; s < INS_STAGES; ++s) mbar_init(&S.bar[s], 1);
        fence_mbar_init();
    }
    if (blockIdx.x == 0 && tid < (int)(head + tail))
        s_extra[tid] = (tid < (int)head) ? keys[tid] : keys[head + body_n + (tid - head)];
    __syncthreads();
    if (blockIdx.x == 0 && wid == 0 && head + tail > 0) {
        const uint32_t k = lane < (int)(head + tail) ? s_extra[lane] : 0u;
        const uint64_t idx = lane < (int)head ? (uint64_t)lane : head + body_n + (lane - head);
        insert_group<AGG, LPK>(D, S, k, (int)(head + tail), false, ROUTE_PRELOAD, idx, D.seed, D.fm_low, 0u);
    }

    // keys per tile (<= INS_TILE, a multiple of 4 so that every TMA copy stays 16-byte sized
    // and aligned): small chunks take smaller tiles to spread over more CTAs
    const uint64_t tile = (D.ins_tile && D.ins_tile <= (uint32_t)INS_TILE) ? (D.ins_tile & ~3u) : (uint64_t)INS_TILE;
    const uint64_t ntiles = (body_n + tile - 1) / tile;
    const uint64_t my_tiles = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    auto issue = [&](uint64_t i) {
        const int st = (int)(i % INS_STAGES);
        const uint64_t g = blockIdx.x + i * gridDim.x;
        const uint64_t start = g * tile;
        const uint32_t cnt = (uint32_t)umin64(tile, body_n - start);
        mbar_arrive_expect_tx(&S.bar[st], cnt * 4u);
        tma_bulk_g2s(S.keys + st * INS_TILE, body + start, cnt * 4u, &S.bar[st]);
    };
    if (tid == 0)
        for (uint64_t i = 0; i < umin64(INS_STAGES, my_tiles); ++i) issue(i);

    for (uint64_t i = 0; i < my_tiles; ++i) {
        const int st = (int)(i % INS_STAGES);
        const uint32_t parity = (uint32_t)((i / INS_STAGES) & 1u);
        if (tid == 0) s_ok = mbar_wait_bounded(&S.bar[st], parity) ? 1 : 0;
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) {
                atomicOr(&D.ctl->status, ST_TIMEOUT);
                // wait (bounded) for the copies still in flight before leaving
                for (uint64_t j = i; j < umin64(i + INS_STAGES, my_tiles); ++j)
                    mbar_wait_bounded(&S.bar[j % INS_STAGES], (uint32_t)((j / INS_STAGES) & 1u));
            }
            return;
        }
        for (uint32_t it = 0; it < 64 && !mbar_try_wait(&S.bar[st], parity); ++it) {
        }
        const uint64_t g = blockIdx.x + i * gridDim.x;
        const int cnt = (int)umin64(tile, body_n - g * tile);
        const uint32_t* tk = S.keys + st * INS_TILE;
        const int route = (int)S.misc[2];
        for (int base = wid * 32; base < cnt; base += INS_THREADS) {
            const int c = min(32, cnt - base);
            const uint32_t k = lane < c ? tk[base + lane] : 0u;
            insert_group<AGG, LPK>(D, S, k, c, true, route, head + g * tile + base + lane, D.seed, D.fm_low, 0u);
        }
        __syncthreads();
        if (tid == 0) {  // adaptive: the next tile is fused while under 1/16 of the keys are linked
            if (D.route == 0) S.misc[2] = S.misc[1] * 16u < (uint32_t)cnt ? ROUTE_FUSED : ROUTE_PRELOAD;
            S.misc[1] = 0;
        }
        if (AGG == AGG_BLOCK) {
            drain_table<LPK>(D, S, D.seed, D.fm_low, 0u);
            __syncthreads();
        }
        if (tid == 0 && i + INS_STAGES < my_tiles) {
            fence_proxy_async_smem();
            issue(i + INS_STAGES);
        }
    }
    __syncthreads();
    if (tid == 0 && S.misc[0]) atomicAdd(&D.ctl->dropped, (unsigned long long)S.misc[0]);
}

// ---- ordered replay ---------------------------------------------------------------------

constexpr int SET_SLOTS = 16384;  // words of the repair's dynamic shared memory (64 KiB), reused by
                                  // the phases: flag filter, tile prefix, a resident radix tile,
                                  // the records of a sort-free replay
constexpr int BLOOM_BITS = 17;    // per-block filter of the flagged buckets: 2^17 bits (16 KiB)
constexpr int BLOOM_WORDS = (1 << BLOOM_BITS) / 32;
constexpr uint32_t TC_MAX = 128;  // tiles per block in the flag test (grids have >= 148 blocks)
constexpr uint32_t SEMI_TILES = 4;  // radix tiles per block kept as offsets and ranks
static_assert(SEMI_TILES * (REPAIR_THREADS / 32) * 256 * 2 + SEMI_TILES * REPAIR_TILE <= SET_SLOTS * 4,
              "the offsets and ranks of SEMI_TILES tiles fit the shared space");
constexpr uint32_t SCAN_CAP = SET_SLOTS / 2;  // records replayed without a sort (64 KiB of uint2)
constexpr uint32_t NONE = 0xffffffffu;

__device__ __forceinline__ int radix_passes(uint32_t F) {
    if (F <= 1) return 0;
    const int bits = 32 - __clz(F - 1);
    return (bits + 7) / 8;
}

// Is bucket b flagged in this chunk?  A per-block filter in shared memory (one bit per hash
// of each flagged bucket) answers "no" for almost every key with one shared load; a filter
// hit reads the bucket's index word, which pass 1 left at FLAG | slot (flag_bucket).
__device__ __forceinline__ uint32_t bloom_bit(uint32_t b) { return (b * 0x9E3779B1u) >> (32 - BLOOM_BITS); }

__device__ __forceinline__ bool bloom_hit(const uint32_t* sbloom, uint32_t b) {
    const uint32_t h = bloom_bit(b);
    return (sbloom[h >> 5] >> (h & 31)) & 1u;
}

// The slot an index word names, or NONE if its bucket was not flagged in this chunk.
__device__ __forceinline__ uint32_t flag_slot(uint32_t w7, uint32_t F) {
    return ((w7 & FLAG) && (w7 & ~FLAG) < F) ? (w7 & ~FLAG) : NONE;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Accumulate the time since the previous mark into phase k (block 0, thread 0), when profiling.
__device__ __forceinline__ void phase_mark(const MswsDev& D, int k) {
    if (!D.prof) return;  // the timers' global reads and writes would delay block 0 at every barrier
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Ctl* ctl = D.ctl;
        const uint64_t now = globaltimer();
        if (k >= 0) ctl->phase_ns[k] += now - ctl->phase_t;
        ctl->phase_t = now;
    }
}

// End of a repair: the last block to finish (counted on bar_count, which wraps back to 0)
// resets the chunk's counters and the barrier arrivals; no block waits for the others.
__device__ __forceinline__ void finish_repair(Ctl* ctl) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicInc(&ctl->bar_count, gridDim.x - 1) == gridDim.x - 1) {
            __threadfence();
            const uint64_t now = globaltimer();
            ctl->phase_ns[5] += now - ctl->phase_t;
            ctl->phase_t = now;
            ctl->n_flagged = 0;
            ctl->n_records = 0;
            ctl->n_long = 0;
            ctl->bar_arrive = 0;  // every block is past its last grid barrier
            ctl->repairs += 1;
            ctl->link_gen += 1;
            __threadfence();
        }
    }
}

// Batched streams: the stream of window key i (< wpre[n_streams]), i.e. the last s with
// wpre[s] <= i, which is never an empty slice.
__device__ __forceinline__ uint32_t stream_of_window_key(const BatchDev& B, uint32_t i) {
    uint32_t lo = 0, hi = B.n_streams;  // wpre[lo] <= i < wpre[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(B.wpre + mid) <= i)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// The stream whose bucket range holds global bucket g (bases strictly increase).
__device__ __forceinline__ uint32_t stream_of_bucket(const BatchDev& B, uint32_t g) {
    uint32_t lo = 0, hi = B.n_streams;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&B.desc[mid].low_base) <= g)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// The repair's key passes: one sketch whose chunk is `keys[0, n)`, or a batch window whose key
// i lies in stream s at flat index lo[s] + i - wpre[s]; a thread walks window keys in
// increasing order, so the stream cursor only moves forward.
template <bool BATCH>
struct KeyMap {
    uint32_t s = 0;
    __device__ __forceinline__ void start(const BatchDev& B, uint32_t i) {
        if (BATCH) s = stream_of_window_key(B, i);
    }
    __device__ __forceinline__ uint64_t flat(const BatchDev& B, uint32_t i) {
        if constexpr (!BATCH) {
            return i;
        } else {
            while (i >= __ldg(B.wpre + s + 1)) ++s;
            return __ldg(B.lo + s) + (i - __ldg(B.wpre + s));
        }
    }
    // window keys of the current stream end here (exclusive)
    __device__ __forceinline__ uint32_t end(const BatchDev& B) const {
        return BATCH ? __ldg(B.wpre + s + 1) : 0xffffffffu;
    }
    // bucket of a key of the current stream
    __device__ __forceinline__ uint32_t bucket(const MswsDev& D, const BatchDev& B, uint32_t key, uint32_t& hv) const {
        if (!BATCH) {
            hv = key * D.seed;
            return fast_mod(D.fm_low, hv);
        }
        const StreamDesc* sd = B.desc + s;
        hv = key * __ldg(&sd->seed);
        const FastMod fm{__ldg(&sd->fm_low.M), __ldg(&sd->fm_low.d), 0u};
        return __ldg(&sd->low_base) + fast_mod(fm, hv);
    }
};

struct RadixSmem {
    uint32_t whist[REPAIR_THREADS / 32][256];
};

size_t msws_repair_smem() { return (size_t)SET_SLOTS * 4; }

// A tile of REPAIR_TILE records in registers: each of the 16 warps owns 256 consecutive
// records, lane l of warp w holding records t*REPAIR_TILE + w*256 + r*32 + l (r < 8).  All
// eight loads are issued before any is used, so a tile costs one L2 round trip.
constexpr int TILE_ROUNDS = 256 / 32;
__device__ __forceinline__ void tile_load(const uint2* src, uint32_t K, uint32_t t, uint2 (&rec)[TILE_ROUNDS]) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < TILE_ROUNDS; ++r) {
        const uint32_t i = t * REPAIR_TILE + wid * 256 + r * 32 + lane;
        rec[r] = i < K ? __ldcg(&src[i]) : make_uint2(0u, 0u);
    }
}

// The array-order positions of a tile's records, in the layout of tile_load (psrc null: the
// records are still in array order, so a record's position is its index).
__device__ __forceinline__ void tile_load_pos(const uint32_t* psrc, uint32_t K, uint32_t t,
                                              uint32_t (&pos)[TILE_ROUNDS]) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < TILE_ROUNDS; ++r) {
        const uint32_t i = t * REPAIR_TILE + wid * 256 + r * 32 + lane;
        pos[r] = psrc ? (i < K ? __ldcg(psrc + i) : 0u) : i;
    }
}

// Per-warp counts of the tile's records by the 8-bit digit at `shift`.
__device__ __forceinline__ void tile_count(RadixSmem& rs, const uint2 (&rec)[TILE_ROUNDS], uint32_t K, uint32_t t,
                                           int shift) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < 256 * (REPAIR_THREADS / 32); d += REPAIR_THREADS) (&rs.whist[0][0])[d] = 0;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < TILE_ROUNDS; ++r) {
        const uint32_t i = t * REPAIR_TILE + wid * 256 + r * 32 + lane;
        const bool v = i < K;
        const uint32_t d = v ? (rec[r].x >> shift) & 0xffu : 256u + lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (v && lane == __ffs(peers) - 1) rs.whist[wid][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
}

// ---- per-bucket replay (one warp per flagged bucket; lane i keeps counter i) ------------
// The chunk's keys of a flagged bucket, in array order, are replayed with the sequential
// semantics of device_sketch_v3.h:88-191: the pre-chunk counters are restored (final word
// minus the packed sum of the chunk's increments, mod 2^32), the first key that sees a
// selected counter above LIMIT is found (the low->high switch of :160-190), the bucket is
// linked there (atomic_malloc, :69-85) and that key and all later ones count high.

// Occurrences of counter c (lane c) among the 32 masks of the warp: seven warp sums of the
// masks expanded to one byte per counter (a byte counts at most 32, so no carries).
__device__ __forceinline__ uint32_t group_counts(uint32_t m) {
    const int lane = threadIdx.x & 31;
    uint32_t mine = 0;
#pragma unroll
    for (int w = 0; w < 7; ++w) {
        const uint32_t t = __reduce_add_sync(0xffffffffu, expand_nibble((m >> (4 * w)) & 0xfu));
        if ((lane >> 2) == w) mine = t;
    }
    return lane < LOW_COUNTERS ? (mine >> (8 * (lane & 3))) & 0xffu : 0u;
}

// Lane c accumulates the occurrences of counter c among the 32 masks of the warp.
__device__ __forceinline__ void count_counters(uint32_t m, uint32_t& T) { T += group_counts(m); }

// Pre-chunk counter of lane i from the bucket's final words and the chunk totals T.
__device__ __forceinline__ uint32_t pre_counters(const uint32_t* wp, uint32_t T) {
    const int lane = threadIdx.x & 31;
    const uint32_t fw = lane < 7 ? __ldcg(wp + lane) : 0u;
    uint32_t sw = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) sw += __shfl_sync(0xffffffffu, T, (4 * (lane & 7) + k) & 31) << (8 * k);
    const uint32_t pwi = __shfl_sync(0xffffffffu, fw - sw, (lane >> 2) & 7);
    return lane < LOW_COUNTERS ? (pwi >> (8 * (lane & 3))) & 0xffu : 0u;
}

// 32 consecutive records (mask m, 0 for lanes that are not this bucket's): returns the lane
// of the first record that sees a selected counter above LIMIT, or -1; `cur` advances over
// the records before it (all 32 when none triggers).
__device__ __forceinline__ int link_step(uint32_t m, uint32_t& cur) {
    const int lane = threadIdx.x & 31;
    // The last record with counter c sees cur + (occurrences - 1): when that stays within
    // LIMIT for every counter, no record of the group switches.
    const uint32_t tot = group_counts(m);
    if (!__any_sync(0xffffffffu, tot && cur + tot > LIMIT + 1)) {
        cur += tot;
        return -1;
    }
    const uint32_t lt = lanemask_lt();
    bool trig = false;
    uint32_t inc = 0;
#pragma unroll
    for (int c = 0; c < LOW_COUNTERS; ++c) {
        const uint32_t bal = __ballot_sync(0xffffffffu, (m >> c) & 1u);
        const uint32_t cc = __shfl_sync(0xffffffffu, cur, c);
        if (((m >> c) & 1u) && cc + __popc(bal & lt) > LIMIT) trig = true;
        if (lane == c) inc = __popc(bal);
    }
    const uint32_t tb = __ballot_sync(0xffffffffu, trig);
    if (!tb) {
        cur += inc;
        return -1;
    }
    const int j = __ffs(tb) - 1;
    const uint32_t before = (1u << j) - 1u;
#pragma unroll
    for (int c = 0; c < LOW_COUNTERS; ++c) {
        const uint32_t bal = __ballot_sync(0xffffffffu, (m >> c) & 1u);
        if (lane == c) cur += __popc(bal & before);
    }
    return j;
}

// Where the replay of one flagged bucket ended (per lane c: counter c).
struct ReplayOut {
    bool found;        // a key switched the bucket to the high level
    uint32_t L;        // that key's record: index into the records the replay read
    uint32_t n_after;  // the bucket's keys at or after the switch
    uint32_t n_total;  // the bucket's keys in the chunk
    uint32_t T;        // the chunk's increments of counter c
    uint32_t P;        // counter c before the chunk
    uint32_t cur;      // counter c when the switch happens (final low value)
    uint32_t mL;       // the switching key's mask
};

// Increments of high counter `lane` in the new high bucket: the switching key's and all
// later keys'.
__device__ __forceinline__ uint32_t high_increments(const MswsDev& D, const ReplayOut& o) {
    const int lane = threadIdx.x & 31;
    uint32_t H = o.T - (o.cur - o.P);
    if (D.compat_v3) {  // device_sketch_v3.h:187: the switching key lands on bit % 8
        if (lane < LOW_COUNTERS && ((o.mL >> lane) & 1u)) H -= 1u;
        if (lane < 8) H += __popc(o.mL & (0x01010101u << lane));
    }
    return H;
}

// The low counters at the switch, packed back into words 0..6 of bucket b.
__device__ __forceinline__ void write_low_words(const MswsDev& D, uint32_t b, uint32_t cur) {
    const int lane = threadIdx.x & 31;
    uint32_t word = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) word |= __shfl_sync(0xffffffffu, cur, (4 * (lane & 7) + k) & 31) << (8 * k);
    if (lane < 7) __stcg(D.low + (uint64_t)b * LOW_WORDS + lane, word);
}

// Replay slot s from its segment of the slot-sorted records (no writes).
__device__ __forceinline__ ReplayOut replay_sorted(const MswsDev& D, const uint2* sorted, uint32_t s, uint32_t F,
                                                  uint32_t K, uint32_t b) {
    const int lane = threadIdx.x & 31;
    const uint32_t beg = __ldcg(D.seg_beg + s);
    const uint32_t end = (s + 1 < F) ? __ldcg(D.seg_beg + s + 1) : K;
    ReplayOut o;
    o.T = 0;
    if (s < D.long_cap) {
        o.T = lane < LOW_COUNTERS ? __ldcg(D.totals + (uint64_t)s * LOW_COUNTERS + lane) : 0u;
    } else {
        for (uint32_t g = beg; g < end; g += 32) count_counters((g + lane < end) ? __ldcg(&sorted[g + lane].y) : 0u, o.T);
    }
    o.P = pre_counters(D.low + (uint64_t)b * LOW_WORDS, o.T);
    o.cur = o.P;
    o.mL = 0;
    uint32_t L = NONE;
    // four groups of 32 records loaded per step, so a long segment costs one L2 round trip
    // per 128 records
    constexpr int GR = 4;
    for (uint32_t g0 = beg; g0 < end && L == NONE; g0 += 32 * GR) {
        uint32_t mm[GR];
#pragma unroll
        for (int q = 0; q < GR; ++q) {
            const uint32_t i = g0 + 32 * q + lane;
            mm[q] = i < end ? __ldcg(&sorted[i].y) : 0u;
        }
#pragma unroll
        for (int q = 0; q < GR; ++q) {
            if (L == NONE && g0 + 32 * q < end) {  // warp-uniform
                const int j = link_step(mm[q], o.cur);
                if (j >= 0) {
                    L = g0 + 32 * q + j;
                    o.mL = __shfl_sync(0xffffffffu, mm[q], j);
                }
            }
        }
    }
    o.found = L != NONE;
    o.L = L;
    o.n_after = o.found ? end - L : 0u;
    o.n_total = end - beg;
    return o;
}

// Replay slot s straight from the chunk's records in array order (all K of them staged in
// shared memory; no writes): steps of 32 records without one of this slot skip after one
// ballot.  The slot's counter totals and record count come from the write phase (slots <
// long_cap).
__device__ __forceinline__ ReplayOut replay_scan(const MswsDev& D, const uint2* srec, uint32_t s, uint32_t K,
                                                uint32_t b) {
    const int lane = threadIdx.x & 31;
    ReplayOut o;
    o.T = 0;
    o.n_total = 0;
    if (s < D.long_cap) {  // accumulated while the records were written
        o.T = lane < LOW_COUNTERS ? __ldcg(D.totals + (uint64_t)s * LOW_COUNTERS + lane) : 0u;
        o.n_total = __ldcg(D.seg_beg + s);
    } else {
        for (uint32_t g = 0; g < K; g += 32) {
            const uint2 r = g + lane < K ? srec[g + lane] : make_uint2(NONE, 0u);
            const bool hit = r.x == s;
            const uint32_t hb = __ballot_sync(0xffffffffu, hit);
            if (!hb) continue;
            o.n_total += __popc(hb);
            count_counters(hit ? r.y : 0u, o.T);
        }
    }
    o.P = pre_counters(D.low + (uint64_t)b * LOW_WORDS, o.T);
    o.cur = o.P;
    o.mL = 0;
    o.found = false;
    o.L = NONE;
    uint32_t before = 0;
    for (uint32_t g = 0; g < K; g += 32) {
        const uint2 r = g + lane < K ? srec[g + lane] : make_uint2(NONE, 0u);
        const bool hit = r.x == s;
        const uint32_t hb = __ballot_sync(0xffffffffu, hit);
        if (!hb) continue;
        const uint32_t m = hit ? r.y : 0u;
        const int j = link_step(m, o.cur);
        if (j >= 0) {
            o.found = true;
            o.L = g + j;
            before += __popc(hb & ((1u << j) - 1u));
            o.mL = __shfl_sync(0xffffffffu, m, j);
            break;
        }
        before += __popc(hb);
    }
    o.n_after = o.found ? o.n_total - before : 0u;
    return o;
}

// After the replay of slot s (bucket b): a bucket that did not switch is final (word 7 back
// to 0).  One that switched records its switch position `pos` (array order of the chunk's
// records) for the link order; when its slot has a totals row (s < long_cap) the low words
// are written now and the high increments wait in that row, otherwise the bucket is replayed
// again once its high id is known.
template <bool BATCH>
__device__ __forceinline__ void settle_bucket(const MswsDev& D, const BatchDev& B, unsigned long long gen, uint32_t s,
                                              uint32_t b, const ReplayOut& o, uint32_t pos) {
    const int lane = threadIdx.x & 31;
    if (o.found) {
        if (s < D.long_cap) {
            const uint32_t H = high_increments(D, o);
            if (lane < LOW_COUNTERS) __stcg(D.totals + (uint64_t)s * LOW_COUNTERS + lane, H);
            write_low_words(D, b, o.cur);
        }
        if (lane == 0) {
            __stcg(D.sw + s, make_uint2(pos, o.n_after));
            atomicOr(D.sw_bits + (pos >> 5), 1u << (pos & 31));
            atomicAdd(D.sw_cnt + pos / SW_BLOCK, 1u);
            if (BATCH) {  // the stream's first switch position of this repair, and its allocator
                const uint32_t st = stream_of_bucket(B, b);  // (nothing writes it before the barrier)
                atomicMax(B.first + st, (gen << 32) | (unsigned long long)(~pos));
                __stcg(D.sw_base + s, __ldcg(B.next_id + st));
            }
        }
    } else {
        if (lane == 0) __stcg(D.sw + s, make_uint2(NONE, 0u));
        if (lane == 7) __stcg(D.low + (uint64_t)b * LOW_WORDS + 7, 0u);  // every key added low
    }
    if (lane == 0) {
        atomicAdd(&D.ctl->repaired_buckets, 1ull);
        atomicAdd(&D.ctl->repaired_keys, (unsigned long long)o.n_total);
    }
}

// Link bucket b to high id `id` (global; ok: inside the pool) with high increments H, or
// saturate it when the pool has run out (its n_after keys are dropped).
__device__ __forceinline__ void link_bucket(const MswsDev& D, uint32_t b, uint32_t id, bool ok, uint32_t H,
                                            uint32_t n_after) {
    const int lane = threadIdx.x & 31;
    if (ok) {
        __stcg(D.high + (uint64_t)(id - START) * HIGH_WORDS + lane, H);
    } else if (lane == 0) {
        atomicOr(&D.ctl->status, ST_POOL_FULL);
        atomicAdd(&D.ctl->dropped, (unsigned long long)n_after);
    }
    if (lane == 7) __stcg(D.low + (uint64_t)b * LOW_WORDS + 7, ok ? id : SATURATED);
}

// Rank of switch position p among all switch positions of the chunk (the result in every
// lane): the exclusive prefix `spre` of the per-SW_BLOCK counts, plus the set bits before p
// in its block of 128 words.
__device__ __forceinline__ uint32_t switch_rank(const MswsDev& D, const uint32_t* spre, uint32_t p) {
    const int lane = threadIdx.x & 31;
    const uint32_t q = p / SW_BLOCK, w = p >> 5;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < (int)(SW_BLOCK / 32 / 32); ++k) {
        const uint32_t wi = q * (SW_BLOCK / 32) + k * 32 + lane;
        if (wi < w) c += __popc(__ldcg(D.sw_bits + wi));
    }
    if (lane == 0) c += __popc(__ldcg(D.sw_bits + w) & ((1u << (p & 31)) - 1u));
    return spre[q] + __reduce_add_sync(0xffffffffu, c);
}

// The same rank in a chunk of at most SCAN_CAP records: the set bits of all switch words
// before p, eight loads per lane in flight, with no prefix of the per-block counts.
__device__ __forceinline__ uint32_t switch_rank_small(const MswsDev& D, uint32_t p) {
    static_assert(SCAN_CAP / 32 == 8 * 32, "eight switch words per lane");
    const int lane = threadIdx.x & 31;
    const uint32_t w = p >> 5;
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t wi = k * 32 + lane;
        v[k] = wi < w ? __ldcg(D.sw_bits + wi) : (wi == w ? __ldcg(D.sw_bits + w) & ((1u << (p & 31)) - 1u) : 0u);
    }
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) c += __popc(v[k]);
    return __reduce_add_sync(0xffffffffu, c);
}

// What the replay of a warp's first slot leaves in registers for the link phase, which
// would otherwise read it back: the bucket, the switch (position, keys from it on) and
// the high increments of lane c.
struct SlotCache {
    uint32_t s = NONE;  // the slot (NONE: nothing cached)
    uint32_t b = 0, pos = NONE, n_after = 0, H = 0;
};

__device__ __forceinline__ SlotCache slot_cache(const MswsDev& D, uint32_t s, uint32_t b, const ReplayOut& o,
                                                uint32_t pos) {
    SlotCache c;
    c.s = s;
    c.b = b;
    c.pos = o.found ? pos : NONE;
    c.n_after = o.found ? o.n_after : 0u;
    c.H = o.found ? high_increments(D, o) : 0u;
    return c;
}

// The 8 keys of the chunk from position `base` (a multiple of 8) and their skip bits; km is
// left at base's stream.  Two 16-byte loads when the keys are whole, contiguous (one
// stream) and aligned; keys past n read as 0 (the caller skips them).
template <bool BATCH>
__device__ __forceinline__ void repair_tile_keys(const uint32_t* __restrict__ keys, uint64_t n, const MswsDev& D,
                                                 const BatchDev& B, uint64_t base, uint32_t (&k)[8], uint32_t& skip8,
                                                 KeyMap<BATCH>& km) {
    uint64_t f0 = 0;
    if (base < n) {
        km.start(B, (uint32_t)base);
        f0 = km.flat(B, (uint32_t)base);
    }
    const bool whole = base + 8 <= n && base + 8 <= km.end(B);
    if (whole && !(reinterpret_cast<uintptr_t>(keys + f0) & 15u)) {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(keys + f0));
        const uint4 c = __ldg(reinterpret_cast<const uint4*>(keys + f0) + 1);
        k[0] = a.x, k[1] = a.y, k[2] = a.z, k[3] = a.w, k[4] = c.x, k[5] = c.y, k[6] = c.z, k[7] = c.w;
    } else if (whole) {
#pragma unroll
        for (int j = 0; j < 8; ++j) k[j] = __ldg(keys + f0 + j);
    } else {
        KeyMap<BATCH> kl = km;
#pragma unroll
        for (int j = 0; j < 8; ++j) k[j] = base + j < n ? __ldg(keys + kl.flat(B, (uint32_t)(base + j))) : 0u;
    }
    skip8 = (D.skip && base < n) ? (__ldg(D.skip + (base >> 5)) >> (base & 31)) & 0xffu : 0u;
}

// Link a bucket that switched: its high increments wait in its totals row, or (no row) the
// bucket is replayed again by `rerun` now that its id is known.
template <typename Rerun>
__device__ __forceinline__ void finish_link(const MswsDev& D, uint32_t s, uint32_t b, uint32_t id, bool ok,
                                            uint32_t n_after, Rerun& rerun, const SlotCache& sc) {
    const int lane = threadIdx.x & 31;
    uint32_t H;
    if (s < D.long_cap && s == sc.s) {
        H = sc.H;
    } else if (s < D.long_cap) {
        H = lane < LOW_COUNTERS ? __ldcg(D.totals + (uint64_t)s * LOW_COUNTERS + lane) : 0u;
    } else {
        const ReplayOut o = rerun(s, b);
        write_low_words(D, b, o.cur);
        H = high_increments(D, o);
        n_after = o.n_after;
    }
    link_bucket(D, b, id, ok, H, n_after);
}

// The link order of the chunk's switched buckets.  A bucket's rank is the number of switch
// positions before its own (array order of the records), so the r-th switching key of the
// chunk gets id next_id + r, as one-key-at-a-time insertion hands them out
// (atomic_malloc, device_sketch_v3.h:69-85); once the pool is used up the remaining buckets
// saturate.  Batched streams rank within their stream (each has its own allocator): the
// replay recorded the stream's first switch position (generation-tagged atomicMax) and its
// allocator before the barrier, and a bucket's rank in its stream is its rank minus that
// position's.  one_block: every slot lives in block 0 and only it runs this.
template <bool BATCH, typename Rerun>
__device__ __forceinline__ void link_phase(const MswsDev& D, const BatchDev& B, uint32_t F, uint32_t K,
                                           uint32_t base_id, unsigned long long gen, bool one_block, Rerun rerun,
                                           uint32_t* s_small, uint32_t* s_big, const SlotCache& sc) {
    Ctl* ctl = D.ctl;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int NW = REPAIR_THREADS / 32;
    const uint32_t nq = (K + SW_BLOCK - 1) / SW_BLOCK;  // K <= 2^26: at most 16384 counts
    uint32_t* spre = nq <= 64 ? s_small : s_big;        // the sort-free replay (K <= SCAN_CAP) keeps
                                                        // its records in s_big
    // one sketch, few records: ranks straight from the switch bits, no prefix of the counts
    const bool small = !BATCH && K <= SCAN_CAP;
    uint32_t nfound = 0;
    if (!small) {
        for (uint32_t i = tid; i < nq; i += REPAIR_THREADS) spre[i] = __ldcg(D.sw_cnt + i);
        __syncthreads();
        nfound = block_scan_smem(spre, nq);
    } else if (blockIdx.x == 0 && tid == 0) {
        for (uint32_t i = 0; i < nq; ++i) nfound += __ldcg(D.sw_cnt + i);
    }
    for (uint32_t s = blockIdx.x * NW + wid; s < F; s += gridDim.x * NW) {
        const bool cached = s == sc.s;
        const uint2 w = cached ? make_uint2(sc.pos, sc.n_after) : __ldcg(D.sw + s);
        if (w.x == NONE) continue;  // warp-uniform
        const uint32_t b = cached ? sc.b : __ldcg(D.flag_list + s);
        const uint32_t rank = small ? switch_rank_small(D, w.x) : switch_rank(D, spre, w.x);
        if (!BATCH) {
            const uint32_t id = base_id + rank;
            finish_link(D, s, b, id, (uint64_t)(id - START) < D.n_high, w.y, rerun, sc);
            continue;
        }
        // batched streams: the rank among the stream's own switches (its positions are
        // contiguous in the window) on top of the stream's allocator read before the barrier
        uint32_t st = 0, fp = 0;
        if (lane == 0) {
            st = stream_of_bucket(B, b);
            fp = ~(uint32_t)__ldcg(B.first + st);
        }
        st = __shfl_sync(0xffffffffu, st, 0);
        fp = __shfl_sync(0xffffffffu, fp, 0);
        const uint32_t own = __ldcg(D.sw_base + s) + (rank - switch_rank(D, spre, fp));
        const uint32_t nh = __ldg(&B.desc[st].n_high);
        const bool ok = (uint64_t)(own - START) < nh;
        finish_link(D, s, b, own + __ldg(&B.desc[st].high_base), ok, w.y, rerun, sc);
        if (lane == 0) {
            atomicMax(B.next_id + st, (uint32_t)min((unsigned long long)own + 1ull, (unsigned long long)START + nh));
            if (!ok) atomicOr(B.status + st, ST_POOL_FULL);
        }
    }
    if (!BATCH && blockIdx.x == 0 && tid == 0) {  // the allocator stops at the pool's end, as the oracle's
        const unsigned long long nid = min((unsigned long long)base_id + nfound, (unsigned long long)START + D.n_high);
        if (nid > base_id) ctl->next_id = (uint32_t)nid;
    }
}

// BATCH: `keys` is the batch's flat key array and the chunk is the window the plan kernel
// described (B.wpre, B.lo); n is read from the window (the launch's own n is ignored).
template <bool BATCH>
__global__ void __launch_bounds__(REPAIR_THREADS, 2) k_msws_repair(const uint32_t* __restrict__ keys, uint64_t n,
                                                                MswsDev D, BatchDev B) {
    __shared__ RadixSmem rs;
    __shared__ uint32_t s_dbase[256];  // radix pass: first output position of each digit
    __shared__ uint32_t s_acc_base[256];  // radix pass, several tiles per block: a tile's digit bases
    __shared__ uint32_t s_acc[2][LOW_COUNTERS];
    __shared__ uint32_t s_acc_slot[2];
    __shared__ uint32_t s_tc[TC_MAX];       // phase 1: counts of this block's tiles, by round
    __shared__ uint32_t s_swpre[64];        // link order: prefix of the switch counts (small chunks)
    extern __shared__ __align__(16) uint32_t s_set[];
    griddep_wait();  // pass 1 has ended (its flags, tables and counters are final)
    Ctl* ctl = D.ctl;
    const uint32_t F = min(__ldcg(&ctl->n_flagged), D.flag_cap);
    if (F == 0) return;
    // Read before the first grid barrier; only the link phase, after it, writes them.
    const uint32_t base_id = __ldcg(&ctl->next_id);
    const unsigned long long gen = (unsigned long long)__ldcg(&ctl->link_gen) + 1ull;
    phase_mark(D, -1);
    if (BATCH) n = __ldcg(B.win + 1);

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int NW = REPAIR_THREADS / 32;
    constexpr int PER = REPAIR_TILE / REPAIR_THREADS;  // 8 consecutive keys per thread
    static_assert(PER == 8, "8 keys per thread: two 16-byte loads, one byte of skip bits");
    const uint32_t ntk = (uint32_t)((n + REPAIR_TILE - 1) / REPAIR_TILE);
    // the tile-count prefix of phase 2 lives in the SET_SLOTS words of shared memory: chunks of at most
    // SET_SLOTS tiles (2^26 keys; the host rejects larger max_batch); uniform, so every block
    // leaves before any barrier
    if (ntk > (uint32_t)SET_SLOTS || ntk > TC_MAX * gridDim.x) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->status, ST_CAPACITY);
        return;
    }
    const uint32_t nthreads = gridDim.x * REPAIR_THREADS;
    const uint32_t gtid = blockIdx.x * REPAIR_THREADS + tid;

    // Phase 0: the flagged buckets' filter in every block; zero the totals.
    uint32_t* sbloom = s_set;
    for (int i = tid; i < BLOOM_WORDS; i += REPAIR_THREADS) sbloom[i] = 0u;
    __syncthreads();
    for (uint32_t s0 = tid; s0 < F; s0 += 8 * REPAIR_THREADS) {  // eight loads in flight
        uint32_t fb[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) fb[u] = s0 + u * REPAIR_THREADS < F ? __ldcg(D.flag_list + s0 + u * REPAIR_THREADS) : NONE;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (fb[u] != NONE) {
                const uint32_t h = bloom_bit(fb[u]);
                atomicOr(sbloom + (h >> 5), 1u << (h & 31));
            }
        }
    }
    for (int i = tid; i < TC_MAX; i += REPAIR_THREADS) s_tc[i] = 0u;
    __syncthreads();
    const uint32_t ntot = min(F, D.long_cap);
    for (uint32_t i = gtid; i < ntot * LOW_COUNTERS; i += nthreads) __stcg(D.totals + i, 0u);
    for (uint32_t i = gtid; i < ntot; i += nthreads) __stcg(D.seg_beg + i, 0u);  // record counts (scan mode)
    phase_mark(D, 8);

    // Phase 1: the keys of flagged buckets, per tile of the chunk.  Each warp owns 256
    // consecutive keys of a tile (8 per lane) and stages their records at its own place, so
    // no block-wide synchronisation happens per tile: the warp's record count goes to wcnt
    // (the histogram buffer, unused until the radix passes) and into the tile's count in
    // shared memory.
    uint32_t* wcnt = D.hist;  // [ntk][NW]
    const uint32_t seed = D.seed;      // one sketch (not batched): its hash and bucket count
    const FastMod fm_low = D.fm_low;
    auto test_tile = [&](uint32_t t, uint32_t rk, const uint32_t (&k)[PER], uint32_t skip8, KeyMap<BATCH> km) {
        const uint64_t base = (uint64_t)t * REPAIR_TILE + (uint64_t)tid * PER;
        const uint32_t nv = base >= n ? 0u : (uint32_t)umin64(PER, n - base);
        const uint32_t live = ((1u << nv) - 1u) & ~skip8;  // keys of the chunk, not skipped
        // the filter first for all eight keys, then their index words (filter hits only) as
        // eight independent loads in flight together, then the slots
        uint32_t hit = 0, cand = 0, slot[PER];
        KeyMap<BATCH> km0 = km;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            slot[j] = 0u;
            if ((live >> j) & 1u) {
                uint32_t b;
                if constexpr (BATCH) {
                    km.flat(B, (uint32_t)(base + j));  // moves the cursor to key j's stream
                    uint32_t hv;
                    b = km.bucket(D, B, k[j], hv);
                } else {
                    b = fast_mod(fm_low, k[j] * seed);
                }
                if (bloom_hit(sbloom, b)) {
                    cand |= 1u << j;
                    slot[j] = b;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < PER; ++j)
            slot[j] = ((cand >> j) & 1u) ? __ldcg(D.low + (uint64_t)slot[j] * LOW_WORDS + 7) : 0u;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            slot[j] = ((cand >> j) & 1u) ? flag_slot(slot[j], F) : NONE;
            if (slot[j] != NONE) hit |= 1u << j;
        }
        const uint32_t hc = __popc(hit);
        uint32_t x = hc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        uint32_t pos = x - hc;
        const uint32_t wtot = __shfl_sync(0xffffffffu, x, 31);
        if (lane == 0) {
            __stcg(wcnt + (uint64_t)t * NW + wid, wtot);
            if (wtot) atomicAdd(s_tc + rk, wtot);
        }
        // the hit keys' (slot, mask) records in array order, staged at the warp's own place
        // in rec[1] (its keys start at t * REPAIR_TILE + wid * 256 < n, so the stage stays
        // inside)
        if (hit) {
            uint2* stage = D.rec[1] + (uint64_t)t * REPAIR_TILE + wid * 256;
#pragma unroll
            for (int j = 0; j < PER; ++j) {
                if ((hit >> j) & 1u) {
                    uint32_t hv;
                    if constexpr (BATCH) {
                        km0.flat(B, (uint32_t)(base + j));
                        km0.bucket(D, B, k[j], hv);
                    } else {
                        hv = k[j] * seed;
                    }
                    __stcg(stage + pos, make_uint2(slot[j], __ldg(D.masks + fast_mod(D.fm_mask, hv))));
                    ++pos;
                }
            }
        }
    };
    const uint32_t my_tiles = blockIdx.x < ntk ? (ntk - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    {
        // the next tile's keys are loaded before the current tile is tested
        uint32_t k[PER], skip8 = 0;
        KeyMap<BATCH> km;
        if (my_tiles) repair_tile_keys<BATCH>(keys, n, D, B, (uint64_t)blockIdx.x * REPAIR_TILE + tid * PER, k, skip8, km);
        for (uint32_t i = 0; i < my_tiles; ++i) {
            const uint32_t t = blockIdx.x + i * gridDim.x;
            uint32_t kn[PER] = {}, skipn = 0;
            KeyMap<BATCH> kmn;
            if (i + 1 < my_tiles)
                repair_tile_keys<BATCH>(keys, n, D, B, (uint64_t)(t + gridDim.x) * REPAIR_TILE + tid * PER, kn, skipn,
                                        kmn);
            test_tile(t, i, k, skip8, km);
#pragma unroll
            for (int j = 0; j < PER; ++j) k[j] = kn[j];
            skip8 = skipn;
            km = kmn;
        }
    }
    __syncthreads();
    for (uint32_t r = tid; blockIdx.x + r * gridDim.x < ntk; r += REPAIR_THREADS)
        __stcg(D.tile_counts + blockIdx.x + r * gridDim.x, s_tc[r]);
    if (!grid_barrier(ctl)) return;
    phase_mark(D, 0);
    // Phase 2: every block scans the tile counts itself (exclusive, in shared memory — the
    // flag filter is not needed after phase 1), which gives its tiles' record offsets
    // and the record total K without another grid barrier.
    uint32_t* spre = s_set;
    for (uint32_t i0 = tid; i0 < ntk; i0 += 4 * REPAIR_THREADS) {  // four loads in flight
        uint32_t v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = i0 + u * REPAIR_THREADS < ntk ? __ldcg(D.tile_counts + i0 + u * REPAIR_THREADS) : 0u;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (i0 + u * REPAIR_THREADS < ntk) spre[i0 + u * REPAIR_THREADS] = v[u];
    }
    __syncthreads();
    const uint32_t K = block_scan_smem(spre, ntk);
    if (blockIdx.x == 0 && tid == 0) __stcg(&ctl->n_records, K);
    phase_mark(D, 1);
    // Few records (K <= SCAN_CAP): the replay scans them unsorted, and the per-slot counter
    // totals and record counts it needs are accumulated here with global atomics.
    const bool scan_mode = K <= SCAN_CAP;
    {  // the link order's switch bits and counts: positions lie below K
        const uint32_t nsw = (K + 31) >> 5, nswc = (K + SW_BLOCK - 1) / SW_BLOCK;
        for (uint32_t i = gtid; i < nsw; i += nthreads) __stcg(D.sw_bits + i, 0u);
        for (uint32_t i = gtid; i < nswc; i += nthreads) __stcg(D.sw_cnt + i, 0u);
    }
    // Phase 3: the staged records of every tile move to their place in array order, one warp
    // per tile: the tile's 16 region counts, scanned in the warp, place record i of the tile
    // in region r (the first whose running count exceeds i) at offset i - (counts before r).
    for (uint32_t t = blockIdx.x * NW + wid; t < ntk; t += gridDim.x * NW) {
        const uint32_t beg = spre[t], cnt = (t + 1 < ntk ? spre[t + 1] : K) - beg;
        if (cnt == 0) continue;  // warp-uniform
        const uint32_t v = lane < NW ? __ldcg(wcnt + (uint64_t)t * NW + lane) : 0u;
        uint32_t x = v;  // inclusive running count over the regions
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const uint2* stage = D.rec[1] + (uint64_t)t * REPAIR_TILE;
        for (uint32_t i0 = 0; i0 < cnt; i0 += 32) {  // warp-uniform trip count
            const uint32_t i = i0 + lane;
            uint32_t lo = 0, hi = NW - 1;  // region of record i: x[lo - 1] <= i < x[lo]
#pragma unroll
            for (int it = 0; it < 4; ++it) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__shfl_sync(0xffffffffu, x, mid) > i) hi = mid;
                else lo = mid + 1;
            }
            const uint32_t before = __shfl_sync(0xffffffffu, x - v, lo);
            if (i >= cnt) continue;
            const uint2 r = __ldcg(stage + lo * 256 + (i - before));
            __stcg(D.rec[0] + beg + i, r);
            if (scan_mode && r.x < D.long_cap) {
                for (uint32_t mm = r.y; mm; mm &= mm - 1)
                    atomicAdd(D.totals + (uint64_t)r.x * LOW_COUNTERS + (__ffs(mm) - 1), 1u);
                atomicAdd(D.seg_beg + r.x, 1u);
            }
        }
    }
    if (!grid_barrier(ctl)) return;
    phase_mark(D, 2);

    // Few records: no sort.  Every block that replays a slot stages all K records in shared
    // memory (the flag filter is no longer needed; the 64 KiB hold SCAN_CAP records)
    // and each warp scans them for its slot in array order.
    // The switch position of a record is its index here (array order).
    const bool one_block = F <= (uint32_t)NW;  // every slot in block 0: no grid barrier to link
    SlotCache sc;  // the replay of the warp's first slot, kept for the link phase (one sketch)
    if (scan_mode) {
        uint2* srec = reinterpret_cast<uint2*>(s_set);
        if (blockIdx.x * NW < F) {
            for (uint32_t i = tid; i < K; i += REPAIR_THREADS) srec[i] = __ldcg(D.rec[0] + i);
            __syncthreads();
            for (uint32_t s = blockIdx.x * NW + wid; s < F; s += gridDim.x * NW) {
                const uint32_t b = __ldcg(D.flag_list + s);
                const ReplayOut o = replay_scan(D, srec, s, K, b);
                settle_bucket<BATCH>(D, B, gen, s, b, o, o.L);
                if (!BATCH && s == blockIdx.x * NW + wid) sc = slot_cache(D, s, b, o, o.L);
            }
        }
        phase_mark(D, 5);
        if (one_block) {
            if (blockIdx.x != 0) {
                finish_repair(ctl);
                return;
            }
            __syncthreads();
        } else if (!grid_barrier(ctl)) {
            return;
        }
        auto rerun = [&](uint32_t s, uint32_t b) { return replay_scan(D, srec, s, K, b); };
        link_phase<BATCH>(D, B, F, K, base_id, gen, one_block, rerun, s_swpre, s_set, sc);
        phase_mark(D, 9);
        finish_repair(ctl);
        return;
    }

    // Phase 4: stable LSD radix sort of the records by slot, 8 bits per pass.
    const int npass = radix_passes(F);
    const uint32_t ntr = (K + REPAIR_TILE - 1) / REPAIR_TILE;
    const uint2* sorted = D.rec[npass & 1];
    // One tile per block (up to gridDim.x * REPAIR_TILE records): the count keeps the tile's
    // records, each record's rank within its warp's run of its digit, and the per-warp digit
    // offsets in shared memory, so the scatter needs neither a reload nor a recount.
    const bool resident = ntr <= gridDim.x;
    uint2* srec = reinterpret_cast<uint2*>(s_set);   // [REPAIR_TILE]
    uint32_t* srank = s_set + 2 * REPAIR_TILE;        // [REPAIR_TILE]
    uint32_t* spos = s_set + 3 * REPAIR_TILE;         // [REPAIR_TILE] the records' array-order positions
    static_assert(4 * REPAIR_TILE <= SET_SLOTS, "resident tile fits the shared space");
    // Up to SEMI_TILES tiles per block: the count keeps, per tile, the per-warp digit offsets
    // (u16: below REPAIR_TILE) and each record's in-warp rank (u8: a warp holds 256 records);
    // the scatter reloads the records but does not recount them.
    const uint32_t tiles_here = blockIdx.x < ntr ? (ntr - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const bool semi = !resident && ntr <= SEMI_TILES * gridDim.x;
    uint16_t* swoff = reinterpret_cast<uint16_t*>(s_set);                                    // [q][NW][256]
    uint8_t* srank8 = reinterpret_cast<uint8_t*>(s_set) + SEMI_TILES * NW * 256 * 2;        // [q][REPAIR_TILE]
    for (int p = 0; p < npass; ++p) {
        const uint2* src = D.rec[p & 1];
        uint2* dst = D.rec[(p + 1) & 1];
        // record positions in array order: the identity before the first pass
        const uint32_t* psrc = p ? D.rpos[p & 1] : nullptr;
        uint32_t* pdst = D.rpos[(p + 1) & 1];
        const int shift = 8 * p;
        if (resident) {
            if (blockIdx.x < ntr) {
                const uint32_t t = blockIdx.x;
                uint2 rec[TILE_ROUNDS];
                uint32_t pos[TILE_ROUNDS];
                tile_load(src, K, t, rec);
                tile_load_pos(psrc, K, t, pos);
                for (int d = tid; d < 256 * NW; d += REPAIR_THREADS) (&rs.whist[0][0])[d] = 0;
                __syncthreads();
#pragma unroll
                for (int r = 0; r < TILE_ROUNDS; ++r) {
                    const uint32_t li = wid * 256 + r * 32 + lane;
                    const bool v = t * REPAIR_TILE + li < K;
                    const uint32_t d = v ? (rec[r].x >> shift) & 0xffu : 256u + lane;
                    const uint32_t peers = __match_any_sync(0xffffffffu, d);
                    const uint32_t before = v ? rs.whist[wid][d] : 0u;
                    __syncwarp();
                    if (v && lane == __ffs(peers) - 1) rs.whist[wid][d] = before + __popc(peers);
                    __syncwarp();
                    srec[li] = rec[r];
                    srank[li] = before + __popc(peers & lanemask_lt());
                    spos[li] = pos[r];
                }
                __syncthreads();
                for (int d = tid; d < 256; d += REPAIR_THREADS) {  // per-warp offsets, tile total
                    uint32_t run = 0;
                    for (int w = 0; w < NW; ++w) {
                        const uint32_t x = rs.whist[w][d];
                        rs.whist[w][d] = run;
                        run += x;
                    }
                    __stcg(D.hist + (uint64_t)d * ntr + t, run);
                }
                __syncthreads();
            }
        } else if (semi) {
            for (uint32_t q = 0; q < tiles_here; ++q) {
                const uint32_t t = blockIdx.x + q * gridDim.x;
                uint2 rec[TILE_ROUNDS];
                tile_load(src, K, t, rec);
                for (int d = tid; d < 256 * NW; d += REPAIR_THREADS) (&rs.whist[0][0])[d] = 0;
                __syncthreads();
#pragma unroll
                for (int r = 0; r < TILE_ROUNDS; ++r) {
                    const uint32_t li = wid * 256 + r * 32 + lane;
                    const bool v = t * REPAIR_TILE + li < K;
                    const uint32_t d = v ? (rec[r].x >> shift) & 0xffu : 256u + lane;
                    const uint32_t peers = __match_any_sync(0xffffffffu, d);
                    const uint32_t before = v ? rs.whist[wid][d] : 0u;
                    __syncwarp();
                    if (v && lane == __ffs(peers) - 1) rs.whist[wid][d] = before + __popc(peers);
                    __syncwarp();
                    srank8[q * REPAIR_TILE + li] = (uint8_t)(before + __popc(peers & lanemask_lt()));
                }
                __syncthreads();
                for (int d = tid; d < 256; d += REPAIR_THREADS) {  // per-warp offsets, tile total
                    uint32_t run = 0;
                    for (int w = 0; w < NW; ++w) {
                        const uint32_t x = rs.whist[w][d];
                        swoff[(q * NW + w) * 256 + d] = (uint16_t)run;
                        run += x;
                    }
                    __stcg(D.hist + (uint64_t)d * ntr + t, run);
                }
                __syncthreads();
            }
        } else {
            for (uint32_t t = blockIdx.x; t < ntr; t += gridDim.x) {  // per-tile digit counts
                uint2 rec[TILE_ROUNDS];
                tile_load(src, K, t, rec);
                tile_count(rs, rec, K, t, shift);
                for (int d = tid; d < 256; d += REPAIR_THREADS) {
                    uint32_t s = 0;
                    for (int w = 0; w < NW; ++w) s += rs.whist[w][d];
                    __stcg(D.hist + (uint64_t)d * ntr + t, s);
                }
                __syncthreads();
            }
        }
        if (!grid_barrier(ctl)) return;
        phase_mark(D, 6);
        // one warp per digit scans its row of tile counts (exclusive, in place) and stores the
        // digit's total; then every block forms the 256 digit bases itself
        uint32_t* dtot = D.hist + 256ull * D.max_tiles;
        for (uint32_t d = blockIdx.x * NW + wid; d < 256; d += gridDim.x * NW) {
            uint32_t* row = D.hist + (uint64_t)d * ntr;
            uint32_t run = 0;
            for (uint32_t t0 = 0; t0 < ntr; t0 += 128) {  // four rows of 32 counts in flight
                uint32_t v4[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t t = t0 + u * 32 + lane;
                    v4[u] = t < ntr ? __ldcg(row + t) : 0u;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t t = t0 + u * 32 + lane, v = v4[u];
                    uint32_t x = v;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (t < ntr) __stcg(row + t, run + x - v);
                    run += __shfl_sync(0xffffffffu, x, 31);
                }
            }
            if (lane == 0) __stcg(dtot + d, run);
        }
        if (!grid_barrier(ctl)) return;
        phase_mark(D, 7);
        {
            uint32_t total;
            const uint32_t ex = block_exclusive_scan(tid < 256 ? __ldcg(dtot + tid) : 0u, &total);
            if (tid < 256) s_dbase[tid] = ex;
            __syncthreads();
        }
        if (resident) {
            if (blockIdx.x < ntr) {
                const uint32_t t = blockIdx.x;
                for (int d = tid; d < 256; d += REPAIR_THREADS) s_dbase[d] += __ldcg(D.hist + (uint64_t)d * ntr + t);
                __syncthreads();
#pragma unroll
                for (int r = 0; r < TILE_ROUNDS; ++r) {
                    const uint32_t li = wid * 256 + r * 32 + lane;
                    if (t * REPAIR_TILE + li < K) {
                        const uint2 rec = srec[li];
                        const uint32_t d = (rec.x >> shift) & 0xffu;
                        const uint32_t to = s_dbase[d] + rs.whist[wid][d] + srank[li];
                        __stcg(dst + to, rec);
                        __stcg(pdst + to, spos[li]);
                    }
                }
                __syncthreads();
            }
        }
        if (semi) {
            for (uint32_t q = 0; q < tiles_here; ++q) {
                const uint32_t t = blockIdx.x + q * gridDim.x;
                uint2 rec[TILE_ROUNDS];
                uint32_t pos[TILE_ROUNDS];
                tile_load(src, K, t, rec);
                tile_load_pos(psrc, K, t, pos);
                uint32_t* sbase = s_acc_base;  // this tile's first position of each digit
                for (int d = tid; d < 256; d += REPAIR_THREADS) sbase[d] = s_dbase[d] + __ldcg(D.hist + (uint64_t)d * ntr + t);
                __syncthreads();
#pragma unroll
                for (int r = 0; r < TILE_ROUNDS; ++r) {
                    const uint32_t li = wid * 256 + r * 32 + lane;
                    if (t * REPAIR_TILE + li < K) {
                        const uint32_t d = (rec[r].x >> shift) & 0xffu;
                        const uint32_t to = sbase[d] + swoff[(q * NW + wid) * 256 + d] + srank8[q * REPAIR_TILE + li];
                        __stcg(dst + to, rec[r]);
                        __stcg(pdst + to, pos[r]);
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t t = blockIdx.x; t < ntr && !resident && !semi; t += gridDim.x) {  // stable scatter
            uint2 rec[TILE_ROUNDS];
            uint32_t pos[TILE_ROUNDS];
            tile_load(src, K, t, rec);
            tile_load_pos(psrc, K, t, pos);
            tile_count(rs, rec, K, t, shift);
            for (int d = tid; d < 256; d += REPAIR_THREADS) {
                uint32_t run = s_dbase[d] + __ldcg(D.hist + (uint64_t)d * ntr + t);
                for (int w = 0; w < NW; ++w) {
                    const uint32_t x = rs.whist[w][d];
                    rs.whist[w][d] = run;
                    run += x;
                }
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < TILE_ROUNDS; ++r) {
                const uint32_t i = t * REPAIR_TILE + wid * 256 + r * 32 + lane;
                const bool v = i < K;
                const uint32_t d = v ? (rec[r].x >> shift) & 0xffu : 256u + lane;
                const uint32_t peers = __match_any_sync(0xffffffffu, d);
                if (v) {
                    const uint32_t rank = rs.whist[wid][d] + __popc(peers & lanemask_lt());
                    __stcg(dst + rank, rec[r]);
                    __stcg(pdst + rank, pos[r]);
                }
                __syncwarp();
                if (v && lane == __ffs(peers) - 1) rs.whist[wid][d] += __popc(peers);
                __syncwarp();
            }
            __syncthreads();
        }
        if (!grid_barrier(ctl)) return;
        phase_mark(D, 3);
    }

    // Phase 5: segment starts, and per-counter totals of slots < long_cap; each block a
    // contiguous record range whose first and last slot accumulate in shared memory.
    for (uint32_t i = gtid; i < K; i += nthreads) {
        const uint32_t s = __ldcg(&sorted[i].x);
        if (i == 0 || __ldcg(&sorted[i - 1].x) != s) __stcg(D.seg_beg + s, i);
    }
    {
        const uint32_t per = ((K + gridDim.x - 1) / gridDim.x + 31) & ~31u;
        const uint32_t beg = min(K, blockIdx.x * per), end = min(K, beg + per);
        if (tid < 2 * LOW_COUNTERS) (&s_acc[0][0])[tid] = 0;
        if (tid == 0) {
            s_acc_slot[0] = beg < end ? __ldcg(&sorted[beg].x) : NONE;
            s_acc_slot[1] = beg < end ? __ldcg(&sorted[end - 1].x) : NONE;
        }
        __syncthreads();
        for (uint32_t g = beg + wid * 32; g < end; g += REPAIR_THREADS) {
            const uint32_t i = g + lane;
            const bool v = i < end;
            const uint2 rec = v ? __ldcg(&sorted[i]) : make_uint2(NONE, 0u);
            const bool use = v && rec.x < D.long_cap;
            const uint32_t peers = __match_any_sync(0xffffffffu, rec.x);
            const bool leader = lane == __ffs(peers) - 1;
            const int sl = rec.x == s_acc_slot[0] ? 0 : (rec.x == s_acc_slot[1] ? 1 : -1);
            for (int c = 0; c < LOW_COUNTERS; ++c) {
                const uint32_t bal = __ballot_sync(0xffffffffu, use && ((rec.y >> c) & 1u));
                const uint32_t cnt = __popc(bal & peers);
                if (use && leader && cnt) {
                    if (sl >= 0)
                        atomicAdd(&s_acc[sl][c], cnt);
                    else
                        atomicAdd(D.totals + (uint64_t)rec.x * LOW_COUNTERS + c, cnt);
                }
            }
        }
        __syncthreads();
        if (tid < 2 * LOW_COUNTERS) {
            const int sl = tid / LOW_COUNTERS, c = tid % LOW_COUNTERS;
            const uint32_t s = s_acc_slot[sl];
            const bool dup = (sl == 1 && s == s_acc_slot[0]);
            const uint32_t v = s_acc[sl][c];
            if (s < D.long_cap && !dup && v) atomicAdd(D.totals + (uint64_t)s * LOW_COUNTERS + c, v);
        }
    }
    if (!grid_barrier(ctl)) return;
    phase_mark(D, 4);

    // Phase 6: replay each flagged bucket in array order, one warp per slot; then link the
    // switched buckets in the array order of their switching keys (the records' positions
    // before the sort travelled through the radix passes in rpos).
    const uint32_t* fpos = npass ? D.rpos[npass & 1] : nullptr;
    for (uint32_t s = blockIdx.x * NW + wid; s < F; s += gridDim.x * NW) {
        const uint32_t b = __ldcg(D.flag_list + s);
        const ReplayOut o = replay_sorted(D, sorted, s, F, K, b);
        const uint32_t pos = o.found ? (fpos ? __ldcg(fpos + o.L) : o.L) : 0u;
        settle_bucket<BATCH>(D, B, gen, s, b, o, pos);
        if (!BATCH && s == blockIdx.x * NW + wid) sc = slot_cache(D, s, b, o, pos);
    }
    phase_mark(D, 5);
    if (one_block) {
        if (blockIdx.x != 0) {
            finish_repair(ctl);
            return;
        }
        __syncthreads();
    } else if (!grid_barrier(ctl)) {
        return;
    }
    auto rerun = [&](uint32_t s, uint32_t b) { return replay_sorted(D, sorted, s, F, K, b); };
    link_phase<BATCH>(D, B, F, K, base_id, gen, one_block, rerun, s_swpre, s_set, sc);
    phase_mark(D, 9);
    finish_repair(ctl);
}

// ---- query ----------------------------------------------------------------------------

constexpr int QRY_THREADS = 256;
constexpr int QRY_KPT = 4;

// The estimate from a key's low bucket words u (word 7 the index) and mask m, h4 holding its
// first four selected high counters when the bucket is linked (calculation_s2_search,
// device_sketch_v3.h:340-357, 397-402; search_high :293-307, 364-395): min over the selected
// 8-bit counters, plus the min over the selected high counters if linked.
__device__ __forceinline__ uint32_t msws_estimate(const MswsDev& D, const uint32_t (&u)[8], uint32_t m,
                                                  const uint32_t (&h4)[4]) {
    uint32_t acc = 0xffffffffu;
#pragma unroll
    for (int w = 0; w < 7; ++w) {
        const uint32_t sel = expand_nibble((m >> (4 * w)) & 0xfu) * 0xffu;
        acc = __vminu4(acc, u[w] | ~sel);
    }
    acc = __vminu4(acc, acc >> 16);
    const uint32_t lo = min(acc & 0xffu, (acc >> 8) & 0xffu);
    const uint32_t ptr = u[7];
    if (!(ptr > START && (uint64_t)(ptr - START) < D.n_high)) return lo;
    uint32_t hi = min(min(h4[0], h4[1]), min(h4[2], h4[3]));
    uint32_t mm = m;
#pragma unroll
    for (int i = 0; i < 4; ++i) mm &= mm - 1;
    const uint32_t* hb = D.high + (uint64_t)(ptr - START) * HIGH_WORDS;
    for (; mm; mm &= mm - 1) hi = min(hi, __ldg(hb + (__ffs(mm) - 1)));  // masks of more than four counters
    return lo + hi;
}

__device__ __forceinline__ uint32_t msws_lookup(const MswsDev& D, const uint32_t* s_masks, uint32_t key,
                                                uint32_t seed, const FastMod& fm_low, uint32_t base) {
    const uint32_t hv = key * seed;
    const uint32_t b = base + fast_mod(fm_low, hv);
    const uint32_t m = s_masks[fast_mod(D.fm_mask, hv)];
    const uint4* bp = reinterpret_cast<const uint4*>(D.low + (uint64_t)b * LOW_WORDS);
    const uint4 a = __ldg(bp), c = __ldg(bp + 1);
    const uint32_t u[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
    // min over the selected bytes (calculation_s2_search, device_sketch_v3.h:340-357,397-402)
    uint32_t acc = 0xffffffffu;
#pragma unroll
    for (int w = 0; w < 7; ++w) {
        const uint32_t sel = expand_nibble((m >> (4 * w)) & 0xfu) * 0xffu;
        acc = __vminu4(acc, u[w] | ~sel);
    }
    acc = __vminu4(acc, acc >> 16);
    const uint32_t lo = min(acc & 0xffu, (acc >> 8) & 0xffu);
    const uint32_t ptr = u[7];
    uint32_t hi = 0;
    if (ptr > START && (uint64_t)(ptr - START) < D.n_high) {  // search_high, device_sketch_v3.h:293-307, 364-395
        // the first four selected counters as independent loads (no loop: the lookups of a
        // thread's keys interleave), the rest of a wider mask after them
        const uint32_t* hb = D.high + (uint64_t)(ptr - START) * HIGH_WORDS;
        uint32_t mm = m, h4[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            h4[i] = mm ? __ldg(hb + (__ffs(mm) - 1)) : 0xffffffffu;
            mm &= mm - 1;
        }
        hi = min(min(h4[0], h4[1]), min(h4[2], h4[3]));
        for (; mm; mm &= mm - 1) hi = min(hi, __ldg(hb + (__ffs(mm) - 1)));
    }
    return lo + hi;
}

__global__ void __launch_bounds__(QRY_THREADS) k_msws_query(const uint32_t* __restrict__ keys, uint64_t n,
                                                            uint32_t* __restrict__ out, MswsDev D) {
    extern __shared__ __align__(16) uint32_t s_masks[];
    griddep_wait();  // the previous kernel (an insert or its replay) has ended
    griddep_launch_dependents();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t base = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t k[QRY_KPT], r[QRY_KPT];
    // the first keys are loaded while the mask table is staged
#pragma unroll
    for (int j = 0; j < QRY_KPT; ++j) {
        const uint64_t i = base + j * stride;
        k[j] = i < n ? __ldcs(keys + i) : 0u;
    }
    for (uint32_t i = threadIdx.x; i < D.n_masks; i += blockDim.x) s_masks[i] = __ldg(D.masks + i);
    __syncthreads();
    for (; base < n; base += stride * QRY_KPT) {
        if (base != (uint64_t)blockIdx.x * blockDim.x + threadIdx.x) {
#pragma unroll
            for (int j = 0; j < QRY_KPT; ++j) {
                const uint64_t i = base + j * stride;
                k[j] = i < n ? __ldcs(keys + i) : 0u;
            }
        }
        // the low buckets of all QRY_KPT keys first, then the high counters of the linked ones,
        // so the loads of the thread's keys are in flight together at each level
        uint4 la[QRY_KPT], lc[QRY_KPT];
        uint32_t m[QRY_KPT];
#pragma unroll
        for (int j = 0; j < QRY_KPT; ++j) {
            const uint32_t hv = k[j] * D.seed;
            const uint4* bp = reinterpret_cast<const uint4*>(D.low + (uint64_t)fast_mod(D.fm_low, hv) * LOW_WORDS);
            m[j] = s_masks[fast_mod(D.fm_mask, hv)];
            la[j] = __ldg(bp);
            lc[j] = __ldg(bp + 1);
        }
        uint32_t h4[QRY_KPT][4];
#pragma unroll
        for (int j = 0; j < QRY_KPT; ++j) {
            const uint32_t ptr = lc[j].w;
            const bool linked = ptr > START && (uint64_t)(ptr - START) < D.n_high;
            const uint32_t* hb = D.high + (uint64_t)(linked ? ptr - START : 0u) * HIGH_WORDS;
            uint32_t mm = m[j];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                h4[j][i] = (linked && mm) ? __ldg(hb + (__ffs(mm) - 1)) : 0xffffffffu;
                mm &= mm - 1;
            }
        }
#pragma unroll
        for (int j = 0; j < QRY_KPT; ++j) {
            const uint32_t u[8] = {la[j].x, la[j].y, la[j].z, la[j].w, lc[j].x, lc[j].y, lc[j].z, lc[j].w};
            r[j] = msws_estimate(D, u, m[j], h4[j]);
        }
#pragma unroll
        for (int j = 0; j < QRY_KPT; ++j) {
            const uint64_t i = base + j * stride;
            if (i < n) __stcs(out + i, r[j]);
        }
    }
}

// Learned split query: exact count of a key in the heavy table (if admitted) plus the MSWS
// estimate (its occurrences before admission live in the sketch).
__global__ void __launch_bounds__(QRY_THREADS) k_learned_query(const uint32_t* __restrict__ keys, uint64_t n,
                                                               TableDev T, uint32_t* __restrict__ out, MswsDev D) {
    extern __shared__ __align__(16) uint32_t s_masks[];
    for (uint32_t i = threadIdx.x; i < D.n_masks; i += blockDim.x) s_masks[i] = __ldg(D.masks + i);
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t key = __ldcs(keys + i);
        uint32_t r = msws_lookup(D, s_masks, key, D.seed, D.fm_low, 0u);
        const int s = table_find(T.keys, T.slots, key);
        if (s >= 0) r += __ldcg(T.counts + s);
        __stcs(out + i, r);
    }
}

cudaError_t learned_query(const uint32_t* d_keys, uint64_t n, const TableDev& T, const MswsDev& D, const MswsLaunch& L,
                          uint32_t* d_out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + QRY_THREADS - 1) / QRY_THREADS;
    const int grid = (int)std::min<uint64_t>((uint64_t)L.query_grid, std::max<uint64_t>(1ull, want));
    k_learned_query<<<grid, QRY_THREADS, (size_t)D.n_masks * 4, st>>>(d_keys, n, T, d_out, D);
    return cudaGetLastError();
}

// ---- batched streams -------------------------------------------------------------------
// Many per-stream sketches (StreamDesc) in one arena.  A call covers the window [c0, c1) of
// the caller's flat key array, stream s being keys[key_off[s], key_off[s+1]).  Work items
// are tiles of at most INS_TILE keys of one stream; every size is read on the device, so
// the launch sequence can be recorded once in a CUDA graph and replayed on new contents.

// One block: each stream's slice of the window (flat mode: the stream clipped to [c0, c1);
// else for streams in [s_lo, s_hi) its keys [rel_lo, rel_hi) from its start), its tile count
// and the prefix sums of tiles and keys; reset the work queue.  Offsets that are not
// non-decreasing from 0 latch ST_BAD_OFFSETS and empty the window; strict (flat) mode
// latches ST_CAPACITY if the keys run past c1.
__global__ void __launch_bounds__(1024) k_batch_plan(BatchDev B, BatchWindow W, uint32_t strict, Ctl* ctl) {
    const uint32_t S = B.n_streams;
    bool bad = false;
    for (uint32_t s = threadIdx.x; s < S; s += blockDim.x)
        bad |= __ldcg(B.key_off + s + 1) < __ldcg(B.key_off + s);
    bad = __syncthreads_or(bad) || __ldcg(B.key_off) != 0;
    const uint64_t total = __ldcg(B.key_off + S);
    const uint64_t e = bad ? W.c0 : umin64(W.c1, total);
    const uint64_t b0 = umin64(W.c0, e);
    for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
        const uint64_t o0 = __ldcg(B.key_off + s), o1 = __ldcg(B.key_off + s + 1);
        uint64_t lo, hi;
        if (bad) {
            lo = hi = 0;
        } else if (W.flat) {
            lo = umin64(e, max(o0, b0));
            hi = umin64(e, max(o1, lo));
        } else if (s >= W.s_lo && s < W.s_hi) {
            const uint64_t len = o1 - o0;
            lo = o0 + umin64(W.rel_lo, len);
            hi = o0 + umin64(W.rel_hi, len);
        } else {
            lo = hi = o0;
        }
        B.lo[s] = lo;
        B.hi[s] = hi;
        B.item_off[s] = (uint32_t)((hi - lo + INS_TILE - 1) / INS_TILE);
        B.wpre[s] = (uint32_t)(hi - lo);
    }
    __syncthreads();
    // the same work items in the grouped (size-class) order of the pass-1 launches
    for (uint32_t k = threadIdx.x; k < S; k += blockDim.x) {
        const uint32_t s = __ldg(B.cls_streams + k);
        B.cls_item_off[k] = B.item_off[s];
    }
    __syncthreads();
    const uint32_t items = block_scan_array(B.item_off, S);
    const uint32_t keys = block_scan_array(B.wpre, S);
    block_scan_array(B.cls_item_off, S);
    for (uint32_t c = threadIdx.x; c < MAX_SIZE_CLASSES; c += blockDim.x) B.work[c] = 0;
    if (threadIdx.x == 0) {
        B.item_off[S] = items;
        B.cls_item_off[S] = items;
        B.wpre[S] = keys;
        B.win[0] = 0;
        B.win[1] = keys;
        if (bad) atomicOr(&ctl->status, ST_BAD_OFFSETS);
        if (strict && !bad && total > W.c1) atomicOr(&ctl->status, ST_CAPACITY);
    }
}

// The stream of work item `it` (< item_off[n_streams]): the last s with item_off[s] <= it.
// Called by a whole warp: each step probes 32 evenly spaced offsets, so 512 streams take two
// dependent loads instead of nine.
__device__ __forceinline__ uint32_t stream_of_item_warp(const BatchDev& B, uint32_t it) {
    const int lane = threadIdx.x & 31;
    uint32_t lo = 0, hi = B.n_streams;  // item_off[lo] <= it; the answer lies in [lo, hi)
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + lane * step;
        const bool le = idx < hi && __ldcg(B.item_off + idx) <= it;
        const uint32_t bal = __ballot_sync(0xffffffffu, le);  // lane 0 always holds
        const uint32_t last = 31 - __clz(bal);
        lo += last * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// The grouped index k in [k_lo, k_hi) whose items hold work item `it` (cls_item_off[k] <=
// it), by a whole warp as stream_of_item_warp.
__device__ __forceinline__ uint32_t group_of_item_warp(const BatchDev& B, uint32_t it, uint32_t k_lo, uint32_t k_hi) {
    const int lane = threadIdx.x & 31;
    uint32_t lo = k_lo, hi = k_hi;
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + lane * step;
        const bool le = idx < hi && __ldcg(B.cls_item_off + idx) <= it;
        const uint32_t bal = __ballot_sync(0xffffffffu, le);  // lane 0 always holds
        const uint32_t last = 31 - __clz(bal);
        lo += last * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// Pass 1 over a batch: a persistent grid pulls tiles from the work queue; a tile's keys
// all belong to one stream, so they hash with its descriptor and the tile's shared-memory
// merge table never mixes sketches.  Everything after hashing is the single-sketch pass 1.
// One launch covers the streams [k_lo, k_hi) of the size-class grouped order (work counter
// `cls`), so each size class runs with its own lanes per key.
template <int AGG, int LPK>
__global__ void __launch_bounds__(INS_THREADS, INS_MIN_CTAS) k_batch_insert(const uint32_t* __restrict__ keys, MswsDev D,
                                                                 BatchDev B, uint32_t k_lo, uint32_t k_hi,
                                                                 uint32_t cls) {
    extern __shared__ __align__(128) uint8_t smem[];
    const InsShared S = ins_carve(smem, D.n_masks);
    __shared__ uint32_t s_item, s_stream;
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    for (uint32_t i = tid; i < D.n_masks; i += blockDim.x) S.masks[i] = __ldg(D.masks + i);
    for (int i = tid; i < AGG_SLOTS; i += blockDim.x) {
        S.akey[i] = AGG_EMPTY;
        S.acnt[i] = 0;
    }
    if (tid == 0) {
        S.misc[0] = 0;
        S.misc[1] = 0;
        S.misc[2] = D.route == 2 ? ROUTE_FUSED : ROUTE_PRELOAD;
    }
    const uint32_t item_lo = __ldcg(B.cls_item_off + k_lo), n_items = __ldcg(B.cls_item_off + k_hi);
    for (;;) {
        if (wid == 0) {  // warp 0 takes the next work item and finds its stream
            uint32_t it = 0;
            if (lane == 0) it = item_lo + atomicAdd(B.work + cls, 1u);
            it = __shfl_sync(0xffffffffu, it, 0);
            uint32_t s = 0, first = 0;
            if (it < n_items) {
                const uint32_t k = group_of_item_warp(B, it, k_lo, k_hi);
                s = __ldg(B.cls_streams + k);
                first = __ldcg(B.cls_item_off + k);
            }
            if (lane == 0) {
                s_item = it - first;  // the item's index within its stream
                s_stream = it < n_items ? s : 0xffffffffu;
            }
        }
        __syncthreads();
        if (s_stream == 0xffffffffu) break;
        const uint32_t s = s_stream;
        const uint32_t it_local = s_item;
        const StreamDesc* sd = B.desc + s;
        const uint32_t seed = __ldg(&sd->seed), base = __ldg(&sd->low_base);
        const FastMod fm{__ldg(&sd->fm_low.M), __ldg(&sd->fm_low.d), 0u};
        const uint64_t t0 = __ldcg(B.lo + s) + (uint64_t)it_local * INS_TILE;
        const int cnt = (int)umin64(INS_TILE, __ldcg(B.hi + s) - t0);
        const int route = (int)S.misc[2];
        for (int b = wid * 32; b < cnt; b += INS_THREADS) {
            const int c = min(32, cnt - b);
            const uint32_t k = lane < c ? __ldcs(keys + t0 + b + lane) : 0u;
            insert_group<AGG, LPK>(D, S, k, c, true, route, 0, seed, fm, base);
        }
        __syncthreads();
        if (tid == 0) {
            if (D.route == 0) S.misc[2] = S.misc[1] * 16u < (uint32_t)cnt ? ROUTE_FUSED : ROUTE_PRELOAD;
            S.misc[1] = 0;
        }
        if (AGG == AGG_BLOCK) drain_table<LPK>(D, S, seed, fm, base);
        __syncthreads();
    }
    if (tid == 0 && S.misc[0]) atomicAdd(&D.ctl->dropped, (unsigned long long)S.misc[0]);
}

// Query over a batch: static tiles, each stream's keys with its own descriptor.
__global__ void __launch_bounds__(QRY_THREADS) k_batch_query(const uint32_t* __restrict__ keys,
                                                             uint32_t* __restrict__ out, MswsDev D, BatchDev B) {
    extern __shared__ __align__(16) uint32_t s_masks[];
    __shared__ uint32_t s_stream;
    for (uint32_t i = threadIdx.x; i < D.n_masks; i += blockDim.x) s_masks[i] = __ldg(D.masks + i);
    const uint32_t n_items = __ldcg(B.item_off + B.n_streams);
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
        if (threadIdx.x < 32) {
            const uint32_t s = stream_of_item_warp(B, it);
            if (threadIdx.x == 0) s_stream = s;
        }
        __syncthreads();
        const uint32_t s = s_stream;
        __syncthreads();
        const StreamDesc* sd = B.desc + s;
        const uint32_t seed = __ldg(&sd->seed), base = __ldg(&sd->low_base);
        const FastMod fm{__ldg(&sd->fm_low.M), __ldg(&sd->fm_low.d), 0u};
        const uint64_t t0 = __ldcg(B.lo + s) + (uint64_t)(it - __ldcg(B.item_off + s)) * INS_TILE;
        const uint32_t cnt = (uint32_t)umin64(INS_TILE, __ldcg(B.hi + s) - t0);
        constexpr int PER = INS_TILE / QRY_THREADS;
        uint32_t k[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const uint32_t i = threadIdx.x + j * QRY_THREADS;
            k[j] = i < cnt ? __ldcs(keys + t0 + i) : 0u;
        }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const uint32_t i = threadIdx.x + j * QRY_THREADS;
            const uint32_t r = msws_lookup(D, s_masks, k[j], seed, fm, base);
            if (i < cnt) __stcs(out + t0 + i, r);
        }
    }
}

// ---- launchers ----------------------------------------------------------------------------

// Pass-1 kernels by aggregation mode and lanes per key (1, 2, 4, 8, 16, 32).
int lpk_index(int lpk) {
    return lpk == 4 ? 0 : lpk == 16 ? 2 : lpk == 32 ? 3 : lpk == 2 ? 4 : lpk == 1 ? 5 : 1;
}

template <int AGG>
const void* ins_fn(int li, bool batch) {
    switch (li) {
        case 0: return batch ? (const void*)k_batch_insert<AGG, 4> : (const void*)k_msws_insert<AGG, 4>;
        case 2: return batch ? (const void*)k_batch_insert<AGG, 16> : (const void*)k_msws_insert<AGG, 16>;
        case 3: return batch ? (const void*)k_batch_insert<AGG, 32> : (const void*)k_msws_insert<AGG, 32>;
        case 4: return batch ? (const void*)k_batch_insert<AGG, 2> : (const void*)k_msws_insert<AGG, 2>;
        case 5: return batch ? (const void*)k_batch_insert<AGG, 1> : (const void*)k_msws_insert<AGG, 1>;
        default: return batch ? (const void*)k_batch_insert<AGG, 8> : (const void*)k_msws_insert<AGG, 8>;
    }
}

const void* ins_fn(int agg, int li, bool batch) {
    return agg == AGG_BLOCK ? ins_fn<AGG_BLOCK>(li, batch)
           : agg == AGG_WARP ? ins_fn<AGG_WARP>(li, batch)
                             : ins_fn<AGG_NONE>(li, batch);
}

// Persistent pass-1 grid: ctas_per_sm CTAs per SM (0 = as many as fit), at most the occupancy.
int ins_grid(const MswsLaunch& L, int agg, int li) {
    const int occ = std::max(1, L.ins_occ[agg][li]);
    const int per = L.ctas_per_sm > 0 ? std::min(L.ctas_per_sm, occ) : occ;
    return L.num_sms * per;
}

cudaError_t msws_configure(int device, uint32_t n_masks, MswsLaunch* L) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    L->num_sms = prop.multiProcessorCount;
    // The dynamic shared-memory cap is a per-kernel attribute shared by every sketch of the
    // process: set it for the largest mask table (16384 words); the launch passes the actual size.
    const size_t ins_smem = msws_insert_smem(n_masks);
    for (int agg = 0; agg < 3; ++agg)
        for (int li = 0; li < LPK_VARIANTS; ++li)
            for (int batch = 0; batch < 2; ++batch) {
                const void* fn = ins_fn(agg, li, batch != 0);
                e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)msws_insert_smem(16384));
                if (e != cudaSuccess) return e;
                if (!batch) {
                    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&L->ins_occ[agg][li], fn, INS_THREADS, ins_smem);
                    if (e != cudaSuccess) return e;
                }
            }
    e = cudaFuncSetAttribute((const void*)k_msws_query, cudaFuncAttributeMaxDynamicSharedMemorySize, 16384 * 4);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void*)k_learned_query, cudaFuncAttributeMaxDynamicSharedMemorySize, 16384 * 4);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void*)k_batch_query, cudaFuncAttributeMaxDynamicSharedMemorySize, 16384 * 4);
    if (e != cudaSuccess) return e;
    int occ = 0;
    L->insert_grid = prop.multiProcessorCount * std::max(1, L->ins_occ[AGG_BLOCK][1]);
    for (const void* fn : {(const void*)k_msws_repair<false>, (const void*)k_msws_repair<true>}) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msws_repair_smem());
        if (e != cudaSuccess) return e;
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_msws_repair<true>, REPAIR_THREADS, msws_repair_smem());
    if (e != cudaSuccess) return e;
    int occ_single = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_single, k_msws_repair<false>, REPAIR_THREADS,
                                                      msws_repair_smem());
    occ = std::min(occ, occ_single);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    L->repair_grid = prop.multiProcessorCount * (occ < 2 ? occ : 2);
    L->query_grid = prop.multiProcessorCount * 8;
    return cudaSuccess;
}

// Launch with programmatic stream serialization: the kernel may be scheduled while the
// previous kernel of the stream drains (hiding the launch gap between the dependent passes);
// each kernel launched this way calls griddep_wait() before it reads what a kernel writes.
// A driver that refuses the attribute next to a cooperative launch gets the plain one.
cudaError_t launch_pdl(const void* fn, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void** args,
                       bool cooperative) {
    static bool coop_pdl_refused = false;
    if (cooperative && coop_pdl_refused) return cudaLaunchCooperativeKernel(fn, grid, block, args, smem, st);
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    at[1].id = cudaLaunchAttributeCooperative;
    at[1].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = cooperative ? 2 : 1;
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    if (e == cudaSuccess || !cooperative) return e;
    (void)cudaGetLastError();  // a refused configuration is not sticky
    coop_pdl_refused = true;
    return cudaLaunchCooperativeKernel(fn, grid, block, args, smem, st);
}

cudaError_t msws_insert_pass(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, int agg,
                             cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const size_t smem = msws_insert_smem(D.n_masks);
    const int li = lpk_index(L.lanes_per_key);
    MswsDev Dc = D;
    // Waves of one tile per CTA, tiles of at most T keys; the keys spread evenly over the
    // tiles of that many waves, so the last wave leaves no CTA idle (a 943,718-key chunk with
    // T = 1024 on 592 CTAs: 1,180 tiles of 800 keys instead of 922 of 1024).  Tiles stay
    // multiples of 4 keys for the 16-byte TMA copies.
    const uint64_t T = (L.tile_keys >= 256 && L.tile_keys <= INS_TILE) ? (uint64_t)L.tile_keys : (uint64_t)INS_TILE;
    const uint64_t G = (uint64_t)ins_grid(L, agg, li);
    const uint64_t waves = (n + G * T - 1) / (G * T);
    const uint64_t even = (((n + waves * G - 1) / (waves * G)) + 3) & ~3ull;
    Dc.ins_tile = (uint32_t)std::min<uint64_t>(T, std::max<uint64_t>(256ull, even));
    const uint64_t tiles = (n + Dc.ins_tile - 1) / Dc.ins_tile;
    const int grid = (int)std::min<uint64_t>(G, std::max<uint64_t>(1ull, tiles));
    void* args[] = {(void*)&d_keys, (void*)&n, (void*)&Dc};
    return launch_pdl(ins_fn(agg, li, false), dim3(grid), dim3(INS_THREADS), smem, st, args, false);
}

cudaError_t msws_repair(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    MswsDev Dc = D;
    BatchDev Bn{};
    void* args[] = {(void*)&d_keys, (void*)&n, (void*)&Dc, (void*)&Bn};
    return launch_pdl((const void*)k_msws_repair<false>, dim3(L.repair_grid), dim3(REPAIR_THREADS), msws_repair_smem(),
                      st, args, true);
}

cudaError_t batch_plan(const BatchDev& B, Ctl* ctl, const BatchWindow& W, bool strict, cudaStream_t st) {
    k_batch_plan<<<1, 1024, 0, st>>>(B, W, strict ? 1u : 0u, ctl);
    return cudaGetLastError();
}

cudaError_t batch_insert_pass(const uint32_t* d_keys, const MswsDev& D, const BatchDev& B, const MswsLaunch& L,
                              int agg, int lanes_per_key, uint32_t k_lo, uint32_t k_hi, uint32_t cls, cudaStream_t st) {
    const size_t smem = msws_insert_smem(D.n_masks);
    const int li = lpk_index(lanes_per_key);
    MswsDev Dc = D;
    BatchDev Bc = B;
    void* args[] = {(void*)&d_keys, (void*)&Dc, (void*)&Bc, (void*)&k_lo, (void*)&k_hi, (void*)&cls};
    return cudaLaunchKernel(ins_fn(agg, li, true), dim3(ins_grid(L, agg, li)), dim3(INS_THREADS), args, smem, st);
}

// d_keys: the caller's flat key array (the window is described by the plan).
cudaError_t batch_repair(const uint32_t* d_window, const MswsDev& D, const BatchDev& B, const MswsLaunch& L,
                         cudaStream_t st) {
    MswsDev Dc = D;
    BatchDev Bc = B;
    uint64_t n = 0;  // read from the window on the device
    void* args[] = {(void*)&d_window, (void*)&n, (void*)&Dc, (void*)&Bc};
    return cudaLaunchCooperativeKernel((const void*)k_msws_repair<true>, dim3(L.repair_grid), dim3(REPAIR_THREADS),
                                       args, msws_repair_smem(), st);
}

cudaError_t batch_query(const uint32_t* d_keys, uint32_t* d_out, const MswsDev& D, const BatchDev& B,
                        const MswsLaunch& L, cudaStream_t st) {
    k_batch_query<<<L.query_grid, QRY_THREADS, (size_t)D.n_masks * 4, st>>>(d_keys, d_out, D, B);
    return cudaGetLastError();
}

cudaError_t msws_query(const uint32_t* d_keys, uint64_t n, uint32_t* d_out, const MswsDev& D, const MswsLaunch& L,
                       cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + QRY_THREADS * QRY_KPT - 1) / (QRY_THREADS * QRY_KPT);
    const int grid = (int)umin64((uint64_t)L.query_grid, std::max<uint64_t>(1ull, want));
    MswsDev Dc = D;
    void* args[] = {(void*)&d_keys, (void*)&n, (void*)&d_out, (void*)&Dc};
    return launch_pdl((const void*)k_msws_query, dim3(grid), dim3(QRY_THREADS), (size_t)D.n_masks * 4, st, args, false);
}

}  // namespace qsb
