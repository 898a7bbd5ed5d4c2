// qs_learned.cu — routing of the learned heavy-hitter split: exact-table lookups, hit counting,
// the per-chunk skip bitmap for the sketch, table admission, and distinct-key extraction.
#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {

constexpr int RT_THREADS = 256;
constexpr int RT_TILE = 2048;
constexpr int RT_MAP = 1024;  // per-CTA map merging hits on the same table slot

// Per tile of 2048 keys (warp w, round r: keys [r*256 + w*32, +32) of the tile, so each warp
// writes whole 32-bit words of the skip bitmap): keys found in the exact table count there
// (merged per tile in shared memory) and are marked in the skip bitmap.  While R.collect is
// set, the others are gathered once per warp into a per-tile shared list that is appended to
// the miss list with one global reservation per tile (the list's order is unspecified).
__global__ void __launch_bounds__(RT_THREADS) k_route(const uint32_t* __restrict__ keys, uint64_t n, TableDev T,
                                                      RouteDev R) {
    __shared__ uint32_t mslot[RT_MAP], mcnt[RT_MAP];
    __shared__ uint32_t smiss[RT_TILE];
    __shared__ uint32_t s_nmiss, s_base;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < RT_MAP; i += RT_THREADS) {
        mslot[i] = 0xffffffffu;
        mcnt[i] = 0;
    }
    if (tid == 0) s_nmiss = 0;
    __syncthreads();
    for (uint64_t t0 = (uint64_t)blockIdx.x * RT_TILE; t0 < n; t0 += (uint64_t)gridDim.x * RT_TILE) {
        for (int r = 0; r < RT_TILE / RT_THREADS; ++r) {
            const uint64_t i = t0 + r * RT_THREADS + wid * 32 + lane;
            const bool v = i < n;
            const uint32_t key = v ? __ldcs(keys + i) : 0u;
            const int s = v ? table_find(T.keys, T.slots, key) : -1;
            const bool hit = s >= 0;
            const uint32_t hb = __ballot_sync(0xffffffffu, hit);
            if (lane == 0 && t0 + r * RT_THREADS + wid * 32 < n) R.skip[(i >> 5)] = hb;
            // hits: merge equal slots of the warp, then of the tile
            if (hb) {
                const uint32_t hp = __match_any_sync(0xffffffffu, hit ? (uint32_t)s : 0xffffffffu) & hb;
                if (hit && lane == __ffs(hp) - 1) {
                    const uint32_t c = __popc(hp);
                    uint32_t h = mix32((uint32_t)s) & (RT_MAP - 1);
                    bool done = false;
                    for (int p = 0; p < 16 && !done; ++p, h = (h + 1) & (RT_MAP - 1)) {
                        const uint32_t prev = atomicCAS(mslot + h, 0xffffffffu, (uint32_t)s);
                        if (prev == 0xffffffffu || prev == (uint32_t)s) {
                            atomicAdd(mcnt + h, c);
                            done = true;
                        }
                    }
                    if (!done) atomicAdd(T.counts + s, c);
                }
            }
            if (R.collect) {  // misses: one entry per distinct key of the warp
                const bool miss = v && !hit;
                const uint32_t mb = __ballot_sync(0xffffffffu, miss);
                const uint32_t mp = __match_any_sync(0xffffffffu, miss ? key : 0u) & mb;
                const bool lead = miss && lane == __ffs(mp) - 1;
                const uint32_t lb = __ballot_sync(0xffffffffu, lead);
                uint32_t base = 0;
                if (lane == 0 && lb) base = atomicAdd(&s_nmiss, (uint32_t)__popc(lb));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (lead) smiss[base + __popc(lb & lanemask_lt())] = key;
            }
        }
        __syncthreads();
        for (int i = tid; i < RT_MAP; i += RT_THREADS) {
            if (mslot[i] != 0xffffffffu) {
                atomicAdd(T.counts + mslot[i], mcnt[i]);
                mslot[i] = 0xffffffffu;
                mcnt[i] = 0;
            }
        }
        if (R.collect) {
            if (tid == 0) s_base = s_nmiss ? atomicAdd(R.n_misses, s_nmiss) : 0u;
            __syncthreads();
            const uint32_t cnt = s_nmiss;
            for (uint32_t i = tid; i < cnt; i += RT_THREADS) R.misses[s_base + i] = smiss[i];
            __syncthreads();
            if (tid == 0) s_nmiss = 0;
        }
        __syncthreads();
    }
}

// Admit keys into the exact table in the given order, one thread, so the result does not
// depend on scheduling: a key takes the first free slot along its sector probe sequence
// (the sequence table_find follows) while the table holds fewer than max_fill keys.
__global__ void k_table_admit(TableDev T, const uint32_t* __restrict__ sorted, uint32_t count) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t fill = *T.fill;
    const uint32_t nsec = T.slots / TBL_SECTOR;
    for (uint32_t j = 0; j < count && fill < T.max_fill; ++j) {
        const uint32_t key = sorted[j];
        if (key == TBL_EMPTY) continue;
        const uint32_t s0 = mix32(key) & (nsec - 1);
        bool done = false;
        for (int p = 0; p < TBL_SECTOR_PROBES && !done; ++p) {
            uint32_t* sk = T.keys + (uint64_t)((s0 + p) & (nsec - 1)) * TBL_SECTOR;
            for (int q = 0; q < TBL_SECTOR && !done; ++q) {
                if (sk[q] == key) {
                    done = true;
                } else if (sk[q] == TBL_EMPTY) {
                    sk[q] = key;
                    T.counts[(sk - T.keys) + q] = 0;
                    ++fill;
                    done = true;
                }
            }
        }
    }
    *T.fill = fill;
}

// Distinct keys: insert into an open-addressing set, then gather the occupied slots.
__global__ void k_set_insert(const uint32_t* __restrict__ keys, uint64_t n, uint32_t* set, uint32_t slots,
                             uint32_t* overflow) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t key = keys[i];
        if (key == 0xffffffffu) continue;
        uint32_t h = mix32(key) & (slots - 1);
        bool ok = false;
        for (uint32_t p = 0; p < 4096; ++p, h = (h + 1) & (slots - 1)) {
            const uint32_t prev = atomicCAS(set + h, 0xffffffffu, key);
            if (prev == 0xffffffffu || prev == key) {
                ok = true;
                break;
            }
        }
        if (!ok) atomicAdd(overflow, 1u);
    }
}

__global__ void k_set_gather(const uint32_t* __restrict__ set, uint32_t slots, uint32_t* out, uint32_t* count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
        const uint32_t k = set[i];
        if (k != 0xffffffffu) out[atomicAdd(count, 1u)] = k;
    }
}

cudaError_t route_chunk(const uint32_t* d_keys, uint64_t n, const TableDev& T, const RouteDev& R, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t tiles = (n + RT_TILE - 1) / RT_TILE;
    const int grid = (int)std::min<uint64_t>(tiles, 148ull * 8);
    k_route<<<grid, RT_THREADS, 0, st>>>(d_keys, n, T, R);
    return cudaGetLastError();
}

cudaError_t table_admit(const TableDev& T, const uint32_t* d_sorted, uint32_t count, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    k_table_admit<<<1, 1, 0, st>>>(T, d_sorted, count);
    return cudaGetLastError();
}

cudaError_t distinct_keys(const uint32_t* d_keys, uint64_t n, uint32_t* d_set, uint32_t set_slots, uint32_t* d_out,
                          uint32_t* d_count, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_set, 0xff, (size_t)set_slots * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, 8, st);
    if (e != cudaSuccess) return e;
    k_set_insert<<<148 * 8, 256, 0, st>>>(d_keys, n, d_set, set_slots, d_count + 1);
    k_set_gather<<<148 * 8, 256, 0, st>>>(d_set, set_slots, d_out, d_count);
    return cudaGetLastError();
}

}  // namespace qsb
