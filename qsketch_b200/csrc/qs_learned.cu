// qs_learned.cu — the learned heavy-hitter split's routing (exact-table lookups, hit counting,
// the per-chunk skip bitmap for the sketch), host-side table admission, and the training set
// (distinct warm-up keys, per-epoch example order).
#include <cub/cub.cuh>

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

// Admission into the exact table, on the host over a mirror of the table's key array (the
// device array changes only by admission): in the given order, a key takes the first free
// slot along its sector probe sequence — the sequence table_find follows — while the table
// holds fewer than max_fill keys.  Returns the new fill; the caller uploads the mirror.
uint32_t table_admit_host(uint32_t* keys, uint32_t slots, const uint32_t* order, uint32_t count, uint32_t fill,
                          uint32_t max_fill) {
    const uint32_t nsec = slots / TBL_SECTOR;
    for (uint32_t j = 0; j < count && fill < max_fill; ++j) {
        const uint32_t key = order[j];
        if (key == TBL_EMPTY) continue;
        const uint32_t s0 = mix32(key) & (nsec - 1);
        bool done = false;
        for (int p = 0; p < TBL_SECTOR_PROBES && !done; ++p) {
            uint32_t* sk = keys + (uint64_t)((s0 + p) & (nsec - 1)) * TBL_SECTOR;
            for (int q = 0; q < TBL_SECTOR && !done; ++q) {
                if (sk[q] == key) {
                    done = true;
                } else if (sk[q] == TBL_EMPTY) {
                    sk[q] = key;  // its count slot is still 0: slots are never vacated
                    ++fill;
                    done = true;
                }
            }
        }
    }
    return fill;
}


cudaError_t route_chunk(const uint32_t* d_keys, uint64_t n, const TableDev& T, const RouteDev& R, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t tiles = (n + RT_TILE - 1) / RT_TILE;
    const int grid = (int)std::min<uint64_t>(tiles, 148ull * 8);
    k_route<<<grid, RT_THREADS, 0, st>>>(d_keys, n, T, R);
    return cudaGetLastError();
}


// A seeded bijection of [0, n): a 4-round Feistel network on 2h bits (4^h >= n), walked
// until it lands below n (each step is itself a bijection of [0, 4^h), so the walk is one
// of [0, n)).  Expected walk length <= 4.
struct FeistelPerm {
    uint32_t h, mask, n, k[4];
    __device__ __forceinline__ uint32_t step(uint32_t x) const {
        uint32_t l = x >> h, r = x & mask;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t t = l ^ (mix32(r ^ k[i]) & mask);
            l = r;
            r = t;
        }
        return (l << h) | r;
    }
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const {
        uint32_t x = step(i);
        while (x >= n) x = step(x);
        return x;
    }
};

// Training examples of one epoch in a seeded order: out[i] = in[perm(i)].
__global__ void k_permute_examples(const uint32_t* __restrict__ keys, const uint8_t* __restrict__ labels,
                                   FeistelPerm P, uint32_t* __restrict__ okeys, uint8_t* __restrict__ olabels) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const uint32_t j = P(i);
        okeys[i] = __ldg(keys + j);
        olabels[i] = __ldg(labels + j);
    }
}

cudaError_t permute_examples(const uint32_t* d_keys, const uint8_t* d_labels, uint32_t n, uint64_t seed,
                             uint32_t* d_okeys, uint8_t* d_olabels, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    FeistelPerm P;
    P.n = n;
    P.h = 1;
    while ((1ull << (2 * P.h)) < n) ++P.h;
    P.mask = (1u << P.h) - 1u;
    for (int i = 0; i < 4; ++i) P.k[i] = mix32((uint32_t)(seed >> (16 * (i & 1))) ^ (0x9E3779B9u * (i + 1)));
    k_permute_examples<<<148 * 8, 256, 0, st>>>(d_keys, d_labels, P, d_okeys, d_olabels);
    return cudaGetLastError();
}

// Distinct keys in ascending order: a device radix sort into d_tmp (n words), then unique into
// d_out; *d_count (device) receives how many.  The scratch of the two passes is allocated here.
cudaError_t distinct_sorted(const uint32_t* d_keys, uint32_t n, uint32_t* d_tmp, uint32_t* d_out, uint32_t* d_count,
                            cudaStream_t st) {
    size_t b1 = 0, b2 = 0;
    cudaError_t e = cub::DeviceRadixSort::SortKeys(nullptr, b1, d_keys, d_tmp, n, 0, 32, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(nullptr, b2, d_tmp, d_out, d_count, n, st);
    if (e != cudaSuccess) return e;
    void* scratch = nullptr;
    e = cudaMalloc(&scratch, std::max<size_t>(std::max(b1, b2), 16));
    if (e != cudaSuccess) return e;
    e = cub::DeviceRadixSort::SortKeys(scratch, b1, d_keys, d_tmp, n, 0, 32, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(scratch, b2, d_tmp, d_out, d_count, n, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(scratch);
    return e;
}


}  // namespace qsb
