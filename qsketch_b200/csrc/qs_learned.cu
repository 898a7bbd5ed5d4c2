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
// d_out; *d_count (device) receives how many.
cudaError_t distinct_sorted(const uint32_t* d_keys, uint32_t n, uint32_t* d_tmp, uint32_t* d_out, uint32_t* d_count,
                            TrainScratch& S, cudaStream_t st) {
    size_t b1 = 0, b2 = 0;
    cudaError_t e = cub::DeviceRadixSort::SortKeys(nullptr, b1, d_keys, d_tmp, n, 0, 32, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(nullptr, b2, d_tmp, d_out, d_count, n, st);
    if (e == cudaSuccess) e = S.ensure(std::max(b1, b2));
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(S.p, b1, d_keys, d_tmp, n, 0, 32, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(S.p, b2, d_tmp, d_out, d_count, n, st);
    return e;
}

// ---- training set and admission on the device ------------------------------------------------
// Scratch for the device-wide sorts and selections, grown on demand.
cudaError_t TrainScratch::ensure(size_t bytes) {
    if (bytes <= size) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    size = 0;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) size = bytes;
    return e;
}
TrainScratch::~TrainScratch() {
    if (p) cudaFree(p);
}

// Reserve the scratch of every sort and selection of a training on n keys, so training
// allocates nothing.
cudaError_t train_scratch_reserve(TrainScratch& S, uint32_t n, uint32_t set_slots) {
    (void)set_slots;
    size_t b = 0, m = 0;
    const uint32_t* u = nullptr;
    uint32_t* o = nullptr;
    const uint8_t* f = nullptr;
    uint8_t* o8 = nullptr;
    const float* fz = nullptr;
    float* oz = nullptr;
    cudaError_t e = cub::DeviceRadixSort::SortKeys(nullptr, b, u, o, n, 0, 32);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(nullptr, b, u, o, o, n);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeysDescending(nullptr, b, u, o, n, 0, 32);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, b, u, f, o, o, n);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, b, f, f, o8, o, n);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, b, fz, f, oz, o, n);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(nullptr, b, fz, oz, n, 0, 32);
    m = std::max(m, b);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairsDescending(nullptr, b, u, o, u, o, n, 0, 32);
    m = std::max(m, b);
    return e == cudaSuccess ? S.ensure(m) : e;
}

// The k-th largest (k >= 1) of n values: a descending device radix sort into d_tmp (n words),
// then element k-1 read back.
cudaError_t kth_largest(const uint32_t* d_in, uint32_t n, uint32_t k, uint32_t* d_tmp, TrainScratch& S,
                        uint32_t* h_out, cudaStream_t st) {
    size_t b = 0;
    cudaError_t e = cub::DeviceRadixSort::SortKeysDescending(nullptr, b, d_in, d_tmp, n, 0, 32, st);
    if (e == cudaSuccess) e = S.ensure(b);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeysDescending(S.p, b, d_in, d_tmp, n, 0, 32, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, d_tmp + (k - 1), 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

// Labels of the distinct warm-up keys (heavy: estimate >= thr) and their count.
__global__ void k_label(const uint32_t* __restrict__ est, uint32_t n, uint32_t thr, uint8_t* __restrict__ lab,
                        uint32_t* __restrict__ npos) {
    uint32_t c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint8_t l = __ldg(est + i) >= thr ? 1 : 0;
        lab[i] = l;
        c += l;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(npos, c);
}

// The training sample: every labelled-heavy key and the light keys whose seeded hash (murmur3
// finaliser of key ^ seed) falls below `cut` (a rate in 2^-32 units).
__global__ void k_sample(const uint32_t* __restrict__ keys, const uint8_t* __restrict__ lab, uint32_t n,
                         uint32_t seed, uint64_t cut, uint8_t* __restrict__ take) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t h = __ldg(keys + i) ^ seed;
        h ^= h >> 16;
        h *= 0x85EBCA6Bu;
        h ^= h >> 13;
        h *= 0xC2B2AE35u;
        h ^= h >> 16;
        take[i] = (lab[i] || (uint64_t)h < cut) ? 1 : 0;
    }
}

cudaError_t label_keys(const uint32_t* d_est, uint32_t n, uint32_t thr, uint8_t* d_lab, uint32_t* d_npos,
                       cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_npos, 0, 4, st);
    if (e != cudaSuccess || n == 0) return e;
    k_label<<<148 * 4, 256, 0, st>>>(d_est, n, thr, d_lab, d_npos);
    return cudaGetLastError();
}

// The training set in ascending key order: keys and labels of the sample (stable selection);
// *d_count receives its size.
cudaError_t training_set(const uint32_t* d_keys, const uint8_t* d_lab, uint32_t n, uint32_t seed, uint64_t cut,
                         uint8_t* d_take, uint32_t* d_tkeys, uint8_t* d_tlab, uint32_t* d_count, TrainScratch& S,
                         cudaStream_t st) {
    if (n) k_sample<<<148 * 4, 256, 0, st>>>(d_keys, d_lab, n, seed, cut, d_take);
    cudaError_t e = cudaGetLastError();
    size_t b1 = 0, b2 = 0;
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, b1, d_keys, d_take, d_tkeys, d_count, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, b2, d_lab, d_take, d_tlab, d_count, n, st);
    if (e == cudaSuccess) e = S.ensure(std::max(b1, b2));
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(S.p, b2, d_lab, d_take, d_tlab, d_count, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(S.p, b1, d_keys, d_take, d_tkeys, d_count, n, st);
    return e;
}

// Eligibility and confusion counts of the trained network on the labelled keys: pred = z >=
// zthr; counts[0..2] += true positives, false positives, false negatives.
__global__ void k_predict(const float* __restrict__ z, const uint8_t* __restrict__ lab, uint32_t n, float zthr,
                          uint8_t* __restrict__ pred, uint32_t* __restrict__ counts) {
    uint32_t tp = 0, fp = 0, fn = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool p = z[i] >= zthr, l = lab[i] != 0;
        pred[i] = p ? 1 : 0;
        tp += p && l;
        fp += p && !l;
        fn += !p && l;
    }
    tp = __reduce_add_sync(0xffffffffu, tp);
    fp = __reduce_add_sync(0xffffffffu, fp);
    fn = __reduce_add_sync(0xffffffffu, fn);
    if ((threadIdx.x & 31) == 0) {
        if (tp) atomicAdd(counts + 0, tp);
        if (fp) atomicAdd(counts + 1, fp);
        if (fn) atomicAdd(counts + 2, fn);
    }
}

// The logit below which `quantile` (0..1) of the labelled-heavy keys fall: their logits
// selected and sorted ascending, element floor(quantile * (npos - 1)) read back.
cudaError_t positive_logit_quantile(const float* d_z, const uint8_t* d_lab, uint32_t n, uint32_t npos,
                                    double quantile, float* d_tmp, float* d_tmp2, uint32_t* d_count,
                                    TrainScratch& S, float* h_out, cudaStream_t st) {
    size_t b1 = 0, b2 = 0;
    cudaError_t e = cub::DeviceSelect::Flagged(nullptr, b1, d_z, d_lab, d_tmp, d_count, n, st);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(nullptr, b2, d_tmp, d_tmp2, npos, 0, 32, st);
    if (e == cudaSuccess) e = S.ensure(std::max(b1, b2));
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(S.p, b1, d_z, d_lab, d_tmp, d_count, n, st);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(S.p, b2, d_tmp, d_tmp2, npos, 0, 32, st);
    const uint32_t at = (uint32_t)std::floor(quantile * (double)(npos - 1));
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, d_tmp2 + at, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

cudaError_t predict_keys(const float* d_z, const uint8_t* d_lab, uint32_t n, float zthr, uint8_t* d_pred,
                         uint32_t* d_counts, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_counts, 0, 12, st);
    if (e != cudaSuccess || n == 0) return e;
    k_predict<<<148 * 4, 256, 0, st>>>(d_z, d_lab, n, zthr, d_pred, d_counts);
    return cudaGetLastError();
}

// The predicted-heavy keys ranked by the sketch's estimate, highest first, ties in ascending
// key order (the keys come in ascending order and the descending radix sort is stable):
// d_okeys receives them, *d_count how many.
cudaError_t rank_predicted(const uint32_t* d_keys, const uint32_t* d_est, const uint8_t* d_pred, uint32_t n,
                           uint32_t* d_hkeys, uint32_t* d_hest, uint32_t* d_okeys, uint32_t* d_oest,
                           uint32_t* d_count, TrainScratch& S, uint32_t* h_count, cudaStream_t st) {
    size_t b1 = 0, b2 = 0, b3 = 0;
    cudaError_t e = cub::DeviceSelect::Flagged(nullptr, b1, d_keys, d_pred, d_hkeys, d_count, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, b2, d_est, d_pred, d_hest, d_count, n, st);
    if (e == cudaSuccess) e = S.ensure(std::max(b1, b2));
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(S.p, b2, d_est, d_pred, d_hest, d_count, n, st);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(S.p, b1, d_keys, d_pred, d_hkeys, d_count, n, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_count, d_count, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess || *h_count == 0) return e;
    const uint32_t H = *h_count;
    e = cub::DeviceRadixSort::SortPairsDescending(nullptr, b3, d_hest, d_oest, d_hkeys, d_okeys, H, 0, 32, st);
    if (e == cudaSuccess) e = S.ensure(b3);
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairsDescending(S.p, b3, d_hest, d_oest, d_hkeys, d_okeys, H, 0, 32, st);
    return e;
}

}  // namespace qsb
