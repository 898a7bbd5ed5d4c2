// qs_shard.cu — routing for a bucket-sharded sketch across GPUs.
//
// A key's whole MSWS state is one low bucket and the high bucket it may link to
// (device_sketch_v3.h:228, :119, :185), so the sketch shards by bucket: bucket b belongs to
// shard floor(b * G / n_low), G contiguous ranges.  Before an insert or a query each rank
// partitions its batch by owner shard — stably, so every shard receives each rank's keys in
// their array order — and exchanges the parts with one all-to-all; the owner then applies
// them to its sketch in (rank, array) order, which is the order of the concatenated batches.
// Query estimates return with a second all-to-all and go back to their array positions.
//
// k_shard_count / k_shard_scan / k_shard_scatter form a stable counting sort by shard: a
// tile of SH_TILE keys per block, 16 consecutive keys per thread, per-(shard, tile) counts
// scanned shard-major, then each thread writes its keys after the keys of earlier threads of
// its tile and of earlier tiles.
#include "../../include/qsketch_c.h"
#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {

constexpr int SH_THREADS = 256;
constexpr int SH_PER = 16;
constexpr uint32_t SH_TILE = SH_THREADS * SH_PER;  // 4096 keys
constexpr uint32_t SH_MAX_SHARDS = 32;

// Owner of a key: its MSWS bucket hv % n_low (hv = key * seed), buckets in G contiguous ranges.
__device__ __forceinline__ uint32_t shard_of(uint32_t key, uint32_t seed, const FastMod& fm, uint64_t n_low,
                                             uint32_t G) {
    const uint64_t b = fast_mod(fm, key * seed);
    return (uint32_t)((b * G) / n_low);
}

// counts[g * ntiles + t] = keys of tile t owned by shard g.
__global__ void __launch_bounds__(SH_THREADS) k_shard_count(const uint32_t* __restrict__ keys, uint64_t n,
                                                            uint32_t seed, FastMod fm, uint64_t n_low, uint32_t G,
                                                            uint32_t* __restrict__ counts, uint32_t ntiles) {
    __shared__ uint32_t s_cnt[SH_MAX_SHARDS];
    const uint32_t t = blockIdx.x;
    for (uint32_t g = threadIdx.x; g < G; g += SH_THREADS) s_cnt[g] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)t * SH_TILE;
    for (uint32_t j = threadIdx.x; j < SH_TILE; j += SH_THREADS) {  // coalesced: counts only
        const uint64_t i = base + j;
        if (i < n) atomicAdd(&s_cnt[shard_of(__ldg(keys + i), seed, fm, n_low, G)], 1u);
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += SH_THREADS) counts[(uint64_t)g * ntiles + t] = s_cnt[g];
}

// One block: exclusive scan of counts (shard-major) in place; shard_counts[g] = keys of shard g.
__global__ void __launch_bounds__(1024) k_shard_scan(uint32_t* counts, uint32_t ntiles, uint32_t G,
                                                     uint32_t* shard_counts) {
    const uint32_t len = G * ntiles;
    const uint32_t per = (len + blockDim.x - 1) / blockDim.x;
    const uint32_t beg = min(len, threadIdx.x * per), end = min(len, beg + per);
    uint32_t sum = 0;
    for (uint32_t i = beg; i < end; ++i) sum += counts[i];
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, &total);
    for (uint32_t i = beg; i < end; ++i) {
        const uint32_t v = counts[i];
        counts[i] = run;
        run += v;
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < G; g += blockDim.x) {
        const uint32_t lo = counts[g * ntiles];
        const uint32_t hi = g + 1 < G ? counts[(g + 1) * ntiles] : total;
        shard_counts[g] = hi - lo;
    }
}

// Stable scatter: out[offset] = key, perm[offset] = its index in the batch (if perm).
__global__ void __launch_bounds__(SH_THREADS) k_shard_scatter(const uint32_t* __restrict__ keys, uint64_t n,
                                                              uint32_t seed, FastMod fm, uint64_t n_low, uint32_t G,
                                                              const uint32_t* __restrict__ offsets, uint32_t ntiles,
                                                              uint32_t* __restrict__ out, uint32_t* __restrict__ perm) {
    __shared__ uint32_t s_cnt[SH_MAX_SHARDS][SH_THREADS];  // per shard, per thread: its keys, then their prefix
    __shared__ uint32_t s_base[SH_MAX_SHARDS];
    const uint32_t t = blockIdx.x, tid = threadIdx.x;
    const uint64_t first = (uint64_t)t * SH_TILE + (uint64_t)tid * SH_PER;
    uint32_t k[SH_PER], own[SH_PER];
#pragma unroll
    for (int j = 0; j < SH_PER; ++j) {
        const uint64_t i = first + j;
        k[j] = i < n ? __ldg(keys + i) : 0u;
        own[j] = i < n ? shard_of(k[j], seed, fm, n_low, G) : SH_MAX_SHARDS;
    }
    for (uint32_t g = 0; g < G; ++g) s_cnt[g][tid] = 0;
#pragma unroll
    for (int j = 0; j < SH_PER; ++j)
        if (own[j] < G) ++s_cnt[own[j]][tid];
    for (uint32_t g = tid; g < G; g += SH_THREADS) s_base[g] = offsets[(uint64_t)g * ntiles + t];
    for (uint32_t g = 0; g < G; ++g) {  // exclusive prefix over the tile's threads, per shard
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(s_cnt[g][tid], &total);
        s_cnt[g][tid] = ex;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SH_PER; ++j) {
        const uint32_t g = own[j];
        if (g < G) {
            const uint32_t dst = s_base[g] + s_cnt[g][tid]++;
            out[dst] = k[j];
            if (perm) perm[dst] = (uint32_t)(first + j);
        }
    }
}

// out[perm[i]] = in[i]: estimates of a partitioned batch back to their array positions.
__global__ void k_shard_unpartition(const uint32_t* __restrict__ in, const uint32_t* __restrict__ perm, uint64_t n,
                                    uint32_t* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[__ldg(perm + i)] = __ldg(in + i);
}

}  // namespace qsb

using namespace qsb;

extern "C" qs_status qs_shard_partition(const uint32_t* d_keys, size_t n, uint32_t hash_seed, uint64_t n_low,
                                        uint32_t n_shards, uint32_t* d_out, uint32_t* d_perm, uint32_t* d_scratch,
                                        uint32_t* d_shard_counts, void* stream) {
    if (n_shards == 0 || n_shards > SH_MAX_SHARDS || n_low == 0 || n_low > 0xffffffffull || hash_seed == 0)
        return set_last_error("qs_shard_partition: n_shards in [1, 32], n_low in [1, 2^32), hash_seed != 0"),
               QS_ERR_INVALID_ARG;
    if (n > 0xffffffffull) return set_last_error("qs_shard_partition: at most 2^32 - 1 keys"), QS_ERR_CAPACITY;
    if ((n && (!d_keys || !d_out)) || !d_scratch || !d_shard_counts)
        return set_last_error("qs_shard_partition: null pointer"), QS_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t ntiles = (uint32_t)std::max<uint64_t>(1, (n + SH_TILE - 1) / SH_TILE);
    const FastMod fm = make_fastmod((uint32_t)n_low);
    if (n) k_shard_count<<<ntiles, SH_THREADS, 0, st>>>(d_keys, n, hash_seed, fm, n_low, n_shards, d_scratch, ntiles);
    else cudaMemsetAsync(d_scratch, 0, (size_t)n_shards * ntiles * 4, st);
    k_shard_scan<<<1, 1024, 0, st>>>(d_scratch, ntiles, n_shards, d_shard_counts);
    if (n)
        k_shard_scatter<<<ntiles, SH_THREADS, 0, st>>>(d_keys, n, hash_seed, fm, n_low, n_shards, d_scratch, ntiles,
                                                       d_out, d_perm);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return QS_ERR_CUDA;
    }
    return QS_OK;
}

extern "C" size_t qs_shard_scratch_words(size_t n, uint32_t n_shards) {
    return (size_t)n_shards * std::max<size_t>(1, (n + SH_TILE - 1) / SH_TILE);
}

extern "C" qs_status qs_shard_unpartition(const uint32_t* d_in, const uint32_t* d_perm, size_t n, uint32_t* d_out,
                                          void* stream) {
    if (n && (!d_in || !d_perm || !d_out)) return set_last_error("qs_shard_unpartition: null pointer"), QS_ERR_INVALID_ARG;
    if (!n) return QS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = (int)std::min<uint64_t>(148 * 8, (n + 255) / 256);
    k_shard_unpartition<<<grid, 256, 0, st>>>(d_in, d_perm, n, d_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return QS_ERR_CUDA;
    }
    return QS_OK;
}
