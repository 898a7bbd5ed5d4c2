// qs_cm.cu — plain count-min ("thread sketch", Algorithm 1 of the paper), the in-GPU
// baseline.  Reference: include/sketch/device_sketch/device_sketch_v0.h
//   insert_kernel :13-55 (thread per key, m rows, atomicAdd), search_kernel :58-101 (min).
// Row j hashes with its own seed: hv = key * seed[j], column hv % n (:48-52, :94-97).
// Counter additions commute, so any schedule gives the sequential result.
#include "qs_kernels.h"

namespace qsb {

constexpr int CM_THREADS = 256;

template <int AGG>
__global__ void __launch_bounds__(CM_THREADS) k_cm_insert(const uint32_t* __restrict__ keys, uint64_t n, CmDev D) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? __ldcs(keys + i) : 0u;
        uint32_t c = valid ? 1u : 0u;
        if (AGG) {
            const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
            const uint32_t peers = __match_any_sync(0xffffffffu, key) & vmask;
            c = (valid && lane == __ffs(peers) - 1) ? (uint32_t)__popc(peers) : 0u;
        }
        if (c) {
            for (uint32_t j = 0; j < D.rows; ++j) {
                const uint32_t col = fast_mod(D.fm, key * D.seeds[j]);
                atomicAdd(D.table + (uint64_t)j * D.n + col, c);
            }
        }
    }
}

// CM_QPT keys per thread in flight: every row's counter of all of them is loaded before any
// is used, so a thread waits one L2 round trip per CM_QPT keys instead of per key.
constexpr int CM_QPT = 4;

__global__ void __launch_bounds__(CM_THREADS) k_cm_query(const uint32_t* __restrict__ keys, uint64_t n,
                                                         uint32_t* __restrict__ out, CmDev D) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += stride * CM_QPT) {
        uint32_t key[CM_QPT], c[CM_QPT];
#pragma unroll
        for (int q = 0; q < CM_QPT; ++q) {
            const uint64_t i = base + q * stride;
            key[q] = i < n ? __ldcs(keys + i) : 0u;
            c[q] = 0xffffffffu;
        }
        for (uint32_t j = 0; j < D.rows; ++j) {
            const uint32_t sd = D.seeds[j];
            const uint32_t* row = D.table + (uint64_t)j * D.n;
            uint32_t v[CM_QPT];
#pragma unroll
            for (int q = 0; q < CM_QPT; ++q) v[q] = __ldg(row + fast_mod(D.fm, key[q] * sd));
#pragma unroll
            for (int q = 0; q < CM_QPT; ++q) c[q] = min(c[q], v[q]);
        }
#pragma unroll
        for (int q = 0; q < CM_QPT; ++q) {
            const uint64_t i = base + q * stride;
            if (i < n) __stcs(out + i, c[q]);
        }
    }
}

// ---- one-level bucket sketch (the reference's warp sketch, device_sketch_v1.h:50-61, 135-158,
// and sub-warp sketch, device_sketch_v2.h:54-64, 156-185): bucket b = hv % n of `rows` u32 counters, the
// key's mask word (bit i selects counter i) from the table at hv % H; insert adds 1 to every
// selected counter, query is their minimum.  Counter additions commute, so any schedule gives
// the sequential result.
template <int AGG>
__global__ void __launch_bounds__(CM_THREADS) k_bucket_insert(const uint32_t* __restrict__ keys, uint64_t n,
                                                              CmDev D) {
    extern __shared__ __align__(16) uint32_t s_masks[];
    for (uint32_t i = threadIdx.x; i < D.n_masks; i += blockDim.x) s_masks[i] = __ldg(D.masks + i);
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? __ldcs(keys + i) : 0u;
        uint32_t c = valid ? 1u : 0u;
        if (AGG) {
            const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
            const uint32_t peers = __match_any_sync(0xffffffffu, key) & vmask;
            c = (valid && lane == __ffs(peers) - 1) ? (uint32_t)__popc(peers) : 0u;
        }
        if (c) {
            const uint32_t hv = key * D.seeds[0];
            uint32_t* bucket = D.table + (uint64_t)fast_mod(D.fm, hv) * D.rows;
            for (uint32_t m = s_masks[fast_mod(D.fm_mask, hv)]; m; m &= m - 1) atomicAdd(bucket + (__ffs(m) - 1), c);
        }
    }
}

__global__ void __launch_bounds__(CM_THREADS) k_bucket_query(const uint32_t* __restrict__ keys, uint64_t n,
                                                             uint32_t* __restrict__ out, CmDev D) {
    extern __shared__ __align__(16) uint32_t s_masks[];
    for (uint32_t i = threadIdx.x; i < D.n_masks; i += blockDim.x) s_masks[i] = __ldg(D.masks + i);
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += stride * CM_QPT) {
        uint32_t c[CM_QPT], m[CM_QPT];
        const uint32_t* bucket[CM_QPT];
#pragma unroll
        for (int q = 0; q < CM_QPT; ++q) {
            const uint64_t i = base + q * stride;
            const uint32_t hv = (i < n ? __ldcs(keys + i) : 0u) * D.seeds[0];
            bucket[q] = D.table + (uint64_t)fast_mod(D.fm, hv) * D.rows;
            m[q] = s_masks[fast_mod(D.fm_mask, hv)];
            c[q] = 0xffffffffu;
        }
        // up to 32 counters per mask; the loads of all CM_QPT keys' first counters go together
        for (;;) {
            bool any = false;
            uint32_t v[CM_QPT];
#pragma unroll
            for (int q = 0; q < CM_QPT; ++q) {
                v[q] = m[q] ? __ldg(bucket[q] + (__ffs(m[q]) - 1)) : 0xffffffffu;
                any |= m[q] != 0;
            }
            if (!any) break;
#pragma unroll
            for (int q = 0; q < CM_QPT; ++q) {
                c[q] = min(c[q], v[q]);
                m[q] &= m[q] - 1;
            }
        }
#pragma unroll
        for (int q = 0; q < CM_QPT; ++q) {
            const uint64_t i = base + q * stride;
            if (i < n) __stcs(out + i, c[q]);
        }
    }
}

// Mask tables above 12288 words need the opt-in dynamic shared memory.
static cudaError_t bucket_smem(const void* fn, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t cm_insert(const uint32_t* d_keys, uint64_t n, const CmDev& D, int agg, int grid, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + CM_THREADS - 1) / CM_THREADS;
    const int g = (int)std::min<uint64_t>((uint64_t)grid, std::max<uint64_t>(1, want));
    if (D.masks) {
        const size_t smem = (size_t)D.n_masks * 4;
        const void* fn = agg ? (const void*)k_bucket_insert<1> : (const void*)k_bucket_insert<0>;
        cudaError_t e = bucket_smem(fn, smem);
        if (e != cudaSuccess) return e;
        if (agg)
            k_bucket_insert<1><<<g, CM_THREADS, smem, st>>>(d_keys, n, D);
        else
            k_bucket_insert<0><<<g, CM_THREADS, smem, st>>>(d_keys, n, D);
        return cudaGetLastError();
    }
    if (agg)
        k_cm_insert<1><<<g, CM_THREADS, 0, st>>>(d_keys, n, D);
    else
        k_cm_insert<0><<<g, CM_THREADS, 0, st>>>(d_keys, n, D);
    return cudaGetLastError();
}

cudaError_t cm_query(const uint32_t* d_keys, uint64_t n, uint32_t* d_out, const CmDev& D, int grid, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + (uint64_t)CM_THREADS * CM_QPT - 1) / ((uint64_t)CM_THREADS * CM_QPT);
    const int g = (int)std::min<uint64_t>((uint64_t)grid, std::max<uint64_t>(1, want));
    if (D.masks) {
        const size_t smem = (size_t)D.n_masks * 4;
        cudaError_t e = bucket_smem((const void*)k_bucket_query, smem);
        if (e != cudaSuccess) return e;
        k_bucket_query<<<g, CM_THREADS, smem, st>>>(d_keys, n, d_out, D);
        return cudaGetLastError();
    }
    k_cm_query<<<g, CM_THREADS, 0, st>>>(d_keys, n, d_out, D);
    return cudaGetLastError();
}

}  // namespace qsb
