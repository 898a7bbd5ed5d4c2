// qs_remove.cu — REMOVE: one occurrence of each key taken out of the sketch.
//
// The reference has no deletion code; its paper defines deletion as the insertion with a
// subtraction (doc/main.tex:232, "increase or decrease the count variables").  For the
// two-level MSWS the bucket's level decides where a removal lands: a linked bucket's selected
// high counters lose one, an unlinked bucket's selected 8-bit low counters lose one, each
// floored at 0; a saturated bucket drops the removal (counted).  Removals never link or
// unlink a bucket, so within one call the result per counter is max(0, value - removals)
// whatever the order of the keys: a saturating subtraction per word, applied by a CAS loop
// after equal keys of a warp are merged (one update of c removals instead of c updates).
// Count-min: each row's counter loses one, floored at 0.
#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {

constexpr int RM_THREADS = 256;
constexpr uint32_t RM_TRIES = 1u << 22;  // CAS attempts per word before giving up (ST_TIMEOUT)

// Per-byte saturating subtraction of `dec` from *w; false if the CAS never won.
__device__ __forceinline__ bool sat_sub_bytes(uint32_t* w, uint32_t dec) {
    uint32_t old = __ldcg(w);
    for (uint32_t it = 0; it < RM_TRIES; ++it) {
        const uint32_t nw = __vsubus4(old, dec);
        if (nw == old) return true;  // every selected byte already 0
        const uint32_t prev = atomicCAS(w, old, nw);
        if (prev == old) return true;
        old = prev;
    }
    return false;
}

// Saturating subtraction of c from the u32 counter *p; false if the CAS never won.
__device__ __forceinline__ bool sat_sub_u32(uint32_t* p, uint32_t c) {
    uint32_t old = __ldcg(p);
    for (uint32_t it = 0; it < RM_TRIES; ++it) {
        const uint32_t nw = old > c ? old - c : 0u;
        if (nw == old) return true;
        const uint32_t prev = atomicCAS(p, old, nw);
        if (prev == old) return true;
        old = prev;
    }
    return false;
}

__global__ void __launch_bounds__(RM_THREADS) k_msws_remove(const uint32_t* __restrict__ keys, uint64_t n,
                                                            MswsDev D) {
    extern __shared__ __align__(16) uint32_t s_masks[];
    for (uint32_t i = threadIdx.x; i < D.n_masks; i += blockDim.x) s_masks[i] = __ldg(D.masks + i);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    bool ok = true;
    uint32_t dropped = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {  // warp-uniform
        const uint64_t i = base + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? __ldcs(keys + i) : 0u;
        const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
        const uint32_t peers = __match_any_sync(0xffffffffu, key) & vmask;
        if (!valid || lane != __ffs(peers) - 1) continue;
        const uint32_t c = __popc(peers);  // equal keys: one bucket, one mask
        const uint32_t hv = key * D.seed;
        const uint32_t b = fast_mod(D.fm_low, hv);
        const uint32_t m = s_masks[fast_mod(D.fm_mask, hv)];
        uint32_t* wp = D.low + (uint64_t)b * LOW_WORDS;
        const uint32_t ptr = __ldcg(wp + 7);
        if (ptr == SATURATED) {
            dropped += c;
        } else if (ptr > START && (uint64_t)(ptr - START) < D.n_high) {
            uint32_t* hb = D.high + (uint64_t)(ptr - START) * HIGH_WORDS;
            for (uint32_t mm = m; mm; mm &= mm - 1) ok &= sat_sub_u32(hb + (__ffs(mm) - 1), c);
        } else {
#pragma unroll
            for (int w = 0; w < 7; ++w) {
                const uint32_t nib = (m >> (4 * w)) & 0xfu;
                if (nib) ok &= sat_sub_bytes(wp + w, expand_nibble(nib) * c);
            }
        }
    }
    if (!ok) atomicOr(&D.ctl->status, ST_TIMEOUT);
    if (dropped) atomicAdd(&D.ctl->dropped, (unsigned long long)dropped);
}

__global__ void __launch_bounds__(RM_THREADS) k_cm_remove(const uint32_t* __restrict__ keys, uint64_t n, CmDev D,
                                                          uint32_t* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    bool ok = true;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? __ldcs(keys + i) : 0u;
        const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
        const uint32_t peers = __match_any_sync(0xffffffffu, key) & vmask;
        if (!valid || lane != __ffs(peers) - 1) continue;
        const uint32_t c = __popc(peers);
        if (D.masks) {  // one-level bucket sketch: the selected counters of the key's bucket
            const uint32_t hv = key * D.seeds[0];
            uint32_t* bucket = D.table + (uint64_t)fast_mod(D.fm, hv) * D.rows;
            for (uint32_t mm = __ldg(D.masks + fast_mod(D.fm_mask, hv)); mm; mm &= mm - 1)
                ok &= sat_sub_u32(bucket + (__ffs(mm) - 1), c);
            continue;
        }
        for (uint32_t j = 0; j < D.rows; ++j)
            ok &= sat_sub_u32(D.table + (uint64_t)j * D.n + fast_mod(D.fm, key * D.seeds[j]), c);
    }
    if (!ok && status) atomicOr(status, ST_TIMEOUT);
}

cudaError_t msws_remove(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + RM_THREADS - 1) / RM_THREADS;
    const int grid = (int)std::min<uint64_t>((uint64_t)L.num_sms * 8, std::max<uint64_t>(1, want));
    const size_t smem = (size_t)D.n_masks * 4;
    if (smem > 48 * 1024) {  // mask tables above 12288 words need the opt-in shared memory
        const cudaError_t e = cudaFuncSetAttribute((const void*)k_msws_remove,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_msws_remove<<<grid, RM_THREADS, smem, st>>>(d_keys, n, D);
    return cudaGetLastError();
}

cudaError_t cm_remove(const uint32_t* d_keys, uint64_t n, const CmDev& D, int grid, uint32_t* d_status,
                      cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + RM_THREADS - 1) / RM_THREADS;
    const int g = (int)std::min<uint64_t>((uint64_t)grid, std::max<uint64_t>(1, want));
    k_cm_remove<<<g, RM_THREADS, 0, st>>>(d_keys, n, D, d_status);
    return cudaGetLastError();
}

}  // namespace qsb
