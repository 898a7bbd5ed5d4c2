// qs_device.cuh — PTX helpers (mbarrier, TMA bulk copy), bounded waits, block scans.
#pragma once
#include "qs_common.cuh"

namespace qsb {

// ---- bounded waits -------------------------------------------------------------------
// Every spin in this library gives up after about a second and latches ST_TIMEOUT.
constexpr uint32_t SPIN_LIMIT = 1u << 23;  // iterations of ~128 ns sleeps (~1 s)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// TMA bulk copy global -> this CTA's shared memory (no tensor map, no multicast).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void tma_bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase; false after SPIN_LIMIT tries.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(64);
    }
    return false;
}

// ---- programmatic dependent launch ---------------------------------------------------
// A kernel launched with programmatic stream serialization may start while the previous
// kernel of its stream is still running; griddep_wait() returns once that kernel has
// completed and its writes are visible (at once for a kernel launched without it), so every
// such kernel calls it before it reads anything a kernel writes, and before it can return.
// griddep_launch_dependents() lets the next such kernel be scheduled before this one ends.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---- grid barrier for cooperative launches (bounded) ---------------------------------
// All blocks of the grid are co-resident (cudaLaunchCooperativeKernel).  Arrivals count up in
// one 64-bit word that is never reset: thread 0 of each block fences the block's writes and
// adds 1, and the count before its add gives the barrier's end, the next multiple of the
// grid size; it then polls the count with acquire loads until it gets there (the last block
// to arrive at once).  One returning atomic per block and no second hop through a generation
// word.  Returns false (and latches ST_TIMEOUT) if the other blocks do not arrive within the
// spin limit.
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_barrier(Ctl* ctl, uint32_t limit = SPIN_LIMIT) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned long long g = gridDim.x;
        const unsigned long long end = (atomicAdd(&ctl->bar_arrive, 1ull) / g + 1ull) * g;
        int ok = 1;
        uint32_t it = 0;
        while (ld_acquire_gpu_u64(&ctl->bar_arrive) < end) {
            if (++it > limit) {
                ok = 0;
                atomicOr(&ctl->status, ST_TIMEOUT);
                break;
            }
            if (it > 256) __nanosleep(64);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---- block-wide scans ------------------------------------------------------------------
// Exclusive scan of one value per thread (blockDim.x <= 1024, multiple of 32).
// Returns the exclusive prefix; *total receives the block sum (all threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_total;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < nw ? s_warp[lane] : 0u;
        uint32_t u = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, u, o);
            if (lane >= o) u += y;
        }
        if (lane < nw) s_warp[lane] = u - t;
        if (lane == 31) s_total = u;
    }
    __syncthreads();
    const uint32_t r = s_warp[wid] + x - v;
    *total = s_total;
    __syncthreads();
    return r;
}

// Exclusive scan in place of a shared-memory array a[0..len) by one block; returns the total
// (all threads).  Each thread owns a contiguous run.
__device__ __forceinline__ uint32_t block_scan_smem(uint32_t* a, uint32_t len) {
    const uint32_t per = (len + blockDim.x - 1) / blockDim.x;
    const uint32_t beg = min(len, threadIdx.x * per);
    const uint32_t end = min(len, beg + per);
    uint32_t sum = 0;
    for (uint32_t i = beg; i < end; ++i) sum += a[i];
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, &total);
    for (uint32_t i = beg; i < end; ++i) {
        const uint32_t t = a[i];
        a[i] = run;
        run += t;
    }
    __syncthreads();
    return total;
}

// Exclusive scan in place of a global array a[0..len) by one block; returns the total.
// a must be 16-byte aligned; each thread owns a run of a multiple of 4 entries.
__device__ __forceinline__ uint32_t block_scan_array(uint32_t* a, uint32_t len) {
    const uint32_t per = ((len + blockDim.x - 1) / blockDim.x + 3) & ~3u;
    const uint32_t beg = min(len, threadIdx.x * per);
    const uint32_t end = min(len, beg + per);
    uint32_t sum = 0, i = beg;
#pragma unroll 4
    for (; i + 4 <= end; i += 4) {
        const uint4 v = __ldcg(reinterpret_cast<const uint4*>(a + i));
        sum += v.x + v.y + v.z + v.w;
    }
    for (; i < end; ++i) sum += __ldcg(a + i);
    uint32_t total;
    uint32_t run = block_exclusive_scan(sum, &total);
    i = beg;
#pragma unroll 4
    for (; i + 4 <= end; i += 4) {
        const uint4 v = __ldcg(reinterpret_cast<const uint4*>(a + i));
        uint4 o;
        o.x = run;
        run += v.x;
        o.y = run;
        run += v.y;
        o.z = run;
        run += v.z;
        o.w = run;
        run += v.w;
        __stcg(reinterpret_cast<uint4*>(a + i), o);
    }
    for (; i < end; ++i) {
        const uint32_t t = __ldcg(a + i);
        __stcg(a + i, run);
        run += t;
    }
    return total;
}

// ---- exact table of the learned split -----------------------------------------------------
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

// The exact table is bucketized: 8 keys per 32-byte sector; a key hashes to a sector and
// probes up to 8 sectors linearly, stopping at a sector with a free slot.  One lookup is one
// or two 32 B loads at the loads a 75 %-full table sees.
constexpr int TBL_SECTOR = 8;
constexpr int TBL_SECTOR_PROBES = 8;

// Slot of `key`, or -1.
__device__ __forceinline__ int table_find(const uint32_t* keys, uint32_t slots, uint32_t key) {
    if (key == 0xffffffffu) return -1;
    const uint32_t nsec = slots / TBL_SECTOR;
    const uint32_t s0 = mix32(key) & (nsec - 1);
    for (int p = 0; p < TBL_SECTOR_PROBES; ++p) {
        const uint32_t sec = (s0 + p) & (nsec - 1);
        const uint4* q = reinterpret_cast<const uint4*>(keys + (uint64_t)sec * TBL_SECTOR);
        const uint4 a = __ldg(q), b = __ldg(q + 1);
        const uint32_t k[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        bool empty = false;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (k[j] == key) return (int)(sec * TBL_SECTOR + j);
            empty |= k[j] == 0xffffffffu;
        }
        if (empty) return -1;
    }
    return -1;
}

}  // namespace qsb
