// qs_aux.cu — synthetic key streams, exact-count histograms, error metrics and the
// roofline probes used by the benchmark.  None of this is on the insert/query path.
#include <cmath>
#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// One xorshift64* step (Vigna 2016) from a splitmix64-scrambled counter state, so key i
// depends only on (seed, i).
__device__ __forceinline__ uint32_t xorshift_key(uint64_t seed, uint64_t i) {
    uint64_t x = splitmix64(seed ^ (i * 0xD1B54A32D192ED03ull)) | 1ull;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    return (uint32_t)((x * 0x2545F4914F6CDD1Dull) >> 32);
}

__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t i, uint32_t attempt) {
    const uint64_t x = splitmix64(seed * 0x9E3779B97F4A7C15ull + i * 0xA24BAED4963EE407ull + attempt);
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

// Seeded bijection of u32 (xor, odd multiplies and xor-shifts are each invertible), so
// distinct ranks map to distinct keys.
__host__ __device__ __forceinline__ uint32_t rank_to_key(uint32_t r, uint64_t ps) {
    const uint32_t k0 = (uint32_t)ps, k1 = (uint32_t)(ps >> 32) | 1u;
    uint32_t x = r ^ k0;
    x *= 0x9E3779B1u;
    x ^= x >> 15;
    x *= k1;
    x ^= x >> 13;
    x *= 0x85EBCA6Bu;
    x ^= x >> 16;
    return x + (k0 >> 3);
}

// Rejection-inversion sampling of a Zipf(s) law on ranks 1..N (W. Hoermann and
// G. Derflinger, "Rejection-inversion to generate variates from monotone discrete
// distributions", ACM TOMACS 6(3), 1996).  H is an antiderivative of h(x) = x^-s.
struct ZipfParams {
    double s, hx1, hxn, sconst, N;
};

__host__ __device__ __forceinline__ double zh(double x, double s) { return exp(-s * log(x)); }
__host__ __device__ __forceinline__ double zhelper1(double x) {  // log(1+x)/x
    return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x));
}
__host__ __device__ __forceinline__ double zhelper2(double x) {  // (exp(x)-1)/x
    return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x * (1.0 / 3.0) * (1.0 + 0.25 * x));
}
__host__ __device__ __forceinline__ double zH(double x, double s) {
    const double lx = log(x);
    return zhelper2((1.0 - s) * lx) * lx;
}
__host__ __device__ __forceinline__ double zHinv(double y, double s) {
    double t = y * (1.0 - s);
    if (t < -1.0) t = -1.0;
    return exp(zhelper1(t) * y);
}

__global__ void k_gen_keys(uint32_t kind, uint64_t seed, ZipfParams zp, uint64_t perm_seed, uint32_t* keys,
                           uint32_t* ranks, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (kind == 0) {
            keys[i] = xorshift_key(seed, i);
            continue;
        }
        double k = 1.0;
        for (uint32_t a = 0; a < 64; ++a) {  // expected < 1.1 attempts; bounded
            const double u = zp.hxn + uniform01(seed, i, a) * (zp.hx1 - zp.hxn);
            const double x = zHinv(u, zp.s);
            k = floor(x + 0.5);
            if (k < 1.0) k = 1.0;
            if (k > zp.N) k = zp.N;
            if (k - x <= zp.sconst || u >= zH(k + 0.5, zp.s) - zh(k, zp.s)) break;
        }
        const uint32_t r = (uint32_t)k - 1u;
        keys[i] = rank_to_key(r, perm_seed);
        if (ranks) ranks[i] = r;
    }
}

// Seeded bijection of 16-bit values (odd multiplies mod 2^16 and xor-shifts invert).
__device__ __forceinline__ uint32_t perm16(uint32_t r, uint32_t k) {
    uint32_t x = (r ^ k) & 0xffffu;
    x = (x * 0x9E35u) & 0xffffu;
    x ^= x >> 7;
    x = (x * (((k >> 16) | 1u) & 0xffffu)) & 0xffffu;
    x ^= x >> 9;
    x = (x * 0x6A27u) & 0xffffu;
    return x ^ (x >> 8);
}

// key = class << 16 | suffix: class rank ~ Zipf(s_class) over n_class classes (the class id
// is its rank), suffix rank ~ Zipf(s_suffix) over 2^16 mapped by the class's own permutation.
__global__ void k_gen_class_keys(uint64_t seed, ZipfParams zc, ZipfParams zs, uint64_t perm_seed, uint32_t* keys,
                                 uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double kc = 1.0, ks = 1.0;
        for (uint32_t a = 0; a < 64; ++a) {
            const double u = zc.hxn + uniform01(seed, i, a) * (zc.hx1 - zc.hxn);
            const double x = zHinv(u, zc.s);
            kc = fmin(fmax(floor(x + 0.5), 1.0), zc.N);
            if (kc - x <= zc.sconst || u >= zH(kc + 0.5, zc.s) - zh(kc, zc.s)) break;
        }
        for (uint32_t a = 0; a < 64; ++a) {
            const double u = zs.hxn + uniform01(seed ^ 0x5851F42D4C957F2Dull, i, a) * (zs.hx1 - zs.hxn);
            const double x = zHinv(u, zs.s);
            ks = fmin(fmax(floor(x + 0.5), 1.0), zs.N);
            if (ks - x <= zs.sconst || u >= zH(ks + 0.5, zs.s) - zh(ks, zs.s)) break;
        }
        const uint32_t c = (uint32_t)kc - 1u, r = (uint32_t)ks - 1u;
        const uint32_t k = (uint32_t)splitmix64(perm_seed ^ ((uint64_t)c << 20));
        keys[i] = (c << 16) | perm16(r, k);
    }
}

__global__ void k_gen_rank_keys(uint64_t perm_seed, uint64_t first, uint32_t* keys, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        keys[i] = rank_to_key((uint32_t)(first + i), perm_seed);
}

__global__ void k_rank_histogram(const uint32_t* ranks, uint64_t n, uint32_t* hist, uint64_t n_ranks) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool v = i < n;
        const uint32_t r = v ? ranks[i] : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, r);
        if (v && r < n_ranks && lane == __ffs(peers) - 1) atomicAdd(hist + r, (uint32_t)__popc(peers));
    }
}

__global__ void k_error_metrics(const uint32_t* est, const uint32_t* exact, uint64_t n, double* acc) {
    double rel = 0, ratio = 0, cnt = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t a = exact[i];
        if (!a) continue;
        const double e = est[i], ad = a;
        rel += fabs(e - ad) / ad;
        ratio += e / ad;
        cnt += 1;
    }
    for (int o = 16; o; o >>= 1) {
        rel += __shfl_down_sync(0xffffffffu, rel, o);
        ratio += __shfl_down_sync(0xffffffffu, ratio, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc + 0, rel);
        atomicAdd(acc + 1, ratio);
        atomicAdd(acc + 2, cnt);
    }
}

static ZipfParams make_zipf(double s, uint64_t n_ranks) {
    ZipfParams z;
    z.s = s;
    z.N = (double)n_ranks;
    z.hx1 = zH(1.5, s) - 1.0;
    z.hxn = zH(z.N + 0.5, s);
    z.sconst = 2.0 - zHinv(zH(2.5, s) - zh(2.0, s), s);
    return z;
}

cudaError_t gen_keys(uint32_t kind, uint64_t seed, uint64_t n_ranks, double s, uint64_t perm_seed, uint32_t* d_keys,
                     uint32_t* d_ranks, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    ZipfParams z = make_zipf(s > 0 ? s : 1.0, n_ranks ? n_ranks : 1);
    k_gen_keys<<<148 * 8, 256, 0, st>>>(kind, seed, z, perm_seed, d_keys, d_ranks, n);
    return cudaGetLastError();
}

cudaError_t gen_class_keys(uint64_t seed, uint32_t n_class, double s_class, double s_suffix, uint64_t perm_seed,
                           uint32_t* d_keys, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_gen_class_keys<<<148 * 8, 256, 0, st>>>(seed, make_zipf(s_class, n_class), make_zipf(s_suffix, 1u << 16),
                                              perm_seed, d_keys, n);
    return cudaGetLastError();
}

cudaError_t gen_rank_keys(uint64_t perm_seed, uint64_t first, uint32_t* d_keys, uint64_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_gen_rank_keys<<<148 * 8, 256, 0, st>>>(perm_seed, first, d_keys, n);
    return cudaGetLastError();
}

cudaError_t rank_histogram(const uint32_t* d_ranks, uint64_t n, uint32_t* d_hist, uint64_t n_ranks, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_rank_histogram<<<148 * 8, 256, 0, st>>>(d_ranks, n, d_hist, n_ranks);
    return cudaGetLastError();
}

cudaError_t error_metrics(const uint32_t* d_est, const uint32_t* d_exact, uint64_t n, double* d_acc,
                          cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_error_metrics<<<148 * 4, 256, 0, st>>>(d_est, d_exact, n, d_acc);
    return cudaGetLastError();
}

// ---- roofline probes ---------------------------------------------------------------------
// kind 0: random 32 B sectors, a sub-warp of 8 lanes per sector, 3 lanes issue red.add.u32
//         on 3 distinct words (the MSWS insert's atomic pattern) -> sectors/s
// kind 1: random 32 B sector loads, thread per sector (the query's access) -> sectors/s
// kind 2: streaming 16 B loads over the buffer -> bytes/s
// kind 3: kind 0 with returning atom.add and a prior load of the sector's last word
// kind 4: one returning atom.add instruction per sector: 3 words + add 0 to the last word
// kind 5: kind 0 after a prior load of the sector's last word
__device__ __forceinline__ uint32_t probe_mix(uint32_t x) {
    x *= 0x9E3779B1u;
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

__global__ void k_probe(uint32_t kind, uint32_t* buf, uint64_t nsec, uint64_t nops, uint32_t* sink) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, w = lane & 7;
    uint32_t acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += stride) {
        if (kind == 0 || kind == 3 || kind == 4 || kind == 5) {
            const uint32_t key = (uint32_t)(i >> 3);
            const uint32_t h = probe_mix(key);
            const uint64_t s = ((uint64_t)h * nsec) >> 32;
            const uint32_t word = (w + (h & 7)) % 7;  // lanes 0..2 -> 3 distinct words of 0..6
            if (kind == 0) {
                if (w < 3) atomicAdd(buf + s * 8 + word, 1u);
            } else if (kind == 4) {
                if (w < 3 || w == 7) acc += atomicAdd(buf + s * 8 + (w == 7 ? 7u : word), w == 7 ? 0u : 1u);
            } else if (kind == 5) {
                const uint32_t v = __ldcg(buf + s * 8 + 7);
                if (w < 3 && v != 0xdeadbeefu) atomicAdd(buf + s * 8 + word, 1u);
            } else {
                const uint32_t v = __ldcg(buf + s * 8 + 7);
                if (w < 3 && v != 0xdeadbeefu) acc += atomicAdd(buf + s * 8 + word, 1u);
            }
        } else if (kind == 7) {  // every lane its own random sector, one red per lane
            const uint32_t h = probe_mix((uint32_t)i);
            const uint64_t s = ((uint64_t)h * nsec) >> 32;
            atomicAdd(buf + s * 8 + (h >> 29), 1u);
        } else if (kind == 1) {
            const uint32_t h = probe_mix((uint32_t)i);
            const uint64_t s = ((uint64_t)h * nsec) >> 32;
            const uint4* p = reinterpret_cast<const uint4*>(buf + s * 8);
            const uint4 a = __ldg(p), b = __ldg(p + 1);
            acc += a.x ^ b.w ^ a.y ^ b.z;
        } else {
            const uint4* p = reinterpret_cast<const uint4*>(buf);
            const uint4 a = __ldcs(p + (i % (nsec * 2)));
            acc += a.x ^ a.w;
        }
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;
}

// kind 6: `nops` grid-wide barriers of the replay kernel's form (bounded waits) in one
// cooperative launch of 512-thread blocks, two per SM
__global__ void __launch_bounds__(512) k_probe_barrier(Ctl* ctl, uint64_t nops) {
    for (uint64_t i = 0; i < nops; ++i)
        if (!grid_barrier(ctl)) return;
}

// kind 8 (failure path): one barrier that block 0 never reaches, waited for at most `limit`
// polls; every other block gives up, latches ST_TIMEOUT and returns.
__global__ void __launch_bounds__(512) k_probe_barrier_absent(Ctl* ctl, uint32_t limit) {
    if (blockIdx.x == 0) return;
    grid_barrier(ctl, limit);
}

// Launch kind 8 and report its latched status: cudaErrorLaunchTimeout when the waits gave up
// (the expected outcome), cudaSuccess if they did not.
cudaError_t probe_barrier_timeout(uint64_t limit) {
    Ctl* ctl = nullptr;
    int dev = 0, sms = 148, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_probe_barrier_absent, 512, 0);
    if (e == cudaSuccess && occ < 1) e = cudaErrorInvalidConfiguration;
    if (e == cudaSuccess) e = cudaMalloc(&ctl, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaMemset(ctl, 0, sizeof(Ctl));
    uint32_t lim = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(limit, 1), SPIN_LIMIT);
    if (e == cudaSuccess) {
        void* args[] = {&ctl, &lim};
        e = cudaLaunchCooperativeKernel((const void*)k_probe_barrier_absent, dim3(sms * std::min(occ, 2)), dim3(512),
                                        args, 0, nullptr);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    Ctl h{};
    if (e == cudaSuccess) e = cudaMemcpy(&h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && (h.status & ST_TIMEOUT)) e = cudaErrorLaunchTimeout;
    if (ctl) cudaFree(ctl);
    return e;
}

cudaError_t probe_barrier(uint64_t ops, double* ops_per_s) {
    Ctl* ctl = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int dev = 0, sms = 148, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_probe_barrier, 512, 0);
    if (e == cudaSuccess && occ < 1) e = cudaErrorInvalidConfiguration;
    if (e == cudaSuccess) e = cudaMalloc(&ctl, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaMemset(ctl, 0, sizeof(Ctl));
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const int grid = sms * std::min(occ, 2);
    float best = 1e30f;
    for (int r = 0; r < 4 && e == cudaSuccess; ++r) {
        uint64_t n = r ? ops : 16;  // the first launch warms up
        void* args[] = {&ctl, &n};
        cudaEventRecord(a);
        e = cudaLaunchCooperativeKernel((const void*)k_probe_barrier, dim3(grid), dim3(512), args, 0, nullptr);
        cudaEventRecord(b);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (r && ms > 0 && ms < best) best = ms;
    }
    Ctl h{};
    if (e == cudaSuccess) e = cudaMemcpy(&h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && (h.status & ST_TIMEOUT)) e = cudaErrorLaunchTimeout;
    if (e == cudaSuccess) *ops_per_s = (double)ops / (best * 1e-3);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (ctl) cudaFree(ctl);
    return e;
}

cudaError_t probe(uint32_t kind, uint64_t bytes, uint64_t ops, double* ops_per_s) {
    if (kind == 6) return ops ? probe_barrier(ops, ops_per_s) : cudaErrorInvalidValue;
    if (kind == 8) {
        *ops_per_s = 0.0;
        return probe_barrier_timeout(ops);
    }
    if (kind > 7 || kind == 6 || bytes < 64) return cudaErrorInvalidValue;
    uint32_t* buf = nullptr;
    uint32_t* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&buf, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&sink, 64);
    if (e == cudaSuccess) e = cudaMemset(buf, 0, bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const uint64_t nsec = bytes / 32;
    if (kind == 2) ops = nsec * 2 * 4;  // four passes of 16 B loads
    const uint64_t thread_ops = (kind == 0 || (kind >= 3 && kind <= 5)) ? ops * 8 : ops;  // 8 lanes per sector
    float best = 1e30f;
    if (e == cudaSuccess) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = sms * 8;
        k_probe<<<grid, 256>>>(kind, buf, nsec, thread_ops / 4, sink);
        for (int r = 0; r < 5 && e == cudaSuccess; ++r) {
            cudaEventRecord(a);
            k_probe<<<grid, 256>>>(kind, buf, nsec, thread_ops, sink);
            cudaEventRecord(b);
            e = cudaEventSynchronize(b);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
            if (ms > 0 && ms < best) best = ms;
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e == cudaSuccess) *ops_per_s = (kind == 2 ? (double)ops * 16.0 : (double)ops) / (best * 1e-3);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (buf) cudaFree(buf);
    if (sink) cudaFree(sink);
    return e;
}

}  // namespace qsb
