// ref_shim.cu — TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own
// library sources (lib/hashmask.cu, lib/qsketch.cu, lib/default.cu, read in place from the
// reference checkout) into oracle/_ref/libqsref.so, so that tests can pin the oracle's
// restatements against the reference's code.  Nothing in the product links this.
//
// The reference seeds its engines from /dev/urandom (include/tool/tool.h:192-204); these
// entry points reseed them with an integer first, which makes them deterministic.
#include <qsketch.h>

#include <algorithm>
#include <cstring>
#include <vector>

extern "C" {

// generate_hashmask (lib/hashmask.cu:32-83) on cpu_tool<uint>.eng reseeded with rng_seed.
int ref_generate_hashmask(unsigned int rng_seed, size_t n, size_t m_bits, size_t ones,
                          size_t padding, unsigned char *out) {
    qsketch::cpu_tool<unsigned int>.eng.seed(rng_seed);
    unsigned char *t = qsketch::generate_hashmask(nullptr, n, m_bits, ones, padding);
    size_t bytes = n * ((m_bits + 7) / 8);
    memcpy(out, t, bytes);
    delete[] t;
    return 0;
}

// The seed draw of Device_Seed::resize (device_sketch.h:290): gpu_tool<Seed_T>.random
// draws on the host with CPU_Tools::random (include/tool/tool.h:206-220) before copying;
// the host half is called here directly.
int ref_draw_seeds(unsigned int rng_seed, size_t count, unsigned int *out) {
    qsketch::gpu_tool<unsigned int>.eng.seed(rng_seed);
    unsigned int *t = qsketch::gpu_tool<unsigned int>.qsketch::CPU_Tools<unsigned int>::random(
        nullptr, count, 1u, std::numeric_limits<unsigned int>::max());
    memcpy(out, t, count * sizeof(unsigned int));
    delete[] t;
    return 0;
}

// find_greatest_prime (lib/qsketch.cu:50-115).
unsigned long long ref_find_greatest_prime(unsigned long long upper_bound) {
    return qsketch::find_greatest_prime((size_t)upper_bound);
}

// Unordered_Map (include/sketch/host_sketch/host_sketch.h:15-63): exact counts of
// `queries` after inserting `keys`.
int ref_exact_counts(const unsigned int *keys, size_t n, const unsigned int *queries, size_t nq,
                     unsigned int *out) {
    qsketch::Unordered_Map<unsigned int, unsigned int> um;
    um.insert(const_cast<unsigned int *>(keys), n);
    um.search(const_cast<unsigned int *>(queries), nq, out);
    return 0;
}

}  // extern "C"

// ---- the reference's own sketch kernels, run on the GPU ------------------------------------
// These construct the reference's classes and call their own insert/search, so the oracle's
// restatement of the insert/query semantics can be pinned against the reference's kernels.
// Both take host arrays and copy them to and from the device around the reference's calls.

namespace {
using RefHash = qsketch::hash_mul_add<unsigned int, unsigned int, unsigned int>;
using RefMsws = qsketch::Sketch_GPU_Sub_Warp_Level<unsigned int, unsigned int, unsigned int, unsigned int, RefHash>;
using RefCm = qsketch::Sketch_GPU_Thread<unsigned int, unsigned int, unsigned int, unsigned int, RefHash>;

// The reference launches 65536 one-warp blocks (lib/default.cu:46-49) and gives each warp
// ceil(n / 65536) consecutive keys (device_sketch_v3.h:572).  Its four 8-lane sub-warps step
// through a warp's keys together and meet in full-warp shuffles and votes
// (device_sketch_v3.h:110-131, 364-398), so every warp's share must be a multiple of 4 keys,
// or some lanes would wait in a shuffle the others never reach.
bool warp_shares_whole(size_t n) {
    const size_t warps = 65536;
    const size_t per = (n + warps - 1) / warps;
    return n % 4 == 0 && per % 4 == 0;
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};
}  // namespace

extern "C" {

// Sketch_GPU_Sub_Warp_Level(n_low, 8, n_high, 32, 1, 1021) (device_sketch_v3.h:544-563) with
// its engines reseeded (hash seed: gpu_tool<uint>, mask table: cpu_tool<uint>), then its own
// insert(keys) (:570-599) and search(queries) (:600-632).  Returns the seed and the mask table
// it drew, the estimates and (if h_low is not null) the low table.
//
// Only inputs on which the reference kernel is well defined are run: every warp's share of
// keys and of queries a multiple of 4 (see warp_shares_whole), and no low counter above 128
// after the insert, checked on the host before any launch.  Above 128 the reference links a
// high bucket through atomic_malloc (device_sketch_v3.h:69-85), whose wait has no bound and
// whose result depends on the thread schedule.  Returns -1 when the inputs are refused, a CUDA
// error code when a CUDA call fails, 0 on success.
int ref_msws_gpu(unsigned int seed_rng, unsigned int mask_rng, size_t n_low, size_t n_high,
                 const unsigned int *h_keys, size_t n, const unsigned int *h_queries, size_t nq,
                 unsigned int *h_counts, unsigned int *h_low, unsigned int *seed_out,
                 unsigned char *masks_out) {
    const size_t H = 1021;
    if (n_low == 0 || n_low > (1ull << 28) || n_high < 2 || !warp_shares_whole(n) || !warp_shares_whole(nq))
        return -1;
    qsketch::gpu_tool<unsigned int>.eng.seed(seed_rng);
    qsketch::cpu_tool<unsigned int>.eng.seed(mask_rng);
    RefMsws sk(n_low, 8, n_high, 32, 1, H);
    unsigned int seed = 0;
    if (cudaMemcpy(&seed, sk.ds.seed, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return (int)cudaGetLastError();
    std::vector<unsigned char> masks(H * 4);
    if (cudaMemcpy(masks.data(), sk.hash_mask_table, H * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return (int)cudaGetLastError();
    // Host check: the final value of every low counter if no bucket ever links.
    {
        std::vector<unsigned int> cnt(n_low * 28, 0);
        for (size_t i = 0; i < n; ++i) {
            const unsigned int hv = h_keys[i] * seed;
            const size_t b = hv % n_low;
            unsigned int m;
            memcpy(&m, masks.data() + (hv % H) * 4, 4);
            for (int c = 0; c < 28; ++c)
                if ((m >> c) & 1u)
                    if (++cnt[b * 28 + c] > 128) return -1;
        }
    }
    DevBuf dk, dq, dc;
    if (cudaMalloc(&dk.p, std::max<size_t>(n, 1) * 4) != cudaSuccess ||
        cudaMalloc(&dq.p, std::max<size_t>(nq, 1) * 4) != cudaSuccess ||
        cudaMalloc(&dc.p, std::max<size_t>(nq, 1) * 4) != cudaSuccess)
        return (int)cudaGetLastError();
    if (cudaMemcpy(dk.p, h_keys, n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dq.p, h_queries, nq * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return (int)cudaGetLastError();
    if (n) sk.insert(static_cast<unsigned int *>(dk.p), n);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    if (nq) sk.search(static_cast<unsigned int *>(dq.p), nq, static_cast<unsigned int *>(dc.p));
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h_counts, dc.p, nq * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h_low) e = cudaMemcpy(h_low, sk.dht_low.table, n_low * 8 * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    *seed_out = seed;
    memcpy(masks_out, masks.data(), H * 4);
    return 0;
}

// Sketch_GPU_Thread(n, m, 1) (device_sketch_v0.h:121-131) with gpu_tool<uint> reseeded, then
// its own insert(keys) (:140-161) and search(queries) (:162-189).  Counter additions commute,
// so any input is well defined.  Returns the m seeds it drew, the estimates and (if h_table is
// not null) the m*n counters.
int ref_cm_gpu(unsigned int seed_rng, size_t n, size_t m, const unsigned int *h_keys, size_t nk,
               const unsigned int *h_queries, size_t nq, unsigned int *h_counts, unsigned int *h_table,
               unsigned int *seeds_out) {
    if (n == 0 || m == 0 || m > 64) return -1;
    qsketch::gpu_tool<unsigned int>.eng.seed(seed_rng);
    RefCm sk(n, m, 1);
    DevBuf dk, dq, dc;
    if (cudaMalloc(&dk.p, std::max<size_t>(nk, 1) * 4) != cudaSuccess ||
        cudaMalloc(&dq.p, std::max<size_t>(nq, 1) * 4) != cudaSuccess ||
        cudaMalloc(&dc.p, std::max<size_t>(nq, 1) * 4) != cudaSuccess)
        return (int)cudaGetLastError();
    if (cudaMemcpy(dk.p, h_keys, nk * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dq.p, h_queries, nq * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return (int)cudaGetLastError();
    if (nk) sk.insert(static_cast<unsigned int *>(dk.p), nk);
    if (nq) sk.search(static_cast<unsigned int *>(dq.p), nq, static_cast<unsigned int *>(dc.p));
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h_counts, dc.p, nq * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h_table) e = cudaMemcpy(h_table, sk.dht_low.table, n * m * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(seeds_out, sk.ds.seed, m * 4, cudaMemcpyDeviceToHost);
    return (int)e;
}

}  // extern "C"
