// Exercises include/qsketch_b200.hpp the way the reference's drivers use their classes
// (src/test.cu:340-393): construct, insert a device key buffer, search, clear.
//   host_api_driver <keys.bin> <queries.bin> <masks.bin> <out.bin> <n_low> <n_high> <hash_seed>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "qsketch_b200.hpp"

static std::vector<unsigned char> slurp(const char* path) {
    std::vector<unsigned char> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    unsigned char buf[1 << 16];
    size_t r;
    while ((r = std::fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + r);
    std::fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc != 8) {
        std::fprintf(stderr, "usage: %s keys queries masks out n_low n_high hash_seed\n", argv[0]);
        return 2;
    }
    auto keys = slurp(argv[1]), queries = slurp(argv[2]), masks = slurp(argv[3]);
    const size_t nk = keys.size() / 4, nq = queries.size() / 4;
    qs_params p;
    qs_params_default(&p);
    p.n_low = std::strtoull(argv[5], nullptr, 10);
    p.n_high = std::strtoull(argv[6], nullptr, 10);
    p.hash_seed = (uint32_t)std::strtoul(argv[7], nullptr, 10);
    p.hash_mask_table_sz = (uint32_t)(masks.size() / 4);
    p.mask_table = masks.data();
    unsigned int *d_keys = nullptr, *d_q = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_keys, keys.size() + 4) != cudaSuccess || cudaMalloc(&d_q, queries.size() + 4) != cudaSuccess ||
        cudaMalloc(&d_out, queries.size() + 4) != cudaSuccess)
        return 3;
    cudaMemcpy(d_keys, keys.data(), keys.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_q, queries.data(), queries.size(), cudaMemcpyHostToDevice);
    try {
        qsketch_b200::Sketch_GPU_Sub_Warp_Level map(p);
        qsketch_b200::Sketch<unsigned int, unsigned int>& s = map;
        if (s.insert(d_keys, nk / 2) != 0 || s.insert(d_keys + nk / 2, nk - nk / 2) != 0) return 4;
        if (s.search(d_q, nq, d_out) != 0) return 5;
        if (map.sync() != QS_OK) return 6;
        std::vector<unsigned int> out(nq);
        cudaMemcpy(out.data(), d_out, nq * 4, cudaMemcpyDeviceToHost);
        FILE* f = std::fopen(argv[4], "wb");
        std::fwrite(out.data(), 4, nq, f);
        std::fclose(f);
        s.clear();
        if (s.search(d_q, nq, d_out) != 0 || map.sync() != QS_OK) return 7;
        cudaMemcpy(out.data(), d_out, nq * 4, cudaMemcpyDeviceToHost);
        for (unsigned int x : out)
            if (x != 0) return 8;  // cleared sketch estimates 0 everywhere
        std::printf("inserted %zu searched %zu ok; linked %llu\n", nk, nq,
                    (unsigned long long)map.stats().linked_buckets);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 9;
    }
    cudaFree(d_keys);
    cudaFree(d_q);
    cudaFree(d_out);
    return 0;
}
