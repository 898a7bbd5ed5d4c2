// ref_shim.cu — TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own
// library sources (lib/hashmask.cu, lib/qsketch.cu, lib/default.cu, read in place from the
// reference checkout) into oracle/_ref/libqsref.so, so that tests can pin the oracle's
// restatements against the reference's code.  Nothing in the product links this.
//
// The reference seeds its engines from /dev/urandom (include/tool/tool.h:192-204); these
// entry points reseed them with an integer first, which makes them deterministic.
#include <qsketch.h>

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
