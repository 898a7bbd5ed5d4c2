// qsketch_b200.hpp — C++ host interface over the C ABI (qsketch_c.h), with the names and
// argument meaning of the reference's classes, so reference callers switch by changing the
// include and the namespace:
//
//   qsketch::Sketch<Key_T, Count_T>          reference include/sketch/sketch.h:5-28
//   qsketch::Sketch_GPU_Sub_Warp_Level       reference device_sketch_v3.h:526-634
//       (n_low, m_low, n_high, m_high, seed_sz, n_hash_mask_table)
//   qsketch::Sketch_GPU_Thread (n, m, seed_sz)  reference device_sketch_v0.h:105-191
//   qsketch::find_greatest_prime             reference lib/qsketch.cu:50-115
//
// Key_T = Count_T = unsigned int, as in the reference drivers (src/main.cu:3-6).  insert()
// and search() take device pointers and return 0 like the reference; unlike the reference
// (include/qsketch.h:104-105) a failure is not ignored: they return the non-zero qs_status.
// Calls are stream-ordered on `stream()` (default: the legacy stream), not synchronous;
// sync() waits and reports the latched device status.
#ifndef QSKETCH_B200_HPP
#define QSKETCH_B200_HPP

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "qsketch_c.h"

namespace qsketch_b200 {

inline std::string last_error() { return std::string(qs_last_error_string()); }

inline size_t find_greatest_prime(size_t upper_bound) { return (size_t)qs_find_greatest_prime(upper_bound); }

template <typename Key_T, typename Count_T>
struct Sketch {
    virtual int insert(Key_T* keys, size_t keys_sz) = 0;
    virtual int search(Key_T* keys, size_t keys_sz, Count_T* counts) = 0;
    virtual void clear() = 0;
    virtual ~Sketch() {}
};

// Owns one qs_sketch handle.
class Sketch_GPU : public Sketch<unsigned int, unsigned int> {
   public:
    int insert(unsigned int* keys, size_t keys_sz) override { return qs_insert(h_, keys, keys_sz, stream_); }
    int search(unsigned int* keys, size_t keys_sz, unsigned int* counts) override {
        return qs_query(h_, keys, keys_sz, counts, stream_);
    }
    void clear() override { qs_clear(h_, stream_); }
    // Host-buffer variants (copies pipelined with the kernels inside the library).
    int insert_host(const unsigned int* keys, size_t keys_sz) { return qs_insert_host(h_, keys, keys_sz); }
    int search_host(const unsigned int* keys, size_t keys_sz, unsigned int* counts) {
        return qs_query_host(h_, keys, keys_sz, counts);
    }
    int sync() { return qs_sync(h_, stream_); }
    qs_stats stats() {
        qs_stats s{};
        qs_get_stats(h_, &s);
        return s;
    }
    void set_stream(void* stream) { stream_ = stream; }
    void* stream() const { return stream_; }
    qs_sketch* handle() const { return h_; }
    ~Sketch_GPU() override { qs_destroy(h_); }
    Sketch_GPU(const Sketch_GPU&) = delete;
    Sketch_GPU& operator=(const Sketch_GPU&) = delete;

   protected:
    Sketch_GPU() = default;
    void create(const qs_params& p) {
        if (qs_create(&p, &h_) != QS_OK) throw std::runtime_error("qs_create: " + last_error());
    }
    qs_sketch* h_ = nullptr;
    void* stream_ = nullptr;
};

// The MSWS "Level" sketch.  The reference seeds its hash multiplier and mask table from
// /dev/urandom; here `seed_rng` / `mask_rng` seed the same draws reproducibly.
class Sketch_GPU_Sub_Warp_Level : public Sketch_GPU {
   public:
    Sketch_GPU_Sub_Warp_Level(size_t n_low, size_t m_low = 8, size_t n_high = 1024, size_t m_high = 32,
                              size_t seed_sz = 1, size_t n_hash_mask_table = 1021, uint32_t seed_rng = 1,
                              uint32_t mask_rng = 1) {
        qs_params p;
        qs_params_default(&p);
        p.kind = QS_KIND_MSWS;
        p.n_low = n_low;
        p.m_low = (uint32_t)m_low;
        p.n_high = n_high;
        p.m_high = (uint32_t)m_high;
        p.seed_sz = (uint32_t)seed_sz;
        p.hash_mask_table_sz = (uint32_t)n_hash_mask_table;
        p.seed_rng = seed_rng;
        p.mask_rng = mask_rng;
        create(p);
    }
    explicit Sketch_GPU_Sub_Warp_Level(const qs_params& p) { create(p); }

    // Sketch_GPU::number_of_buckets (device_sketch.h:371-376).
    static size_t number_of_buckets(size_t insert_keys_sz, size_t m, double factor) {
        return (size_t)qs_number_of_buckets(insert_keys_sz, m, factor, 3);
    }
};

// The plain count-min ("thread sketch").
class Sketch_GPU_Thread : public Sketch_GPU {
   public:
    Sketch_GPU_Thread(size_t n, size_t m, size_t seed_sz = 1, uint32_t seed_rng = 1) {
        qs_params p;
        qs_params_default(&p);
        p.kind = QS_KIND_PLAIN_CM;
        p.n_low = n;
        p.m_low = (uint32_t)m;
        p.seed_sz = (uint32_t)seed_sz;
        p.seed_rng = seed_rng;
        create(p);
    }
    // device_sketch_v0.h:133-138: find_greatest_prime(keys / factor).
    static size_t number_of_buckets(size_t insert_keys_sz, size_t /*m*/, double factor) {
        return find_greatest_prime((size_t)(insert_keys_sz / factor));
    }
};

}  // namespace qsketch_b200

#endif  // QSKETCH_B200_HPP
