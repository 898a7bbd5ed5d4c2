// qs_noalloc.cu — qs_msws_insert_noalloc: the MSWS insert for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs inside an engine which owns all device memory (a fixed arena
// set up at start-up, for instance) and may not call cudaMalloc/cudaFree while it serves —
// those calls synchronise the device and fragment the arena.  Such a caller keeps the sketch
// tables in its own memory and passes them in; the only working memory this insert needs
// beyond its inputs and outputs, the scratch of the ordered replay, lives in the file-scope
// array below, which every GPU that loads the library holds until the process exits.
//
// Limits (checked before anything runs; larger requests get QS_ERR_CAPACITY):
//   at most QS_NOALLOC_MAX_KEYS keys per call and QS_NOALLOC_MAX_BUCKETS low buckets.
// Sharing: every call on a device uses the same scratch array and leaves its contents
// behind; the call clears what must start at zero.  Calls whose work overlaps on the GPU
// (other streams, other host threads, without ordering between them) race on the array and
// corrupt each other's results — order them.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/qsketch_c.h"
#include "qs_kernels.h"

namespace qsb {

constexpr uint64_t NA_MAX_KEYS = QS_NOALLOC_MAX_KEYS;
constexpr uint64_t NA_MAX_BUCKETS = QS_NOALLOC_MAX_BUCKETS;
constexpr uint64_t NA_TILES = NA_MAX_KEYS / REPAIR_TILE;
constexpr uint64_t NA_TOTAL_SLOTS = 4096;

// Scratch layout (bytes), each part 256-byte aligned.
constexpr uint64_t na_align(uint64_t x) { return (x + 255) & ~uint64_t(255); }
constexpr uint64_t NA_OFF_REC0 = 0;
constexpr uint64_t NA_OFF_REC1 = NA_OFF_REC0 + na_align(NA_MAX_KEYS * 8);
constexpr uint64_t NA_OFF_FLAGS = NA_OFF_REC1 + na_align(NA_MAX_KEYS * 8);
constexpr uint64_t NA_OFF_SEG = NA_OFF_FLAGS + na_align(NA_MAX_KEYS * 4);
constexpr uint64_t NA_OFF_TILES = NA_OFF_SEG + na_align(NA_MAX_KEYS * 4);
constexpr uint64_t NA_OFF_HIST = NA_OFF_TILES + na_align(NA_TILES * 4);
constexpr uint64_t NA_OFF_TOTALS = NA_OFF_HIST + na_align(256 * NA_TILES * 4 + 256 * 4);  // + digit totals
constexpr uint64_t NA_OFF_RPOS0 = NA_OFF_TOTALS + na_align(NA_TOTAL_SLOTS * LOW_COUNTERS * 4);
constexpr uint64_t NA_OFF_RPOS1 = NA_OFF_RPOS0 + na_align(NA_MAX_KEYS * 4);
constexpr uint64_t NA_OFF_SW = NA_OFF_RPOS1 + na_align(NA_MAX_KEYS * 4);
constexpr uint64_t NA_OFF_SWBASE = NA_OFF_SW + na_align(NA_MAX_KEYS * 8);
constexpr uint64_t NA_OFF_SWBITS = NA_OFF_SWBASE + na_align(NA_MAX_KEYS * 4);
constexpr uint64_t NA_OFF_SWCNT = NA_OFF_SWBITS + na_align(NA_MAX_KEYS / 8);
constexpr uint64_t NA_BYTES = NA_OFF_SWCNT + na_align(NA_MAX_KEYS / SW_BLOCK * 4 + 4);
static_assert(NA_BYTES <= QS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the documented size");
static_assert(sizeof(Ctl) <= QS_MSWS_STATE_BYTES, "control block exceeds the caller's state block");

// The scratch.  In host code `na_scratch` is only a stand-in symbol, not a device address:
// host code must use the address cudaGetSymbolAddress returns (na_setup below).
static __device__ __align__(256) unsigned char na_scratch[QS_NOALLOC_SCRATCH_BYTES];

// A fresh sketch is all-zero tables and an all-zero state block; the first call starts the
// bump allocator at 1025 (device_sketch.h:107-111).  Every call resets the per-call counters.
__global__ void k_noalloc_begin(Ctl* st) {
    if (st->next_id == 0) st->next_id = FIRST_ID;
    st->n_flagged = 0;
    st->n_records = 0;
    st->n_long = 0;
    st->bar_count = 0;
    st->bar_arrive = 0;
}

struct NaDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;
    uint32_t n_masks = 0;  // mask-table size the launch geometry below was computed for
    MswsLaunch launch{};
};

constexpr int NA_MAX_DEVICES = 64;
NaDevice na_devices[NA_MAX_DEVICES];
std::mutex na_mutex;

// Once per device, with that device current: resolve the scratch array's device address.
// The launch geometry (pass-1 occupancy depends on the shared-memory copy of the mask table)
// is recomputed whenever the mask-table size differs from the previous call's; that is
// host-side work only.  The caller gets a copy of the geometry, taken under the lock.
static qs_status na_setup(int dev, uint32_t n_masks, unsigned char** scratch, MswsLaunch* launch, char* err,
                          size_t errlen) {
    std::lock_guard<std::mutex> lk(na_mutex);
    NaDevice& d = na_devices[dev];
    if (!d.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, na_scratch);
        if (e != cudaSuccess) {
            snprintf(err, errlen, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            return e == cudaErrorNoKernelImageForDevice ? QS_ERR_NO_DEVICE : QS_ERR_CUDA;
        }
        d.scratch = static_cast<unsigned char*>(p);
        d.ready = true;
    }
    if (d.n_masks != n_masks) {
        cudaError_t e = msws_configure(dev, n_masks, &d.launch);
        if (e != cudaSuccess) {
            d.n_masks = 0;
            snprintf(err, errlen, "kernel configuration: %s", cudaGetErrorString(e));
            return QS_ERR_CUDA;
        }
        d.n_masks = n_masks;
    }
    *scratch = d.scratch;
    *launch = d.launch;
    return QS_OK;
}

}  // namespace qsb

using namespace qsb;

extern "C" qs_status qs_msws_insert_noalloc(uint32_t* d_low, uint64_t n_low, uint32_t* d_high, uint64_t n_high,
                                            void* d_state, const uint32_t* d_masks, uint32_t n_masks,
                                            uint32_t hash_seed, uint32_t flags, const uint32_t* d_keys, size_t n,
                                            void* stream) {
    char err[320];
    if (!d_low || !d_high || !d_state || !d_masks || (!d_keys && n))
        return set_last_error("qs_msws_insert_noalloc: null pointer"), QS_ERR_INVALID_ARG;
    if (n_low == 0 || n_high < 2 || n_high > (1ull << 30) || n_masks == 0 || n_masks > 16384 || hash_seed == 0)
        return set_last_error("qs_msws_insert_noalloc: n_low, n_high, n_masks or hash_seed out of range"),
               QS_ERR_INVALID_ARG;
    if (n > NA_MAX_KEYS || n_low > NA_MAX_BUCKETS) {
        snprintf(err, sizeof err,
                 "qs_msws_insert_noalloc: %zu keys / %llu buckets exceed the fixed scratch (at most %llu keys per "
                 "call and %llu low buckets); split the call or use qs_create/qs_insert",
                 n, (unsigned long long)n_low, (unsigned long long)NA_MAX_KEYS, (unsigned long long)NA_MAX_BUCKETS);
        return set_last_error(err), QS_ERR_CAPACITY;
    }
    if ((reinterpret_cast<uintptr_t>(d_keys) | reinterpret_cast<uintptr_t>(d_low) |
         reinterpret_cast<uintptr_t>(d_high) | reinterpret_cast<uintptr_t>(d_masks)) & 3u)
        return set_last_error("qs_msws_insert_noalloc: pointers must be 4-byte aligned"), QS_ERR_INVALID_ARG;
    // The state block holds 64-bit counters updated with 64-bit atomics.
    if (reinterpret_cast<uintptr_t>(d_state) & (QS_MSWS_STATE_ALIGN - 1))
        return set_last_error("qs_msws_insert_noalloc: the state block must be 16-byte aligned"), QS_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(d_low) & 31u)
        return set_last_error("qs_msws_insert_noalloc: the low table must be 32-byte aligned"), QS_ERR_INVALID_ARG;
    if (n == 0) return QS_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES)
        return set_last_error("qs_msws_insert_noalloc: no current CUDA device"), QS_ERR_NO_DEVICE;
    unsigned char* sc = nullptr;
    MswsLaunch launch{};
    qs_status s = na_setup(dev, n_masks, &sc, &launch, err, sizeof err);
    if (s != QS_OK) return set_last_error(err), s;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MswsDev D{};
    D.low = d_low;
    D.high = d_high;
    D.masks = d_masks;
    D.ctl = static_cast<Ctl*>(d_state);
    D.n_low = n_low;
    D.n_high = n_high;
    D.fm_low = make_fastmod((uint32_t)n_low);
    D.fm_mask = make_fastmod(n_masks);
    D.seed = hash_seed;
    D.n_masks = n_masks;
    D.compat_v3 = (flags & QS_FLAG_COMPAT_V3) ? 1u : 0u;
    D.route = 1;
    D.flag_cap = (uint32_t)std::min<uint64_t>(n_low, NA_MAX_KEYS);
    D.max_tiles = (uint32_t)NA_TILES;
    D.long_cap = (uint32_t)std::min<uint64_t>(D.flag_cap, NA_TOTAL_SLOTS);
    D.rec[0] = reinterpret_cast<uint2*>(sc + NA_OFF_REC0);
    D.rec[1] = reinterpret_cast<uint2*>(sc + NA_OFF_REC1);
    D.flag_list = reinterpret_cast<uint32_t*>(sc + NA_OFF_FLAGS);
    D.seg_beg = reinterpret_cast<uint32_t*>(sc + NA_OFF_SEG);
    D.tile_counts = reinterpret_cast<uint32_t*>(sc + NA_OFF_TILES);
    D.hist = reinterpret_cast<uint32_t*>(sc + NA_OFF_HIST);
    D.totals = reinterpret_cast<uint32_t*>(sc + NA_OFF_TOTALS);
    D.rpos[0] = reinterpret_cast<uint32_t*>(sc + NA_OFF_RPOS0);
    D.rpos[1] = reinterpret_cast<uint32_t*>(sc + NA_OFF_RPOS1);
    D.sw = reinterpret_cast<uint2*>(sc + NA_OFF_SW);
    D.sw_base = reinterpret_cast<uint32_t*>(sc + NA_OFF_SWBASE);
    D.sw_bits = reinterpret_cast<uint32_t*>(sc + NA_OFF_SWBITS);
    D.sw_cnt = reinterpret_cast<uint32_t*>(sc + NA_OFF_SWCNT);

    // Every scratch part is written before it is read.
    k_noalloc_begin<<<1, 1, 0, st>>>(D.ctl);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = msws_insert_pass(d_keys, n, D, launch, 2, st);
    if (e == cudaSuccess) e = msws_repair(d_keys, n, D, launch, st);
    if (e != cudaSuccess) {
        snprintf(err, sizeof err, "qs_msws_insert_noalloc: %s", cudaGetErrorString(e));
        return set_last_error(err), QS_ERR_CUDA;
    }
    return QS_OK;
}
