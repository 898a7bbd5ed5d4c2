// qs_kernels.h — host-side launchers of the sm_100a kernels (internal to libqsketch).
#pragma once
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include "qs_common.cuh"

namespace qsb {

constexpr int LPK_VARIANTS = 6;  // lanes per key 4, 8, 16, 32, 2, 1 (index order of lpk_index)

struct MswsLaunch {
    int num_sms;
    int insert_grid;
    int repair_grid;
    int query_grid;
    int ins_occ[3][6];       // resident pass-1 CTAs per SM by [aggregation][lanes-per-key index]
    int lanes_per_key = 8;   // pass-1 lanes per key: 1, 2, 4, 8, 16 or 32
    int ctas_per_sm = 0;     // pass-1 CTAs per SM, 0 = as many as fit
    int tile_keys = 2048;    // pass-1 keys per tile: 256, 512, 1024 or 2048
};

size_t msws_insert_smem(uint32_t n_masks);
cudaError_t msws_configure(int device, uint32_t n_masks, MswsLaunch* L);
// Pass 1 (packed atomics + crossing detection) and the ordered repair of one chunk of at
// most max_batch keys; the repair exits at once when nothing crossed.
// Batched streams (StreamDesc / BatchDev in qs_common.cuh).
cudaError_t batch_plan(const BatchDev& B, Ctl* ctl, const BatchWindow& W, bool strict, cudaStream_t st);
// Pass 1 of the streams [k_lo, k_hi) of the size-class grouped order (work counter cls).
cudaError_t batch_insert_pass(const uint32_t* d_keys, const MswsDev& D, const BatchDev& B, const MswsLaunch& L,
                              int agg, int lanes_per_key, uint32_t k_lo, uint32_t k_hi, uint32_t cls, cudaStream_t st);
cudaError_t batch_repair(const uint32_t* d_window, const MswsDev& D, const BatchDev& B, const MswsLaunch& L,
                         cudaStream_t st);
cudaError_t batch_query(const uint32_t* d_keys, uint32_t* d_out, const MswsDev& D, const BatchDev& B,
                        const MswsLaunch& L, cudaStream_t st);
cudaError_t msws_insert_pass(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, int agg,
                             cudaStream_t st);
cudaError_t msws_repair(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, cudaStream_t st);
cudaError_t msws_query(const uint32_t* d_keys, uint64_t n, uint32_t* d_out, const MswsDev& D, const MswsLaunch& L,
                       cudaStream_t st);

cudaError_t cm_insert(const uint32_t* d_keys, uint64_t n, const CmDev& D, int agg, int grid, cudaStream_t st);
// REMOVE (qs_remove.cu): one occurrence of each key out, counters floored at 0.
cudaError_t msws_remove(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, cudaStream_t st);
cudaError_t cm_remove(const uint32_t* d_keys, uint64_t n, const CmDev& D, int grid, uint32_t* d_status,
                      cudaStream_t st);
cudaError_t cm_query(const uint32_t* d_keys, uint64_t n, uint32_t* d_out, const CmDev& D, int grid, cudaStream_t st);

cudaError_t gen_keys(uint32_t kind, uint64_t seed, uint64_t n_ranks, double s, uint64_t perm_seed, uint32_t* d_keys,
                     uint32_t* d_ranks, uint64_t n, cudaStream_t st);
cudaError_t gen_rank_keys(uint64_t perm_seed, uint64_t first, uint32_t* d_keys, uint64_t n, cudaStream_t st);
cudaError_t gen_class_keys(uint64_t seed, uint32_t n_class, double s_class, double s_suffix, uint64_t perm_seed,
                           uint32_t* d_keys, uint64_t n, cudaStream_t st);
cudaError_t rank_histogram(const uint32_t* d_ranks, uint64_t n, uint32_t* d_hist, uint64_t n_ranks, cudaStream_t st);
cudaError_t error_metrics(const uint32_t* d_est, const uint32_t* d_exact, uint64_t n, double* d_acc,
                          cudaStream_t st);
cudaError_t probe(uint32_t kind, uint64_t bytes, uint64_t ops, double* ops_per_s);

// Text returned by qs_last_error_string() on this host thread.
void set_last_error(const char* text);

// ---- learned split: MLP 32 -> 128 -> 128 -> 1 ---------------------------------------------
constexpr uint32_t MLP_W1_N = 128 * 32, MLP_W2_N = 128 * 128;
constexpr uint32_t MLP_BF16_PARAMS = MLP_W1_N + MLP_W2_N;           // W1 | W2 in bf16
constexpr uint32_t MLP_PARAMS = MLP_BF16_PARAMS + 128 + 128 + 128 + 1;  // + b1 | b2 | w3 | b3

struct MlpDev {
    __nv_bfloat16* W1;  // bf16 copies, W2 = W1 + MLP_W1_N
    __nv_bfloat16* W2;
    float* params;      // fp32 master: W1 | W2 | b1 | b2 | w3 | b3
    float *b1, *b2, *w3, *b3;
    float* grads;       // same layout
    float *gW1, *gW2, *gb1, *gb2, *g3, *gb3;
    float *adam_m, *adam_v;
    float* partials;    // MLP_MAX_TILES * MLP_PARTIAL_STRIDE per-tile gradients (fixed-order reduction)
    float* ploss;       // MLP_MAX_TILES tile losses
    uint32_t* status;   // ST_TIMEOUT once a tensor-core wait gave up
};
constexpr uint32_t MLP_TILE_EXAMPLES = 128;  // examples per CTA tile (the MMAs' M)
constexpr uint32_t MLP_PARTIAL_STRIDE = (MLP_PARAMS + 3u) & ~3u;  // floats per tile partial: 16-byte rows
constexpr uint32_t MLP_MAX_TILES = 256;      // tiles per backward launch

// Launch with programmatic stream serialization (the kernel waits with griddep_wait before
// it reads what the previous kernel of the stream wrote); cooperative launches keep that
// property.
cudaError_t launch_pdl(const void* fn, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void** args,
                       bool cooperative);
size_t mlp_smem_bytes();
size_t mlp_fwd_smem_bytes();
cudaError_t mlp_configure();
cudaError_t mlp_forward(const uint32_t* d_keys, uint64_t n, const MlpDev& M, float* d_logits, cudaStream_t st);
cudaError_t mlp_backward(const uint32_t* d_keys, const uint8_t* d_labels, uint64_t n, float pos_weight,
                         float inv_batch, const MlpDev& M, float* d_loss, cudaStream_t st);
cudaError_t mlp_adam(const MlpDev& M, uint32_t step, float lr, cudaStream_t st);
// One Adam step on a batch of n examples: the backward pass, then the tile reduction fused
// with the update, *d_loss set to the batch's loss sum (same arithmetic, in the same order,
// as mlp_backward into a zeroed loss followed by mlp_adam).
cudaError_t mlp_train_step(const uint32_t* d_keys, const uint8_t* d_labels, uint64_t n, float pos_weight,
                           float inv_batch, const MlpDev& M, float* d_loss, uint32_t step, float lr, cudaStream_t st);
cudaError_t mlp_refresh_bf16(const MlpDev& M, cudaStream_t st);

// ---- learned split: exact table of heavy keys and routing -----------------------------------
constexpr uint32_t TBL_EMPTY = 0xffffffffu;
constexpr int TBL_PROBES = 32;

struct TableDev {
    uint32_t* keys;    // slots, TBL_EMPTY when free
    uint32_t* counts;  // exact counts of the admitted keys
    uint32_t slots;    // power of two
    uint32_t max_fill; // admission stops at this many keys
    uint32_t* fill;    // device counter of admitted keys
};

struct RouteDev {
    uint32_t* skip;         // 1 bit per key of the chunk: counted in the exact table
    uint32_t* misses;       // distinct-per-warp keys that missed the table (unordered)
    uint32_t* n_misses;
    uint32_t* cand_keys;    // candidate set (open addressing), TBL_EMPTY when free
    uint32_t cand_slots;    // power of two
    uint32_t* n_cand;
    uint32_t* cand_list;    // admitted-order list of candidates
    float z_threshold;      // a key is a candidate when its logit is >= this
    uint32_t collect;       // k_route fills `misses` only while this is set
};

cudaError_t route_chunk(const uint32_t* d_keys, uint64_t n, const TableDev& T, const RouteDev& R, cudaStream_t st);
cudaError_t classify_misses(const MlpDev& M, const RouteDev& R, uint64_t max_misses, cudaStream_t st);
uint32_t table_admit_host(uint32_t* keys, uint32_t slots, const uint32_t* order, uint32_t count, uint32_t fill,
                          uint32_t max_fill);
cudaError_t learned_query(const uint32_t* d_keys, uint64_t n, const TableDev& T, const MswsDev& D, const MswsLaunch& L,
                          uint32_t* d_out, cudaStream_t st);
// Device scratch of the training-set and admission sorts (grown on demand, freed with it).
struct TrainScratch {
    void* p = nullptr;
    size_t size = 0;
    cudaError_t ensure(size_t bytes);
    ~TrainScratch();
};
cudaError_t distinct_sorted(const uint32_t* d_keys, uint32_t n, uint32_t* d_tmp, uint32_t* d_out, uint32_t* d_count,
                            TrainScratch& S, cudaStream_t st);
// Training examples in a seeded order (a Feistel-network bijection of [0, n)).
cudaError_t permute_examples(const uint32_t* d_keys, const uint8_t* d_labels, uint32_t n, uint64_t seed,
                             uint32_t* d_okeys, uint8_t* d_olabels, cudaStream_t st);

cudaError_t train_scratch_reserve(TrainScratch& S, uint32_t n, uint32_t set_slots);
cudaError_t kth_largest(const uint32_t* d_in, uint32_t n, uint32_t k, uint32_t* d_tmp, TrainScratch& S,
                        uint32_t* h_out, cudaStream_t st);
cudaError_t label_keys(const uint32_t* d_est, uint32_t n, uint32_t thr, uint8_t* d_lab, uint32_t* d_npos,
                       cudaStream_t st);
cudaError_t training_set(const uint32_t* d_keys, const uint8_t* d_lab, uint32_t n, uint32_t seed, uint64_t cut,
                         uint8_t* d_take, uint32_t* d_tkeys, uint8_t* d_tlab, uint32_t* d_count, TrainScratch& S,
                         cudaStream_t st);
cudaError_t positive_logit_quantile(const float* d_z, const uint8_t* d_lab, uint32_t n, uint32_t npos,
                                    double quantile, float* d_tmp, float* d_tmp2, uint32_t* d_count,
                                    TrainScratch& S, float* h_out, cudaStream_t st);
cudaError_t predict_keys(const float* d_z, const uint8_t* d_lab, uint32_t n, float zthr, uint8_t* d_pred,
                         uint32_t* d_counts, cudaStream_t st);
cudaError_t rank_predicted(const uint32_t* d_keys, const uint32_t* d_est, const uint8_t* d_pred, uint32_t n,
                           uint32_t* d_hkeys, uint32_t* d_hest, uint32_t* d_okeys, uint32_t* d_oest,
                           uint32_t* d_count, TrainScratch& S, uint32_t* h_count, cudaStream_t st);

}  // namespace qsb
