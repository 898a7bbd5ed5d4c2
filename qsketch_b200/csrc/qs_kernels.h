// qs_kernels.h — host-side launchers of the sm_100a kernels (internal to libqsketch).
#pragma once
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>
#include "qs_common.cuh"

namespace qsb {

struct MswsLaunch {
    int num_sms;
    int insert_grid;
    int repair_grid;
    int query_grid;
};

size_t msws_insert_smem(uint32_t n_masks);
cudaError_t msws_configure(int device, uint32_t n_masks, MswsLaunch* L);
// Pass 1 (packed atomics + crossing detection) and the ordered repair of one chunk of at
// most max_batch keys; the repair exits at once when nothing crossed.
cudaError_t msws_insert_pass(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, int agg,
                             cudaStream_t st);
cudaError_t msws_repair(const uint32_t* d_keys, uint64_t n, const MswsDev& D, const MswsLaunch& L, cudaStream_t st);
cudaError_t msws_query(const uint32_t* d_keys, uint64_t n, uint32_t* d_out, const MswsDev& D, const MswsLaunch& L,
                       cudaStream_t st);

cudaError_t cm_insert(const uint32_t* d_keys, uint64_t n, const CmDev& D, int agg, int grid, cudaStream_t st);
cudaError_t cm_query(const uint32_t* d_keys, uint64_t n, uint32_t* d_out, const CmDev& D, int grid, cudaStream_t st);

cudaError_t gen_keys(uint32_t kind, uint64_t seed, uint64_t n_ranks, double s, uint64_t perm_seed, uint32_t* d_keys,
                     uint32_t* d_ranks, uint64_t n, cudaStream_t st);
cudaError_t gen_rank_keys(uint64_t perm_seed, uint64_t first, uint32_t* d_keys, uint64_t n, cudaStream_t st);
cudaError_t rank_histogram(const uint32_t* d_ranks, uint64_t n, uint32_t* d_hist, uint64_t n_ranks, cudaStream_t st);
cudaError_t error_metrics(const uint32_t* d_est, const uint32_t* d_exact, uint64_t n, double* d_acc,
                          cudaStream_t st);
cudaError_t probe(uint32_t kind, uint64_t bytes, uint64_t ops, double* ops_per_s);

// Text returned by qs_last_error_string() on this host thread.
void set_last_error(const char* text);

}  // namespace qsb
