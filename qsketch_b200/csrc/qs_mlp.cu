// qs_mlp.cu — the heavy-hitter classifier of the learned split: an MLP 32 -> 128 -> 128 -> 1
// over the 32 bits of a key (feature x_i = +1 if bit i is set, else -1), ReLU hidden layers,
// BF16 weights and activations, FP32 accumulation on the tensor cores, weighted binary
// cross-entropy.  Forward, backward and the Adam update are written here.
//
// Numerics (the CPU oracle in oracle/mlp.py mirrors the rounding points):
//   W1, W2 bf16; b1, b2, w3, b3 fp32;  h1 = bf16(relu(fp32(x W1^T) + b1));
//   h2 = bf16(relu(fp32(h1 W2^T) + b2));  z = fp32 sum_j h2_j w3_j + b3.
//   dz = (sigmoid(z) - y) * wt / B, wt = pos_weight for positives;  g3 += h2 dz; gb3 += dz;
//   dh2 = bf16(dz * w3 * [h2 > 0]);  gW2 += dh2^T h1;  gb2 += dh2;
//   dh1 = bf16(fp32(dh2 W2) * [h1 > 0]);  gW1 += dh1^T x;  gb1 += dh1.
#include <mma.h>
#include <cuda_bf16.h>

#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {
using namespace nvcuda;

constexpr int MLP_IN = 32, MLP_H = 128;
constexpr int MLP_T = 64;  // examples per CTA tile
constexpr int MLP_THREADS = 256;

struct MlpSmem {
    __nv_bfloat16 W1[MLP_H * MLP_IN];   // row-major [out][in]
    __nv_bfloat16 W2[MLP_H * MLP_H];    // row-major [out][in]
    __nv_bfloat16 X[MLP_T * MLP_IN];
    __nv_bfloat16 H1[MLP_T * MLP_H];
    __nv_bfloat16 H2[MLP_T * MLP_H];
    __nv_bfloat16 D2[MLP_T * MLP_H];    // dh2
    __nv_bfloat16 D1[MLP_T * MLP_H];    // dh1
    float F[MLP_H * MLP_H];             // fp32 staging: activations [T][128] or weight grads [128][128]
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    float z[MLP_T], dz[MLP_T];
};

size_t mlp_smem_bytes() { return sizeof(MlpSmem); }

__device__ __forceinline__ void load_weights(MlpSmem& S, const MlpDev& M) {
    for (int i = threadIdx.x; i < MLP_H * MLP_IN; i += blockDim.x) S.W1[i] = M.W1[i];
    for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) S.W2[i] = M.W2[i];
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
        S.b1[i] = M.b1[i];
        S.b2[i] = M.b2[i];
        S.w3[i] = M.w3[i];
    }
}

__device__ __forceinline__ void load_features(MlpSmem& S, const uint32_t* keys, uint64_t base, uint64_t n) {
    for (int i = threadIdx.x; i < MLP_T * MLP_IN; i += blockDim.x) {
        const int r = i / MLP_IN, c = i % MLP_IN;
        const uint64_t k = base + r;
        const uint32_t key = k < n ? keys[k] : 0u;
        S.X[i] = __float2bfloat16(((key >> c) & 1u) ? 1.0f : -1.0f);
    }
}

// C[T x 128] (fp32, into S.F, row-major ld 128) = A[T x K] (row-major bf16, ld K) * B where
// B is W^T: W row-major [128][K] read as a col-major K x 128 matrix.
template <int K>
__device__ __forceinline__ void gemm_xwT(MlpSmem& S, const __nv_bfloat16* A, const __nv_bfloat16* W) {
    const int warp = threadIdx.x >> 5;
    // 4 row tiles x 8 col tiles of 16x16; 8 warps -> 4 tiles each
    for (int t = warp; t < (MLP_T / 16) * (MLP_H / 16); t += MLP_THREADS / 32) {
        const int tr = t / (MLP_H / 16), tc = t % (MLP_H / 16);
        wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
        wmma::fill_fragment(acc, 0.0f);
#pragma unroll
        for (int k = 0; k < K; k += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> b;
            wmma::load_matrix_sync(a, A + tr * 16 * K + k, K);
            wmma::load_matrix_sync(b, W + tc * 16 * K + k, K);
            wmma::mma_sync(acc, a, b, acc);
        }
        wmma::store_matrix_sync(S.F + tr * 16 * MLP_H + tc * 16, acc, MLP_H, wmma::mem_row_major);
    }
}

// Forward pass of one tile; leaves h1, h2 in shared memory and z in S.z.
__device__ __forceinline__ void forward_tile(MlpSmem& S, const MlpDev& M) {
    gemm_xwT<MLP_IN>(S, S.X, S.W1);
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_T * MLP_H; i += blockDim.x)
        S.H1[i] = __float2bfloat16(fmaxf(S.F[i] + S.b1[i % MLP_H], 0.0f));
    __syncthreads();
    gemm_xwT<MLP_H>(S, S.H1, S.W2);
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_T * MLP_H; i += blockDim.x)
        S.H2[i] = __float2bfloat16(fmaxf(S.F[i] + S.b2[i % MLP_H], 0.0f));
    __syncthreads();
    // z = h2 . w3 + b3: a warp per row
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < MLP_T; r += MLP_THREADS / 32) {
        float s = 0.0f;
        for (int j = lane; j < MLP_H; j += 32) s += __bfloat162float(S.H2[r * MLP_H + j]) * S.w3[j];
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) S.z[r] = s + *M.b3;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_forward(const uint32_t* __restrict__ keys, uint64_t n, MlpDev M,
                                                             float* __restrict__ logits) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
    load_weights(S, M);
    for (uint64_t base = (uint64_t)blockIdx.x * MLP_T; base < n; base += (uint64_t)gridDim.x * MLP_T) {
        load_features(S, keys, base, n);
        __syncthreads();
        forward_tile(S, M);
        for (int r = threadIdx.x; r < MLP_T; r += blockDim.x)
            if (base + r < n) logits[base + r] = S.z[r];
        __syncthreads();
    }
}

// Classify the keys that missed the exact table; keys predicted heavy (z >= threshold) join the
// candidate set (deduplicated; order of arrival does not matter, admission sorts them).
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_classify(MlpDev M, RouteDev R, uint64_t max_misses) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
    const uint64_t n = min((uint64_t)__ldcg(R.n_misses), max_misses);
    if ((uint64_t)blockIdx.x * MLP_T >= n) return;
    load_weights(S, M);
    for (uint64_t base = (uint64_t)blockIdx.x * MLP_T; base < n; base += (uint64_t)gridDim.x * MLP_T) {
        load_features(S, R.misses, base, n);
        __syncthreads();
        forward_tile(S, M);
        if (threadIdx.x < MLP_T && base + threadIdx.x < n && S.z[threadIdx.x] >= R.z_threshold) {
            const uint32_t key = R.misses[base + threadIdx.x];
            if (key != 0xffffffffu) {
                uint32_t h = mix32(key) & (R.cand_slots - 1);
                for (uint32_t p = 0; p < 64; ++p, h = (h + 1) & (R.cand_slots - 1)) {  // a full set drops
                    const uint32_t prev = atomicCAS(R.cand_keys + h, 0xffffffffu, key);
                    if (prev == 0xffffffffu) {
                        const uint32_t at = atomicAdd(R.n_cand, 1u);
                        if (at < R.cand_slots) R.cand_list[at] = key;
                        break;
                    }
                    if (prev == key) break;
                }
            }
        }
        __syncthreads();
    }
}

// dW (fp32, S.F as [128][ldb]) = A^T B with A [T x 128] row-major bf16 (read col-major) and
// B [T x N] row-major bf16; N = 128 or 32.
template <int N>
__device__ __forceinline__ void gemm_aT_b(MlpSmem& S, const __nv_bfloat16* A, const __nv_bfloat16* B) {
    const int warp = threadIdx.x >> 5;
    for (int t = warp; t < (MLP_H / 16) * (N / 16); t += MLP_THREADS / 32) {
        const int tr = t / (N / 16), tc = t % (N / 16);
        wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
        wmma::fill_fragment(acc, 0.0f);
#pragma unroll
        for (int k = 0; k < MLP_T; k += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> a;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> b;
            wmma::load_matrix_sync(a, A + k * MLP_H + tr * 16, MLP_H);
            wmma::load_matrix_sync(b, B + k * N + tc * 16, N);
            wmma::mma_sync(acc, a, b, acc);
        }
        wmma::store_matrix_sync(S.F + tr * 16 * N + tc * 16, acc, N, wmma::mem_row_major);
    }
}

// Gradients of the weighted BCE over examples [tile0*64, ...): CTA b handles tile tile0+b and
// writes its partial gradient (fp32, MLP_PARAMS) to partials + b*MLP_PARAMS and its loss sum
// to ploss[b]; k_mlp_reduce then adds the partials in tile order, so the result does not
// depend on scheduling.
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_backward(const uint32_t* __restrict__ keys,
                                                              const uint8_t* __restrict__ labels, uint64_t n,
                                                              uint64_t tile0, float pos_weight, float inv_batch,
                                                              MlpDev M, float* __restrict__ partials,
                                                              float* __restrict__ ploss) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float* G = partials + (uint64_t)blockIdx.x * MLP_PARAMS;
    float* gW1 = G;
    float* gW2 = G + MLP_W1_N;
    float* gb1 = G + MLP_BF16_PARAMS;
    float* gb2 = gb1 + MLP_H;
    float* g3 = gb2 + MLP_H;
    float* gb3 = g3 + MLP_H;
    const uint64_t base = (tile0 + blockIdx.x) * MLP_T;
    load_weights(S, M);
    load_features(S, keys, base, n);
    __syncthreads();
    forward_tile(S, M);
    // loss and dz
    float lsum = 0.0f, dzsum = 0.0f;
    if (tid < MLP_T) {
        const uint64_t i = base + tid;
        float dz = 0.0f;
        if (i < n) {
            const float z = S.z[tid];
            const float y = labels[i] ? 1.0f : 0.0f;
            const float w = labels[i] ? pos_weight : 1.0f;
            const float p = 1.0f / (1.0f + __expf(-z));
            const float l = fmaxf(z, 0.0f) - z * y + log1pf(__expf(-fabsf(z)));  // log(1+e^-|z|) form
            lsum = w * l;
            dz = (p - y) * w * inv_batch;
        }
        S.dz[tid] = dz;
        dzsum = dz;
    }
    __shared__ float s_red[2][2];
    if (warp < 2) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
            dzsum += __shfl_xor_sync(0xffffffffu, dzsum, o);
        }
        if (lane == 0) {
            s_red[warp][0] = lsum;
            s_red[warp][1] = dzsum;
        }
    }
    __syncthreads();
    if (tid == 0) {
        ploss[blockIdx.x] = s_red[0][0] + s_red[1][0];
        *gb3 = s_red[0][1] + s_red[1][1];
    }
    // dh2, g3
    for (int i = tid; i < MLP_T * MLP_H; i += blockDim.x) {
        const int r = i / MLP_H, j = i % MLP_H;
        const float h = __bfloat162float(S.H2[i]);
        S.D2[i] = __float2bfloat16(h > 0.0f ? S.dz[r] * S.w3[j] : 0.0f);
    }
    for (int j = tid; j < MLP_H; j += blockDim.x) {
        float g = 0.0f;
        for (int r = 0; r < MLP_T; ++r) g += __bfloat162float(S.H2[r * MLP_H + j]) * S.dz[r];
        g3[j] = g;
    }
    __syncthreads();
    // gb2 = colsum(dh2); gW2 = dh2^T h1
    for (int j = tid; j < MLP_H; j += blockDim.x) {
        float g = 0.0f;
        for (int r = 0; r < MLP_T; ++r) g += __bfloat162float(S.D2[r * MLP_H + j]);
        gb2[j] = g;
    }
    gemm_aT_b<MLP_H>(S, S.D2, S.H1);
    __syncthreads();
    for (int i = tid; i < MLP_H * MLP_H; i += blockDim.x) gW2[i] = S.F[i];
    __syncthreads();
    // dh1 = (dh2 W2) * [h1 > 0]: B = W2 row-major [128][128] used as is
    for (int t = warp; t < (MLP_T / 16) * (MLP_H / 16); t += MLP_THREADS / 32) {
        const int tr = t / (MLP_H / 16), tc = t % (MLP_H / 16);
        wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
        wmma::fill_fragment(acc, 0.0f);
#pragma unroll
        for (int k = 0; k < MLP_H; k += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> b;
            wmma::load_matrix_sync(a, S.D2 + tr * 16 * MLP_H + k, MLP_H);
            wmma::load_matrix_sync(b, S.W2 + k * MLP_H + tc * 16, MLP_H);
            wmma::mma_sync(acc, a, b, acc);
        }
        wmma::store_matrix_sync(S.F + tr * 16 * MLP_H + tc * 16, acc, MLP_H, wmma::mem_row_major);
    }
    __syncthreads();
    for (int i = tid; i < MLP_T * MLP_H; i += blockDim.x)
        S.D1[i] = __float2bfloat16(__bfloat162float(S.H1[i]) > 0.0f ? S.F[i] : 0.0f);
    __syncthreads();
    for (int j = tid; j < MLP_H; j += blockDim.x) {
        float g = 0.0f;
        for (int r = 0; r < MLP_T; ++r) g += __bfloat162float(S.D1[r * MLP_H + j]);
        gb1[j] = g;
    }
    gemm_aT_b<MLP_IN>(S, S.D1, S.X);
    __syncthreads();
    for (int i = tid; i < MLP_H * MLP_IN; i += blockDim.x) gW1[i] = S.F[i];
}

// grads += sum over tiles (in order) of the partial gradients; *loss += sum of the tile losses.
__global__ void k_mlp_reduce(const float* __restrict__ partials, const float* __restrict__ ploss, uint32_t tiles,
                             float* __restrict__ grads, float* __restrict__ loss) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_PARAMS; i += gridDim.x * blockDim.x) {
        float s = grads[i];
        for (uint32_t t = 0; t < tiles; ++t) s += partials[(uint64_t)t * MLP_PARAMS + i];
        grads[i] = s;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float s = *loss;
        for (uint32_t t = 0; t < tiles; ++t) s += ploss[t];
        *loss = s;
    }
}

// Adam (Kingma & Ba 2015) on the fp32 master parameters; refreshes the bf16 copies and
// clears the gradients.  Parameters are one flat fp32 array: W1 | W2 | b1 | b2 | w3 | b3.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       uint32_t count, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ w_bf16, uint32_t n_bf16) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        g[i] = 0.0f;
        if (i < n_bf16) w_bf16[i] = __float2bfloat16(pi);
    }
}

__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ w, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        w[i] = __float2bfloat16(p[i]);
}

cudaError_t mlp_configure() {
    cudaError_t e = cudaFuncSetAttribute((const void*)k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mlp_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void*)k_mlp_classify, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mlp_smem_bytes());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute((const void*)k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)mlp_smem_bytes());
}

cudaError_t mlp_forward(const uint32_t* d_keys, uint64_t n, const MlpDev& M, float* d_logits, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t tiles = (n + MLP_T - 1) / MLP_T;
    const int grid = (int)std::min<uint64_t>(tiles, 148ull * 8);
    k_mlp_forward<<<grid, MLP_THREADS, mlp_smem_bytes(), st>>>(d_keys, n, M, d_logits);
    return cudaGetLastError();
}

cudaError_t classify_misses(const MlpDev& M, const RouteDev& R, uint64_t max_misses, cudaStream_t st) {
    if (max_misses == 0) return cudaSuccess;
    const uint64_t tiles = (max_misses + MLP_T - 1) / MLP_T;
    const int grid = (int)std::min<uint64_t>(tiles, 148ull);
    k_mlp_classify<<<grid, MLP_THREADS, mlp_smem_bytes(), st>>>(M, R, max_misses);
    return cudaGetLastError();
}

cudaError_t mlp_backward(const uint32_t* d_keys, const uint8_t* d_labels, uint64_t n, float pos_weight,
                         float inv_batch, const MlpDev& M, float* d_loss, cudaStream_t st) {
    const uint64_t tiles = (n + MLP_T - 1) / MLP_T;
    for (uint64_t t0 = 0; t0 < tiles; t0 += MLP_MAX_TILES) {
        const uint32_t nt = (uint32_t)std::min<uint64_t>(MLP_MAX_TILES, tiles - t0);
        k_mlp_backward<<<nt, MLP_THREADS, mlp_smem_bytes(), st>>>(d_keys, d_labels, n, t0, pos_weight, inv_batch, M,
                                                                   M.partials, M.ploss);
        k_mlp_reduce<<<82, 256, 0, st>>>(M.partials, M.ploss, nt, M.grads, d_loss);
    }
    return cudaGetLastError();
}

cudaError_t mlp_adam(const MlpDev& M, uint32_t step, float lr, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<64, 256, 0, st>>>(M.params, M.grads, M.adam_m, M.adam_v, MLP_PARAMS, lr, b1, b2, eps, c1, c2, M.W1,
                               MLP_BF16_PARAMS);
    return cudaGetLastError();
}

cudaError_t mlp_refresh_bf16(const MlpDev& M, cudaStream_t st) {
    k_to_bf16<<<64, 256, 0, st>>>(M.params, M.W1, MLP_BF16_PARAMS);
    return cudaGetLastError();
}

}  // namespace qsb
