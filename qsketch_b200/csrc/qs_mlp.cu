// qs_mlp.cu — the heavy-hitter classifier of the learned split: an MLP 32 -> 128 -> 128 -> 1
// over the 32 bits of a key (feature x_i = +1 if bit i is set, else -1), ReLU hidden layers,
// BF16 weights and activations, FP32 accumulation on the 5th-generation tensor cores
// (tcgen05.mma, operands in shared memory, accumulators in tensor memory), weighted binary
// cross-entropy.  Forward, backward and the Adam update are written here.  A CTA takes a
// tile of 128 examples, one thread per example row (its TMEM lane); one thread issues the
// MMAs and commits them to an mbarrier the block waits on.
//
// Numerics (the CPU oracle in oracle/mlp.py mirrors the rounding points):
//   W1, W2 bf16; b1, b2, w3, b3 fp32;  h1 = bf16(relu(fp32(x W1^T) + b1));
//   h2 = bf16(relu(fp32(h1 W2^T) + b2));  z = fp32 sum_j h2_j w3_j + b3.
//   dz = (sigmoid(z) - y) * wt / B, wt = pos_weight for positives;  g3 += h2 dz; gb3 += dz;
//   dh2 = bf16(dz * w3 * [h2 > 0]);  gW2 += dh2^T h1;  gb2 += dh2;
//   dh1 = bf16(fp32(dh2 W2) * [h1 > 0]);  gW1 += dh1^T x;  gb1 += dh1.
#include <cuda_bf16.h>

#include "qs_device.cuh"
#include "qs_kernels.h"

namespace qsb {

constexpr int MLP_IN = 32, MLP_H = 128;
constexpr int MLP_T = 128;        // examples per CTA tile: the MMAs' M
constexpr int MLP_THREADS = 128;  // one thread per example row (its TMEM lane)
constexpr int XC = 48;            // X' columns: the 32 features, a ones column (gb1), zeros to a multiple of 16
constexpr int HC = 144;           // H1' columns: the 128 activations, a ones column (gb2), zeros
static_assert(MLP_T == MLP_TILE_EXAMPLES, "the host sizes the backward launches by this tile");

// ---- tcgen05 operands ----------------------------------------------------------------------
// A R x C bf16 matrix in shared memory as 8 x 8 core matrices: element (r, c) at byte
//   (r/8)*(C*16) + (c/8)*128 + (r%8)*16 + (c%8)*2,
// each 16-byte row of a core matrix holding 8 consecutive columns.  Read with C as the K
// dimension this is the canonical K-major layout without swizzle (8-element K chunks 128 B
// apart, 8-row groups C*16 B apart); read with C as the M or N dimension and R as K, it is the
// canonical MN-major layout (MN chunks 128 B apart, 8-row K groups C*16 B apart).  So each
// activation is stored once and serves both orientations (forward and weight-gradient GEMMs).
__host__ __device__ constexpr uint32_t cm_off(uint32_t r, uint32_t c, uint32_t C) {
    return (r >> 3) * (C * 16u) + (c >> 3) * 128u + (r & 7u) * 16u + (c & 7u) * 2u;
}

// Shared-memory matrix descriptor (tcgen05, no swizzle): start address, leading and stride
// byte offsets in 16-byte units, version 1 (bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo, uint32_t sbo) {
    const uint32_t a = smem_addr(p);
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K slice s (16 elements) of a matrix whose C columns are its K dimension.
__device__ __forceinline__ uint64_t desc_kmajor(const uint8_t* base, uint32_t C, int s) {
    return smem_desc(base + s * 256, 128u, C * 16u);
}
// K slice s (rows 16s .. 16s+15) of a matrix whose rows are its K dimension and whose C
// columns are its M or N dimension.
__device__ __forceinline__ uint64_t desc_mnmajor(const uint8_t* base, uint32_t C, int s) {
    return smem_desc(base + (uint32_t)s * 32u * C, C * 16u, 128u);
}
// Instruction descriptor, kind::f16: bf16 A and B, fp32 D, A/B major (0 K, 1 MN), N, M.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N, uint32_t a_mn, uint32_t b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D (TMEM) = A * B (+ D when acc), one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
// The mbarrier completes once every MMA this thread issued before has finished.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Whole warp: ncols TMEM columns (a power of two >= 32), their address written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 16 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32w .. 32w+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}
// 8 values as bf16 into the 16-byte core row of (r, c..c+7).
__device__ __forceinline__ void st_chunk(uint8_t* base, uint32_t r, uint32_t c, uint32_t C, const float* v) {
    *reinterpret_cast<uint4*>(base + cm_off(r, c, C)) =
        make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]), pack_bf16x2(v[6], v[7]));
}

// TMEM columns: forward accumulators, then the backward products in the same space.
constexpr uint32_t TM_ACC1 = 0, TM_ACC2 = 128;   // x W1^T, h1 W2^T            [t][128]
constexpr uint32_t TM_DH1 = 0, TM_GW1 = 128;     // dh2 W2 [t][128], dh1^T x'  [i][48]
constexpr uint32_t TM_GW2 = 256;                 // dh2^T h1'                  [j][144]

struct TcFwd {
    uint8_t X[MLP_T * XC * 2];       // x' [t][48]: the features, ones, zeros
    uint8_t W1[MLP_H * MLP_IN * 2];  // W1 [out][in]
    uint8_t W2[MLP_H * MLP_H * 2];   // W2 [out][in]
    uint8_t H1[MLP_T * HC * 2];      // h1' [t][144]: the activations, ones, zeros
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    uint64_t bar;
    uint32_t tmem;
};
struct TcBwd {
    TcFwd f;
    alignas(128) uint8_t D2[MLP_T * MLP_H * 2];  // dh2 [t][128]
    uint8_t D1[MLP_T * MLP_H * 2];               // dh1 [t][128]
    float g3[MLP_THREADS / 32][MLP_H];
    float red[MLP_THREADS / 32][2];
};
static_assert(offsetof(TcFwd, W1) % 128 == 0 && offsetof(TcFwd, W2) % 128 == 0 && offsetof(TcFwd, H1) % 128 == 0 &&
                  offsetof(TcBwd, D2) % 128 == 0 && offsetof(TcBwd, D1) % 128 == 0,
              "operand tiles 128-byte aligned");

size_t mlp_smem_bytes() { return sizeof(TcBwd); }
size_t mlp_fwd_smem_bytes() { return sizeof(TcFwd); }

// Weights and biases into shared memory (thread t: row t of W1 and W2).
__device__ __forceinline__ void tc_load_weights(TcFwd& S, const MlpDev& M) {
    const int t = threadIdx.x;
    const uint4* w1 = reinterpret_cast<const uint4*>(M.W1) + t * (MLP_IN / 8);
    const uint4* w2 = reinterpret_cast<const uint4*>(M.W2) + t * (MLP_H / 8);
#pragma unroll
    for (int q = 0; q < MLP_IN / 8; ++q) *reinterpret_cast<uint4*>(S.W1 + cm_off(t, 8 * q, MLP_IN)) = __ldg(w1 + q);
#pragma unroll 4
    for (int q = 0; q < MLP_H / 8; ++q) *reinterpret_cast<uint4*>(S.W2 + cm_off(t, 8 * q, MLP_H)) = __ldg(w2 + q);
    S.b1[t] = M.b1[t];
    S.b2[t] = M.b2[t];
    S.w3[t] = M.w3[t];
}

// Row t of x': the 32 key bits as +1 / -1, a one, zeros (a row past n: key 0).
__device__ __forceinline__ void tc_load_features(TcFwd& S, uint32_t key) {
    const int t = threadIdx.x;
    float v[8];
#pragma unroll
    for (int q = 0; q < MLP_IN / 8; ++q) {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = ((key >> (8 * q + i)) & 1u) ? 1.0f : -1.0f;
        st_chunk(S.X, t, 8 * q, XC, v);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = i == 0 ? 1.0f : 0.0f;
    st_chunk(S.X, t, MLP_IN, XC, v);
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = 0.0f;
    st_chunk(S.X, t, MLP_IN + 8, XC, v);
}

// Shared-memory operands written by this block become visible to the tensor cores, and the
// TMEM reads before it are ordered, for the MMAs one thread issues next.
__device__ __forceinline__ void tc_publish() {
    tc_fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    tc_fence_after();
}

// Wait for the MMAs committed to S.bar (phase `ph`, flipped); false (in every thread) after the
// bounded spin.
__device__ __forceinline__ bool tc_wait(TcFwd& S, uint32_t& ph) {
    const bool ok = __syncthreads_and(mbar_wait_bounded(&S.bar, ph));  // the same answer in every thread
    ph ^= 1u;
    tc_fence_after();
    return ok;
}

// Forward of the tile in S.X: h1' into S.H1 (from x W1^T + b1, ReLU, bf16) and the logit of
// this thread's row.  The accumulators stay in TMEM (h1 W2^T at TM_ACC2 for the backward).
// Returns false if an MMA did not complete.
__device__ __forceinline__ bool tc_forward(TcFwd& S, const MlpDev& M, uint32_t& ph, float& z) {
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t lane_base = S.tmem + ((uint32_t)(warp * 32) << 16);
    tc_publish();
    if (t == 0) {
        const uint32_t id = idesc_bf16(MLP_T, MLP_H, 0, 0);
#pragma unroll
        for (int s = 0; s < MLP_IN / 16; ++s)
            umma_bf16(S.tmem + TM_ACC1, desc_kmajor(S.X, XC, s), desc_kmajor(S.W1, MLP_IN, s), id, s > 0);
        umma_commit(&S.bar);
    }
    if (!tc_wait(S, ph)) return false;
    float v[16];
#pragma unroll 1
    for (int q = 0; q < MLP_H / 16; ++q) {
        tmem_ld16(lane_base + TM_ACC1 + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i] + S.b1[16 * q + i], 0.0f);
        st_chunk(S.H1, t, 16 * q, HC, v);
        st_chunk(S.H1, t, 16 * q + 8, HC, v + 8);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = i == 0 ? 1.0f : 0.0f;
    st_chunk(S.H1, t, MLP_H, HC, v);
    st_chunk(S.H1, t, MLP_H + 8, HC, v + 8);
    tc_publish();
    if (t == 0) {
        const uint32_t id = idesc_bf16(MLP_T, MLP_H, 0, 0);
#pragma unroll
        for (int s = 0; s < MLP_H / 16; ++s)
            umma_bf16(S.tmem + TM_ACC2, desc_kmajor(S.H1, HC, s), desc_kmajor(S.W2, MLP_H, s), id, s > 0);
        umma_commit(&S.bar);
    }
    if (!tc_wait(S, ph)) return false;
    float acc = 0.0f;
#pragma unroll 1
    for (int q = 0; q < MLP_H / 16; ++q) {
        tmem_ld16(lane_base + TM_ACC2 + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; ++i)
            acc += __bfloat162float(__float2bfloat16(fmaxf(v[i] + S.b2[16 * q + i], 0.0f))) * S.w3[16 * q + i];
    }
    z = acc + *M.b3;
    return true;
}

// Block setup of the tcgen05 kernels: the mbarrier, ncols TMEM columns (warp 0), the weights.
__device__ __forceinline__ void tc_setup(TcFwd& S, const MlpDev& M, uint32_t ncols) {
    if (threadIdx.x == 0) {
        mbar_init(&S.bar, 1);
        fence_mbar_init();
    }
    if (threadIdx.x < 32) tmem_alloc(&S.tmem, ncols);
    tc_load_weights(S, M);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__device__ __forceinline__ void tc_teardown(TcFwd& S, uint32_t ncols) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32) tmem_dealloc(S.tmem, ncols);
}

__global__ void __launch_bounds__(MLP_THREADS) k_mlp_forward(const uint32_t* __restrict__ keys, uint64_t n, MlpDev M,
                                                             float* __restrict__ logits) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    TcFwd& S = *reinterpret_cast<TcFwd*>(smem_raw);
    tc_setup(S, M, 256);
    uint32_t ph = 0;
    bool ok = true;
    for (uint64_t base = (uint64_t)blockIdx.x * MLP_T; base < n && ok; base += (uint64_t)gridDim.x * MLP_T) {
        const uint64_t i = base + threadIdx.x;
        tc_load_features(S, i < n ? __ldg(keys + i) : 0u);
        float z = 0.0f;
        ok = tc_forward(S, M, ph, z);
        if (ok && i < n) logits[i] = z;
    }
    if (!ok && threadIdx.x == 0) atomicOr(M.status, ST_TIMEOUT);
    tc_teardown(S, 256);
}

// Classify the keys that missed the exact table; keys predicted heavy (z >= threshold) join the
// candidate set (deduplicated; order of arrival does not matter, admission sorts them).
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_classify(MlpDev M, RouteDev R, uint64_t max_misses) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    TcFwd& S = *reinterpret_cast<TcFwd*>(smem_raw);
    const uint64_t n = min((uint64_t)__ldcg(R.n_misses), max_misses);
    if ((uint64_t)blockIdx.x * MLP_T >= n) return;
    tc_setup(S, M, 256);
    uint32_t ph = 0;
    bool ok = true;
    for (uint64_t base = (uint64_t)blockIdx.x * MLP_T; base < n && ok; base += (uint64_t)gridDim.x * MLP_T) {
        const uint64_t i = base + threadIdx.x;
        const uint32_t key = i < n ? R.misses[i] : 0u;
        tc_load_features(S, key);
        float z = 0.0f;
        ok = tc_forward(S, M, ph, z);
        if (ok && i < n && z >= R.z_threshold && key != 0xffffffffu) {
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
    if (!ok && threadIdx.x == 0) atomicOr(M.status, ST_TIMEOUT);
    tc_teardown(S, 256);
}

// Gradients of the weighted BCE over examples [tile0*128, ...): CTA b handles tile tile0+b and
// writes its partial gradient (fp32, MLP_PARAMS) to partials + b*MLP_PARTIAL_STRIDE (16-byte
// aligned rows for the vector stores) and its loss sum
// to ploss[b]; k_mlp_reduce then adds the partials in tile order, so the result does not
// depend on scheduling.  Products on the tensor cores (fp32 in TMEM):
//   gW2 | gb2 = dh2^T [h1 | 1]   (A = dh2 read MN-major, B = h1' read MN-major)
//   dh1       = dh2 W2           (A = dh2 K-major, B = W2 read MN-major)
//   gW1 | gb1 = dh1^T [x | 1]    (A = dh1 MN-major, B = x' MN-major)
// g3 = h2^T dz and gb3 = sum dz in fp32 on the CUDA cores.
__global__ void __launch_bounds__(MLP_THREADS) k_mlp_backward(const uint32_t* __restrict__ keys,
                                                              const uint8_t* __restrict__ labels, uint64_t n,
                                                              uint64_t tile0, float pos_weight, float inv_batch,
                                                              MlpDev M, float* __restrict__ partials,
                                                              float* __restrict__ ploss) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    TcBwd& B = *reinterpret_cast<TcBwd*>(smem_raw);
    TcFwd& S = B.f;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    float* G = partials + (uint64_t)blockIdx.x * MLP_PARTIAL_STRIDE;
    const uint64_t base = (tile0 + blockIdx.x) * MLP_T;
    const uint64_t i = base + t;
    griddep_wait();  // the previous step's update of the weights has ended
    tc_setup(S, M, 512);
    const uint32_t lane_base = S.tmem + ((uint32_t)(warp * 32) << 16);
    tc_load_features(S, i < n ? __ldg(keys + i) : 0u);
    uint32_t ph = 0;
    float z = 0.0f;
    bool ok = tc_forward(S, M, ph, z);
    // loss and dz of this row
    float lsum = 0.0f, dz = 0.0f;
    if (i < n) {
        const float y = labels[i] ? 1.0f : 0.0f;
        const float w = labels[i] ? pos_weight : 1.0f;
        const float p = 1.0f / (1.0f + __expf(-z));
        lsum = w * (fmaxf(z, 0.0f) - z * y + log1pf(__expf(-fabsf(z))));  // log(1+e^-|z|) form
        dz = (p - y) * w * inv_batch;
    }
    // dh2 = bf16(dz * w3 * [h2 > 0]) into B.D2; g3 = sum over rows of h2 * dz (per warp, then
    // over the warps)
    float v[16];
#pragma unroll 1
    for (int q = 0; q < MLP_H / 16 && ok; ++q) {
        tmem_ld16(lane_base + TM_ACC2 + 16 * q, v);
        float d[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int c = 16 * q + k;
            const float h2 = __bfloat162float(__float2bfloat16(fmaxf(v[k] + S.b2[c], 0.0f)));
            d[k] = h2 > 0.0f ? dz * S.w3[c] : 0.0f;
            float g = h2 * dz;
#pragma unroll
            for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
            if (lane == 0) B.g3[warp][c] = g;
        }
        st_chunk(B.D2, t, 16 * q, MLP_H, d);
        st_chunk(B.D2, t, 16 * q + 8, MLP_H, d + 8);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        dz += __shfl_xor_sync(0xffffffffu, dz, o);
    }
    if (lane == 0) {
        B.red[warp][0] = lsum;
        B.red[warp][1] = dz;
    }
    tc_publish();
    if (ok && t == 0) {
        const uint32_t id_gw2 = idesc_bf16(MLP_H, HC, 1, 1), id_dh1 = idesc_bf16(MLP_T, MLP_H, 0, 1);
#pragma unroll
        for (int s = 0; s < MLP_T / 16; ++s)
            umma_bf16(S.tmem + TM_GW2, desc_mnmajor(B.D2, MLP_H, s), desc_mnmajor(S.H1, HC, s), id_gw2, s > 0);
#pragma unroll
        for (int s = 0; s < MLP_H / 16; ++s)
            umma_bf16(S.tmem + TM_DH1, desc_kmajor(B.D2, MLP_H, s), desc_mnmajor(S.W2, MLP_H, s), id_dh1, s > 0);
        umma_commit(&S.bar);
    }
    if (ok) ok = tc_wait(S, ph);
    // dh1 = bf16(fp32(dh2 W2) * [h1 > 0]) into B.D1 (h1 > 0 read back from S.H1)
#pragma unroll 1
    for (int q = 0; q < MLP_H / 16 && ok; ++q) {
        tmem_ld16(lane_base + TM_DH1 + 16 * q, v);
        const uint4 h_lo = *reinterpret_cast<const uint4*>(S.H1 + cm_off(t, 16 * q, HC));
        const uint4 h_hi = *reinterpret_cast<const uint4*>(S.H1 + cm_off(t, 16 * q + 8, HC));
        const uint32_t hw[8] = {h_lo.x, h_lo.y, h_lo.z, h_lo.w, h_hi.x, h_hi.y, h_hi.z, h_hi.w};
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const uint32_t bits = (hw[k >> 1] >> (16 * (k & 1))) & 0xffffu;  // bf16 h1 > 0: sign clear, not zero
            v[k] = (bits != 0u && bits < 0x8000u) ? v[k] : 0.0f;
        }
        st_chunk(B.D1, t, 16 * q, MLP_H, v);
        st_chunk(B.D1, t, 16 * q + 8, MLP_H, v + 8);
    }
    tc_publish();
    if (ok && t == 0) {
        const uint32_t id = idesc_bf16(MLP_H, XC, 1, 1);
#pragma unroll
        for (int s = 0; s < MLP_T / 16; ++s)
            umma_bf16(S.tmem + TM_GW1, desc_mnmajor(B.D1, MLP_H, s), desc_mnmajor(S.X, XC, s), id, s > 0);
        umma_commit(&S.bar);
    }
    if (ok) ok = tc_wait(S, ph);
    // this thread's row of gW2 | gb2 (row j = t) and of gW1 | gb1 (row i = t)
    float* gW1 = G;
    float* gW2 = G + MLP_W1_N;
    float* gb1 = G + MLP_BF16_PARAMS;
    float* gb2 = gb1 + MLP_H;
    float* g3 = gb2 + MLP_H;
    float* gb3 = g3 + MLP_H;
#pragma unroll 1
    for (int q = 0; q < HC / 16 && ok; ++q) {
        tmem_ld16(lane_base + TM_GW2 + 16 * q, v);
        if (q < MLP_H / 16) {
            float4* dst = reinterpret_cast<float4*>(gW2 + (uint64_t)t * MLP_H + 16 * q);
#pragma unroll
            for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        } else {
            gb2[t] = v[0];
        }
    }
#pragma unroll 1
    for (int q = 0; q < XC / 16 && ok; ++q) {
        tmem_ld16(lane_base + TM_GW1 + 16 * q, v);
        if (q < MLP_IN / 16) {
            float4* dst = reinterpret_cast<float4*>(gW1 + (uint64_t)t * MLP_IN + 16 * q);
#pragma unroll
            for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
        } else {
            gb1[t] = v[0];
        }
    }
    __syncthreads();
    float gs = 0.0f;
#pragma unroll
    for (int w = 0; w < MLP_THREADS / 32; ++w) gs += B.g3[w][t];
    g3[t] = gs;
    if (t == 0) {
        float l = 0.0f, d = 0.0f;
#pragma unroll
        for (int w = 0; w < MLP_THREADS / 32; ++w) l += B.red[w][0], d += B.red[w][1];
        ploss[blockIdx.x] = l;
        *gb3 = d;
        if (!ok) atomicOr(M.status, ST_TIMEOUT);
    }
    tc_teardown(S, 512);
}

// grads += sum over tiles (in order) of the partial gradients; *loss += sum of the tile losses.
__global__ void k_mlp_reduce(const float* __restrict__ partials, const float* __restrict__ ploss, uint32_t tiles,
                             float* __restrict__ grads, float* __restrict__ loss) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_PARAMS; i += gridDim.x * blockDim.x) {
        float s = grads[i];
        for (uint32_t t = 0; t < tiles; ++t) s += partials[(uint64_t)t * MLP_PARTIAL_STRIDE + i];
        grads[i] = s;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float s = *loss;
        for (uint32_t t = 0; t < tiles; ++t) s += ploss[t];
        *loss = s;
    }
}

// One training step's reduction and update: grads[i] plus the tiles' partials of parameter
// i (in tile order), then Adam as k_adam does, gradients left cleared; *loss = the tiles'
// loss sum.  The next step's backward may be scheduled at once (it waits for this kernel).
__global__ void k_mlp_reduce_adam(const float* __restrict__ partials, const float* __restrict__ ploss,
                                  uint32_t tiles, float* __restrict__ loss, float* __restrict__ p,
                                  float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, uint32_t count,
                                  float lr, float b1, float b2, float eps, float c1, float c2,
                                  __nv_bfloat16* __restrict__ w_bf16, uint32_t n_bf16) {
    griddep_wait();
    griddep_launch_dependents();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        for (uint32_t t = 0; t < tiles; ++t) gi += partials[(uint64_t)t * MLP_PARTIAL_STRIDE + i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        g[i] = 0.0f;
        if (i < n_bf16) w_bf16[i] = __float2bfloat16(pi);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float s = 0.0f;
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
                                         (int)mlp_fwd_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void*)k_mlp_classify, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mlp_fwd_smem_bytes());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute((const void*)k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)mlp_smem_bytes());
}

// Forward grids hold two blocks per SM (256 TMEM columns each); the backward one per SM (512).
cudaError_t mlp_forward(const uint32_t* d_keys, uint64_t n, const MlpDev& M, float* d_logits, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const uint64_t tiles = (n + MLP_T - 1) / MLP_T;
    const int grid = (int)std::min<uint64_t>(tiles, 148ull * 2);
    k_mlp_forward<<<grid, MLP_THREADS, mlp_fwd_smem_bytes(), st>>>(d_keys, n, M, d_logits);
    return cudaGetLastError();
}

cudaError_t classify_misses(const MlpDev& M, const RouteDev& R, uint64_t max_misses, cudaStream_t st) {
    if (max_misses == 0) return cudaSuccess;
    const uint64_t tiles = (max_misses + MLP_T - 1) / MLP_T;
    const int grid = (int)std::min<uint64_t>(tiles, 148ull * 2);
    k_mlp_classify<<<grid, MLP_THREADS, mlp_fwd_smem_bytes(), st>>>(M, R, max_misses);
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

cudaError_t mlp_train_step(const uint32_t* d_keys, const uint8_t* d_labels, uint64_t n, float pos_weight,
                           float inv_batch, const MlpDev& M, float* d_loss, uint32_t step, float lr, cudaStream_t st) {
    const uint64_t tiles = (n + MLP_T - 1) / MLP_T;
    if (tiles > MLP_MAX_TILES) {  // several backward launches accumulate into the gradients
        cudaError_t e = cudaMemsetAsync(d_loss, 0, 4, st);
        if (e == cudaSuccess) e = mlp_backward(d_keys, d_labels, n, pos_weight, inv_batch, M, d_loss, st);
        if (e == cudaSuccess) e = mlp_adam(M, step, lr, st);
        return e;
    }
    uint32_t nt = (uint32_t)std::max<uint64_t>(1ull, tiles);
    uint64_t tile0 = 0;
    MlpDev Mc = M;
    float* partials = M.partials;
    float* ploss = M.ploss;
    void* bargs[] = {(void*)&d_keys, (void*)&d_labels, (void*)&n, (void*)&tile0, (void*)&pos_weight, (void*)&inv_batch,
                     (void*)&Mc, (void*)&partials, (void*)&ploss};
    cudaError_t e = launch_pdl((const void*)k_mlp_backward, dim3(nt), dim3(MLP_THREADS), mlp_smem_bytes(), st, bargs,
                               false);
    if (e != cudaSuccess) return e;
    float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    float* params = M.params;
    float* grads = M.grads;
    float* am = M.adam_m;
    float* av = M.adam_v;
    uint32_t count = MLP_PARAMS, n_bf16 = MLP_BF16_PARAMS;
    __nv_bfloat16* w = M.W1;
    void* rargs[] = {(void*)&partials, (void*)&ploss, (void*)&nt, (void*)&d_loss, (void*)&params, (void*)&grads,
                     (void*)&am, (void*)&av, (void*)&count, (void*)&lr, (void*)&b1, (void*)&b2, (void*)&eps,
                     (void*)&c1, (void*)&c2, (void*)&w, (void*)&n_bf16};
    return launch_pdl((const void*)k_mlp_reduce_adam, dim3(82), dim3(256), 0, st, rargs, false);
}

cudaError_t mlp_refresh_bf16(const MlpDev& M, cudaStream_t st) {
    k_to_bf16<<<64, 256, 0, st>>>(M.params, M.W1, MLP_BF16_PARAMS);
    return cudaGetLastError();
}

}  // namespace qsb
