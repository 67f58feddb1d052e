// BF16 inference of the sequence encoder on the 5th-generation tensor cores: the embedding path
// of the learned proposals (the fp32 kernels of encoder.cu stay the training reference).
//
// A chunk of sequences is laid out as tiles of 4 sequences x 32 positions = 128 rows.  Every
// 128-wide activation lives in HBM as bf16 in the tcgen05 operand layout: per tile two 16 KB
// blocks (columns 0-63, 64-127), row r at r*128 bytes, the 16-byte unit u of a row stored at
// u ^ (r & 7) (the 128-byte swizzle).  One bulk copy of a tile's 32 KB is then a ready K-major
// A operand, and an output tile staged in shared memory leaves with one bulk store.
//
// Layers (the fp32 model's, with bf16 activations and fp32 accumulation):
//   conv1      gather of W1 rows by residue code (CUDA cores)  -> h1
//   conv2      one GEMM h1 x [W2_-1 | W2_0 | W2_+1] (N = 384) whose epilogue shifts the three
//              column blocks by -1 / 0 / +1 rows inside each sequence (a sequence is one warp's
//              32 TMEM lanes, so the shift is a warp shuffle), adds b2, applies ReLU, adds the
//              h1 skip and masks the padding                      -> h
//   2 x attention: one fused kernel per layer (attn_layer_kernel): QKV, the block-diagonal
//              scores, softmax, P V and the Wo projection with the residual, all on the tensor
//              cores with the intermediates in TMEM and shared memory      -> h'
//   pool       mean over the valid positions, x Wout + bout, unit length -> embedding
// Both tensor-core kernels are persistent (one CTA per SM): the weights are bulk-copied into
// shared memory once, activation tiles stream in by bulk copy, one thread issues tcgen05.mma
// (M = 128, N = 128 per instruction, K = 16) into TMEM, and 8 epilogue warps drain the
// accumulators with tcgen05.ld.  Every wait is bounded.
#include <cuda_bf16.h>

#include <cstring>
#include <vector>

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>

#include "common.cuh"
#include "encoder_layout.cuh"
#include "tc.cuh"

namespace stb {

namespace {

using namespace enc;

constexpr int kTileRows = 128;
constexpr int kTileBytes = kTileRows * kW * 2;  // 32 KB
constexpr int kSeqPerTile = kTileRows / kP;     // 4

// Byte offset of the 16-byte unit u (columns 8u .. 8u+7) of row r in the tiled layout.
__host__ __device__ __forceinline__ int64_t unit_off(int64_t r, int u) {
    const int rr = int(r & 127);
    return (r >> 7) * kTileBytes + (u >> 3) * 16384 + rr * 128 + (((u & 7) ^ (rr & 7)) << 4);
}

union Pack8 {
    uint4 v;
    __nv_bfloat162 h[4];
};

// ------------------------------------------------------------------------ weights ----------
// B operand [N x 128] bf16, tiled like activations (N/128 row blocks x 2 column blocks):
//   mode 0 (conv2): B[n][c] = W2[(n / 128) * 128 + c][n % 128]   (block o = n / 128 maps h1[t+o-1])
//   mode 1:         B[n][c] = W[c][n] for W [128][N] row-major  (Wqkv, Wo)
__global__ void prep_weights_kernel(const float* __restrict__ W, int N, int mode,
                                    __nv_bfloat16* __restrict__ out) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N * kW) return;
    const int n = idx / kW, c = idx % kW;
    const float v = mode == 0 ? W[((n >> 7) * kW + c) * kW + (n & 127)] : W[int64_t(c) * N + n];
    const int64_t byte = ((n >> 7) * 2 + (c >> 6)) * 16384 + (n & 127) * 128 +
                         ((((c & 63) >> 3) ^ (n & 7)) << 4) + (c & 7) * 2;
    out[byte / 2] = __float2bfloat16_rn(v);
}

// ------------------------------------------------------------------------- conv1 -----------
// One CTA per tile, one thread per row: h1[t] = relu(b1 + sum_o W1[o][code(t+o-1)]) for t < L
// (neighbours outside [0, L) contribute nothing), zero rows past L.
__global__ void __launch_bounds__(128) conv1_bf16_kernel(const uint8_t* __restrict__ bytes,
                                                         const int64_t* __restrict__ off,
                                                         const int32_t* __restrict__ lens,
                                                         int64_t first,
                                                         const float* __restrict__ prm,
                                                         uint8_t* __restrict__ h1) {
    constexpr int kStride = 3 * kA + 1;  // W1 transposed to [j][o*24 + code], padded
    __shared__ float w1t[kW * kStride];
    __shared__ float b1[kW];
    for (int i = threadIdx.x; i < 3 * kA * kW; i += blockDim.x) {
        const int oc = i / kW, j = i % kW;
        w1t[j * kStride + oc] = prm[oW1 + i];
    }
    for (int j = threadIdx.x; j < kW; j += blockDim.x) b1[j] = prm[ob1 + j];
    __syncthreads();
    const int64_t tile = blockIdx.x;
    const int r = threadIdx.x, seq = int(tile) * kSeqPerTile + r / kP, t = r % kP;
    const int L = lens[seq];
    int cm = -1, c0 = -1, cp = -1;
    if (t < L) {
        const uint8_t* p = bytes + off[first + seq];
        c0 = p[t];
        if (t >= 1) cm = p[t - 1];
        if (t + 1 < L) cp = p[t + 1];
    }
    const int64_t row = tile * kTileRows + r;
#pragma unroll 1
    for (int u = 0; u < 16; ++u) {
        Pack8 pk;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float a[2] = {0.f, 0.f};
            if (c0 >= 0) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int j = u * 8 + e * 2 + q;
                    const float* w = w1t + j * kStride;
                    float v = b1[j] + w[kA + c0];
                    if (cm >= 0) v += w[cm];
                    if (cp >= 0) v += w[2 * kA + cp];
                    a[q] = fmaxf(v, 0.f);
                }
            }
            pk.h[e] = __floats2bfloat162_rn(a[0], a[1]);
        }
        *reinterpret_cast<uint4*>(h1 + unit_off(row, u)) = pk.v;
    }
}

// -------------------------------------------------------------------------- GEMM ------------
struct GemmArgs {
    const uint8_t* a;            // tiled activations (tiles x 32 KB)
    const __nv_bfloat16* w;      // tiled weights (N x 128)
    const float* bias;           // fp32 (conv2: b2)
    uint8_t* out;                // tiled activations
    const int32_t* lens;         // tiles x 4
    int64_t tiles;
    unsigned long long* err;
};

constexpr int kGemmThreads = 320;  // warp 0 loads, warp 1 issues MMAs, warps 2-9 drain
constexpr int kGemmStages = 2;

struct Conv2Shape {
    static constexpr int N = 384;
    static constexpr int kW_ = N * kW * 2;                         // weight bytes
    static constexpr int kSmA = kW_;                               // A ring
    static constexpr int kSmOut = kSmA + kGemmStages * kTileBytes; // output staging tile
    static constexpr int kSmBar = kSmOut + kTileBytes;
    static constexpr size_t kSmem = size_t(kSmBar) + 128 + 1024;
};

__device__ __forceinline__ float bf16_at(const uint8_t* tile, int r, int c) {
    const int u = c >> 3;
    const int64_t o = (u >> 3) * 16384 + r * 128 + (((u & 7) ^ (r & 7)) << 4) + (c & 7) * 2;
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + o));
}

__global__ void __launch_bounds__(kGemmThreads, 1) conv2_gemm_kernel(GemmArgs g) {
    using S = Conv2Shape;
    constexpr int N = S::N, NB = N / 128;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((uintptr_t(smem_raw) + 1023) & ~uintptr_t(1023));
    // barriers: 0 weights, 1-2 A full, 3-4 A empty (8 arrivals), 5 acc full, 6 acc empty
    // (8 arrivals), 7 MMA drain, 8-9 epilogue rendezvous before / after the tile store
    // (8 arrivals; bounded waits, unlike a named barrier)
    const uint32_t bar0 = smem_u32(smem + S::kSmBar);
    auto BAR = [&](int i) { return bar0 + 8u * uint32_t(i); };
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + S::kSmBar + 96);
    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + S::kSmBar + 100);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        bar_init(BAR(0), 1);
        for (int s = 0; s < kGemmStages; ++s) {
            bar_init(BAR(1 + s), 1);
            bar_init(BAR(3 + s), 8);
        }
        bar_init(BAR(5), 1);
        bar_init(BAR(6), 8);
        bar_init(BAR(7), 1);
        bar_init(BAR(8), 8);
        bar_init(BAR(9), 8);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_smem();
    }
    if (warp == 1) tmem_alloc(smem_u32(s_tmem), 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t sW = smem_u32(smem), sA = smem_u32(smem + S::kSmA);

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------------------------ loads ---------
        bar_expect_tx(BAR(0), uint32_t(S::kW_));
        bulk_load(sW, g.w, uint32_t(S::kW_), BAR(0));
        uint32_t stage = 0, phase = 0, issued = 0, par = 0;
        for (int64_t tile = blockIdx.x; tile < g.tiles; tile += gridDim.x) {
            if (!bar_wait(BAR(3 + stage), phase ^ 1u, s_abort, g.err)) break;
            bar_expect_tx(BAR(1 + stage), kTileBytes);
            bulk_load(sA + stage * kTileBytes, g.a + tile * kTileBytes, kTileBytes, BAR(1 + stage));
            issued |= 1u << stage;
            par = phase ? (par | (1u << stage)) : (par & ~(1u << stage));
            if (++stage == kGemmStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        bar_drain(BAR(0), 0);
        for (int s = 0; s < kGemmStages; ++s)
            if (issued & (1u << s)) bar_drain(BAR(1 + s), (par >> s) & 1u);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------------------------- MMAs ---------
        constexpr uint32_t idesc = idesc_bf16(128, 128);
        uint32_t stage = 0, phase = 0, accphase = 0;
        if (bar_wait(BAR(0), 0, s_abort, g.err)) {
            for (int64_t tile = blockIdx.x; tile < g.tiles; tile += gridDim.x) {
                if (!bar_wait(BAR(6), accphase ^ 1u, s_abort, g.err) ||
                    !bar_wait(BAR(1 + stage), phase, s_abort, g.err))
                    break;
                tc_fence_after();
                const uint32_t a = sA + stage * kTileBytes;
#pragma unroll
                for (int nb = 0; nb < NB; ++nb) {
#pragma unroll
                    for (int kc = 0; kc < 2; ++kc) {
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            tc_mma(tmem + uint32_t(nb) * 128u,
                                   sw128_desc(a + kc * 16384 + kk * 32),
                                   sw128_desc(sW + (nb * 2 + kc) * 16384 + kk * 32), idesc,
                                   (kc | kk) ? 1u : 0u);
                        }
                    }
                }
                tc_commit(BAR(5));
                if (++stage == kGemmStages) {
                    stage = 0;
                    phase ^= 1u;
                }
                accphase ^= 1u;
            }
        }
        tc_commit(BAR(7));
        bar_drain(BAR(7), 0);
    } else if (warp >= 2) {
        // ------------------------------------------------------------------ drain ---------
        const int ew = warp - 2, quarter = warp & 3, half = ew >> 2;
        const int r = quarter * 32 + lane;
        const uint32_t tl = tmem + (uint32_t(quarter * 32) << 16);
        uint8_t* stage_out = smem + S::kSmOut;
        uint32_t stage = 0, phase = 0, accphase = 0, rv = 0;
        for (int64_t tile = blockIdx.x; tile < g.tiles; tile += gridDim.x) {
            if (!bar_wait_own(BAR(5), accphase, g.err)) break;
            tc_fence_after();
            const int L = g.lens[tile * kSeqPerTile + quarter];
            const bool valid = lane < L;
            const uint8_t* a_tile = smem + S::kSmA + stage * kTileBytes;
            {
#pragma unroll 1
                for (int gi = 0; gi < 2; ++gi) {
                    const int c0 = half * 64 + gi * 32;
                    uint32_t y0[32], y1[32], y2[32];
                    __syncwarp();
                    tmem_ld32(tl + uint32_t(c0), y0);
                    tmem_ld32(tl + 128u + uint32_t(c0), y1);
                    tmem_ld32(tl + 256u + uint32_t(c0), y2);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        Pack8 pk;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            float o2[2];
#pragma unroll
                            for (int q = 0; q < 2; ++q) {
                                const int j = u * 8 + e * 2 + q;
                                const float up = __shfl_up_sync(0xffffffffu, __uint_as_float(y0[j]), 1);
                                const float dn = __shfl_down_sync(0xffffffffu, __uint_as_float(y2[j]), 1);
                                const float pre = (lane > 0 ? up : 0.f) + __uint_as_float(y1[j]) +
                                                  (lane < 31 ? dn : 0.f) + g.bias[c0 + j];
                                o2[q] = valid ? bf16_at(a_tile, r, c0 + j) + fmaxf(pre, 0.f) : 0.f;
                            }
                            pk.h[e] = __floats2bfloat162_rn(o2[0], o2[1]);
                        }
                        const int uu = (c0 >> 3) + u;
                        *reinterpret_cast<uint4*>(stage_out + unit_off(r, uu)) = pk.v;
                    }
                }
            }
            tc_fence_before();
            {
                // all 8 warps' rows are in the staging tile -> one bulk store -> staging free
                fence_async_smem();
                __syncwarp();
                if (lane == 0) bar_arrive(BAR(8));
                if (!bar_wait_own(BAR(8), rv, g.err)) break;
                if (ew == 0 && lane == 0) {
                    bulk_store(g.out + tile * kTileBytes, smem_u32(stage_out), kTileBytes);
                    bulk_store_drain();
                }
                __syncwarp();
                if (lane == 0) bar_arrive(BAR(9));
                if (!bar_wait_own(BAR(9), rv, g.err)) break;
                rv ^= 1u;
            }
            __syncwarp();
            if (lane == 0) {
                bar_arrive(BAR(6));
                bar_arrive(BAR(3 + stage));
            }
            if (++stage == kGemmStages) {
                stage = 0;
                phase ^= 1u;
            }
            accphase ^= 1u;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_free(tmem, 512);
    }
}

// ------------------------------------------------------------- attention layer ------------
// One attention layer fused on the tensor cores, per tile of 4 sequences (128 rows):
//   MMA 1  QKV = h Wqkv                (TMEM columns 0-383: q | k | v)
//   drain  q + bq -> X, k + bk -> Y    (bf16 operand tiles in shared memory)
//   MMA 2  S = X Y^T                   (columns 384-511; only the four 32 x 32 diagonal blocks,
//                                       one per sequence, are used)
//   drain  row t of sequence s: softmax over its keys u < L of S[t][32s + u] / sqrt(128) -> the
//          row of P (zero outside the diagonal block, zero rows t >= L) -> X;
//          v + bv transposed -> Y
//   MMA 3  O = P V                     (columns 384-511)
//   drain  O -> X
//   MMA 4  Y' = O Wo                   (columns 0-127)
//   drain  h' = (h + Y' + bo) masked to t < L -> staging (Y) -> one bulk store
// Warp 0 loads (weights once, then one h tile per tile), warp 1 issues the MMAs, warps 2-9
// drain (warp % 4 = TMEM lane quarter = sequence, (warp - 2) / 4 = column half).
struct LayerArgs {
    const uint8_t* h;            // tiled input
    const __nv_bfloat16* wqkv;   // tiled [384 x 128]
    const __nv_bfloat16* wo;     // tiled [128 x 128]
    // Biases by value: the drain warps read them with warp-uniform indices, which the kernel
    // parameter space (constant bank) serves without a global-memory round trip.
    float bqkv[3 * 128];
    float bo[128];
    uint8_t* out;                // tiled output
    const int32_t* lens;
    int64_t tiles;
    unsigned long long* err;
};

constexpr int kLySmWqkv = 0;
constexpr int kLySmWo = kLySmWqkv + 3 * kW * kW * 2;     // 96 KB
constexpr int kLySmA = kLySmWo + kW * kW * 2;            // 128 KB
constexpr int kLySmX = kLySmA + kTileBytes;
constexpr int kLySmY = kLySmX + kTileBytes;
constexpr int kLySmBar = kLySmY + kTileBytes;            // 224 KB
constexpr size_t kLySmem = size_t(kLySmBar) + 128 + 1024;

// Writes 8 consecutive values (columns 8u..8u+7 of row r) as one 16-byte unit of a tiled operand.
__device__ __forceinline__ void put_unit(uint8_t* tile, int r, int u, const float (&v)[8]) {
    Pack8 pk;
#pragma unroll
    for (int e = 0; e < 4; ++e) pk.h[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
    *reinterpret_cast<uint4*>(tile + unit_off(r, u)) = pk.v;
}

__global__ void __launch_bounds__(kGemmThreads, 1) attn_layer_kernel(const __grid_constant__ LayerArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((uintptr_t(smem_raw) + 1023) & ~uintptr_t(1023));
    // barriers: 0 weights, 1 h full, 2 h empty (8), 3 QKV done, 4 Q/K staged (8), 5 S done,
    // 6 P/V staged (8), 7 O done, 8 O staged (8), 9 Y' done, 10-11 store rendezvous (8),
    // 12 MMA drain
    const uint32_t bar0 = smem_u32(smem + kLySmBar);
    auto BAR = [&](int i) { return bar0 + 8u * uint32_t(i); };
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + kLySmBar + 112);
    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + kLySmBar + 116);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        const uint32_t counts[13] = {1, 1, 8, 1, 8, 1, 8, 1, 8, 1, 8, 8, 1};
        for (int b = 0; b < 13; ++b) bar_init(BAR(b), counts[b]);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_smem();
    }
    if (warp == 1) tmem_alloc(smem_u32(s_tmem), 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t sWqkv = smem_u32(smem + kLySmWqkv), sWo = smem_u32(smem + kLySmWo);
    const uint32_t sA = smem_u32(smem + kLySmA), sX = smem_u32(smem + kLySmX),
                   sY = smem_u32(smem + kLySmY);
    constexpr uint32_t idesc = idesc_bf16(128, 128);
    // D (+)= A B^T for one 128 x 128 x 128 block: 2 column blocks x 4 K=16 steps
    auto mma_block = [&](uint32_t d, uint32_t a, uint32_t b) {
#pragma unroll
        for (int kc = 0; kc < 2; ++kc)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                tc_mma(d, sw128_desc(a + kc * 16384 + kk * 32), sw128_desc(b + kc * 16384 + kk * 32),
                       idesc, (kc | kk) ? 1u : 0u);
    };

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------------------------ loads ---------
        bar_expect_tx(BAR(0), uint32_t(4 * kW * kW * 2));
        bulk_load(sWqkv, g.wqkv, uint32_t(3 * kW * kW * 2), BAR(0));
        bulk_load(sWo, g.wo, uint32_t(kW * kW * 2), BAR(0));
        uint32_t ph = 0;
        bool issued = false;
        for (int64_t tile = blockIdx.x; tile < g.tiles; tile += gridDim.x) {
            if (!bar_wait(BAR(2), ph ^ 1u, s_abort, g.err)) break;
            bar_expect_tx(BAR(1), kTileBytes);
            bulk_load(sA, g.h + tile * kTileBytes, kTileBytes, BAR(1));
            issued = true;
            ph ^= 1u;
        }
        bar_drain(BAR(0), 0);
        if (issued) bar_drain(BAR(1), ph ^ 1u);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------------------------- MMAs ---------
        uint32_t ph = 0;
        if (bar_wait(BAR(0), 0, s_abort, g.err)) {
            for (int64_t tile = blockIdx.x; tile < g.tiles; tile += gridDim.x) {
                if (!bar_wait(BAR(1), ph, s_abort, g.err)) break;
                tc_fence_after();
#pragma unroll
                for (int nb = 0; nb < 3; ++nb)
                    mma_block(tmem + uint32_t(nb) * 128u, sA, sWqkv + nb * 2 * 16384);
                tc_commit(BAR(3));
                if (!bar_wait(BAR(4), ph, s_abort, g.err)) break;
                tc_fence_after();
                mma_block(tmem + 384u, sX, sY);
                tc_commit(BAR(5));
                if (!bar_wait(BAR(6), ph, s_abort, g.err)) break;
                tc_fence_after();
                mma_block(tmem + 384u, sX, sY);
                tc_commit(BAR(7));
                if (!bar_wait(BAR(8), ph, s_abort, g.err)) break;
                tc_fence_after();
                mma_block(tmem, sX, sWo);
                tc_commit(BAR(9));
                ph ^= 1u;
            }
        }
        tc_commit(BAR(12));
        bar_drain(BAR(12), 0);
    } else if (warp >= 2) {
        // ------------------------------------------------------------------ drain ---------
        const int ew = warp - 2, quarter = warp & 3, half = ew >> 2;
        const int r = quarter * 32 + lane;
        const uint32_t tl = tmem + (uint32_t(quarter * 32) << 16);
        uint8_t* X = smem + kLySmX;
        uint8_t* Y = smem + kLySmY;
        const uint8_t* A = smem + kLySmA;
        uint32_t ph = 0;
        // hands the staged operands to the MMA thread
        auto handoff = [&](int b) {
            fence_async_smem();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(BAR(b));
        };
        // A phase's two 32-column groups (this warp's columns half * 64 .. + 63 from `base`):
        // both TMEM loads in flight together, then each group handed to use(y, c0).
        auto two_groups = [&](uint32_t base, auto&& use) {
            uint32_t y0[32], y1[32];
            __syncwarp();
            tmem_ld32_issue(base + uint32_t(half * 64), y0);
            tmem_ld32_issue(base + uint32_t(half * 64 + 32), y1);
            tmem_ld32_wait(y0);
            use(y0, half * 64);
            tmem_ld32_wait(y1);
            use(y1, half * 64 + 32);
        };
        for (int64_t tile = blockIdx.x; tile < g.tiles; tile += gridDim.x) {
            const int L = g.lens[tile * kSeqPerTile + quarter];
            const bool valid = lane < L;
            // ---- q, k -> X, Y
            if (!bar_wait_own(BAR(3), ph, g.err)) break;
            tc_fence_after();
#pragma unroll 1
            for (int part = 0; part < 2; ++part) {  // 0: q -> X, 1: k -> Y
                uint8_t* dst = part ? Y : X;
                two_groups(tl + uint32_t(part * 128), [&](const uint32_t (&y)[32], int c0) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float v[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e)
                            v[e] = __uint_as_float(y[u * 8 + e]) + g.bqkv[part * 128 + c0 + u * 8 + e];
                        put_unit(dst, r, (c0 >> 3) + u, v);
                    }
                });
            }
            handoff(4);
            // ---- softmax rows -> P (X); v transposed -> Y
            if (!bar_wait_own(BAR(5), ph, g.err)) break;
            tc_fence_after();
            {
                uint32_t sv[32];
                __syncwarp();
                tmem_ld32(tl + 384u + uint32_t(quarter * 32), sv);
                float a[32];
                float mx = -INFINITY;
#pragma unroll
                for (int u = 0; u < 32; ++u) {
                    a[u] = u < L ? __uint_as_float(sv[u]) * 0.08838834764831845f : -INFINITY;
                    mx = fmaxf(mx, a[u]);
                }
                float sum = 0.f;
#pragma unroll
                for (int u = 0; u < 32; ++u) {
                    a[u] = u < L ? expf(a[u] - mx) : 0.f;
                    sum += a[u];
                }
                const float inv = valid ? 1.f / sum : 0.f;
#pragma unroll
                for (int u = 0; u < 32; ++u) a[u] *= inv;
                // this warp's 64 columns of the P row: the diagonal block or zeros
#pragma unroll
                for (int u8 = 0; u8 < 8; ++u8) {
                    const int col = half * 64 + u8 * 8;
                    float v[8];
                    const bool mine = (col >> 5) == quarter;
#pragma unroll
                    for (int e = 0; e < 8; ++e) v[e] = mine ? a[(col & 31) + e] : 0.f;
                    put_unit(X, r, col >> 3, v);
                }
            }
            two_groups(tl + 256u, [&](const uint32_t (&y)[32], int c0) {  // value dimensions d
                // V^T as a K-major operand: row d, column (k) = this thread's row r
                const int kc = r >> 6, k8 = (r & 63) >> 3, ke = r & 7;
#pragma unroll
                for (int e = 0; e < 32; ++e) {
                    const int d = c0 + e;
                    const float v = __uint_as_float(y[e]) + g.bqkv[256 + d];
                    *reinterpret_cast<__nv_bfloat16*>(Y + kc * 16384 + d * 128 + ((k8 ^ (d & 7)) << 4) +
                                                      ke * 2) = __float2bfloat16_rn(v);
                }
            });
            handoff(6);
            // ---- O -> X
            if (!bar_wait_own(BAR(7), ph, g.err)) break;
            tc_fence_after();
            two_groups(tl + 384u, [&](const uint32_t (&y)[32], int c0) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    float v[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) v[e] = __uint_as_float(y[u * 8 + e]);
                    put_unit(X, r, (c0 >> 3) + u, v);
                }
            });
            handoff(8);
            // ---- h' = h + O Wo + bo (masked) -> staging Y -> bulk store
            if (!bar_wait_own(BAR(9), ph, g.err)) break;
            tc_fence_after();
            two_groups(tl, [&](const uint32_t (&y)[32], int c0) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int uu = (c0 >> 3) + u;
                    Pack8 in;
                    in.v = *reinterpret_cast<const uint4*>(A + unit_off(r, uu));
                    float v[8];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float2 h = __bfloat1622float2(in.h[e]);
                        const int j = u * 8 + 2 * e;
                        v[2 * e] = valid ? h.x + __uint_as_float(y[j]) + g.bo[c0 + j] : 0.f;
                        v[2 * e + 1] = valid ? h.y + __uint_as_float(y[j + 1]) + g.bo[c0 + j + 1] : 0.f;
                    }
                    put_unit(Y, r, uu, v);
                }
            });
            tc_fence_before();
            fence_async_smem();
            __syncwarp();
            if (lane == 0) bar_arrive(BAR(10));
            if (!bar_wait_own(BAR(10), ph, g.err)) break;
            if (ew == 0 && lane == 0) {
                bulk_store(g.out + tile * kTileBytes, sY, kTileBytes);
                bulk_store_drain();
            }
            __syncwarp();
            if (lane == 0) bar_arrive(BAR(11));
            if (!bar_wait_own(BAR(11), ph, g.err)) break;
            // the h tile, X, Y and all TMEM columns are free for the next tile
            __syncwarp();
            if (lane == 0) bar_arrive(BAR(2));
            ph ^= 1u;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_free(tmem, 512);
    }
}

// ------------------------------------------------------------------ pool + output ----------
// One warp per sequence: mean of the valid rows (4 columns per lane), e = pool Wout + bout,
// z = e / |e|; layout 0: fp32 [n][64]; layout 1: bf16 with row r's 16-byte chunks at chunk ^ (r & 7).
__global__ void pool_out_bf16_kernel(const uint8_t* __restrict__ h, const int32_t* __restrict__ lens,
                                     int S, const float* __restrict__ prm, int64_t first, int layout,
                                     void* __restrict__ out) {
    const int s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (s >= S) return;
    const int L = lens[s];
    const int u = lane >> 1, half = lane & 1;
    float p[4] = {0.f, 0.f, 0.f, 0.f};
    for (int t = 0; t < L; ++t) {
        const uint2 v = *reinterpret_cast<const uint2*>(h + unit_off(int64_t(s) * kP + t, u) + half * 8);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
        p[0] += a.x;
        p[1] += a.y;
        p[2] += b.x;
        p[3] += b.y;
    }
    const float invL = L > 0 ? 1.f / float(L) : 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] *= invL;
    const float* Wout = prm + oWout;
    float e0 = prm[obout + lane], e1 = prm[obout + 32 + lane];
#pragma unroll 4
    for (int d = 0; d < kW; ++d) {
        const int src = d >> 2, k = d & 3;
        const float pk = k == 0 ? p[0] : k == 1 ? p[1] : k == 2 ? p[2] : p[3];
        const float pd = __shfl_sync(0xffffffffu, pk, src);
        e0 = fmaf(pd, Wout[d * kE + lane], e0);
        e1 = fmaf(pd, Wout[d * kE + 32 + lane], e1);
    }
    float ss = e0 * e0 + e1 * e1;
#pragma unroll
    for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const float n = sqrtf(fmaxf(ss, 1e-30f));
    const float z0 = e0 / n, z1 = e1 / n;
    const int64_t row = first + s;
    if (layout == 0) {
        float* o = static_cast<float*>(out) + row * kE;
        o[lane] = z0;
        o[32 + lane] = z1;
        return;
    }
    __nv_bfloat16* o = static_cast<__nv_bfloat16*>(out) + row * kE;
    auto pos = [&](int dim) { return (((dim >> 3) ^ int(row & 7)) << 3) | (dim & 7); };
    o[pos(lane)] = __float2bfloat16_rn(z0);
    o[pos(32 + lane)] = __float2bfloat16_rn(z1);
}

struct Bf16State {
    int64_t version = -1;
    DevBuf w2, wqkv[2], wo[2], lens, h1, ha, hb;
    std::vector<float> bias[2];  // per layer: bqkv (384) then bo (128), host copies
};

void launch_conv2(const GemmArgs& g, int sms, cudaStream_t st) {
    ensure_smem_limit(reinterpret_cast<const void*>(conv2_gemm_kernel), Conv2Shape::kSmem);
    const int grid = int(std::min<int64_t>(g.tiles, sms));
    conv2_gemm_kernel<<<grid, kGemmThreads, Conv2Shape::kSmem, st>>>(g);
    STB_CUDA(cudaGetLastError());
}

void launch_layer(const LayerArgs& g, int sms, cudaStream_t st) {
    ensure_smem_limit(reinterpret_cast<const void*>(attn_layer_kernel), kLySmem);
    const int grid = int(std::min<int64_t>(g.tiles, sms));
    attn_layer_kernel<<<grid, kGemmThreads, kLySmem, st>>>(g);
    STB_CUDA(cudaGetLastError());
}

}  // namespace

// Embeddings of every sequence of `set` through the bf16 tensor-core path.  `prm` is the fp32
// parameter array on the device and `version` identifies its contents (the bf16 weight copies
// are rebuilt when it changes).  The caller checked the alphabet and the lengths (1..32).
void encoder_embed_bf16(const float* prm, int64_t version, std::shared_ptr<void>& state,
                        const st_seqset_s& set, void* out, int layout, cudaStream_t st) {
    Context& ctx = context();
    if (!state) state = std::make_shared<Bf16State>();
    auto& B = *static_cast<Bf16State*>(state.get());
    if (B.version != version) {
        auto prep = [&](DevBuf& dst, const float* W, int N, int mode) {
            auto* p = dst.as<__nv_bfloat16>(size_t(N) * kW);
            prep_weights_kernel<<<unsigned(ceil_div(int64_t(N) * kW, 256)), 256, 0, st>>>(W, N, mode, p);
            STB_CUDA(cudaGetLastError());
        };
        prep(B.w2, prm + oW2, 3 * kW, 0);
        for (int l = 0; l < 2; ++l) {
            prep(B.wqkv[l], prm + oL0 + l * kLayer + lWqkv, 3 * kW, 1);
            prep(B.wo[l], prm + oL0 + l * kLayer + lWo, kW, 1);
        }
        note_launch(nullptr, 5);
        for (int l = 0; l < 2; ++l) {  // the layers' biases travel as kernel parameters
            B.bias[l].resize(4 * kW);
            const float* Lp = prm + oL0 + l * kLayer;
            STB_CUDA(cudaMemcpyAsync(B.bias[l].data(), Lp + lbqkv, sizeof(float) * 3 * kW,
                                     cudaMemcpyDeviceToHost, st));
            STB_CUDA(cudaMemcpyAsync(B.bias[l].data() + 3 * kW, Lp + lbo, sizeof(float) * kW,
                                     cudaMemcpyDeviceToHost, st));
        }
        STB_CUDA(cudaStreamSynchronize(st));
        B.version = version;
    }
    constexpr int64_t kChunk = 32768;  // sequences per pass (8,192 tiles)
    const int64_t chunk_tiles = kChunk / kSeqPerTile;
    int32_t* lens = B.lens.as<int32_t>(size_t(kChunk));
    uint8_t* h1 = B.h1.as<uint8_t>(size_t(chunk_tiles) * kTileBytes);
    uint8_t* ha = B.ha.as<uint8_t>(size_t(chunk_tiles) * kTileBytes);
    uint8_t* hb = B.hb.as<uint8_t>(size_t(chunk_tiles) * kTileBytes);
    auto* err = reinterpret_cast<unsigned long long*>(ctx.flags_d + 8);
    for (int64_t first = 0; first < set.count; first += kChunk) {
        const int64_t n = std::min<int64_t>(kChunk, set.count - first);
        const int64_t tiles = ceil_div(n, kSeqPerTile);
        STB_CUDA(cudaMemsetAsync(lens, 0, size_t(tiles) * kSeqPerTile * sizeof(int32_t), st));
        STB_CUDA(cudaMemcpyAsync(lens, set.d_len + first, size_t(n) * sizeof(int32_t),
                                 cudaMemcpyDeviceToDevice, st));
        conv1_bf16_kernel<<<unsigned(tiles), 128, 0, st>>>(set.d_bytes, set.d_off, lens, first, prm, h1);
        STB_CUDA(cudaGetLastError());
        GemmArgs g{};
        g.lens = lens;
        g.tiles = tiles;
        g.err = err;
        g.a = h1;
        g.w = static_cast<const __nv_bfloat16*>(B.w2.ptr);
        g.bias = prm + ob2;
        g.out = ha;
        launch_conv2(g, ctx.num_sms, st);
        uint8_t* hin = ha;
        uint8_t* hout = hb;
        for (int l = 0; l < 2; ++l) {
            LayerArgs la{};
            la.h = hin;
            la.wqkv = static_cast<const __nv_bfloat16*>(B.wqkv[l].ptr);
            la.wo = static_cast<const __nv_bfloat16*>(B.wo[l].ptr);
            std::memcpy(la.bqkv, B.bias[l].data(), sizeof la.bqkv);
            std::memcpy(la.bo, B.bias[l].data() + 3 * kW, sizeof la.bo);
            la.out = hout;
            la.lens = lens;
            la.tiles = tiles;
            la.err = err;
            launch_layer(la, ctx.num_sms, st);
            std::swap(hin, hout);
        }
        pool_out_bf16_kernel<<<unsigned(ceil_div(n, 8)), 256, 0, st>>>(hin, lens, int(n), prm, first,
                                                                      layout, out);
        STB_CUDA(cudaGetLastError());
        note_launch("attn_layer_kernel", 5);
    }
}

}  // namespace stb
