// BF16 tensor-core GEMM with fp32 accumulation for the encoder's training layers:
// C (=, +=) op(A) op(B) with fp32 operands and result (the fp32 master weights and activations
// stay fp32; only the products run in bf16).
//
// Both operands are first packed into the tcgen05 K-major operand layout in bf16: blocks of 128
// rows x 64 k (16 KB), row r at r*128 bytes, the 16-byte unit u of a row at u ^ (r & 7) (the
// 128-byte swizzle), zero outside the matrix.  Packing absorbs the transposes (op(A) is A or
// A^T, the same for B), so the GEMM kernel only ever sees "rows x K" tiles.  One CTA computes
// one 128 x 128 output tile over a range of K chunks: warp 0 bulk-copies A and B chunks through a
// 3-stage shared-memory ring, one thread of warp 1 issues M=128 N=128 K=16 tcgen05.mma into a
// 128-column TMEM accumulator, and warps 2-5 (one TMEM lane quarter each) stage the tile in
// shared memory, from where all six warps store, add or atomically add (split K) it into C with
// coalesced writes.
// Every wait is bounded.
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "tc.cuh"

namespace stb {

namespace {

constexpr int kGT = 128;                 // tile rows (M) and columns (N)
constexpr int kGK = 64;                  // K per chunk: one 128-byte swizzled row
constexpr int kGStages = 3;
constexpr int kGThreads = 192;
constexpr int kBlockB = kGT * kGK * 2;   // 16 KB
constexpr int kGSmBar = kGStages * 2 * kBlockB;
constexpr size_t kGSmem = size_t(kGSmBar) + 128 + 1024;

// Packed operand: op[(tile * kchunks + chunk)][row][unit], value(i, k) = X[i * ld + k] (rows of
// X are the operand's rows).  One thread per 16-byte output unit, in output order: a warp reads
// four 256-byte row pieces and writes 512 contiguous bytes.
__global__ void pack_rows_kernel(const float* __restrict__ X, int ld, int rows, int K, int kchunks,
                                 int64_t units, uint8_t* __restrict__ op) {
    const int64_t pos = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (pos >= units) return;
    const int pu = int(pos & 7);
    const int64_t rowblk = pos >> 3;  // (tile * kchunks + chunk) * 128 + row
    const int row = int(rowblk & 127);
    const int64_t blk = rowblk >> 7;  // tile * kchunks + chunk
    const int chunk = int(blk % kchunks);
    const int64_t i = (blk / kchunks) * kGT + row;
    const int k0 = chunk * kGK + (pu ^ (row & 7)) * 8;
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = (i < rows && k0 + e < K) ? X[i * ld + k0 + e] : 0.f;
    union {
        uint4 q;
        __nv_bfloat162 h[4];
    } pk;
#pragma unroll
    for (int e = 0; e < 4; ++e) pk.h[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
    *reinterpret_cast<uint4*>(op + pos * 16) = pk.q;
}

// The same packed operand from the transpose: value(i, k) = X[k * ld + i].  One 256-thread
// block per (tile, chunk) block: it reads the 64 x 128 fp32 piece of X row by row (coalesced)
// into shared memory and writes the 16 KB block in output order.
__global__ void __launch_bounds__(256) pack_cols_kernel(const float* __restrict__ X, int ld, int rows,
                                                        int K, int kchunks,
                                                        uint8_t* __restrict__ op) {
    __shared__ float t[kGK][kGT + 1];
    const int chunk = int(blockIdx.x % unsigned(kchunks));
    const int64_t i0 = int64_t(blockIdx.x / unsigned(kchunks)) * kGT;
    const int k0 = chunk * kGK;
    for (int idx = threadIdx.x; idx < kGK * kGT; idx += 256) {
        const int kk = idx >> 7, ii = idx & 127;
        const int64_t i = i0 + ii;
        t[kk][ii] = (i < rows && k0 + kk < K) ? X[int64_t(k0 + kk) * ld + i] : 0.f;
    }
    __syncthreads();
    uint8_t* dst = op + int64_t(blockIdx.x) * kBlockB;
    for (int pos = threadIdx.x; pos < kGT * 8; pos += 256) {
        const int row = pos >> 3, u = (pos & 7) ^ (row & 7);
        union {
            uint4 q;
            __nv_bfloat162 h[4];
        } pk;
#pragma unroll
        for (int e = 0; e < 4; ++e)
            pk.h[e] = __floats2bfloat162_rn(t[u * 8 + 2 * e][row], t[u * 8 + 2 * e + 1][row]);
        *reinterpret_cast<uint4*>(dst + pos * 16) = pk.q;
    }
}

struct GemmBf16Args {
    const uint8_t* a;   // packed op(A): mtiles x kchunks blocks
    const uint8_t* b;   // packed op(B): ntiles x kchunks blocks
    int kchunks, chunks_per_split;
    float* C;
    int ldc, M, N;
    int mode;           // 0 store, 1 add, 2 atomic add
    unsigned long long* err;
};

__global__ void __launch_bounds__(kGThreads) gemm_bf16_kernel(GemmBf16Args g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((uintptr_t(smem_raw) + 1023) & ~uintptr_t(1023));
    // barriers: 0-2 full, 3-5 empty, 6 accumulator ready, 7 MMA drain
    const uint32_t bar0 = smem_u32(smem + kGSmBar);
    auto BAR = [&](int i) { return bar0 + 8u * uint32_t(i); };
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + kGSmBar + 64);
    volatile int* s_abort = reinterpret_cast<volatile int*>(smem + kGSmBar + 68);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tn = blockIdx.x, tm = blockIdx.y;
    const int c0 = blockIdx.z * g.chunks_per_split;
    const int c1 = min(g.kchunks, c0 + g.chunks_per_split);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kGStages; ++s) {
            bar_init(BAR(s), 1);
            bar_init(BAR(kGStages + s), 1);
        }
        bar_init(BAR(6), 1);
        bar_init(BAR(7), 1);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_smem();
    }
    if (warp == 1) tmem_alloc(smem_u32(s_tmem), 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t sbase = smem_u32(smem);

    if (warp == 0 && lane == 0) {
        uint32_t stage = 0, phase = 0, issued = 0, par = 0;
        for (int c = c0; c < c1; ++c) {
            if (!bar_wait(BAR(kGStages + stage), phase ^ 1u, s_abort, g.err)) break;
            bar_expect_tx(BAR(stage), 2 * kBlockB);
            const uint32_t dst = sbase + stage * 2 * kBlockB;
            bulk_load(dst, g.a + (int64_t(tm) * g.kchunks + c) * kBlockB, kBlockB, BAR(stage));
            bulk_load(dst + kBlockB, g.b + (int64_t(tn) * g.kchunks + c) * kBlockB, kBlockB, BAR(stage));
            issued |= 1u << stage;
            par = phase ? (par | (1u << stage)) : (par & ~(1u << stage));
            if (++stage == kGStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        for (int s = 0; s < kGStages; ++s)
            if (issued & (1u << s)) bar_drain(BAR(s), (par >> s) & 1u);
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(128, 128);
        uint32_t stage = 0, phase = 0;
        for (int c = c0; c < c1; ++c) {
            if (!bar_wait(BAR(stage), phase, s_abort, g.err)) break;
            tc_fence_after();
            const uint32_t a = sbase + stage * 2 * kBlockB, b = a + kBlockB;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                tc_mma(tmem, sw128_desc(a + kk * 32), sw128_desc(b + kk * 32), idesc,
                       (c > c0 || kk > 0) ? 1u : 0u);
            tc_commit(BAR(kGStages + stage));
            if (++stage == kGStages) {
                stage = 0;
                phase ^= 1u;
            }
        }
        tc_commit(BAR(6));
        tc_commit(BAR(7));
        bar_drain(BAR(7), 0);
    } else if (warp >= 2) {
        const int quarter = warp & 3;
        if (c1 > c0 && bar_wait_own(BAR(6), 0, g.err)) {
            tc_fence_after();
            // The warp's 32 x 128 fp32 quarter goes to the (now idle) ring: TMEM lane r -> tile
            // row quarter * 32 + r, its 16-byte unit u at u ^ (r & 7) (conflict-free both ways).
            float* stage = reinterpret_cast<float*>(smem + quarter * (32 * kGT * 4));
            const uint32_t tl = tmem + (uint32_t(quarter * 32) << 16);
#pragma unroll 1
            for (int grp = 0; grp < 4; ++grp) {
                uint32_t v[32];
                __syncwarp();
                tmem_ld32(tl + uint32_t(grp * 32), v);
#pragma unroll
                for (int t = 0; t < 8; ++t)
                    *reinterpret_cast<uint4*>(stage + lane * kGT + (((grp * 8 + t) ^ (lane & 7)) << 2)) =
                        make_uint4(v[4 * t], v[4 * t + 1], v[4 * t + 2], v[4 * t + 3]);
            }
        } else {
            *s_abort = 1;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_free(tmem, 128);
    }
    if (c1 <= c0 || *s_abort) return;
    // All six warps write the staged tile out, a warp per row at a time (128 consecutive
    // columns per instruction), four rows per batch so that the loads of the add mode overlap.
    const float* stage = reinterpret_cast<const float*>(smem);
    constexpr int kWarps = kGThreads / 32;
#pragma unroll 1
    for (int r0 = warp; r0 < kGT; r0 += 4 * kWarps) {
        float x[4][4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int r = r0 + b * kWarps;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int c = lane + 32 * q;
                x[b][q] = r < kGT ? stage[r * kGT + (((c >> 2) ^ (r & 7)) << 2) + (c & 3)] : 0.f;
            }
        }
        if (g.mode == 1) {
            float y[4][4];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = r0 + b * kWarps, row = tm * kGT + r;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int col = tn * kGT + lane + 32 * q;
                    y[b][q] = (r < kGT && row < g.M && col < g.N) ? g.C[int64_t(row) * g.ldc + col] : 0.f;
                }
            }
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int q = 0; q < 4; ++q) x[b][q] += y[b][q];
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int r = r0 + b * kWarps, row = tm * kGT + r;
            if (r >= kGT || row >= g.M) continue;
            float* crow = g.C + int64_t(row) * g.ldc;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int col = tn * kGT + lane + 32 * q;
                if (col < g.N) {
                    if (g.mode == 2) atomicAdd(crow + col, x[b][q]);
                    else crow[col] = x[b][q];
                }
            }
        }
    }
}

void pack(const float* X, int ld, bool trans, int rows, int K, DevBuf& buf, cudaStream_t st,
          int& tiles, int& kchunks) {
    tiles = int(ceil_div(rows, kGT));
    kchunks = int(ceil_div(K, kGK));
    const int64_t units = int64_t(tiles) * kchunks * kGT * 8;
    uint8_t* op = buf.as<uint8_t>(size_t(units) * 16);
    if (trans)
        pack_cols_kernel<<<unsigned(tiles * kchunks), 256, 0, st>>>(X, ld, rows, K, kchunks, op);
    else
        pack_rows_kernel<<<unsigned(ceil_div(units, 256)), 256, 0, st>>>(X, ld, rows, K, kchunks,
                                                                         units, op);
    STB_CUDA(cudaGetLastError());
}

}  // namespace

// C (=, +=) op(A) op(B) in bf16 with fp32 accumulation.  op(A) is [M x K] (A^T when ta, A being
// [K x M]), op(B) is [K x N] (B^T when tb, B being [N x K]); row-major with leading dimensions.
// Products with a long K and few output tiles are split over K and added atomically, in which
// case C must already hold the value to add to (it is cleared first when !accumulate).
void gemm_bf16(bool ta, bool tb, int M, int N, int K, const float* A, int lda, const float* B,
               int ldb, float* C, int ldc, bool accumulate, cudaStream_t st, int sms) {
    if (M <= 0 || N <= 0) return;
    if (K <= 0) {
        if (!accumulate)
            STB_CUDA(cudaMemset2DAsync(C, sizeof(float) * size_t(ldc), 0, sizeof(float) * size_t(N),
                                       size_t(M), st));
        return;
    }
    Context& ctx = context();
    ensure_smem_limit(reinterpret_cast<const void*>(gemm_bf16_kernel), kGSmem);
    int mtiles, ntiles, kchunks, kb;
    // op(A)[i][k] = ta ? A[k][i] : A[i][k];  op(B)^T[n][k] = tb ? B[n][k] : B[k][n]
    pack(A, lda, ta, M, K, ctx.gemm_a, st, mtiles, kchunks);
    pack(B, ldb, !tb, N, K, ctx.gemm_b, st, ntiles, kb);
    const int tiles = mtiles * ntiles;
    int splits = 1;
    if (tiles < sms && kchunks >= 16) splits = std::min(int(ceil_div(2 * sms, tiles)), kchunks / 4);
    const int cps = int(ceil_div(kchunks, splits));
    splits = int(ceil_div(kchunks, cps));
    const int mode = splits > 1 ? 2 : (accumulate ? 1 : 0);
    if (splits > 1 && !accumulate)
        STB_CUDA(cudaMemsetAsync(C, 0, sizeof(float) * size_t(M) * size_t(ldc), st));
    GemmBf16Args g{};
    g.a = static_cast<const uint8_t*>(ctx.gemm_a.ptr);
    g.b = static_cast<const uint8_t*>(ctx.gemm_b.ptr);
    g.kchunks = kchunks;
    g.chunks_per_split = cps;
    g.C = C;
    g.ldc = ldc;
    g.M = M;
    g.N = N;
    g.mode = mode;
    g.err = reinterpret_cast<unsigned long long*>(ctx.flags_d + 8);
    gemm_bf16_kernel<<<dim3(unsigned(ntiles), unsigned(mtiles), unsigned(splits)), kGThreads, kGSmem,
                       st>>>(g);
    STB_CUDA(cudaGetLastError());
    note_launch("gemm_bf16_kernel", 3);
}

}  // namespace stb
