// Sequence encoder of the learned-proposal path: training (forward, backward, Adam) and the
// embedding of device sequence sets.
//
// The model is fixed: one-hot amino-acid codes padded to 32 positions -> conv k=3 (24->128, ReLU)
// -> conv k=3 (128->128, ReLU, skip) -> 2 x single-head self-attention (d=128, residual) -> mean
// over the valid positions -> linear 128->64 -> unit length.  Parameters are one flat fp32 array
// in the order W1[3][24][128], b1, W2[384][128], b2, (Wqkv[128][384], bqkv, Wo[128][128], bo) x 2,
// Wout[128][64], bout.  Weights, activations, gradients and Adam state are fp32.  The dense
// layers' products run by default on the bf16 tensor cores with fp32 accumulation (gemm_bf16);
// the fp32 precision setting runs them in a tiled SGEMM on CUDA cores instead (128x128x8 tiles,
// 8x8 per thread, split-K for the weight gradients), whose numbers follow the float64
// restatement used as the checker to fp32 rounding.  Per-sequence kernels carry the
// convolutions' gathers, attention, pooling and the pair loss in fp32 either way.
#include <cuda_bf16.h>

#include <cmath>
#include <memory>

#include "common.cuh"
#include "encoder_layout.cuh"

namespace stb {

void gemm_bf16(bool ta, bool tb, int M, int N, int K, const float* A, int lda, const float* B,
               int ldb, float* C, int ldc, bool accumulate, cudaStream_t st, int sms);

namespace {

using namespace enc;
constexpr float kClip = 64.0f;

// ------------------------------------------------------------------------------ SGEMM -------
// C[M x N] (op) = opA(A) * opB(B); A is [M x K] (or [K x M] when TA), B is [K x N] (or [N x K]
// when TB), all row-major with leading dimensions lda/ldb/ldc.  mode 0 stores, 1 adds, 2 adds
// atomically (split-K: gridDim.z slices of K).  Requires lda, ldb multiples of 4 and 16-byte
// aligned bases (all operands here are).
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) sgemm_kernel(int M, int N, int K, const float* __restrict__ A,
                                                    int lda, const float* __restrict__ B, int ldb,
                                                    float* __restrict__ C, int ldc, int kslice,
                                                    int mode) {
    __shared__ __align__(16) float As[2][8][128 + 4];
    __shared__ __align__(16) float Bs[2][8][128 + 4];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * 128, n0 = blockIdx.x * 128;
    const int kb = blockIdx.z * kslice;
    const int ke = min(K, kb + kslice);

    auto load_a = [&](int k0, float4& v) {
        if (!TA) {  // (m, k) at A[m*lda + k]: a row's 8 k as two float4
            const int r = tid >> 1, kq = (tid & 1) * 4;
            const int m = m0 + r, k = k0 + kq;
            v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (m < M) {
                const float* p = A + int64_t(m) * lda + k;
                if (k + 3 < ke) v = *reinterpret_cast<const float4*>(p);
                else {
                    if (k < ke) v.x = p[0];
                    if (k + 1 < ke) v.y = p[1];
                    if (k + 2 < ke) v.z = p[2];
                }
            }
        } else {    // (m, k) at A[k*lda + m]: one k row of 128 m as 32 float4
            const int kr = tid >> 5, mq = (tid & 31) * 4;
            const int k = k0 + kr, m = m0 + mq;
            v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < ke) {
                const float* p = A + int64_t(k) * lda + m;
                if (m + 3 < M) v = *reinterpret_cast<const float4*>(p);
                else {
                    if (m < M) v.x = p[0];
                    if (m + 1 < M) v.y = p[1];
                    if (m + 2 < M) v.z = p[2];
                }
            }
        }
    };
    auto store_a = [&](int buf, const float4& v) {
        if (!TA) {
            const int r = tid >> 1, kq = (tid & 1) * 4;
            As[buf][kq + 0][r] = v.x;
            As[buf][kq + 1][r] = v.y;
            As[buf][kq + 2][r] = v.z;
            As[buf][kq + 3][r] = v.w;
        } else {
            const int kr = tid >> 5, mq = (tid & 31) * 4;
            *reinterpret_cast<float4*>(&As[buf][kr][mq]) = v;
        }
    };
    auto load_b = [&](int k0, float4& v) {
        if (!TB) {  // (k, n) at B[k*ldb + n]
            const int kr = tid >> 5, nq = (tid & 31) * 4;
            const int k = k0 + kr, n = n0 + nq;
            v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < ke) {
                const float* p = B + int64_t(k) * ldb + n;
                if (n + 3 < N) v = *reinterpret_cast<const float4*>(p);
                else {
                    if (n < N) v.x = p[0];
                    if (n + 1 < N) v.y = p[1];
                    if (n + 2 < N) v.z = p[2];
                }
            }
        } else {    // (k, n) at B[n*ldb + k]
            const int r = tid >> 1, kq = (tid & 1) * 4;
            const int n = n0 + r, k = k0 + kq;
            v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (n < N) {
                const float* p = B + int64_t(n) * ldb + k;
                if (k + 3 < ke) v = *reinterpret_cast<const float4*>(p);
                else {
                    if (k < ke) v.x = p[0];
                    if (k + 1 < ke) v.y = p[1];
                    if (k + 2 < ke) v.z = p[2];
                }
            }
        }
    };
    auto store_b = [&](int buf, const float4& v) {
        if (!TB) {
            const int kr = tid >> 5, nq = (tid & 31) * 4;
            *reinterpret_cast<float4*>(&Bs[buf][kr][nq]) = v;
        } else {
            const int r = tid >> 1, kq = (tid & 1) * 4;
            Bs[buf][kq + 0][r] = v.x;
            Bs[buf][kq + 1][r] = v.y;
            Bs[buf][kq + 2][r] = v.z;
            Bs[buf][kq + 3][r] = v.w;
        }
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    float4 ra, rb;
    int buf = 0;
    if (kb < ke) {
        load_a(kb, ra);
        load_b(kb, rb);
        store_a(0, ra);
        store_b(0, rb);
    }
    __syncthreads();
    for (int k0 = kb; k0 < ke; k0 += 8) {
        const bool more = k0 + 8 < ke;
        if (more) {
            load_a(k0 + 8, ra);
            load_b(k0 + 8, rb);
        }
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (more) {
            store_a(buf ^ 1, ra);
            store_b(buf ^ 1, rb);
        }
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int n = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (n >= N) continue;
            float* c = C + int64_t(m) * ldc + n;
            if (mode == 0) *c = acc[i][j];
            else if (mode == 1) *c += acc[i][j];
            else atomicAdd(c, acc[i][j]);
        }
    }
}

// C (=, +=) opA(A) * opB(B).  Weight-gradient products (a long K and a small output) are split
// over K and accumulated atomically into C, which then must hold the value to add to.
template <bool TA, bool TB>
void sgemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
           bool accumulate, cudaStream_t stream, int num_sms) {
    const int tiles = int(ceil_div(M, 128) * ceil_div(N, 128));
    int splits = 1;
    if (tiles < num_sms && K >= 4096) splits = int(std::min<int64_t>(ceil_div(2 * num_sms, tiles), K / 1024));
    int kslice = int(ceil_div(ceil_div(K, splits), 8) * 8);
    splits = int(ceil_div(K, kslice));
    const int mode = splits > 1 ? 2 : (accumulate ? 1 : 0);
    if (splits > 1 && !accumulate) STB_CUDA(cudaMemsetAsync(C, 0, sizeof(float) * size_t(M) * ldc, stream));
    const dim3 grid(unsigned(ceil_div(N, 128)), unsigned(ceil_div(M, 128)), unsigned(splits));
    sgemm_kernel<TA, TB><<<grid, 256, 0, stream>>>(M, N, K, A, lda, B, ldb, C, ldc, kslice, mode);
    STB_CUDA(cudaGetLastError());
    note_launch(nullptr);
}

// The training GEMM in the encoder's chosen precision: bf16 tensor cores (fp32 accumulation)
// or the fp32 SIMT kernel above.
template <bool TA, bool TB>
void mm(bool bf16, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C,
        int ldc, bool accumulate, cudaStream_t stream, int num_sms) {
    if (bf16) gemm_bf16(TA, TB, M, N, K, A, lda, B, ldb, C, ldc, accumulate, stream, num_sms);
    else sgemm<TA, TB>(M, N, K, A, lda, B, ldb, C, ldc, accumulate, stream, num_sms);
}

// ------------------------------------------------------------------------- layer kernels ----
// Row r = s*32 + t; position t of sequence s is valid when t < len[s].  The per-row kernels run
// kRowsPerCta rows per CTA (threadIdx.y) of kW threads (threadIdx.x): R = 32 S is a multiple.
constexpr int kRowsPerCta = 8;
__global__ void conv1_fwd_kernel(const uint8_t* __restrict__ codes, const int32_t* __restrict__ lens,
                                 const float* __restrict__ prm, float* __restrict__ pre1,
                                 float* __restrict__ h1) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    const int L = lens[s];
    float v = 0.f, pre = 0.f;
    if (t < L) {
        pre = prm[ob1 + j];
        for (int o = -1; o <= 1; ++o) {
            const int u = t + o;
            if (u >= 0 && u < L) pre += prm[oW1 + (int64_t(o + 1) * kA + codes[s * kP + u]) * kW + j];
        }
        v = fmaxf(pre, 0.f);
    }
    pre1[r * kW + j] = pre;
    h1[r * kW + j] = v;
}

// x2[r] = [h1[r-1], h1[r], h1[r+1]] within the sequence (zero outside [0, L)).
__global__ void im2col_kernel(const float* __restrict__ h1, const int32_t* __restrict__ lens,
                              float* __restrict__ x2) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    const int L = lens[s];
    const bool in = t < L;
    x2[r * 3 * kW + j] = in && t >= 1 ? h1[(r - 1) * kW + j] : 0.f;
    x2[r * 3 * kW + kW + j] = in ? h1[r * kW + j] : 0.f;
    x2[r * 3 * kW + 2 * kW + j] = in && t + 1 < L ? h1[(r + 1) * kW + j] : 0.f;
}

// h = (h1 + relu(pre2 + b2)) * mask; pre2 keeps the bias added.
__global__ void conv2_out_kernel(float* __restrict__ pre2, const float* __restrict__ h1,
                                 const int32_t* __restrict__ lens, const float* __restrict__ b2,
                                 float* __restrict__ h) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    const float p = pre2[r * kW + j] + b2[j];
    pre2[r * kW + j] = p;
    h[r * kW + j] = t < lens[s] ? h1[r * kW + j] + fmaxf(p, 0.f) : 0.f;
}

__global__ void add_bias_kernel(float* __restrict__ x, const float* __restrict__ b, int cols) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    for (int j = threadIdx.x; j < cols; j += blockDim.x) x[r * cols + j] += b[j];
}

// h_next = (h + y + bo) * mask
__global__ void residual_kernel(const float* __restrict__ h, const float* __restrict__ y,
                                const float* __restrict__ bo, const int32_t* __restrict__ lens,
                                float* __restrict__ out) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    out[r * kW + j] = t < lens[s] ? h[r * kW + j] + y[r * kW + j] + bo[j] : 0.f;
}

// One CTA (256 threads) per sequence: scores, masked softmax, o = a v.  Dynamic shared memory:
// q[32][128], k[32][129], v[32][128], a[32][33].
__global__ void __launch_bounds__(256) attn_fwd_kernel(const float* __restrict__ qkv,
                                                       const int32_t* __restrict__ lens,
                                                       float* __restrict__ a_out,
                                                       float* __restrict__ o_out) {
    extern __shared__ float sm[];
    float* q = sm;
    float* k = q + kP * kW;
    float* v = k + kP * (kW + 1);
    float* a = v + kP * kW;
    const int s = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int L = lens[s];
    const float* base = qkv + int64_t(s) * kP * 3 * kW;
    for (int i = tid; i < kP * kW; i += 256) {
        const int t = i / kW, j = i % kW;
        q[t * kW + j] = base[t * 3 * kW + j];
        k[t * (kW + 1) + j] = base[t * 3 * kW + kW + j];
        v[t * kW + j] = base[t * 3 * kW + 2 * kW + j];
    }
    __syncthreads();
    const float scale = rsqrtf(float(kW));
    {
        // warp w: rows w, w+8, w+16, w+24; lane u: key u.  Each k value feeds four rows.
        const int u = lane;
        float sc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int d = 0; d < kW; ++d) {
            const float kv = k[u * (kW + 1) + d];
#pragma unroll
            for (int i = 0; i < 4; ++i) sc[i] = fmaf(q[(warp + 8 * i) * kW + d], kv, sc[i]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int t = warp + 8 * i;
            const float x = u < L ? sc[i] * scale : -INFINITY;
            float mx = x;
            for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            const float e = u < L ? expf(x - mx) : 0.f;
            float sum = e;
            for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            const float av = t < L ? e / sum : 0.f;
            a[t * (kP + 1) + u] = av;
            a_out[(int64_t(s) * kP + t) * kP + u] = av;
        }
    }
    __syncthreads();
    {
        // warp w: rows 4w..4w+3; lane: columns lane + 32c.  4 x 4 outputs per thread.
        float acc[4][4] = {};
        for (int u = 0; u < L; ++u) {
            float av[4], vv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) av[i] = a[(4 * warp + i) * (kP + 1) + u];
#pragma unroll
            for (int c = 0; c < 4; ++c) vv[c] = v[u * kW + lane + 32 * c];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[i][c] = fmaf(av[i], vv[c], acc[i][c]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                o_out[(int64_t(s) * kP + 4 * warp + i) * kW + lane + 32 * c] = acc[i][c];
    }
}

// Backward of one attention core: from do, q, k, v, a to dqkv.  Shared memory: q, k, v, do
// [32][129] each, a and ds [32][33].
__global__ void __launch_bounds__(256) attn_bwd_kernel(const float* __restrict__ qkv,
                                                       const float* __restrict__ a_in,
                                                       const float* __restrict__ dout,
                                                       const int32_t* __restrict__ lens,
                                                       float* __restrict__ dqkv) {
    extern __shared__ float sm[];
    constexpr int R = kW + 1;
    float* q = sm;
    float* k = q + kP * R;
    float* v = k + kP * R;
    float* dO = v + kP * R;
    float* a = dO + kP * R;
    float* ds = a + kP * (kP + 1);
    const int s = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float* base = qkv + int64_t(s) * kP * 3 * kW;
    for (int i = tid; i < kP * kW; i += 256) {
        const int t = i / kW, j = i % kW;
        q[t * R + j] = base[t * 3 * kW + j];
        k[t * R + j] = base[t * 3 * kW + kW + j];
        v[t * R + j] = base[t * 3 * kW + 2 * kW + j];
        dO[t * R + j] = dout[(int64_t(s) * kP + t) * kW + j];
    }
    for (int i = tid; i < kP * kP; i += 256)
        a[(i / kP) * (kP + 1) + i % kP] = a_in[int64_t(s) * kP * kP + i];
    __syncthreads();
    const float scale = rsqrtf(float(kW));
    {
        // warp w: rows w, w+8, w+16, w+24; lane u: key u.
        const int u = lane;
        float da[4] = {0.f, 0.f, 0.f, 0.f};
        for (int d = 0; d < kW; ++d) {
            const float vv = v[u * R + d];
#pragma unroll
            for (int i = 0; i < 4; ++i) da[i] = fmaf(dO[(warp + 8 * i) * R + d], vv, da[i]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int t = warp + 8 * i;
            const float av = a[t * (kP + 1) + u];
            float dot = da[i] * av;
            for (int o = 16; o; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
            ds[t * (kP + 1) + u] = av * (da[i] - dot) * scale;
        }
    }
    __syncthreads();
    {
        // warp w: rows 4w..4w+3; lane: columns lane + 32c.  Every loaded value feeds four
        // outputs of each of dq, dk, dv.
        float dq[4][4] = {}, dk[4][4] = {}, dv[4][4] = {};
        for (int u = 0; u < kP; ++u) {
            float kv[4], qv[4], ov[4], dr[4], dc[4], ac[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                kv[c] = k[u * R + lane + 32 * c];
                qv[c] = q[u * R + lane + 32 * c];
                ov[c] = dO[u * R + lane + 32 * c];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                dr[i] = ds[(4 * warp + i) * (kP + 1) + u];
                dc[i] = ds[u * (kP + 1) + 4 * warp + i];
                ac[i] = a[u * (kP + 1) + 4 * warp + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    dq[i][c] = fmaf(dr[i], kv[c], dq[i][c]);
                    dk[i][c] = fmaf(dc[i], qv[c], dk[i][c]);
                    dv[i][c] = fmaf(ac[i], ov[c], dv[i][c]);
                }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float* out = dqkv + (int64_t(s) * kP + 4 * warp + i) * 3 * kW;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                out[lane + 32 * c] = dq[i][c];
                out[kW + lane + 32 * c] = dk[i][c];
                out[2 * kW + lane + 32 * c] = dv[i][c];
            }
        }
    }
}

__global__ void pool_kernel(const float* __restrict__ h, const int32_t* __restrict__ lens,
                            float* __restrict__ pool) {
    const int s = blockIdx.x, j = threadIdx.x;
    const int L = lens[s];
    float acc = 0.f;
    for (int t = 0; t < L; ++t) acc += h[(int64_t(s) * kP + t) * kW + j];
    pool[int64_t(s) * kW + j] = acc / float(L);
}

// e += bout; z = e / |e|; nrm = |e|.  One warp per sequence (64 dims, 2 per lane).
__global__ void normalize_kernel(float* __restrict__ e, const float* __restrict__ bout, int S,
                                 float* __restrict__ z, float* __restrict__ nrm) {
    const int s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (s >= S) return;
    float x0 = e[int64_t(s) * kE + lane] + bout[lane];
    float x1 = e[int64_t(s) * kE + 32 + lane] + bout[32 + lane];
    e[int64_t(s) * kE + lane] = x0;
    e[int64_t(s) * kE + 32 + lane] = x1;
    float ss = x0 * x0 + x1 * x1;
    for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const float n = sqrtf(fmaxf(ss, 1e-30f));
    z[int64_t(s) * kE + lane] = x0 / n;
    z[int64_t(s) * kE + 32 + lane] = x1 / n;
    if (lane == 0) nrm[s] = n;
}

// Pair loss over (z[2i], z[2i+1]) and dL/dz; the loss sum is accumulated into *loss.
__global__ void pair_loss_kernel(const float* __restrict__ z, const int32_t* __restrict__ scores,
                                 int pairs, float* __restrict__ dz, float* __restrict__ loss) {
    const int i = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (i >= pairs) return;
    const float* za = z + int64_t(2 * i) * kE;
    const float* zb = za + kE;
    const float d0 = za[lane] - zb[lane], d1 = za[32 + lane] - zb[32 + lane];
    float d = d0 * d0 + d1 * d1;
    for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    const float tgt = fminf(float(scores[i]), kClip) / (kClip * 0.5f);
    const float r = d - tgt;
    const float g = 2.f * r / float(pairs);
    dz[int64_t(2 * i) * kE + lane] = 2.f * g * d0;
    dz[int64_t(2 * i) * kE + 32 + lane] = 2.f * g * d1;
    dz[int64_t(2 * i + 1) * kE + lane] = -2.f * g * d0;
    dz[int64_t(2 * i + 1) * kE + 32 + lane] = -2.f * g * d1;
    if (lane == 0) atomicAdd(loss, r * r / float(pairs));
}

// de = dz / n - e (dz . e) / n^3
__global__ void normalize_bwd_kernel(const float* __restrict__ dz, const float* __restrict__ e,
                                     const float* __restrict__ nrm, int S, float* __restrict__ de) {
    const int s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (s >= S) return;
    const float g0 = dz[int64_t(s) * kE + lane], g1 = dz[int64_t(s) * kE + 32 + lane];
    const float e0 = e[int64_t(s) * kE + lane], e1 = e[int64_t(s) * kE + 32 + lane];
    float dot = g0 * e0 + g1 * e1;
    for (int o = 16; o; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
    const float n = nrm[s];
    const float c = dot / (n * n * n);
    de[int64_t(s) * kE + lane] = g0 / n - e0 * c;
    de[int64_t(s) * kE + 32 + lane] = g1 / n - e1 * c;
}

__global__ void pool_bwd_kernel(const float* __restrict__ dpool, const int32_t* __restrict__ lens,
                                float* __restrict__ dh) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    const int L = lens[s];
    dh[r * kW + j] = t < L ? dpool[int64_t(s) * kW + j] / float(L) : 0.f;
}

__global__ void mask_kernel(float* __restrict__ x, const int32_t* __restrict__ lens) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    if (t >= lens[s]) x[r * kW + j] = 0.f;
}

// dpre2 = dh * (pre2 > 0)
__global__ void relu_bwd_kernel(const float* __restrict__ dh, const float* __restrict__ pre,
                                float* __restrict__ out) {
    const int64_t i = (int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y) * kW + threadIdx.x;
    out[i] = pre[i] > 0.f ? dh[i] : 0.f;
}

// dpre1 = mask * (pre1 > 0) * (dh + dx2[r][W:2W] + dx2[r+1][0:W] + dx2[r-1][2W:3W])
__global__ void col2im_bwd_kernel(const float* __restrict__ dh, const float* __restrict__ dx2,
                                  const float* __restrict__ pre1, const int32_t* __restrict__ lens,
                                  float* __restrict__ dpre1) {
    const int64_t r = int64_t(blockIdx.x) * kRowsPerCta + threadIdx.y;
    const int s = int(r / kP), t = int(r % kP), j = threadIdx.x;
    const int L = lens[s];
    float g = 0.f;
    if (t < L) {
        g = dh[r * kW + j] + dx2[r * 3 * kW + kW + j];
        if (t + 1 < L) g += dx2[(r + 1) * 3 * kW + j];
        if (t >= 1) g += dx2[(r - 1) * 3 * kW + 2 * kW + j];
        if (pre1[r * kW + j] <= 0.f) g = 0.f;
    }
    dpre1[r * kW + j] = g;
}

// dW1[o][code][j] += dpre1[r][j] for the code at t+o, gathered per block of rows in shared
// memory (thread j owns column j, so no conflicts), then added to global memory.
__global__ void __launch_bounds__(128) conv1_bwd_kernel(const float* __restrict__ dpre1,
                                                        const uint8_t* __restrict__ codes,
                                                        const int32_t* __restrict__ lens,
                                                        int64_t rows, int rows_per_block,
                                                        float* __restrict__ dW1,
                                                        float* __restrict__ db1) {
    __shared__ float acc[3 * kA * kW];
    const int j = threadIdx.x;
    for (int i = j; i < 3 * kA * kW; i += 128) acc[i] = 0.f;
    __syncthreads();
    float bsum = 0.f;
    const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
    const int64_t r1 = min(rows, r0 + rows_per_block);
    for (int64_t r = r0; r < r1; ++r) {
        const int s = int(r / kP), t = int(r % kP);
        const int L = lens[s];
        if (t >= L) continue;
        const float g = dpre1[r * kW + j];
        bsum += g;
        for (int o = -1; o <= 1; ++o) {
            const int u = t + o;
            if (u >= 0 && u < L) acc[(int(o + 1) * kA + codes[s * kP + u]) * kW + j] += g;
        }
    }
    __syncthreads();
    for (int i = j; i < 3 * kA * kW; i += 128)
        if (acc[i] != 0.f) atomicAdd(dW1 + i, acc[i]);
    atomicAdd(db1 + j, bsum);
}

// out[c] += sum over rows [blockIdx.x * rows_per_block, ...) of x[r][c] (cols a multiple of 4,
// at most 1024).  blockDim.x = (cols / 4) * G: thread t sums float4 column t % (cols / 4) over
// every G-th row, the G partial sums meet in shared memory, one atomic per column per block.
__global__ void colsum_kernel(const float* __restrict__ x, int64_t rows, int cols,
                              int rows_per_block, float* __restrict__ out) {
    __shared__ float4 part[256];
    const int cq = cols >> 2, G = blockDim.x / cq;
    const int c4 = threadIdx.x % cq, g = threadIdx.x / cq;
    const int64_t r0 = int64_t(blockIdx.x) * rows_per_block;
    const int64_t r1 = min(rows, r0 + rows_per_block);
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4* xv = reinterpret_cast<const float4*>(x);
#pragma unroll 4
    for (int64_t r = r0 + g; r < r1; r += G) {
        const float4 v = xv[r * cq + c4];
        acc.x += v.x;
        acc.y += v.y;
        acc.z += v.z;
        acc.w += v.w;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    if (g == 0) {
        for (int h = 1; h < G; ++h) {
            const float4 v = part[h * cq + c4];
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
        }
        atomicAdd(out + 4 * c4, acc.x);
        atomicAdd(out + 4 * c4 + 1, acc.y);
        atomicAdd(out + 4 * c4 + 2, acc.z);
        atomicAdd(out + 4 * c4 + 3, acc.w);
    }
}

// Column sums of x [rows][cols] added into out (bias gradients).
void colsum(const float* x, int64_t rows, int cols, float* out, cudaStream_t st) {
    const int cq = cols / 4;
    const int threads = cq * std::max(1, 256 / cq);
    constexpr int kRowsPerBlock = 256;
    colsum_kernel<<<unsigned(ceil_div(rows, kRowsPerBlock)), unsigned(threads), 0, st>>>(
        x, rows, cols, kRowsPerBlock, out);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2,
                            float c1, float c2, float eps) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Codes of a device set, padded to 32 positions per sequence (lengths checked by the caller).
__global__ void gather_codes_kernel(const uint8_t* __restrict__ bytes, const int64_t* __restrict__ off,
                                    const int32_t* __restrict__ len, int64_t first, int S,
                                    uint8_t* __restrict__ codes, int32_t* __restrict__ lens) {
    const int s = blockIdx.x, t = threadIdx.x;
    if (s >= S) return;
    const int64_t i = first + s;
    const int L = len[i];
    codes[s * kP + t] = t < L ? bytes[off[i] + t] : 0;
    if (t == 0) lens[s] = L;
}

// Embedding rows out: fp32 [n][64] (layout 0), or bf16 [n][64] with each row's eight 16-byte
// chunks stored at chunk ^ (row & 7) (layout 1) -- the 128-byte-swizzled K-major layout that a
// linear bulk copy into 1024-byte-aligned shared memory turns into a tensor-core operand tile.
__global__ void store_embed_kernel(const float* __restrict__ z, int S, int64_t first, int layout,
                                   void* __restrict__ out) {
    const int s = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (s >= S) return;
    const int64_t row = first + s;
    const float x0 = z[int64_t(s) * kE + lane], x1 = z[int64_t(s) * kE + 32 + lane];
    if (layout == 0) {
        float* o = static_cast<float*>(out) + row * kE;
        o[lane] = x0;
        o[32 + lane] = x1;
        return;
    }
    __nv_bfloat16* o = static_cast<__nv_bfloat16*>(out) + row * kE;
    auto pos = [&](int dim) {
        const int chunk = dim >> 3, within = dim & 7;
        return ((chunk ^ int(row & 7)) << 3) | within;
    };
    o[pos(lane)] = __float2bfloat16_rn(x0);
    o[pos(32 + lane)] = __float2bfloat16_rn(x1);
}

}  // namespace

// ----------------------------------------------------------------------------- model ---------
struct Encoder {
    int device = 0;
    DevBuf params, grads, adam_m, adam_v, loss;
    int64_t step = 0;            // Adam steps taken: also the version of the parameters
    int precision = 1;           // training products: 1 bf16 tensor cores, 0 fp32 SIMT
    std::shared_ptr<void> bf16;  // weights and workspace of the bf16 inference path
    int S_cap = 0;  // sequences the workspace holds
    // forward activations (rows = 32 * S)
    DevBuf codes, lens, scores, pre1, h1, x2, pre2, hA, hB, hC, qkv0, qkv1, a0, a1, o0, o1, y, pool,
        e, z, nrm;
    // backward
    DevBuf dz, de, dpool, dh, dO, dqkv, dx2, dpre;

    void reserve(int S) {
        if (S <= S_cap) return;
        const size_t R = size_t(S) * kP;
        codes.as<uint8_t>(R);
        lens.as<int32_t>(size_t(S));
        scores.as<int32_t>(size_t(S));
        for (DevBuf* b : {&pre1, &h1, &pre2, &hA, &hB, &hC, &o0, &o1, &y, &dh, &dO, &dpre})
            b->as<float>(R * kW);
        for (DevBuf* b : {&x2, &qkv0, &qkv1, &dqkv, &dx2}) b->as<float>(R * 3 * kW);
        a0.as<float>(size_t(S) * kP * kP);
        a1.as<float>(size_t(S) * kP * kP);
        for (DevBuf* b : {&pool, &dpool}) b->as<float>(size_t(S) * kW);
        for (DevBuf* b : {&e, &z, &dz, &de}) b->as<float>(size_t(S) * kE);
        nrm.as<float>(size_t(S));
        S_cap = S;
    }
};

namespace {

float* P(Encoder& m) { return static_cast<float*>(m.params.ptr); }
float* F(DevBuf& b) { return static_cast<float*>(b.ptr); }

size_t attn_fwd_smem() { return sizeof(float) * (kP * kW + kP * (kW + 1) + kP * kW + kP * (kP + 1)); }
size_t attn_bwd_smem() { return sizeof(float) * (4 * kP * (kW + 1) + 2 * kP * (kP + 1)); }

void set_attn_attrs() {
    ensure_smem_limit(reinterpret_cast<const void*>(attn_fwd_kernel), attn_fwd_smem());
    ensure_smem_limit(reinterpret_cast<const void*>(attn_bwd_kernel), attn_bwd_smem());
}

// Forward of S sequences whose padded codes and lengths are in m.codes / m.lens; z in m.z.
void forward(Encoder& m, int S, cudaStream_t st, int sms, bool bf) {
    set_attn_attrs();
    const unsigned R = unsigned(S) * kP;
    const auto* codes = static_cast<const uint8_t*>(m.codes.ptr);
    const auto* lens = static_cast<const int32_t*>(m.lens.ptr);
    float* prm = P(m);
    conv1_fwd_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(codes, lens, prm, F(m.pre1), F(m.h1));
    im2col_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(F(m.h1), lens, F(m.x2));
    mm<false, false>(bf, int(R), kW, 3 * kW, F(m.x2), 3 * kW, prm + oW2, kW, F(m.pre2), kW, false, st, sms);
    conv2_out_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(F(m.pre2), F(m.h1), lens, prm + ob2, F(m.hA));
    float* hin[2] = {F(m.hA), F(m.hB)};
    float* hout[2] = {F(m.hB), F(m.hC)};
    float* qkv[2] = {F(m.qkv0), F(m.qkv1)};
    float* att[2] = {F(m.a0), F(m.a1)};
    float* ob[2] = {F(m.o0), F(m.o1)};
    for (int l = 0; l < 2; ++l) {
        const float* L = prm + oL0 + l * kLayer;
        mm<false, false>(bf, int(R), 3 * kW, kW, hin[l], kW, L + lWqkv, 3 * kW, qkv[l], 3 * kW, false, st, sms);
        add_bias_kernel<<<R / kRowsPerCta, dim3(128, kRowsPerCta), 0, st>>>(qkv[l], L + lbqkv, 3 * kW);
        attn_fwd_kernel<<<unsigned(S), 256, attn_fwd_smem(), st>>>(qkv[l], lens, att[l], ob[l]);
        mm<false, false>(bf, int(R), kW, kW, ob[l], kW, L + lWo, kW, F(m.y), kW, false, st, sms);
        residual_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(hin[l], F(m.y), L + lbo, lens, hout[l]);
    }
    pool_kernel<<<unsigned(S), kW, 0, st>>>(F(m.hC), lens, F(m.pool));
    mm<false, false>(bf, S, kE, kW, F(m.pool), kW, prm + oWout, kE, F(m.e), kE, false, st, sms);
    normalize_kernel<<<unsigned(ceil_div(S, 8)), 256, 0, st>>>(F(m.e), prm + obout, S, F(m.z), F(m.nrm));
    STB_CUDA(cudaGetLastError());
    note_launch(nullptr, 12);
}

// Loss and gradients (into m.grads) of S sequences = S/2 pairs with scores in m.scores.
void loss_backward(Encoder& m, int S, cudaStream_t st, int sms, bool bf) {
    const unsigned R = unsigned(S) * kP;
    const int pairs = S / 2;
    const auto* codes = static_cast<const uint8_t*>(m.codes.ptr);
    const auto* lens = static_cast<const int32_t*>(m.lens.ptr);
    float* prm = P(m);
    float* g = F(m.grads);
    STB_CUDA(cudaMemsetAsync(g, 0, sizeof(float) * kParams, st));
    STB_CUDA(cudaMemsetAsync(m.loss.ptr, 0, sizeof(float), st));
    pair_loss_kernel<<<unsigned(ceil_div(pairs, 8)), 256, 0, st>>>(
        F(m.z), static_cast<const int32_t*>(m.scores.ptr), pairs, F(m.dz), F(m.loss));
    normalize_bwd_kernel<<<unsigned(ceil_div(S, 8)), 256, 0, st>>>(F(m.dz), F(m.e), F(m.nrm), S, F(m.de));
    // e = pool Wout + bout
    mm<true, false>(bf, kW, kE, S, F(m.pool), kW, F(m.de), kE, g + oWout, kE, true, st, sms);
    colsum(F(m.de), S, kE, g + obout, st);
    mm<false, true>(bf, S, kW, kE, F(m.de), kE, prm + oWout, kE, F(m.dpool), kW, false, st, sms);
    pool_bwd_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(F(m.dpool), lens, F(m.dh));
    float* hin[2] = {F(m.hA), F(m.hB)};
    float* qkv[2] = {F(m.qkv0), F(m.qkv1)};
    float* att[2] = {F(m.a0), F(m.a1)};
    float* ob[2] = {F(m.o0), F(m.o1)};
    for (int l = 1; l >= 0; --l) {
        const float* L = prm + oL0 + l * kLayer;
        float* G = g + oL0 + l * kLayer;
        // h_next = (h + o Wo + bo) * mask; dh is already masked
        mm<true, false>(bf, kW, kW, int(R), ob[l], kW, F(m.dh), kW, G + lWo, kW, true, st, sms);
        colsum(F(m.dh), R, kW, G + lbo, st);
        mm<false, true>(bf, int(R), kW, kW, F(m.dh), kW, L + lWo, kW, F(m.dO), kW, false, st, sms);
        attn_bwd_kernel<<<unsigned(S), 256, attn_bwd_smem(), st>>>(qkv[l], att[l], F(m.dO), lens, F(m.dqkv));
        mm<true, false>(bf, kW, 3 * kW, int(R), hin[l], kW, F(m.dqkv), 3 * kW, G + lWqkv, 3 * kW, true, st, sms);
        colsum(F(m.dqkv), R, 3 * kW, G + lbqkv, st);
        // dh_prev = (dh + dqkv Wqkv^T) * mask
        mm<false, true>(bf, int(R), kW, 3 * kW, F(m.dqkv), 3 * kW, L + lWqkv, 3 * kW, F(m.dh), kW, true, st, sms);
        mask_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(F(m.dh), lens);
    }
    // hA = (h1 + relu(pre2)) * mask
    relu_bwd_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(F(m.dh), F(m.pre2), F(m.dpre));
    mm<true, false>(bf, 3 * kW, kW, int(R), F(m.x2), 3 * kW, F(m.dpre), kW, g + oW2, kW, true, st, sms);
    colsum(F(m.dpre), R, kW, g + ob2, st);
    mm<false, true>(bf, int(R), 3 * kW, kW, F(m.dpre), kW, prm + oW2, kW, F(m.dx2), 3 * kW, false, st, sms);
    col2im_bwd_kernel<<<R / kRowsPerCta, dim3(kW, kRowsPerCta), 0, st>>>(F(m.dh), F(m.dx2), F(m.pre1), lens, F(m.dpre));
    conv1_bwd_kernel<<<unsigned(ceil_div(R, 256)), 128, 0, st>>>(F(m.dpre), codes, lens, R, 256,
                                                                 g + oW1, g + ob1);
    STB_CUDA(cudaGetLastError());
    note_launch(nullptr, 16);
}

// The bounded waits of the tensor-core GEMM report through the context's error word 8.
void clear_wait_flag(Context& ctx) {
    STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, sizeof(int64_t), ctx.stream));
}
// Synchronises the stream, then fails if a bounded wait gave up during the step.
void check_wait_flag(Context& ctx) {
    STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, sizeof(int64_t),
                             cudaMemcpyDeviceToHost, ctx.stream));
    STB_CUDA(cudaStreamSynchronize(ctx.stream));
    if (ctx.flags_h[8] != 0)
        fail(ST_ETIMEOUT, "seqtree_b200: a bounded device-side wait gave up (training GEMM)");
}

void upload_batch(Encoder& m, const uint8_t* codes, const int32_t* lens, const int32_t* scores,
                  int S, cudaStream_t st) {
    for (int s = 0; s < S; ++s)
        if (lens[s] < 1 || lens[s] > kP)
            fail(ST_EINVAL, "seqtree_b200: encoder inputs must have 1..32 residues");
    for (int64_t i = 0; i < int64_t(S) * kP; ++i)
        if (codes[i] >= kA) fail(ST_EINVAL, "seqtree_b200: encoder codes must be < 24");
    m.reserve(S);
    h2d(m.codes.ptr, codes, size_t(S) * kP, st);
    h2d(m.lens.ptr, lens, sizeof(int32_t) * size_t(S), st);
    if (scores) h2d(m.scores.ptr, scores, sizeof(int32_t) * size_t(S / 2), st);
}

}  // namespace

int64_t encoder_param_count() { return kParams; }

Encoder* encoder_create(const float* params) {
    auto m = std::make_unique<Encoder>();
    Context& ctx = context();
    m->device = ctx.device;
    m->params.as<float>(kParams);
    m->grads.as<float>(kParams);
    m->adam_m.as<float>(kParams);
    m->adam_v.as<float>(kParams);
    m->loss.as<float>(4);
    STB_CUDA(cudaMemsetAsync(m->adam_m.ptr, 0, sizeof(float) * kParams, ctx.stream));
    STB_CUDA(cudaMemsetAsync(m->adam_v.ptr, 0, sizeof(float) * kParams, ctx.stream));
    if (params) h2d(m->params.ptr, params, sizeof(float) * kParams, ctx.stream);
    else STB_CUDA(cudaMemsetAsync(m->params.ptr, 0, sizeof(float) * kParams, ctx.stream));
    STB_CUDA(cudaStreamSynchronize(ctx.stream));
    return m.release();
}

void encoder_destroy(Encoder* m) {
    if (!m) return;
    for (DevBuf* b : {&m->params, &m->grads, &m->adam_m, &m->adam_v, &m->loss, &m->codes, &m->lens,
                      &m->scores, &m->pre1, &m->h1, &m->x2, &m->pre2, &m->hA, &m->hB, &m->hC,
                      &m->qkv0, &m->qkv1, &m->a0, &m->a1, &m->o0, &m->o1, &m->y, &m->pool, &m->e,
                      &m->z, &m->nrm, &m->dz, &m->de, &m->dpool, &m->dh, &m->dO, &m->dqkv, &m->dx2,
                      &m->dpre})
        b->release();
    delete m;
}

void encoder_params(Encoder& m, float* out) {
    Context& ctx = context();
    STB_CUDA(cudaMemcpyAsync(out, m.params.ptr, sizeof(float) * kParams, cudaMemcpyDeviceToHost,
                             ctx.stream));
    STB_CUDA(cudaStreamSynchronize(ctx.stream));
}

// Precision of the training products: 1 bf16 tensor cores (fp32 accumulation), 0 fp32 SIMT.
void encoder_set_precision(Encoder& m, int precision) {
    if (precision != 0 && precision != 1)
        fail(ST_EINVAL, "seqtree_b200: encoder precision is 0 (fp32) or 1 (bf16)");
    m.precision = precision;
}

// Loss (and optionally the gradient, host) of one batch: S sequences = S/2 pairs.
float encoder_loss_grad(Encoder& m, const uint8_t* codes, const int32_t* lens, const int32_t* scores,
                        int S, float* grad_out) {
    if (S < 2 || S % 2) fail(ST_EINVAL, "seqtree_b200: a batch is an even number of sequences (pairs)");
    Context& ctx = context();
    upload_batch(m, codes, lens, scores, S, ctx.stream);
    clear_wait_flag(ctx);
    forward(m, S, ctx.stream, ctx.num_sms, m.precision == 1);
    loss_backward(m, S, ctx.stream, ctx.num_sms, m.precision == 1);
    float loss = 0.f;
    STB_CUDA(cudaMemcpyAsync(&loss, m.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, ctx.stream));
    if (grad_out)
        STB_CUDA(cudaMemcpyAsync(grad_out, m.grads.ptr, sizeof(float) * kParams,
                                 cudaMemcpyDeviceToHost, ctx.stream));
    check_wait_flag(ctx);
    return loss;
}

// One Adam step (beta 0.9 / 0.999, eps 1e-8) on one batch; returns the batch loss.
float encoder_train_step(Encoder& m, const uint8_t* codes, const int32_t* lens, const int32_t* scores,
                         int S, float lr) {
    if (S < 2 || S % 2) fail(ST_EINVAL, "seqtree_b200: a batch is an even number of sequences (pairs)");
    Context& ctx = context();
    upload_batch(m, codes, lens, scores, S, ctx.stream);
    clear_wait_flag(ctx);
    forward(m, S, ctx.stream, ctx.num_sms, m.precision == 1);
    loss_backward(m, S, ctx.stream, ctx.num_sms, m.precision == 1);
    ++m.step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(m.step)), c2 = 1.f - std::pow(b2, float(m.step));
    adam_kernel<<<unsigned(ctx.num_sms * 4), 256, 0, ctx.stream>>>(
        P(m), F(m.grads), F(m.adam_m), F(m.adam_v), kParams, lr, b1, b2, c1, c2, 1e-8f);
    STB_CUDA(cudaGetLastError());
    note_launch(nullptr);
    float loss = 0.f;
    STB_CUDA(cudaMemcpyAsync(&loss, m.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, ctx.stream));
    check_wait_flag(ctx);
    return loss;
}

void encoder_embed_bf16(const float* prm, int64_t version, std::shared_ptr<void>& state,
                        const st_seqset_s& set, void* out, int layout, cudaStream_t st);

// Embeddings of every sequence of a device set (amino-acid codes, lengths 1..32) into `out`.
void encoder_embed(Encoder& m, const st_seqset_s& set, void* out, int layout, cudaStream_t st) {
    if (set.alphabet != ST_ALPHABET_AA)
        fail(ST_EINVAL, "seqtree_b200: the encoder takes amino-acid sets");
    for (int32_t L : set.h_len)
        if (L < 1 || L > kP) fail(ST_EINVAL, "seqtree_b200: encoder inputs must have 1..32 residues");
    if (layout == 1) {
        encoder_embed_bf16(P(m), m.step, m.bf16, set, out, layout, st);
        return;
    }
    Context& ctx = context();
    constexpr int kChunk = 16384;
    m.reserve(kChunk);
    for (int64_t first = 0; first < set.count; first += kChunk) {
        const int S = int(std::min<int64_t>(kChunk, set.count - first));
        gather_codes_kernel<<<unsigned(S), kP, 0, st>>>(set.d_bytes, set.d_off, set.d_len, first, S,
                                                       static_cast<uint8_t*>(m.codes.ptr),
                                                       static_cast<int32_t*>(m.lens.ptr));
        forward(m, S, st, ctx.num_sms, false);  // layouts 0 and 2: the fp32 forward
        store_embed_kernel<<<unsigned(ceil_div(S, 8)), 256, 0, st>>>(F(m.z), S, first, layout ? 1 : 0,
                                                                    out);
        STB_CUDA(cudaGetLastError());
        note_launch(nullptr, 2);
    }
}

}  // namespace stb
