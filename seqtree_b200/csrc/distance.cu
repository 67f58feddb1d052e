// Dense Hamming and Levenshtein matrices over raw bytes (case-sensitive) on sm_100a.
//
// Reference: seqtree src/distance.cpp:68-109.  Both distances compare bytes for equality only,
// so each call first maps the bytes present in either set to dense codes 0..sigma-1 (any
// bijection preserves equality) and then:
//
//   Hamming (output-write bound): every string is packed at b = 1/2/4/8 bits per symbol into
//   32-bit words; a pair costs one XOR, one fold of each symbol's b bits onto its lowest bit and
//   one POPC per word.  A thread owns four consecutive columns and streams 16-byte stores, so a
//   warp writes 512 contiguous bytes of a row per query.
//
//   Levenshtein (integer-ALU bound): Myers' bit-vector algorithm in Hyyro's formulation for
//   whole-string edit distance.  The ref is the bit pattern (one 64-bit word per lane, n <= 64)
//   and the query is the text, warp-uniform, so the per-character loop never diverges; the
//   pattern-match masks Peq[c] of the 32 lanes live in shared memory as [c][lane].  Lanes own
//   32 consecutive refs, so stores stay coalesced in the original column order.  Longer refs,
//   or more than 64 distinct symbols, take a one-thread-per-pair DP with its row in global
//   scratch (any length).
#include <algorithm>
#include <map>

#include "common.cuh"

namespace stb {

namespace {

// ---------------------------------------------------------------------------- remap ---------
struct ByteLut {
    uint8_t v[256];
};

__global__ void remap_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int64_t n,
                             ByteLut lut) {
    __shared__ uint8_t s[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s[i] = lut.v[i];
    __syncthreads();
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        out[i] = s[in[i]];
}

// Byte-presence bitmap of a set, computed on the device (distinct bytes -> dense codes).
__global__ void presence_kernel(const uint8_t* __restrict__ bytes, int64_t n,
                                unsigned int* __restrict__ present) {
    __shared__ unsigned int s[8];
    if (threadIdx.x < 8) s[threadIdx.x] = 0;
    __syncthreads();
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const uint8_t c = bytes[i];
        atomicOr(&s[c >> 5], 1u << (c & 31));
    }
    __syncthreads();
    if (threadIdx.x < 8 && s[threadIdx.x]) atomicOr(&present[threadIdx.x], s[threadIdx.x]);
}

// Dense codes of a (set, set) pair, cached by the sets' uids so that repeated calls on
// device-resident sets enqueue no host round trip (and can be captured in a CUDA graph).
struct DistCache {
    uint64_t a_uid = 0, b_uid = 0;
    int sigma = 0;
    DevBuf ac, bc;             // codes of a and b
    int packB = 0, packW = 0;  // Hamming packing built for (bits, words); 0 = none
    DevBuf qp, rp;             // packed words
};

DistCache& dist_cache(int device) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<DistCache>> all;
    std::lock_guard<std::mutex> lk(mu);
    auto& p = all[device];
    if (!p) p = std::make_unique<DistCache>();
    return *p;
}

DistCache& compute_codes(st_seqset_s& a, st_seqset_s& b, cudaStream_t stream, Context& ctx) {
    DistCache& dc = dist_cache(ctx.device);
    if (dc.a_uid == a.uid && dc.b_uid == b.uid && a.uid != 0) return dc;
    auto* present = reinterpret_cast<unsigned int*>(ctx.flags_d + 16);
    STB_CUDA(cudaMemsetAsync(present, 0, 32, stream));
    for (st_seqset_s* s : {&a, &b}) {
        if (s->total == 0) continue;
        const unsigned grid = unsigned(std::min<int64_t>(ceil_div(s->total, 256), ctx.num_sms * 4));
        presence_kernel<<<grid, 256, 0, stream>>>(s->d_bytes, s->total, present);
        STB_CUDA(cudaGetLastError());
        note_launch(nullptr);
    }
    STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 16, present, 32, cudaMemcpyDeviceToHost, stream));
    STB_CUDA(cudaStreamSynchronize(stream));
    const auto* bits = reinterpret_cast<const unsigned int*>(ctx.flags_h + 16);
    ByteLut lut;
    std::memset(lut.v, 0, sizeof lut.v);
    int sigma = 0;
    for (int c = 0; c < 256; ++c)
        if (bits[c >> 5] & (1u << (c & 31))) lut.v[c] = uint8_t(sigma++);
    DevBuf* bufs[2] = {&dc.ac, &dc.bc};
    st_seqset_s* sets[2] = {&a, &b};
    for (int t = 0; t < 2; ++t) {
        st_seqset_s* s = sets[t];
        uint8_t* dst = bufs[t]->as<uint8_t>(size_t(s->total) + 64);
        STB_CUDA(cudaMemsetAsync(dst + s->total, 0, 64, stream));
        if (s->total > 0) {
            const unsigned grid = unsigned(std::min<int64_t>(ceil_div(s->total, 256), ctx.num_sms * 4));
            remap_kernel<<<grid, 256, 0, stream>>>(s->d_bytes, dst, s->total, lut);
            STB_CUDA(cudaGetLastError());
            note_launch(nullptr);
        }
    }
    dc.sigma = sigma;
    dc.a_uid = a.uid;
    dc.b_uid = b.uid;
    dc.packB = dc.packW = 0;
    return dc;
}

// ---------------------------------------------------------------------------- Hamming -------
// Pack each string's codes at B bits per symbol into W words (low symbol in low bits).
__global__ void pack_kernel(const uint8_t* __restrict__ codes, const int64_t* __restrict__ off,
                            int64_t count, int L, int B, int W, uint32_t* __restrict__ packed) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint8_t* c = codes + off[s];
    const int per = 32 / B;
    for (int w = 0; w < W; ++w) {
        uint32_t v = 0;
        for (int t = 0; t < per; ++t) {
            const int j = w * per + t;
            if (j < L) v |= uint32_t(c[j]) << (t * B);
        }
        packed[s * W + w] = v;
    }
}

template <int B>
__device__ __forceinline__ uint32_t fold_diff(uint32_t x) {
    if constexpr (B == 1) return x;
    if constexpr (B == 2) return (x | (x >> 1)) & 0x55555555u;
    if constexpr (B == 4) {
        x |= x >> 1;
        x |= x >> 2;
        return x & 0x11111111u;
    }
    x |= x >> 1;
    x |= x >> 2;
    x |= x >> 4;
    return x & 0x01010101u;
}

constexpr int kHamCols = 1024;  // columns per CTA (256 threads x 4)
constexpr int kHamRows = 32;    // query rows per CTA

template <int B, int W>
__global__ void __launch_bounds__(256) hamming_kernel(const uint32_t* __restrict__ qp,
                                                      const uint32_t* __restrict__ rp,
                                                      int64_t N, int64_t K,
                                                      int32_t* __restrict__ out) {
    const int64_t c0 = int64_t(blockIdx.x) * kHamCols + threadIdx.x * 4;
    const int64_t r0 = int64_t(blockIdx.y) * kHamRows;
    const int64_t r1 = (N < r0 + kHamRows ? N : r0 + kHamRows);
    if (c0 >= K) return;
    uint32_t rw[4][W];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int w = 0; w < W; ++w) rw[t][w] = (c0 + t < K) ? __ldg(rp + (c0 + t) * W + w) : 0u;
    const bool full = (c0 + 4 <= K) && ((K & 3) == 0);
    for (int64_t i = r0; i < r1; ++i) {
        uint32_t qw[W];
#pragma unroll
        for (int w = 0; w < W; ++w) qw[w] = __ldg(qp + i * W + w);
        int v[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            int s = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) s += __popc(fold_diff<B>(qw[w] ^ rw[t][w]));
            v[t] = s;
        }
        int32_t* dst = out + i * K + c0;
        if (full) {
            __stcs(reinterpret_cast<int4*>(dst), make_int4(v[0], v[1], v[2], v[3]));
        } else {
#pragma unroll
            for (int t = 0; t < 4; ++t)
                if (c0 + t < K) dst[t] = v[t];
        }
    }
}

// Any word count: same scheme with the words read from memory.
template <int B>
__global__ void __launch_bounds__(256) hamming_kernel_any(const uint32_t* __restrict__ qp,
                                                          const uint32_t* __restrict__ rp,
                                                          int64_t N, int64_t K, int W,
                                                          int32_t* __restrict__ out) {
    const int64_t total = N * K;
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = idx / K, k = idx - i * K;
        int s = 0;
        for (int w = 0; w < W; ++w) s += __popc(fold_diff<B>(qp[i * W + w] ^ rp[k * W + w]));
        out[idx] = s;
    }
}

template <int B>
const char* launch_hamming(const uint32_t* qp, const uint32_t* rp, int64_t N, int64_t K, int W,
                           int32_t* out, cudaStream_t stream, int sms) {
    const dim3 grid(unsigned(ceil_div(K, kHamCols)), unsigned(ceil_div(N, kHamRows)));
    const bool tiled = grid.y <= 65535;
#define STB_HAM(WW)                                                                 \
    if (tiled && W == WW) {                                                         \
        hamming_kernel<B, WW><<<grid, 256, 0, stream>>>(qp, rp, N, K, out);         \
        STB_CUDA(cudaGetLastError());                                               \
        return "hamming_kernel";                                                    \
    }
    STB_HAM(1) STB_HAM(2) STB_HAM(3) STB_HAM(4) STB_HAM(6) STB_HAM(8)
#undef STB_HAM
    const int64_t blocks = std::min<int64_t>(ceil_div(N * K, 256), int64_t(sms) * 16);
    hamming_kernel_any<B><<<unsigned(blocks), 256, 0, stream>>>(qp, rp, N, K, W, out);
    STB_CUDA(cudaGetLastError());
    return "hamming_kernel_any";
}

// ---------------------------------------------------------------------------- Levenshtein ---
constexpr int kLevWarps = 8;
constexpr int kLevRows = 16;  // query rows per CTA

// Pattern = ref (lane), text = query (warp-uniform).  Peq in shared memory as [c][word][lane].
// W = 64-bit words per pattern: one word takes refs up to 64 symbols; longer refs (W = 2, 4, 8)
// run the blocked form, where each word passes its bottom horizontal step (-1, 0 or +1) to the
// next word as the carry into its first row (Myers 1999, "advance_block"): a -1 carry sets the
// match bit of row 0 for the add and shifts a 1 into Mh, a +1 carry shifts a 1 into Ph.  Rows
// past a lane's own ref length act as unmatched rows below the pattern and never reach rows above
// them, so every lane runs all W words and masks its own length at the end.
template <int W>
__global__ void __launch_bounds__(kLevWarps * 32)
levenshtein_kernel(const uint8_t* __restrict__ qc, const int64_t* __restrict__ qoff,
                   const uint8_t* __restrict__ rc, const int64_t* __restrict__ roff, int64_t N,
                   int64_t K, int sigma, int32_t* __restrict__ out) {
    extern __shared__ unsigned long long s_peq[];  // [warp][sigma][W][32]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long* peq = s_peq + size_t(warp) * sigma * W * 32;
    const int64_t k = (int64_t(blockIdx.x) * kLevWarps + warp) * 32 + lane;
    const bool valid = k < K;
    const int64_t kk = valid ? k : (K - 1);
    const uint8_t* r = rc + roff[kk];
    const int n = int(roff[kk + 1] - roff[kk]);
    for (int c = 0; c < sigma * W; ++c) peq[c * 32 + lane] = 0ull;
    for (int j = 0; j < n; ++j) peq[(r[j] * W + (j >> 6)) * 32 + lane] |= 1ull << (j & 63);
    __syncwarp();
    const unsigned long long ones = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
    const int64_t r0 = int64_t(blockIdx.y) * kLevRows;
    const int64_t r1 = (N < r0 + kLevRows ? N : r0 + kLevRows);
    for (int64_t i = r0; i < r1; ++i) {
        const uint8_t* q = qc + qoff[i];
        const int m = int(qoff[i + 1] - qoff[i]);
        // Pv / Mv hold the +1 / -1 vertical steps of the current DP column.  The distance is
        // read once from the last column, D[n][m] = D[0][m] + sum of its steps
        // = m + popc(Pv) - popc(Mv) over the n pattern bits, instead of following the bottom
        // cell through every column (which costs about a fifth of the loop's instructions).
        if constexpr (W > 1) {
            unsigned long long Pv[W], Mv[W];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                Pv[w] = ~0ull;
                Mv[w] = 0ull;
            }
            for (int t = 0; t < m; ++t) {
                const unsigned long long* e = peq + q[t] * W * 32 + lane;
                int h = 1;  // row 0 of the global distance: +1 per text character
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    unsigned long long Eq = e[w * 32];
                    const unsigned long long Xv = Eq | Mv[w];
                    Eq |= h < 0 ? 1ull : 0ull;
                    const unsigned long long Xh = (((Eq & Pv[w]) + Pv[w]) ^ Pv[w]) | Eq;
                    unsigned long long Ph = Mv[w] | ~(Xh | Pv[w]);
                    unsigned long long Mh = Pv[w] & Xh;
                    const int hout = int(Ph >> 63) - int(Mh >> 63);
                    Ph = (Ph << 1) | (h > 0 ? 1ull : 0ull);
                    Mh = (Mh << 1) | (h < 0 ? 1ull : 0ull);
                    Pv[w] = Mh | ~(Xv | Ph);
                    Mv[w] = Ph & Xv;
                    h = hout;
                }
            }
            int score = m;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const int bits = min(64, max(0, n - 64 * w));
                const unsigned long long mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
                score += __popcll(Pv[w] & mask) - __popcll(Mv[w] & mask);
            }
            if (valid) out[i * K + k] = score;
            continue;
        }
        unsigned long long Pv = ones, Mv = 0ull;
        for (int t = 0; t < m; ++t) {
            const unsigned long long Eq = peq[q[t] * 32 + lane];
            const unsigned long long Xv = Eq | Mv;
            const unsigned long long Xh = (((Eq & Pv) + Pv) ^ Pv) | Eq;
            unsigned long long Ph = Mv | ~(Xh | Pv);
            unsigned long long Mh = Pv & Xh;
            Ph = (Ph << 1) | 1ull;
            Mh <<= 1;
            Pv = Mh | ~(Xv | Ph);
            Mv = Ph & Xv;
        }
        const int score = m + __popcll(Pv & ones) - __popcll(Mv & ones);
        if (valid) out[i * K + k] = score;
    }
}

// Any lengths / alphabets: classic single-row DP per (i, k), row kept in global scratch laid
// out [j][thread] so that neighbouring threads touch neighbouring words.
__global__ void __launch_bounds__(256)
levenshtein_dp_kernel(const uint8_t* __restrict__ qc, const int64_t* __restrict__ qoff,
                      const uint8_t* __restrict__ rc, const int64_t* __restrict__ roff, int64_t N,
                      int64_t K, int32_t* __restrict__ scratch, int32_t* __restrict__ out) {
    const int64_t T = int64_t(gridDim.x) * blockDim.x;
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t idx = tid; idx < N * K; idx += T) {
        const int64_t i = idx / K, k = idx - i * K;
        const uint8_t* a = qc + qoff[i];
        const uint8_t* b = rc + roff[k];
        int m = int(qoff[i + 1] - qoff[i]), n = int(roff[k + 1] - roff[k]);
        if (n > m) {  // row over the shorter string (src/distance.cpp:80)
            const uint8_t* t = a; a = b; b = t;
            int u = m; m = n; n = u;
        }
        int32_t v;
        if (n == 0) {
            v = m;
        } else {
            for (int j = 0; j <= n; ++j) scratch[j * T + tid] = j;
            for (int x = 1; x <= m; ++x) {
                int diag = scratch[tid];
                int left = x;
                scratch[tid] = x;
                const uint8_t ax = a[x - 1];
                for (int j = 1; j <= n; ++j) {
                    const int up = scratch[j * T + tid];
                    const int cur = min(min(up + 1, left + 1), diag + (ax == b[j - 1] ? 0 : 1));
                    diag = up;
                    left = cur;
                    scratch[j * T + tid] = cur;
                }
            }
            v = scratch[n * T + tid];
        }
        out[idx] = v;
    }
}

}  // namespace

void hamming_sets(st_seqset_s& a, st_seqset_s& b, int32_t* out_d, cudaStream_t stream) {
    if (a.alphabet != -1 || b.alphabet != -1)
        fail(ST_EINVAL, "seqtree_b200: distance sets must hold raw bytes (alphabet -1)");
    const int64_t N = a.count, K = b.count;
    if (N == 0 || K == 0) return;
    // Every pair must have equal length (src/distance.cpp:68-72).  Report the first mismatched
    // pair in row-major order, as a one-thread reference run would.
    const int32_t L = a.h_len[0];
    int64_t bi = -1, bk = -1;
    bool refs_uniform = true;
    for (int64_t k = 0; k < K; ++k)
        if (b.h_len[size_t(k)] != b.h_len[0]) { refs_uniform = false; break; }
    if (!refs_uniform) {
        for (int64_t k = 0; k < K; ++k)
            if (b.h_len[size_t(k)] != L) { bi = 0; bk = k; break; }
    } else {
        for (int64_t i = 0; i < N; ++i)
            if (a.h_len[size_t(i)] != b.h_len[0]) { bi = i; bk = 0; break; }
    }
    if (bi >= 0)
        fail(ST_EINVAL, "seqtree: hamming distance is only defined for equal-length sequences (got " +
                            std::to_string(a.h_len[size_t(bi)]) + " and " +
                            std::to_string(b.h_len[size_t(bk)]) + ")");
    Context& ctx = context();
    DistCache& dc = compute_codes(a, b, stream, ctx);
    const int sigma = dc.sigma;
    const int B = sigma <= 2 ? 1 : sigma <= 4 ? 2 : sigma <= 16 ? 4 : 8;
    const int per = 32 / B;
    const int W = std::max(1, int(ceil_div(L, per)));
    uint32_t* qp = dc.qp.as<uint32_t>(size_t(N) * W);
    uint32_t* rp = dc.rp.as<uint32_t>(size_t(K) * W);
    if (dc.packB != B || dc.packW != W) {
        const uint8_t* ac = static_cast<uint8_t*>(dc.ac.ptr);
        const uint8_t* bc = static_cast<uint8_t*>(dc.bc.ptr);
        pack_kernel<<<unsigned(ceil_div(N, 256)), 256, 0, stream>>>(ac, a.d_off, N, L, B, W, qp);
        STB_CUDA(cudaGetLastError());
        pack_kernel<<<unsigned(ceil_div(K, 256)), 256, 0, stream>>>(bc, b.d_off, K, L, B, W, rp);
        STB_CUDA(cudaGetLastError());
        note_launch(nullptr, 2);
        dc.packB = B;
        dc.packW = W;
    }
    const char* name;
    switch (B) {
        case 1: name = launch_hamming<1>(qp, rp, N, K, W, out_d, stream, ctx.num_sms); break;
        case 2: name = launch_hamming<2>(qp, rp, N, K, W, out_d, stream, ctx.num_sms); break;
        case 4: name = launch_hamming<4>(qp, rp, N, K, W, out_d, stream, ctx.num_sms); break;
        default: name = launch_hamming<8>(qp, rp, N, K, W, out_d, stream, ctx.num_sms); break;
    }
    note_launch(name);
}

void levenshtein_sets(st_seqset_s& a, st_seqset_s& b, int32_t* out_d, cudaStream_t stream,
                      int64_t r0, int64_t r1) {
    if (a.alphabet != -1 || b.alphabet != -1)
        fail(ST_EINVAL, "seqtree_b200: distance sets must hold raw bytes (alphabet -1)");
    if (r1 < 0) r1 = a.count;
    if (r0 < 0 || r0 > r1 || r1 > a.count) fail(ST_EINVAL, "seqtree_b200: bad row range");
    const int64_t N = r1 - r0, K = b.count;
    if (N == 0 || K == 0) return;
    Context& ctx = context();
    DistCache& dc = compute_codes(a, b, stream, ctx);
    const int sigma = std::max(1, dc.sigma);
    const uint8_t* ac = static_cast<uint8_t*>(dc.ac.ptr);
    const uint8_t* bc = static_cast<uint8_t*>(dc.bc.ptr);
    // rows [r0, r1): their offsets and their block of the result
    const int64_t* aoff = a.d_off + r0;
    out_d += r0 * K;
    const dim3 grid(unsigned(ceil_div(K, kLevWarps * 32)), unsigned(ceil_div(N, kLevRows)));
    // Bit-vector path: refs up to 512 symbols (1, 2, 4 or 8 words) while the Peq table fits.
    const int words = b.max_len <= 64    ? 1
                    : b.max_len <= 128 ? 2
                    : b.max_len <= 256 ? 4
                    : b.max_len <= 512 ? 8
                                       : 0;
    const size_t smem = size_t(kLevWarps) * sigma * std::max(words, 1) * 32 * 8;
    if (words && sigma <= 64 && smem <= size_t(200) * 1024 && grid.y <= 65535) {
        const void* kern = words == 1 ? reinterpret_cast<const void*>(levenshtein_kernel<1>)
                         : words == 2 ? reinterpret_cast<const void*>(levenshtein_kernel<2>)
                         : words == 4 ? reinterpret_cast<const void*>(levenshtein_kernel<4>)
                                      : reinterpret_cast<const void*>(levenshtein_kernel<8>);
        ensure_smem_limit(kern, smem);
        if (words == 1)
            levenshtein_kernel<1><<<grid, kLevWarps * 32, smem, stream>>>(ac, aoff, bc, b.d_off,
                                                                         N, K, sigma, out_d);
        else if (words == 2)
            levenshtein_kernel<2><<<grid, kLevWarps * 32, smem, stream>>>(ac, aoff, bc, b.d_off,
                                                                         N, K, sigma, out_d);
        else if (words == 4)
            levenshtein_kernel<4><<<grid, kLevWarps * 32, smem, stream>>>(ac, aoff, bc, b.d_off,
                                                                         N, K, sigma, out_d);
        else
            levenshtein_kernel<8><<<grid, kLevWarps * 32, smem, stream>>>(ac, aoff, bc, b.d_off,
                                                                         N, K, sigma, out_d);
        STB_CUDA(cudaGetLastError());
        note_launch("levenshtein_kernel");
        return;
    }
    const int shorter_max = std::min(a.max_len, b.max_len);
    const int longer_max = std::max(a.max_len, b.max_len);
    (void)longer_max;
    // Scratch: (shorter+1) words per resident thread, bounded to 2 GiB.
    int64_t threads = std::min<int64_t>(int64_t(ctx.num_sms) * 2048, N * K);
    const int64_t per = int64_t(shorter_max) + 1;
    threads = std::max<int64_t>(256, std::min<int64_t>(threads, (int64_t(1) << 29) / per));
    threads = ceil_div(threads, 256) * 256;
    int32_t* scratch = ctx.work_a.as<int32_t>(size_t(threads) * per);
    levenshtein_dp_kernel<<<unsigned(threads / 256), 256, 0, stream>>>(ac, aoff, bc, b.d_off, N, K,
                                                                       scratch, out_d);
    STB_CUDA(cudaGetLastError());
    note_launch("levenshtein_dp_kernel");
}

}  // namespace stb
