// Dense Gotoh Needleman-Wunsch / Smith-Waterman score and Gram-distance matrices on sm_100a.
//
// Reference: seqtree src/pairwise.cpp:76-125 (three-state recurrence, MAXIMISING, int64 cells,
// sentinel INT64_MIN/4), :273-334 (matrix driver, self-scores for the distance) and :42-49
// (results that do not fit int32 are refused with std::overflow_error naming "score" or
// "distance").
//
// Exact path (this file): one thread per (query, ref) pair running the reference recurrence
// in int64, its single DP row kept in global scratch laid out [column][thread] so that the
// threads of a warp touch consecutive words.  It is exact for any gap magnitude, including the
// 2^31-1 gap costs the reference's tests pin.
#include <algorithm>
#include <climits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <tuple>

#include "common.cuh"

namespace stb {

namespace {

constexpr int64_t kNegInf = INT64_MIN / 4;  // src/pairwise.cpp:37
// Pairs a first-time tuning of per-thread against the wavefront (32- or 64-row buckets) runs
// each variant on.
constexpr int64_t kAlignTunePairs = int64_t(20) * 1000 * 1000;
// Pairs a first-time tuning of the wavefront's row-bucket width runs each variant on.
// A slice much smaller than this holds too few rows per bucket to fill the GPU, and so favours
// the wider buckets (fewer launches) where the whole matrix favours the narrower ones.
constexpr int64_t kWaveTunePairs = int64_t(20) * 1000 * 1000;

__device__ __forceinline__ int64_t gap_run(int64_t L, int32_t open, int32_t extend) {
    return L <= 0 ? 0 : int64_t(open) + (L - 1) * int64_t(extend);
}

__device__ __forceinline__ int64_t max3(int64_t a, int64_t b, int64_t c) {
    return max(a, max(b, c));
}

// Score of one pair; M/X/Y point at this thread's column 0 of each scratch array, stride T.
__device__ int64_t gotoh_pair(const uint8_t* q, int m, const uint8_t* r, int n,
                              const int32_t* s_sim, int A, bool local, int32_t go, int32_t ge,
                              int64_t* M, int64_t* X, int64_t* Y, int64_t T) {
    if (m == 0 || n == 0) return local ? 0 : -gap_run(m ? m : n, go, ge);
    M[0] = 0;
    X[0] = kNegInf;
    Y[0] = kNegInf;
    for (int j = 1; j <= n; ++j) {
        M[j * T] = local ? 0 : kNegInf;
        X[j * T] = kNegInf;
        Y[j * T] = local ? kNegInf : -gap_run(j, go, ge);
    }
    int64_t best = local ? 0 : kNegInf;
    int64_t lm = 0, lx = 0, ly = 0;
    for (int i = 1; i <= m; ++i) {
        int64_t dm = M[0], dx = X[0], dy = Y[0];
        lm = local ? 0 : kNegInf;
        lx = local ? kNegInf : -gap_run(i, go, ge);
        ly = kNegInf;
        M[0] = lm;
        X[0] = lx;
        Y[0] = ly;
        const int32_t* srow = s_sim + q[i - 1] * A;
        for (int j = 1; j <= n; ++j) {
            const int64_t um = M[j * T], ux = X[j * T], uy = Y[j * T];
            int64_t mv = max3(dm, dx, dy) + srow[r[j - 1]];
            if (local && mv < 0) mv = 0;
            const int64_t xv = max3(um - go, ux - ge, uy - go);
            const int64_t yv = max3(lm - go, ly - ge, lx - go);
            M[j * T] = mv;
            X[j * T] = xv;
            Y[j * T] = yv;
            if (local && mv > best) best = mv;
            dm = um;
            dx = ux;
            dy = uy;
            lm = mv;
            lx = xv;
            ly = yv;
        }
    }
    return local ? best : max3(lm, lx, ly);
}

struct ExactArgs {
    const uint8_t* qc;
    const int64_t* qoff;
    const uint8_t* rc;
    const int64_t* roff;
    int64_t N, K;          // self mode: pairs (i, i) for i < N, K ignored
    const int32_t* sim;
    int A;
    int local;
    int32_t go, ge;
    int self;              // 1: write int64 self-scores to self_out
    int dist;              // 1: Gram distance with q_self/r_self
    const int64_t* q_self;
    const int64_t* r_self;
    int64_t* scratch;      // 3 * (nmax+1) * T int64
    int64_t nmax1;
    int32_t* out;
    int64_t* self_out;
    unsigned int* overflow;
};

__global__ void __launch_bounds__(256) gotoh_exact_kernel(const ExactArgs a) {
    extern __shared__ int32_t s_sim[];
    for (int i = threadIdx.x; i < a.A * a.A; i += blockDim.x) s_sim[i] = a.sim[i];
    __syncthreads();
    const int64_t T = int64_t(gridDim.x) * blockDim.x;
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int64_t* M = a.scratch + tid;
    int64_t* X = M + a.nmax1 * T;
    int64_t* Y = X + a.nmax1 * T;
    const int64_t total = a.self ? a.N : a.N * a.K;
    for (int64_t idx = tid; idx < total; idx += T) {
        const int64_t i = a.self ? idx : idx / a.K;
        const int64_t k = a.self ? idx : idx - i * a.K;
        const uint8_t* q = a.qc + a.qoff[i];
        const int m = int(a.qoff[i + 1] - a.qoff[i]);
        const uint8_t* r = a.self ? q : a.rc + a.roff[k];
        const int n = a.self ? m : int(a.roff[k + 1] - a.roff[k]);
        const int64_t s = gotoh_pair(q, m, r, n, s_sim, a.A, a.local != 0, a.go, a.ge, M, X, Y, T);
        if (a.self) {
            a.self_out[idx] = s;
            continue;
        }
        const int64_t v = a.dist ? a.q_self[i] + a.r_self[k] - 2 * s : s;
        if (v < INT32_MIN || v > INT32_MAX) {
            atomicOr(a.overflow, 1u);
            continue;
        }
        a.out[idx] = int32_t(v);
    }
}

int64_t pick_threads(Context& ctx, int64_t work, int64_t per_thread_bytes) {
    int64_t t = std::min<int64_t>(int64_t(ctx.num_sms) * 1024, std::max<int64_t>(work, 1));
    t = std::min<int64_t>(t, std::max<int64_t>(256, (int64_t(1) << 30) / per_thread_bytes));
    return ceil_div(t, 256) * 256;
}

void launch_exact(Context& ctx, ExactArgs a, int64_t work, cudaStream_t stream) {
    const int64_t per = 3 * a.nmax1 * 8;
    const int64_t T = pick_threads(ctx, work, per);
    a.scratch = ctx.work_a.as<int64_t>(size_t(3 * a.nmax1 * T));
    gotoh_exact_kernel<<<unsigned(T / 256), 256, size_t(a.A) * a.A * 4, stream>>>(a);
    STB_CUDA(cudaGetLastError());
    note_launch("gotoh_exact_kernel");
}

// --------------------------------------------------------------------- per-thread path -----
// Short sequences (both sets at most NMAX long): one thread per (query, ref) pair, the whole DP
// row (M, X, Y for ref columns 0..NMAX) in registers, so no scratch memory is touched.  The
// recurrence and its order of evaluation are gotoh_pair's, in int32 with the sentinel kNeg32:
// the host admits a launch only when every legitimate value is bounded by 2^27 in magnitude, so
// sentinel-derived values (>= kNeg32 - 64 * (go + ge) > INT32_MIN) stay below every legitimate
// one and the maxima -- hence the result -- are the int64 recurrence's.  Consecutive threads
// take consecutive refs of one query, so a warp shares the query row and writes 128 contiguous
// bytes.  The three-input maxima are Blackwell DPX instructions.
constexpr int32_t kNeg32 = -(1 << 29);

struct ThreadArgs {
    const uint8_t* qc;
    const int64_t* qoff;
    const uint8_t* rc;
    const int64_t* roff;
    int64_t N, K;
    const int32_t* sim;
    int A;
    int32_t go, ge;
    int self;            // 1: self scores of the query set into self_out
    int64_t* self_out;
    int dist;
    const int64_t* q_self;
    const int64_t* r_self;
    int32_t* out;
    unsigned int* overflow;
};

__device__ __forceinline__ int32_t gap_run32(int L, int32_t open, int32_t extend) {
    return L <= 0 ? 0 : open + (L - 1) * extend;
}

template <int NMAX, bool LOCAL>
__global__ void __launch_bounds__(128) gotoh_thread_kernel(const ThreadArgs a) {
    extern __shared__ int32_t s_sim[];
    for (int i = threadIdx.x; i < a.A * a.A; i += blockDim.x) s_sim[i] = a.sim[i];
    __syncthreads();
    const int64_t total = a.self ? a.N : a.N * a.K;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total; idx += stride) {
        const int64_t i = a.self ? idx : idx / a.K;
        const int64_t k = a.self ? idx : idx - i * a.K;
        const uint8_t* q = a.qc + a.qoff[i];
        const int m = int(a.qoff[i + 1] - a.qoff[i]);
        const uint8_t* r = a.self ? q : a.rc + a.roff[k];
        const int n = a.self ? m : int(a.roff[k + 1] - a.roff[k]);
        int32_t score;
        if (m == 0 || n == 0) {
            score = LOCAL ? 0 : -gap_run32(m ? m : n, a.go, a.ge);
        } else if (!LOCAL && a.ge <= a.go) {
            // Global with gap_extend <= gap_open: the single-H form with every state of (i, j)
            // raised by (i+j) * extend, as in the wavefront kernel -- each gap state is one
            // add-max, borders are the constant extend - open, score = H~(m,n) - (m+n) * extend.
            int rcode[NMAX];
            int32_t H[NMAX + 1], Xr[NMAX + 1];
            const int32_t eo = a.ge - a.go, e2 = 2 * a.ge;
            H[0] = 0;
#pragma unroll
            for (int j = 1; j <= NMAX; ++j) {
                rcode[j - 1] = j <= n ? int(r[j - 1]) : 0;
                H[j] = eo;
                Xr[j] = kNeg32;
            }
            int32_t hn = 0;
            for (int ii = 1; ii <= m; ++ii) {
                int32_t hd = H[0];
                int32_t hl = eo, yl = kNeg32;
                H[0] = eo;
                const int32_t* srow = s_sim + int(q[ii - 1]) * a.A;
#pragma unroll
                for (int j = 1; j <= NMAX; ++j) {
                    if (j <= n) {
                        const int32_t hu = H[j];
                        const int32_t mv = hd + srow[rcode[j - 1]] + e2;
                        const int32_t xv = __viaddmax_s32(hu, eo, Xr[j]);
                        const int32_t yv = __viaddmax_s32(hl, eo, yl);
                        const int32_t hv = __vimax3_s32(mv, xv, yv);
                        hd = hu;
                        H[j] = hv;
                        Xr[j] = xv;
                        hl = hv;
                        yl = yv;
                    }
                }
                hn = hl;
            }
            score = hn - (m + n) * a.ge;
        } else {
            int rcode[NMAX];
            int32_t M[NMAX + 1], X[NMAX + 1], Y[NMAX + 1];
            M[0] = 0;
            X[0] = kNeg32;
            Y[0] = kNeg32;
#pragma unroll
            for (int j = 1; j <= NMAX; ++j) {
                rcode[j - 1] = j <= n ? int(r[j - 1]) : 0;
                M[j] = LOCAL ? 0 : kNeg32;
                X[j] = kNeg32;
                Y[j] = LOCAL ? kNeg32 : -gap_run32(j, a.go, a.ge);
            }
            int32_t best = LOCAL ? 0 : kNeg32;
            int32_t lm = 0, lx = 0, ly = 0;
            for (int ii = 1; ii <= m; ++ii) {
                int32_t dm = M[0], dx = X[0], dy = Y[0];
                lm = LOCAL ? 0 : kNeg32;
                lx = LOCAL ? kNeg32 : -gap_run32(ii, a.go, a.ge);
                ly = kNeg32;
                M[0] = lm;
                X[0] = lx;
                Y[0] = ly;
                const int32_t* srow = s_sim + int(q[ii - 1]) * a.A;
                int32_t em = lm, ex = lx, ey = ly;  // row values at column n
#pragma unroll
                for (int j = 1; j <= NMAX; ++j) {
                    if (j <= n) {
                        const int32_t um = M[j], ux = X[j], uy = Y[j];
                        int32_t mv = __vimax3_s32(dm, dx, dy) + srow[rcode[j - 1]];
                        if (LOCAL) mv = max(mv, 0);
                        const int32_t xv = __viaddmax_s32(max(um, uy), -a.go, ux - a.ge);
                        const int32_t yv = __viaddmax_s32(max(lm, lx), -a.go, ly - a.ge);
                        M[j] = mv;
                        X[j] = xv;
                        Y[j] = yv;
                        if (LOCAL) best = max(best, mv);
                        dm = um;
                        dx = ux;
                        dy = uy;
                        lm = mv;
                        lx = xv;
                        ly = yv;
                        em = mv;
                        ex = xv;
                        ey = yv;
                    }
                }
                lm = em;
                lx = ex;
                ly = ey;
            }
            score = LOCAL ? best : __vimax3_s32(lm, lx, ly);
        }
        if (a.self) {
            a.self_out[idx] = score;
            continue;
        }
        const int64_t v = a.dist ? a.q_self[i] + a.r_self[k] - 2 * int64_t(score) : int64_t(score);
        if (v < INT32_MIN || v > INT32_MAX) {
            atomicOr(a.overflow, 1u);
            continue;
        }
        a.out[idx] = int32_t(v);
    }
}

// Largest legitimate |value| of the recurrence for sequences up to lq / lr long, or -1 when
// the per-thread path does not apply (lengths beyond 32, an empty sequence is fine).
int thread_nmax(const st_seqset_s& qs, const st_seqset_s& rs, const int32_t* sim, int A, int32_t go,
                int32_t ge, bool self_q, bool self_r) {
    int need = rs.max_len;
    if (self_q) need = std::max(need, qs.max_len);
    if (self_r) need = std::max(need, rs.max_len);
    if (need > 32) return -1;
    int64_t smax = 0;
    for (int i = 0; i < A * A; ++i) smax = std::max<int64_t>(smax, std::llabs(int64_t(sim[i])));
    const int64_t span = int64_t(std::max(qs.max_len, rs.max_len)) * 2;
    const int64_t bound = span * (smax + int64_t(go) + int64_t(ge) * span);
    if (bound >= (int64_t(1) << 27)) return -1;
    return need <= 16 ? 16 : 32;
}

void launch_thread(Context& ctx, ThreadArgs a, int nmax, bool local, int64_t work, cudaStream_t stream) {
    const int64_t blocks = std::min<int64_t>(ceil_div(std::max<int64_t>(work, 1), 128),
                                             int64_t(ctx.num_sms) * 16);
    const size_t smem = size_t(a.A) * a.A * 4;
    if (nmax == 16) {
        if (local) gotoh_thread_kernel<16, true><<<unsigned(blocks), 128, smem, stream>>>(a);
        else gotoh_thread_kernel<16, false><<<unsigned(blocks), 128, smem, stream>>>(a);
    } else {
        if (local) gotoh_thread_kernel<32, true><<<unsigned(blocks), 128, smem, stream>>>(a);
        else gotoh_thread_kernel<32, false><<<unsigned(blocks), 128, smem, stream>>>(a);
    }
    STB_CUDA(cudaGetLastError());
    note_launch("gotoh_thread_kernel");
}

// ------------------------------------------------------------------------- wavefront path ---
// Warp-cooperative anti-diagonal wavefront.  A warp scores one query against two refs at once
// (int16x2 halves).  Lane t owns query rows t*R+1 .. t*R+R and at step s processes column
// j = s - t + 1, so the row above its first row (lane t-1's last row, same column) was finished
// one step earlier and arrives by one shuffle, together with the column's two ref residues.
// Cells are updated with DPX max-plus ops on both halves; the substitution scores of a cell pair
// come from one shared-memory word T[q][r1][r2] = s(q,r1) | s(q,r2) << 16, where the extra code
// A pads rows past the query and columns past the shorter ref with NEG.
//
// With gap_extend <= gap_open the vertical gap is max(H_up - open, X_up - extend): H includes X,
// and X_up - open <= X_up - extend, so adding it to the opening term never changes the maximum --
// this is the reference's max(M_up - open, Y_up - open, X_up - extend) (pairwise.cpp:113), and
// likewise for the horizontal gap (:114).  Otherwise (EXACT) the opening terms use max(M, Y) and
// max(M, X) as the reference does.
//
// int16 safety: the host admits a call only when every finite cell lies within +-14000
// (|s| * L + open + extend * (rows + cols) <= 14000, |s| <= 2000); then NEG = -16384 and every
// NEG-derived candidate stays below every finite one without wrapping.
//
// Global mode with gap_extend <= gap_open (OFFSET) keeps every state of cell (i, j) raised by
// (i + j) * extend: H~ = H + (i+j)e, and likewise M~, X~, Y~.  Then
//   X~(i,j) = max(H~(i-1,j) + e - o, X~(i-1,j)),  Y~(i,j) = max(H~(i,j-1) + e - o, Y~(i,j-1)),
//   M~(i,j) = H~(i-1,j-1) + s + 2e,               H~ = max(M~, X~, Y~),
// so each gap state is one add-max instead of two (the 2e rides in the substitution table), and
// every border H~ is the constant e - o (0 at the corner).  The score is H~(m,n) - (m+n)e.  The
// offset is non-negative and at most extend * (rows + cols), which the admission bound above
// already counts, so the raised states stay within +-14000; the gap states only take maxima, so
// NEG never drifts downwards.
constexpr int kWaveThreads = 256;
constexpr uint32_t kNeg2 = 0xC000C000u;  // -16384 in both halves

struct WaveArgs {
    const uint8_t* qc;
    const int64_t* qoff;
    const uint8_t* rc;
    const int64_t* roff;
    const int32_t* qlist;   // queries of this launch (all of one row bucket)
    int64_t nq;
    const int2* rpairs;     // ref pairs of similar length (x == y for an odd one out)
    int64_t nrp;
    const uint32_t* table;  // A1^3 words
    int A1;                 // alphabet size + 1 (the last code pads)
    int32_t go, ge;
    int self;               // 1: each query against itself, int64 result to self_out
    int64_t* self_out;
    int dist;
    const int64_t* q_self;
    const int64_t* r_self;
    int32_t* out;
    int64_t K;
    unsigned int* overflow;
};

__device__ __forceinline__ uint32_t dup2(int v) { return (uint32_t(uint16_t(int16_t(v))) * 0x10001u); }
__device__ __forceinline__ int lo16(uint32_t v) { return int(int16_t(uint16_t(v & 0xFFFFu))); }
__device__ __forceinline__ int hi16(uint32_t v) { return int(int16_t(uint16_t(v >> 16))); }

template <int R, bool LOCAL, bool EXACT>
__global__ void __launch_bounds__(kWaveThreads) gotoh_wave_kernel(const WaveArgs a) {
    extern __shared__ uint32_t s_tab[];
    const int A1 = a.A1, pad = A1 - 1;
    for (int i = threadIdx.x; i < A1 * A1 * A1; i += blockDim.x) s_tab[i] = a.table[i];
    __syncthreads();
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int64_t gwarp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int64_t ntasks = a.self ? a.nq : a.nq * a.nrp;
    const uint32_t mgo2 = dup2(-a.go), mge2 = dup2(-a.ge);
    constexpr bool OFFSET = !LOCAL && !EXACT;
    const uint32_t eo2 = dup2(a.ge - a.go);  // the raised border value, and the gap-open step

    for (int64_t task = gwarp; task < ntasks; task += nwarps) {
        const int64_t qi_idx = a.self ? task : task / a.nrp;
        const int qi = a.qlist[qi_idx];
        int k1 = qi, k2 = qi;
        if (!a.self) {
            const int2 rp = a.rpairs[task - qi_idx * a.nrp];
            k1 = rp.x;
            k2 = rp.y;
        }
        const uint8_t* q = a.qc + a.qoff[qi];
        const int m = int(a.qoff[qi + 1] - a.qoff[qi]);
        const uint8_t* rbase = a.self ? a.qc : a.rc;
        const int64_t* roff = a.self ? a.qoff : a.roff;
        const uint8_t* r1 = rbase + roff[k1];
        const uint8_t* r2 = rbase + roff[k2];
        const int n1 = int(roff[k1 + 1] - roff[k1]);
        const int n2 = int(roff[k2 + 1] - roff[k2]);
        const int nmax = max(n1, n2);

        // Rows of this lane: 1-indexed i = lane*R + r + 1; column 0 state per row.
        uint32_t qb[R], Hl[R], Yl[R], MXl[EXACT ? R : 1];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = lane * R + r;  // 0-indexed query position
            qb[r] = uint32_t((row < m ? q[row] : pad) * A1 * A1);
            const int gr = a.go + row * a.ge;  // gap_run(row + 1)
            Hl[r] = LOCAL ? 0u : (OFFSET ? eo2 : dup2(-gr));
            Yl[r] = kNeg2;
            if constexpr (EXACT) MXl[r] = Hl[r];
        }
        // H[lane*R][0]: the row above this lane's first row, at column 0.
        uint32_t diag = (lane == 0 || LOCAL) ? 0u
                        : (OFFSET ? eo2 : dup2(-(a.go + (lane * R - 1) * a.ge)));
        uint32_t best = 0u, cap = 0u;
        uint32_t outH = 0u, outX = kNeg2, outMY = 0u;
        int outRes = 0;
        const int cap_lane = (m - 1) / R, cap_r = (m - 1) - cap_lane * R;
        const int steps = nmax + 31;
        for (int s = 0; s < steps; ++s) {
            uint32_t upH = __shfl_up_sync(full, outH, 1);
            uint32_t upX = __shfl_up_sync(full, outX, 1);
            uint32_t upMY = EXACT ? __shfl_up_sync(full, outMY, 1) : 0u;
            int res = __shfl_up_sync(full, outRes, 1);
            const int j = s - lane + 1;
            if (lane == 0) {  // the virtual row 0 at column j
                const uint32_t h0 = LOCAL ? 0u : (OFFSET ? eo2 : dup2(-(a.go + (j - 1) * a.ge)));
                upH = h0;
                upX = kNeg2;
                upMY = h0;
                res = (j <= n1 ? int(r1[j - 1]) : pad) | ((j <= n2 ? int(r2[j - 1]) : pad) << 8);
            }
            if (j >= 1 && j <= nmax) {
                const uint32_t col = uint32_t((res & 0xFF) * A1 + (res >> 8));
                const uint32_t top = upH;
                uint32_t d = diag;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const uint32_t sc = s_tab[qb[r] + col];
                    const uint32_t M = LOCAL ? __viaddmax_s16x2_relu(d, sc, kNeg2)
                                             : __viaddmax_s16x2(d, sc, kNeg2);
                    uint32_t X, Y;
                    if constexpr (EXACT) {
                        X = __viaddmax_s16x2(upMY, mgo2, __viaddmax_s16x2(upX, mge2, kNeg2));
                        Y = __viaddmax_s16x2(MXl[r], mgo2, __viaddmax_s16x2(Yl[r], mge2, kNeg2));
                    } else if constexpr (OFFSET) {
                        X = __viaddmax_s16x2(upH, eo2, upX);
                        Y = __viaddmax_s16x2(Hl[r], eo2, Yl[r]);
                    } else {
                        X = __viaddmax_s16x2(upH, mgo2, __viaddmax_s16x2(upX, mge2, kNeg2));
                        Y = __viaddmax_s16x2(Hl[r], mgo2, __viaddmax_s16x2(Yl[r], mge2, kNeg2));
                    }
                    const uint32_t H = __vimax3_s16x2(M, X, Y);
                    if constexpr (LOCAL) best = __vimax3_s16x2(best, M, kNeg2);
                    d = Hl[r];
                    Hl[r] = H;
                    Yl[r] = Y;
                    upH = H;
                    upX = X;
                    if constexpr (EXACT) {
                        MXl[r] = __vimax3_s16x2(M, X, kNeg2);
                        upMY = __vimax3_s16x2(M, Y, kNeg2);
                    }
                }
                diag = top;
                outH = upH;
                outX = upX;
                outMY = upMY;
                outRes = res;
                if (!LOCAL && lane == cap_lane && (j == n1 || j == n2)) {
                    uint32_t h = 0u;
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (r == cap_r) h = Hl[r];
                    if (j == n1) cap = (cap & 0xFFFF0000u) | (h & 0xFFFFu);
                    if (j == n2) cap = (cap & 0xFFFFu) | (h & 0xFFFF0000u);
                }
            }
        }
        int v1, v2;
        if constexpr (LOCAL) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                best = __vimax3_s16x2(best, __shfl_xor_sync(full, best, off), kNeg2);
            v1 = lo16(best);
            v2 = hi16(best);
        } else {
            cap = __shfl_sync(full, cap, cap_lane);
            v1 = lo16(cap);
            v2 = hi16(cap);
            if constexpr (OFFSET) {
                v1 -= (m + n1) * a.ge;
                v2 -= (m + n2) * a.ge;
            }
        }
        if (lane == 0) {
            if (a.self) {
                a.self_out[qi] = v1;
            } else {
                for (int t = 0; t < (k2 != k1 ? 2 : 1); ++t) {
                    const int k = t ? k2 : k1;
                    const int64_t sv = t ? v2 : v1;
                    const int64_t v = a.dist ? a.q_self[qi] + a.r_self[k] - 2 * sv : sv;
                    if (v < INT32_MIN || v > INT32_MAX)
                        atomicOr(a.overflow, 1u);
                    else
                        a.out[int64_t(qi) * a.K + k] = int32_t(v);
                }
            }
        }
    }
}

// Query-pair form of the wavefront, used for the N x K pass.  A CTA holds two queries of one row
// bucket (neighbours in length order) and a chunk of refs taken in length order.  Its shared
// memory holds the pair's substitution profile P[c][r][lane] = s(q1[lane*R + r], c) |
// s(q2[lane*R + r], c) << 16 (NEG past a query's length; + 2 * gap_extend in the raised global
// form), so a lane reads the scores of its R rows at column code c from the words
// c*R*32 + r*32 + lane: one conflict-free 32-bit load per cell pair, at an immediate offset from
// one per-column base.  A warp takes one ref at a time; the ref's codes, pre-multiplied into
// profile offsets, are staged in the warp's slice of shared memory, so every lane reads its own
// column's code without a shuffle.  The recurrence, the int16 safety argument and the raised
// global form are those of gotoh_wave_kernel above.  Only the packing differs: the two halves
// are two queries against one ref, so both end at the ref's last column, and the global score
// of each query is read at its own last row.
constexpr int kQpWarps = 8;
constexpr int kQpMaxRef = 512;  // wave_eligible admits lengths up to 512

struct QpArgs {
    const uint8_t* qc;
    const int64_t* qoff;
    const uint8_t* rc;
    const int64_t* roff;
    const int2* qpairs;      // query pairs of this launch (one row bucket; x == y for a single)
    int64_t nqp;
    const int32_t* rorder;   // every ref, by length
    int64_t K;
    int64_t chunk;           // refs per CTA
    const int32_t* simadd;   // A x A: s(a, b) + add
    int A;
    int32_t go, ge;
    int dist;
    const int64_t* q_self;
    const int64_t* r_self;
    int32_t* out;
    unsigned int* overflow;
};

inline size_t qpair_smem(int A, int R) {
    return size_t(A) * R * 32 * 4 + size_t(kQpWarps) * kQpMaxRef * 2;
}

template <int R, bool LOCAL, bool EXACT>
__global__ void __launch_bounds__(kQpWarps * 32) gotoh_qpair_kernel(const QpArgs a) {
    extern __shared__ uint32_t s_prof[];  // A * R * 32 words, then kQpWarps ref slices
    uint16_t* my_ref = reinterpret_cast<uint16_t*>(s_prof + a.A * R * 32) +
                       (threadIdx.x >> 5) * kQpMaxRef;
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr bool OFFSET = !LOCAL && !EXACT;
    const uint32_t mgo2 = dup2(-a.go), mge2 = dup2(-a.ge);
    const uint32_t eo2 = dup2(a.ge - a.go);
    const int64_t r_lo = int64_t(blockIdx.x) * a.chunk;
    const int64_t r_hi = min(r_lo + a.chunk, a.K);
    const int words = a.A * R * 32;

    for (int64_t p = blockIdx.y; p < a.nqp; p += gridDim.y) {
        const int2 qp = a.qpairs[p];
        const uint8_t* q1 = a.qc + a.qoff[qp.x];
        const uint8_t* q2 = a.qc + a.qoff[qp.y];
        const int m1 = int(a.qoff[qp.x + 1] - a.qoff[qp.x]);
        const int m2 = int(a.qoff[qp.y + 1] - a.qoff[qp.y]);
        __syncthreads();  // every warp is done with the previous pair's profile
        for (int w = threadIdx.x; w < words; w += blockDim.x) {
            const int c = w / (R * 32), rr = (w >> 5) % R, row = (w & 31) * R + rr;
            const int v1 = row < m1 ? a.simadd[int(q1[row]) * a.A + c] : -16384;
            const int v2 = row < m2 ? a.simadd[int(q2[row]) * a.A + c] : -16384;
            s_prof[w] = uint32_t(uint16_t(int16_t(v1))) | (uint32_t(uint16_t(int16_t(v2))) << 16);
        }
        __syncthreads();
        // lane and register of each query's last row
        const int cl1 = (m1 - 1) / R, cr1 = (m1 - 1) - cl1 * R;
        const int cl2 = (m2 - 1) / R, cr2 = (m2 - 1) - cl2 * R;

        for (int64_t t = r_lo + warp; t < r_hi; t += kQpWarps) {
            const int k = a.rorder[t];
            const uint8_t* rs = a.rc + a.roff[k];
            const int n = int(a.roff[k + 1] - a.roff[k]);
            __syncwarp();
            for (int j = lane; j < n; j += 32) my_ref[j] = uint16_t(int(rs[j]) * R * 32);
            __syncwarp();

            // Lane state: H and Y of its R rows at the last column it computed (column 0 to
            // start), the X (and, EXACT, max(M, Y)) of its last row for the lane below, and
            // (EXACT) max(M, X) of each row.
            uint32_t Hl[R], Yl[R], MXl[EXACT ? R : 1];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int row = lane * R + r;
                Hl[r] = LOCAL ? 0u : (OFFSET ? eo2 : dup2(-(a.go + row * a.ge)));
                Yl[r] = kNeg2;
                if constexpr (EXACT) MXl[r] = Hl[r];
            }
            uint32_t diag = (lane == 0 || LOCAL) ? 0u
                            : (OFFSET ? eo2 : dup2(-(a.go + (lane * R - 1) * a.ge)));
            uint32_t Xlast = kNeg2, MYlast = 0u, best = 0u;
            const uint32_t* prof_lane = s_prof + lane;
            const uint16_t* rcol = my_ref - lane;  // rcol[s]: this lane's column j - 1 = s - lane

            // One column of this lane's rows at step s (the lane's column is j = s - lane + 1).
            // Every lane shuffles; `active` lanes update.  The diagonal terms of all rows are
            // formed first, so the old H of a row is dead once its own Y and H are formed.
            auto step = [&](int s, bool active) {
                uint32_t upH = __shfl_up_sync(full, Hl[R - 1], 1);
                uint32_t upX = __shfl_up_sync(full, Xlast, 1);
                uint32_t upMY = EXACT ? __shfl_up_sync(full, MYlast, 1) : 0u;
                if (lane == 0) {  // the virtual row 0 at column j = s + 1
                    const uint32_t h0 = LOCAL ? 0u : (OFFSET ? eo2 : dup2(-(a.go + s * a.ge)));
                    upH = h0;
                    upX = kNeg2;
                    upMY = h0;
                }
                if (!active) return;
                const uint32_t* pc = prof_lane + rcol[s];
                uint32_t M[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const uint32_t dg = r == 0 ? diag : Hl[r - 1];
                    M[r] = LOCAL ? __viaddmax_s16x2_relu(dg, pc[r * 32], kNeg2)
                                 : __viaddmax_s16x2(dg, pc[r * 32], kNeg2);
                }
                diag = upH;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    uint32_t X, Y;
                    if constexpr (EXACT) {
                        X = __viaddmax_s16x2(upMY, mgo2, __viaddmax_s16x2(upX, mge2, kNeg2));
                        Y = __viaddmax_s16x2(MXl[r], mgo2, __viaddmax_s16x2(Yl[r], mge2, kNeg2));
                    } else if constexpr (OFFSET) {
                        X = __viaddmax_s16x2(upH, eo2, upX);
                        Y = __viaddmax_s16x2(Hl[r], eo2, Yl[r]);
                    } else {
                        X = __viaddmax_s16x2(upH, mgo2, __viaddmax_s16x2(upX, mge2, kNeg2));
                        Y = __viaddmax_s16x2(Hl[r], mgo2, __viaddmax_s16x2(Yl[r], mge2, kNeg2));
                    }
                    const uint32_t H = __vimax3_s16x2(M[r], X, Y);
                    if constexpr (EXACT) {
                        MXl[r] = __vimax3_s16x2(M[r], X, kNeg2);
                        upMY = __vimax3_s16x2(M[r], Y, kNeg2);
                    }
                    Hl[r] = H;
                    Yl[r] = Y;
                    upH = H;
                    upX = X;
                }
                if constexpr (LOCAL) {  // the running maximum of M, two rows per operation
#pragma unroll
                    for (int r = 0; r < R; r += 2)
                        best = __vimax3_s16x2(best, M[r], r + 1 < R ? M[r + 1] : kNeg2);
                }
                Xlast = upX;
                MYlast = upMY;
            };
            // Ramp in (lanes start one step apart), steady state (every lane on a column of
            // 1..n: no range test), ramp out.
            int s = 0;
            for (; s < 31; ++s) step(s, s >= lane && s - lane < n);
#pragma unroll 2
            for (; s < n; ++s) step(s, true);
            for (; s < n + 31; ++s) step(s, s - lane < n);

            int v1, v2;
            if constexpr (LOCAL) {
#pragma unroll
                for (int off = 16; off > 0; off >>= 1)
                    best = __vimax3_s16x2(best, __shfl_xor_sync(full, best, off), kNeg2);
                v1 = lo16(best);
                v2 = hi16(best);
            } else {
                // A lane's H registers keep its last column (n) once it has passed it: each
                // query's global score sits in the lane and register of its last row.
                uint32_t c1 = 0u, c2 = 0u;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r == cr1) c1 = Hl[r];
                    if (r == cr2) c2 = Hl[r];
                }
                v1 = lo16(__shfl_sync(full, c1, cl1));
                v2 = hi16(__shfl_sync(full, c2, cl2));
                if constexpr (OFFSET) {
                    v1 -= (m1 + n) * a.ge;
                    v2 -= (m2 + n) * a.ge;
                }
            }
            if (lane == 0) {
                for (int t2 = 0; t2 < (qp.y != qp.x ? 2 : 1); ++t2) {
                    const int qi = t2 ? qp.y : qp.x;
                    const int64_t sv = t2 ? v2 : v1;
                    const int64_t v = a.dist ? a.q_self[qi] + a.r_self[k] - 2 * sv : sv;
                    if (v < INT32_MIN || v > INT32_MAX)
                        atomicOr(a.overflow, 1u);
                    else
                        a.out[int64_t(qi) * a.K + k] = int32_t(v);
                }
            }
        }
    }
}

template <int R>
const void* qpair_kernel_ptr(bool local, bool exact) {
    if (local)
        return exact ? reinterpret_cast<const void*>(gotoh_qpair_kernel<R, true, true>)
                     : reinterpret_cast<const void*>(gotoh_qpair_kernel<R, true, false>);
    return exact ? reinterpret_cast<const void*>(gotoh_qpair_kernel<R, false, true>)
                 : reinterpret_cast<const void*>(gotoh_qpair_kernel<R, false, false>);
}

const void* qpair_kernel(int R, bool local, bool exact) {
    switch (R) {
        case 1: return qpair_kernel_ptr<1>(local, exact);
        case 2: return qpair_kernel_ptr<2>(local, exact);
        case 3: return qpair_kernel_ptr<3>(local, exact);
        case 4: return qpair_kernel_ptr<4>(local, exact);
        case 5: return qpair_kernel_ptr<5>(local, exact);
        case 6: return qpair_kernel_ptr<6>(local, exact);
        case 7: return qpair_kernel_ptr<7>(local, exact);
        case 8: return qpair_kernel_ptr<8>(local, exact);
        case 9: return qpair_kernel_ptr<9>(local, exact);
        case 10: return qpair_kernel_ptr<10>(local, exact);
        case 11: return qpair_kernel_ptr<11>(local, exact);
        case 12: return qpair_kernel_ptr<12>(local, exact);
        case 13: return qpair_kernel_ptr<13>(local, exact);
        case 14: return qpair_kernel_ptr<14>(local, exact);
        case 15: return qpair_kernel_ptr<15>(local, exact);
        default: return qpair_kernel_ptr<16>(local, exact);
    }
}

// Rows per lane of the query-pair kernel: the smallest R with 32 * R >= m, rounded up to a
// multiple of `step` (step 1: 32-row buckets, a query carries fewer than 32 padded rows; step 2:
// 64-row buckets, fewer and larger launches).
int qpair_rows_per_lane(int m, int step = 1) {
    const int r = std::max(1, int((m + 31) / 32));
    return std::min(16, (r + step - 1) / step * step);
}

constexpr int kRowBuckets[] = {2, 4, 6, 8, 10, 12, 14, 16};

int rows_per_lane(int m) {
    for (int r : kRowBuckets)
        if (m <= 32 * r) return r;
    return 0;
}

template <int R>
const void* wave_kernel_ptr(bool local, bool exact) {
    if (local)
        return exact ? reinterpret_cast<const void*>(gotoh_wave_kernel<R, true, true>)
                     : reinterpret_cast<const void*>(gotoh_wave_kernel<R, true, false>);
    return exact ? reinterpret_cast<const void*>(gotoh_wave_kernel<R, false, true>)
                 : reinterpret_cast<const void*>(gotoh_wave_kernel<R, false, false>);
}

const void* wave_kernel(int R, bool local, bool exact) {
    switch (R) {
        case 2: return wave_kernel_ptr<2>(local, exact);
        case 4: return wave_kernel_ptr<4>(local, exact);
        case 6: return wave_kernel_ptr<6>(local, exact);
        case 8: return wave_kernel_ptr<8>(local, exact);
        case 10: return wave_kernel_ptr<10>(local, exact);
        case 12: return wave_kernel_ptr<12>(local, exact);
        case 14: return wave_kernel_ptr<14>(local, exact);
        default: return wave_kernel_ptr<16>(local, exact);
    }
}

// Substitution tables of the wavefront path, per device, and the grid they were built from:
// the packed T[q][r1][r2] words of gotoh_wave_kernel and the A x A s(a, b) + add grid the
// query-pair kernel builds its profiles from.
struct WaveState {
    std::vector<uint8_t> key;
    DevBuf table, simadd;
    // Side streams and events that run the row buckets' launches concurrently (fork / join on
    // the caller's stream), so that one bucket's tail of idle SMs is filled by the next bucket.
    static constexpr int kSide = 4;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr, join[kSide] = {};
    void ensure_streams() {
        if (fork) return;
        for (int i = 0; i < kSide; ++i) {
            STB_CUDA(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
            STB_CUDA(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming));
        }
        STB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    }
};

// Per-set launch plan (depends only on the lengths): the set's indices grouped by rows per
// lane, with the (R, offset, count) of each group; inside each group the sequences sorted by
// length and paired with their neighbour (the query side of the query-pair kernel), with the
// (R, offset, count) of each group's pairs; and every index sorted by length (the ref side).
struct WavePlan {
    uint64_t uid = 0;
    std::vector<std::tuple<int, int64_t, int64_t>> groups, pair_groups[2];
    DevBuf list, qpairs[2], sorted;
};

WavePlan& wave_plan(st_seqset_s& s, Context& ctx, int slot, cudaStream_t stream) {
    std::shared_ptr<void>& holder = s.owns ? s.wave_plan : ctx.tmp_wave_plan[slot];
    if (!holder) holder = std::make_shared<WavePlan>();
    WavePlan& p = *static_cast<WavePlan*>(holder.get());
    if (p.uid == s.uid) return p;
    std::vector<std::vector<int32_t>> b(17);
    for (int64_t i = 0; i < s.count; ++i)
        b[size_t(rows_per_lane(s.h_len[size_t(i)]))].push_back(int32_t(i));
    std::vector<int32_t> all;
    all.reserve(size_t(s.count));
    p.groups.clear();
    for (int R = 1; R <= 16; ++R)
        if (!b[size_t(R)].empty()) {
            p.groups.emplace_back(R, int64_t(all.size()), int64_t(b[size_t(R)].size()));
            all.insert(all.end(), b[size_t(R)].begin(), b[size_t(R)].end());
        }
    auto by_len = [&](int32_t x, int32_t y) { return s.h_len[size_t(x)] < s.h_len[size_t(y)]; };
    std::vector<int32_t> order(static_cast<size_t>(s.count));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), by_len);
    // Query pairs per bucket, for both bucket widths (32 and 64 rows; the tuner picks one).
    std::vector<int32_t> qpairs[2];
    for (int w = 0; w < 2; ++w) {
        qpairs[w].reserve(size_t(s.count) + 34);
        p.pair_groups[w].clear();
        std::vector<std::vector<int32_t>> fine(17);
        for (int64_t i = 0; i < s.count; ++i)
            fine[size_t(qpair_rows_per_lane(s.h_len[size_t(i)], w + 1))].push_back(int32_t(i));
        for (int R = 1; R <= 16; ++R) {
            std::vector<int32_t>& g = fine[size_t(R)];
            if (g.empty()) continue;
            std::stable_sort(g.begin(), g.end(), by_len);
            const int64_t first = int64_t(qpairs[w].size() / 2);
            for (size_t i = 0; i < g.size(); i += 2) {
                qpairs[w].push_back(g[i]);
                qpairs[w].push_back(i + 1 < g.size() ? g[i + 1] : g[i]);
            }
            p.pair_groups[w].emplace_back(R, first, int64_t(qpairs[w].size() / 2) - first);
        }
    }
    // (a pageable-source copy has consumed the host vectors by the time it returns)
    h2d(p.list.as<int32_t>(all.size()), all.data(), all.size() * 4, stream);
    for (int w = 0; w < 2; ++w)
        h2d(p.qpairs[w].as<int32_t>(qpairs[w].size()), qpairs[w].data(), qpairs[w].size() * 4,
            stream);
    h2d(p.sorted.as<int32_t>(order.size()), order.data(), order.size() * 4, stream);
    p.uid = s.uid;
    return p;
}

WaveState& wave_state(int device) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<WaveState>> all;
    std::lock_guard<std::mutex> lk(mu);
    auto& p = all[device];
    if (!p) p = std::make_unique<WaveState>();
    return *p;
}

// Every finite cell of every pair within +-14000 (see the kernel's note), lengths 1..512.
bool wave_eligible(const st_seqset_s& qs, const st_seqset_s& rs, const int32_t* sim, int A,
                   int32_t go, int32_t ge) {
    for (const st_seqset_s* s : {&qs, &rs})
        for (int32_t l : s->h_len)
            if (l < 1) return false;
    if (qs.max_len > 512 || rs.max_len > 512) return false;
    int64_t maxabs = 0;
    for (int i = 0; i < A * A; ++i) maxabs = std::max<int64_t>(maxabs, std::llabs(int64_t(sim[i])));
    if (maxabs > 2000) return false;
    const int64_t rows = 512, cols = std::max(qs.max_len, rs.max_len);
    const int64_t bound = maxabs * rows + int64_t(go) + int64_t(ge) * (rows + cols);
    return bound <= 14000;
}

// Launches one wavefront pass: `list` queries (one row bucket) against `pairs` (or themselves).
void launch_wave(Context& ctx, WaveArgs wa, int R, bool local, bool exact, cudaStream_t stream) {
    const void* kern = wave_kernel(R, local, exact);
    const size_t smem = size_t(wa.A1) * wa.A1 * wa.A1 * 4;
    STB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    STB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWaveThreads, smem));
    const int64_t ntasks = wa.self ? wa.nq : wa.nq * wa.nrp;
    const int64_t warps_per_block = kWaveThreads / 32;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(
        ceil_div(ntasks, warps_per_block), int64_t(ctx.num_sms) * std::max(per_sm, 1)));
    void* args[] = {&wa};
    STB_CUDA(cudaLaunchKernel(kern, dim3(unsigned(blocks)), dim3(kWaveThreads), args, smem, stream));
    note_launch("gotoh_wave_kernel");
}

// Launches one query-pair pass: the pairs of one row bucket against every ref, `chunk` refs per
// CTA column.
void launch_qpair(QpArgs qa, int R, bool local, bool exact, cudaStream_t stream) {
    const void* kern = qpair_kernel(R, local, exact);
    const size_t smem = qpair_smem(qa.A, R);
    ensure_smem_limit(kern, smem);
    const int64_t gx = ceil_div(qa.K, qa.chunk);
    const int64_t gy = std::min<int64_t>(qa.nqp, 65535);
    void* args[] = {&qa};
    STB_CUDA(cudaLaunchKernel(kern, dim3(unsigned(gx), unsigned(gy)), dim3(kQpWarps * 32), args,
                              smem, stream));
    note_launch("gotoh_qpair_kernel");
}

}  // namespace

// The warp-wavefront path for every pair (int16x2 cells; the caller checked wave_eligible).
void align_wave(st_seqset_s& qs, st_seqset_s& rs, const int32_t* similarity, int A, int32_t mode,
                int32_t go, int32_t ge, int32_t dist, int32_t* out_d, unsigned int* ovf,
                cudaStream_t stream, int bucket = 0) {
    Context& ctx = context();
    const int64_t N = qs.count, K = rs.count;
    WaveState& ws = wave_state(ctx.device);
    const int A1 = A + 1;
    {
        // T[(q*A1 + r1)*A1 + r2] = s(q,r1) | s(q,r2) << 16, the pad code scoring NEG; the
        // offset form (global, gap_extend <= gap_open) adds 2 * gap_extend to every finite score.
        const int32_t add = (mode != ST_MODE_LOCAL && ge <= go) ? 2 * ge : 0;
        std::vector<uint8_t> key(size_t(A) * A * 4 + 4);
        std::memcpy(key.data(), similarity, size_t(A) * A * 4);
        std::memcpy(key.data() + size_t(A) * A * 4, &add, 4);
        if (!same_as_last(ws.key, key.data(), key.size())) {
            std::vector<uint32_t> tab(size_t(A1) * A1 * A1);
            auto sv = [&](int x, int y) -> int32_t {
                return (x == A || y == A) ? -16384 : similarity[x * A + y] + add;
            };
            for (int x = 0; x < A1; ++x)
                for (int y1 = 0; y1 < A1; ++y1)
                    for (int y2 = 0; y2 < A1; ++y2)
                        tab[(size_t(x) * A1 + y1) * A1 + y2] =
                            uint32_t(uint16_t(int16_t(sv(x, y1)))) |
                            (uint32_t(uint16_t(int16_t(sv(x, y2)))) << 16);
            std::vector<int32_t> sa(size_t(A) * A);
            for (int x = 0; x < A * A; ++x) sa[size_t(x)] = similarity[x] + add;
            try {
                h2d(ws.table.as<uint32_t>(tab.size()), tab.data(), tab.size() * 4, stream);
                h2d(ws.simadd.as<int32_t>(sa.size()), sa.data(), sa.size() * 4, stream);
            } catch (...) {
                ws.key.clear();  // not uploaded: the next call builds it again
                throw;
            }
        }
    }
    WavePlan& qp = wave_plan(qs, ctx, 0, stream);
    WavePlan& rp = wave_plan(rs, ctx, 1, stream);
    const bool local = mode == ST_MODE_LOCAL;
    const bool exact = ge > go;
    WaveArgs wa{};
    wa.table = static_cast<uint32_t*>(ws.table.ptr);
    wa.A1 = A1;
    wa.go = go;
    wa.ge = ge;
    wa.overflow = ovf;
    wa.K = K;
    int64_t* q_self = nullptr;
    int64_t* r_self = nullptr;
    if (dist) {
        q_self = ctx.work_b.as<int64_t>(size_t(N + K));
        r_self = q_self + N;
        for (int t = 0; t < 2; ++t) {
            const st_seqset_s& s = t == 0 ? qs : rs;
            const WavePlan& p = t == 0 ? qp : rp;
            for (auto& [R, off, cnt] : p.groups) {
                WaveArgs sa = wa;
                sa.qc = s.d_bytes;
                sa.qoff = s.d_off;
                sa.qlist = static_cast<int32_t*>(p.list.ptr) + off;
                sa.nq = cnt;
                sa.self = 1;
                sa.self_out = t == 0 ? q_self : r_self;
                launch_wave(ctx, sa, R, local, exact, stream);
            }
        }
    }
    // The buckets' launches run on side streams forked from (and joined back into) the caller's
    // stream; the longest rows first, so the short buckets fill the long ones' tails.
    ws.ensure_streams();
    const auto& pgroups = qp.pair_groups[bucket];
    const int nside = std::min<int>(WaveState::kSide, int(pgroups.size()));
    STB_CUDA(cudaEventRecord(ws.fork, stream));
    for (int i = 0; i < nside; ++i) STB_CUDA(cudaStreamWaitEvent(ws.side[i], ws.fork, 0));
    int gi = 0;
    for (auto it = pgroups.rbegin(); it != pgroups.rend(); ++it, ++gi) {
        const auto& [R, off, cnt] = *it;
        QpArgs ma{};
        ma.qc = qs.d_bytes;
        ma.qoff = qs.d_off;
        ma.rc = rs.d_bytes;
        ma.roff = rs.d_off;
        ma.qpairs = static_cast<int2*>(qp.qpairs[bucket].ptr) + off;
        ma.nqp = cnt;
        ma.rorder = static_cast<int32_t*>(rp.sorted.ptr);
        ma.K = K;
        ma.chunk = 256;
        ma.simadd = static_cast<int32_t*>(ws.simadd.ptr);
        ma.A = A;
        ma.go = go;
        ma.ge = ge;
        ma.dist = dist;
        ma.q_self = q_self;
        ma.r_self = r_self;
        ma.out = out_d;
        ma.overflow = ovf;
        launch_qpair(ma, R, local, exact, ws.side[gi % nside]);
    }
    for (int i = 0; i < nside; ++i) {
        STB_CUDA(cudaEventRecord(ws.join[i], ws.side[i]));
        STB_CUDA(cudaStreamWaitEvent(stream, ws.join[i], 0));
    }
}

void align_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* similarity, int32_t matrix_size,
                int32_t mode, int32_t go, int32_t ge, int32_t dist, int32_t* out_d,
                cudaStream_t stream) {
    if (go < 0 || ge < 0)
        fail(ST_EINVAL, "seqtree: gap_open and gap_extend must be >= 0 (they are magnitudes, and "
                        "are subtracted)");
    if (qs.alphabet < 0 || qs.alphabet != rs.alphabet)
        fail(ST_EINVAL, "seqtree_b200: alignment sets must be encoded with one alphabet");
    const int A = alphabet_size(qs.alphabet);
    if (!similarity || matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
    if (mode != ST_MODE_GLOBAL && mode != ST_MODE_LOCAL)
        fail(ST_EINVAL, "unknown mode (use 'global' or 'local')");
    const int64_t N = qs.count, K = rs.count;
    if (N == 0 || K == 0) return;
    Context& ctx = context();
    // Word 9 of the context flags: set when a result does not fit int32.
    auto* ovf = reinterpret_cast<unsigned int*>(ctx.flags_d + 9);
    STB_CUDA(cudaMemsetAsync(ovf, 0, 8, stream));

    const int tn = thread_nmax(qs, rs, similarity, A, go, ge, dist != 0, dist != 0);
    const bool wave_ok = wave_eligible(qs, rs, similarity, A, go, ge);
    if (tn > 0) {
        // Short sequences: one thread per pair (registers only) or the warp wavefront, whichever
        // the autotuner measured faster for this shape.
        // the similarity table, uploaded only when it changes (so warmed-up calls capture)
        struct ThreadTable {
            std::vector<uint8_t> key;
            DevBuf sim;
        };
        static std::mutex tmu;
        static std::map<int, std::unique_ptr<ThreadTable>> tables;
        ThreadTable* tt;
        {
            std::lock_guard<std::mutex> lk(tmu);
            auto& slot = tables[ctx.device];
            if (!slot) slot = std::make_unique<ThreadTable>();
            tt = slot.get();
        }
        int32_t* d_sim = tt->sim.as<int32_t>(size_t(A) * A);
        if (!same_as_last(tt->key, similarity, size_t(A) * A * 4)) {
            try {
                h2d(d_sim, similarity, size_t(A) * A * 4, stream);
            } catch (...) {
                tt->key.clear();
                throw;
            }
        }
        auto run_thread = [&](st_seqset_s& q) {
            const int64_t Nq = q.count;
            ThreadArgs t{};
            t.sim = d_sim;
            t.A = A;
            t.go = go;
            t.ge = ge;
            t.overflow = ovf;
            int64_t* q_self = nullptr;
            int64_t* r_self = nullptr;
            if (dist) {
                q_self = ctx.work_b.as<int64_t>(size_t(Nq + K));
                r_self = q_self + Nq;
                for (int side = 0; side < 2; ++side) {
                    const st_seqset_s& s = side == 0 ? q : rs;
                    ThreadArgs b = t;
                    b.qc = s.d_bytes;
                    b.qoff = s.d_off;
                    b.N = s.count;
                    b.self = 1;
                    b.self_out = side == 0 ? q_self : r_self;
                    launch_thread(ctx, b, tn, mode == ST_MODE_LOCAL, s.count, stream);
                }
            }
            t.qc = q.d_bytes;
            t.qoff = q.d_off;
            t.rc = rs.d_bytes;
            t.roff = rs.d_off;
            t.N = Nq;
            t.K = K;
            t.dist = dist;
            t.q_self = q_self;
            t.r_self = r_self;
            t.out = out_d;
            launch_thread(ctx, t, tn, mode == ST_MODE_LOCAL, Nq * K, stream);
        };
        if (!wave_ok) {
            run_thread(qs);
            return;
        }
        const std::string key = "align|" + std::to_string(mode) + "|" + std::to_string(dist) + "|" +
                                std::to_string(A) + "|" + std::to_string(qs.max_len) + "|" +
                                std::to_string(rs.max_len) + "|" + std::to_string(size_bucket(N)) +
                                "|" + std::to_string(size_bucket(K));
        auto variant = [&](int c, st_seqset_s& q) {
            if (c == 0) run_thread(q);
            else align_wave(q, rs, similarity, A, mode, go, ge, dist, out_d, ovf, stream, c - 1);
        };
        // A shape seen for the first time is tuned on its first query rows only (about
        // kAlignTunePairs pairs, written into their own rows of the result); the choice then
        // computes the whole matrix.
        const int64_t slice = std::min<int64_t>(
            N, std::max<int64_t>(64, kAlignTunePairs / std::max<int64_t>(K, 1)));
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        STB_CUDA(cudaStreamIsCapturing(stream, &cs));
        if (slice < N && tuning_enabled() && cs == cudaStreamCaptureStatusNone &&
            tuned_lookup(key) < 0) {
            std::unique_ptr<st_seqset_s> view = row_view(qs, slice);
            tuned_run(key, 3, 0, [&](int c) { variant(c, *view); }, stream);
        }
        tuned_run(key, 3, 0, [&](int c) { variant(c, qs); }, stream);
        return;
    }
    if (wave_ok) {
        // The row-bucket width (32 or 64 rows) is tuned once per shape, on the first query rows
        // (about kWaveTunePairs pairs, written into their own rows of the result).
        const std::string key = "wave|" + std::to_string(mode) + "|" + std::to_string(dist) + "|" +
                                std::to_string(A) + "|" + std::to_string(qs.max_len) + "|" +
                                std::to_string(rs.max_len) + "|" + std::to_string(size_bucket(N)) +
                                "|" + std::to_string(size_bucket(K));
        auto bucketed = [&](int c, st_seqset_s& q) {
            align_wave(q, rs, similarity, A, mode, go, ge, dist, out_d, ovf, stream, c);
        };
        const int64_t slice = std::min<int64_t>(
            N, std::max<int64_t>(64, kWaveTunePairs / std::max<int64_t>(K, 1)));
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        STB_CUDA(cudaStreamIsCapturing(stream, &cs));
        if (slice < N && tuning_enabled() && cs == cudaStreamCaptureStatusNone &&
            tuned_lookup(key) < 0) {
            std::unique_ptr<st_seqset_s> view = row_view(qs, slice);
            tuned_run(key, 2, 0, [&](int c) { bucketed(c, *view); }, stream);
        }
        tuned_run(key, 2, 0, [&](int c) { bucketed(c, qs); }, stream);
        return;
    }

    int32_t* d_sim = ctx.table_buf.as<int32_t>(size_t(A) * A);
    h2d(d_sim, similarity, size_t(A) * A * 4, stream);
    ExactArgs a{};
    a.sim = d_sim;
    a.A = A;
    a.local = mode == ST_MODE_LOCAL;
    a.go = go;
    a.ge = ge;
    a.overflow = ovf;
    int64_t* q_self = nullptr;
    int64_t* r_self = nullptr;
    if (dist) {
        q_self = ctx.work_b.as<int64_t>(size_t(N + K));
        r_self = q_self + N;
        for (int t = 0; t < 2; ++t) {
            st_seqset_s& s = t == 0 ? qs : rs;
            ExactArgs b = a;
            b.qc = s.d_bytes;
            b.qoff = s.d_off;
            b.N = s.count;
            b.self = 1;
            b.self_out = t == 0 ? q_self : r_self;
            b.nmax1 = int64_t(s.max_len) + 1;
            launch_exact(ctx, b, s.count, stream);
        }
    }
    a.qc = qs.d_bytes;
    a.qoff = qs.d_off;
    a.rc = rs.d_bytes;
    a.roff = rs.d_off;
    a.N = N;
    a.K = K;
    a.dist = dist;
    a.q_self = q_self;
    a.r_self = r_self;
    a.out = out_d;
    a.nmax1 = int64_t(rs.max_len) + 1;
    launch_exact(ctx, a, N * K, stream);
}


}  // namespace stb
