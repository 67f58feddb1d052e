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

#include "common.cuh"

namespace stb {

namespace {

constexpr int64_t kNegInf = INT64_MIN / 4;  // src/pairwise.cpp:37

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

}  // namespace

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
    int32_t* d_sim = ctx.table_buf.as<int32_t>(size_t(A) * A);
    STB_CUDA(cudaMemcpyAsync(d_sim, similarity, size_t(A) * A * 4, cudaMemcpyHostToDevice, stream));
    // Word 9 of the context flags: set when a result does not fit int32.
    auto* ovf = reinterpret_cast<unsigned int*>(ctx.flags_d + 9);
    STB_CUDA(cudaMemsetAsync(ovf, 0, 8, stream));

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
