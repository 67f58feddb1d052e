// Batched Gotoh alignment with traceback: seqtree's align_pair (src/pairwise.cpp:141-267) for a
// list of (query, ref) pairs of two device sets -- e.g. the top hits a sparse search or the
// learned proposals produced -- and, further down, its penalty-minimising sibling Index::align
// (src/index.cpp:105-179).
//
// One thread per pair.  The forward pass is the reference's recurrence in int64 (so it is exact
// for any gap cost), its DP row kept in global scratch laid out [column][thread]; every cell
// also stores one direction byte: bits 0-1 the state the match cell came from (M, X, Y or
// stop), bits 2-3 the X (gap in the ref) predecessor, bits 4-5 the Y predecessor, bit 6 "M is 0"
// (the Smith-Waterman stop test).  Ties resolve as the reference's pick(): M, then X only if
// strictly greater, then Y only if strictly greater; the local end cell is the first strictly
// best in row-major order.  The traceback then walks the bytes from the end cell and writes the
// aligned query, aligned ref and ops (M match, S substitution, D gap in the ref, I gap in the
// query) backwards into the pair's output slot; start_out[p] is where they begin.  Pairs with
// an empty side are scored here and marked start -1: their strings are the raw input, which
// the host writes.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace stb {

namespace {

constexpr int64_t kNeg = INT64_MIN / 4;  // src/pairwise.cpp:37
enum : uint8_t { kM = 0, kX = 1, kY = 2, kStop = 3 };

struct TraceArgs {
    const uint8_t* qc;
    const int64_t* qoff;
    const uint8_t* rc;
    const int64_t* roff;
    const int32_t* qi;
    const int32_t* ri;
    int64_t n;
    const int32_t* sim;
    int A;
    int local;
    int32_t go, ge;
    char letters[32];      // code -> symbol
    int64_t* rows;         // 3 * nmax1 * T
    int64_t nmax1;
    uint8_t* dirs;         // dir_cap bytes per thread
    int64_t dir_cap;
    int64_t* score_out;
    int32_t* start_out;
    char* qa_out;
    char* ra_out;
    char* ops_out;
    int64_t out_cap;       // bytes per pair slot (>= m + n)
};

__device__ __forceinline__ int64_t gap_run64(int64_t L, int32_t open, int32_t extend) {
    return L <= 0 ? 0 : int64_t(open) + (L - 1) * int64_t(extend);
}

__device__ __forceinline__ int64_t pick3(int64_t vm, int64_t vx, int64_t vy, uint8_t& who) {
    int64_t v = vm;
    who = kM;
    if (vx > v) {
        v = vx;
        who = kX;
    }
    if (vy > v) {
        v = vy;
        who = kY;
    }
    return v;
}

__global__ void __launch_bounds__(128) align_trace_kernel(const TraceArgs a) {
    extern __shared__ int32_t s_sim[];
    for (int i = threadIdx.x; i < a.A * a.A; i += blockDim.x) s_sim[i] = a.sim[i];
    __syncthreads();
    const int64_t T = int64_t(gridDim.x) * blockDim.x;
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int64_t* M = a.rows + tid;
    int64_t* X = M + a.nmax1 * T;
    int64_t* Y = X + a.nmax1 * T;
    uint8_t* dirs = a.dirs + tid * a.dir_cap;
    for (int64_t p = tid; p < a.n; p += T) {
        const int64_t qi = a.qi[p], ri = a.ri[p];
        const uint8_t* q = a.qc + a.qoff[qi];
        const uint8_t* r = a.rc + a.roff[ri];
        const int m = int(a.qoff[qi + 1] - a.qoff[qi]), n = int(a.roff[ri + 1] - a.roff[ri]);
        const bool local = a.local != 0;
        if (m == 0 || n == 0) {
            a.score_out[p] = local ? 0 : -gap_run64(m ? m : n, a.go, a.ge);
            a.start_out[p] = -1;
            continue;
        }
        const int W = n + 1;
        // row 0
        M[0] = 0;
        X[0] = kNeg;
        Y[0] = kNeg;
        dirs[0] = uint8_t(kStop | (kM << 2) | (kM << 4) | (1 << 6));
        for (int j = 1; j <= n; ++j) {
            M[j * T] = local ? 0 : kNeg;
            X[j * T] = kNeg;
            Y[j * T] = local ? kNeg : -gap_run64(j, a.go, a.ge);
            dirs[j] = uint8_t(kStop | (kM << 2) | ((j > 1 ? kY : kM) << 4) | ((local ? 1 : 0) << 6));
        }
        int64_t best = local ? 0 : kNeg;
        int bi = 0, bj = 0;
        int64_t lm = 0, lx = 0, ly = 0;
        for (int i = 1; i <= m; ++i) {
            int64_t dm = M[0], dx = X[0], dy = Y[0];
            lm = local ? 0 : kNeg;
            lx = local ? kNeg : -gap_run64(i, a.go, a.ge);
            ly = kNeg;
            M[0] = lm;
            X[0] = lx;
            Y[0] = ly;
            uint8_t* drow = dirs + int64_t(i) * W;
            drow[0] = uint8_t(kStop | ((i > 1 ? kX : kM) << 2) | (kM << 4) | ((local ? 1 : 0) << 6));
            const int32_t* srow = s_sim + int(q[i - 1]) * a.A;
            for (int j = 1; j <= n; ++j) {
                const int64_t um = M[j * T], ux = X[j * T], uy = Y[j * T];
                uint8_t wm, wx, wy;
                int64_t mv = pick3(dm, dx, dy, wm) + srow[r[j - 1]];
                if (local && mv < 0) {
                    mv = 0;
                    wm = kStop;
                }
                const int64_t xv = pick3(um - a.go, ux - a.ge, uy - a.go, wx);
                const int64_t yv = pick3(lm - a.go, lx - a.go, ly - a.ge, wy);
                M[j * T] = mv;
                X[j * T] = xv;
                Y[j * T] = yv;
                drow[j] = uint8_t(wm | (wx << 2) | (wy << 4) | ((mv == 0 ? 1 : 0) << 6));
                if (local && mv > best) {
                    best = mv;
                    bi = i;
                    bj = j;
                }
                dm = um;
                dx = ux;
                dy = uy;
                lm = mv;
                lx = xv;
                ly = yv;
            }
        }
        int i, j;
        uint8_t st;
        int64_t pos = a.out_cap;
        char* qa = a.qa_out + p * a.out_cap;
        char* ra = a.ra_out + p * a.out_cap;
        char* ops = a.ops_out + p * a.out_cap;
        if (local) {
            a.score_out[p] = best;
            i = bi;
            j = bj;
            st = kM;
            if (best == 0) {
                a.start_out[p] = int32_t(pos);
                continue;
            }
        } else {
            a.score_out[p] = pick3(lm, lx, ly, st);
            i = m;
            j = n;
        }
        while (i > 0 || j > 0) {
            const uint8_t d = dirs[int64_t(i) * W + j];
            if (st == kM) {
                if (i == 0 || j == 0) break;
                if (local && (d >> 6) & 1) break;
                const char ca = a.letters[q[i - 1]], cb = a.letters[r[j - 1]];
                --pos;
                qa[pos] = ca;
                ra[pos] = cb;
                ops[pos] = ca == cb ? 'M' : 'S';
                st = d & 3;
                --i;
                --j;
                if (st == kStop) break;
            } else if (st == kX) {
                if (i == 0) break;
                --pos;
                qa[pos] = a.letters[q[i - 1]];
                ra[pos] = '-';
                ops[pos] = 'D';
                st = (d >> 2) & 3;
                --i;
            } else {
                if (j == 0) break;
                --pos;
                qa[pos] = '-';
                ra[pos] = a.letters[r[j - 1]];
                ops[pos] = 'I';
                st = (d >> 4) & 3;
                --j;
            }
        }
        a.start_out[p] = int32_t(pos);
    }
}

// ------------------------------------------------------------------ penalty Gotoh (Index::align)
// seqtree's Index::align (src/index.cpp:105-179): global alignment minimising substitution
// penalties (the matrix's penalty grid, or unit cost on codec equality) plus affine gaps, in
// int32 with the reference's kInf = INT32_MAX / 4 borders.  The additions wrap as two's
// complement, which is what the reference's int32 code does for gap costs near 2^29.  Ties
// resolve as its best3(): M, then X only if strictly smaller, then Y only if strictly smaller.
constexpr int32_t kInf32 = INT32_MAX / 4;  // src/index.cpp:127

struct PenaltyArgs {
    const uint8_t* qc;
    const int64_t* qoff;
    const uint8_t* rc;
    const int64_t* roff;
    const int32_t* qi;
    const int32_t* ri;
    int64_t n;
    const int32_t* pen;    // A x A penalty grid; null: unit cost
    int A;
    int32_t go, ge;
    int32_t* rows;         // 3 * nmax1 * T
    int64_t nmax1;
    uint8_t* dirs;         // dir_cap bytes per thread
    int64_t dir_cap;
    int32_t* score_out;
    int32_t* start_out;    // first op in the slot; -2 when the walk left the matrix
    char* ops_out;
    int64_t out_cap;       // bytes per pair slot (>= m + n)
};

__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) {
    return int32_t(uint32_t(a) + uint32_t(b));
}
// go + (L - 1) * ge in wrapping int32 (src/index.cpp:135-136)
__device__ __forceinline__ int32_t gap_run32(int L, int32_t go, int32_t ge) {
    return int32_t(uint32_t(go) + uint32_t(L - 1) * uint32_t(ge));
}
__device__ __forceinline__ int32_t best3(int32_t vm, int32_t vx, int32_t vy, uint8_t& who) {
    int32_t v = vm;
    who = kM;
    if (vx < v) {
        v = vx;
        who = kX;
    }
    if (vy < v) {
        v = vy;
        who = kY;
    }
    return v;
}

__global__ void __launch_bounds__(128) penalty_trace_kernel(const PenaltyArgs a) {
    extern __shared__ int32_t s_pen[];
    if (a.pen)
        for (int i = threadIdx.x; i < a.A * a.A; i += blockDim.x) s_pen[i] = a.pen[i];
    __syncthreads();
    const int64_t T = int64_t(gridDim.x) * blockDim.x;
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int32_t* M = a.rows + tid;
    int32_t* X = M + a.nmax1 * T;
    int32_t* Y = X + a.nmax1 * T;
    uint8_t* dirs = a.dirs + tid * a.dir_cap;
    for (int64_t p = tid; p < a.n; p += T) {
        const int64_t qi = a.qi[p], ri = a.ri[p];
        const uint8_t* q = a.qc + a.qoff[qi];
        const uint8_t* r = a.rc + a.roff[ri];
        const int m = int(a.qoff[qi + 1] - a.qoff[qi]), n = int(a.roff[ri + 1] - a.roff[ri]);
        const int W = n + 1;
        // row 0: M[0][0] = 0, the gap-in-query border on Y, kInf elsewhere
        M[0] = 0;
        X[0] = kInf32;
        Y[0] = kInf32;
        dirs[0] = 0;
        for (int j = 1; j <= n; ++j) {
            M[j * T] = kInf32;
            X[j * T] = kInf32;
            Y[j * T] = gap_run32(j, a.go, a.ge);
            dirs[j] = uint8_t((j > 1 ? kY : kM) << 4);
        }
        for (int i = 1; i <= m; ++i) {
            int32_t dm = M[0], dx = X[0], dy = Y[0];
            int32_t lm = kInf32, lx = gap_run32(i, a.go, a.ge), ly = kInf32;
            M[0] = lm;
            X[0] = lx;
            Y[0] = ly;
            uint8_t* drow = dirs + int64_t(i) * W;
            drow[0] = uint8_t((i > 1 ? kX : kM) << 2);
            const uint8_t qcode = q[i - 1];
            const int32_t* prow = a.pen ? s_pen + int(qcode) * a.A : nullptr;
            for (int j = 1; j <= n; ++j) {
                const int32_t um = M[j * T], ux = X[j * T], uy = Y[j * T];
                const uint8_t rcode = r[j - 1];
                const int32_t sp = prow ? prow[rcode] : (qcode == rcode ? 0 : 1);
                uint8_t wm, wx, wy;
                const int32_t mv = wadd(sp, best3(dm, dx, dy, wm));
                const int32_t xv = best3(wadd(um, a.go), wadd(ux, a.ge), wadd(uy, a.go), wx);
                const int32_t yv = best3(wadd(lm, a.go), wadd(lx, a.go), wadd(ly, a.ge), wy);
                M[j * T] = mv;
                X[j * T] = xv;
                Y[j * T] = yv;
                drow[j] = uint8_t(wm | (wx << 2) | (wy << 4));
                dm = um;
                dx = ux;
                dy = uy;
                lm = mv;
                lx = xv;
                ly = yv;
            }
        }
        uint8_t st;
        a.score_out[p] = best3(M[int64_t(n) * T], X[int64_t(n) * T], Y[int64_t(n) * T], st);
        int i = m, j = n;
        int64_t pos = a.out_cap;
        char* ops = a.ops_out + p * a.out_cap;
        bool left = false;
        while (i > 0 || j > 0) {
            const uint8_t d = dirs[int64_t(i) * W + j];
            if (st == kM) {
                if (i == 0 || j == 0) {
                    left = true;
                    break;
                }
                ops[--pos] = q[i - 1] == r[j - 1] ? 'M' : 'S';
                st = d & 3;
                --i;
                --j;
            } else if (st == kX) {
                if (i == 0) {
                    left = true;
                    break;
                }
                ops[--pos] = 'D';
                st = (d >> 2) & 3;
                --i;
            } else {
                if (j == 0) {
                    left = true;
                    break;
                }
                ops[--pos] = 'I';
                st = (d >> 4) & 3;
                --j;
            }
        }
        a.start_out[p] = left ? -2 : int32_t(pos);
    }
}

const char* symbol_string(int32_t alphabet) {  // src/codec.cpp:9-11
    switch (alphabet) {
        case ST_ALPHABET_AA: return "ARNDCQEGHILKMFPSTWYVBZX*";
        case ST_ALPHABET_NT: return "ACGT";
        default: return "ACGTRYSWKMBDHVN";
    }
}

}  // namespace

// Alignments of the listed pairs; outputs in device memory (scores int64, narrowed by the caller).
void align_pairs_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* qi_d, const int32_t* ri_d,
                      int64_t n, const int32_t* similarity, int32_t matrix_size, int32_t mode,
                      int32_t go, int32_t ge, int64_t* score_d, int32_t* start_d, char* qa_d,
                      char* ra_d, char* ops_d, int64_t out_cap, cudaStream_t stream) {
    if (go < 0 || ge < 0)
        fail(ST_EINVAL, "seqtree: gap_open and gap_extend must be >= 0 (they are magnitudes, and "
                        "are subtracted)");
    if (qs.alphabet < 0 || qs.alphabet != rs.alphabet)
        fail(ST_EINVAL, "seqtree_b200: alignment sets must be encoded with one alphabet");
    const int A = alphabet_size(qs.alphabet);
    if (!similarity || matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
    if (mode != ST_MODE_GLOBAL && mode != ST_MODE_LOCAL)
        fail(ST_EINVAL, "unknown mode (use 'global' or 'local')");
    if (n < 0) fail(ST_EINVAL, "seqtree_b200: negative pair count");
    if (out_cap < int64_t(qs.max_len) + rs.max_len)
        fail(ST_EINVAL, "seqtree_b200: output slots shorter than the longest query + ref");
    if (n == 0) return;
    Context& ctx = context();
    int32_t* d_sim = ctx.table_buf.as<int32_t>(size_t(A) * A);
    h2d(d_sim, similarity, size_t(A) * A * 4, stream);
    TraceArgs a{};
    a.qc = qs.d_bytes;
    a.qoff = qs.d_off;
    a.rc = rs.d_bytes;
    a.roff = rs.d_off;
    a.qi = qi_d;
    a.ri = ri_d;
    a.n = n;
    a.sim = d_sim;
    a.A = A;
    a.local = mode == ST_MODE_LOCAL;
    a.go = go;
    a.ge = ge;
    std::memcpy(a.letters, symbol_string(qs.alphabet), size_t(A));
    a.nmax1 = int64_t(rs.max_len) + 1;
    a.dir_cap = (int64_t(qs.max_len) + 1) * a.nmax1;
    const int64_t per = 3 * a.nmax1 * 8 + a.dir_cap;
    int64_t T = std::min<int64_t>(int64_t(ctx.num_sms) * 1024, n);
    T = std::min<int64_t>(T, std::max<int64_t>(128, (int64_t(1) << 30) / per));
    T = ceil_div(T, 128) * 128;
    a.rows = ctx.work_a.as<int64_t>(size_t(3 * a.nmax1 * T));
    a.dirs = ctx.work_c.as<uint8_t>(size_t(a.dir_cap * T));
    a.score_out = score_d;
    a.start_out = start_d;
    a.qa_out = qa_d;
    a.ra_out = ra_d;
    a.ops_out = ops_d;
    a.out_cap = out_cap;
    align_trace_kernel<<<unsigned(T / 128), 128, size_t(A) * A * 4, stream>>>(a);
    STB_CUDA(cudaGetLastError());
    note_launch("align_trace_kernel");
}

// Index::align of the listed pairs (penalty grid `penalty` of `matrix_size`^2 entries, or unit
// cost when null); scores, op-slot starts and ops in device memory.
void penalty_align_pairs_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* qi_d,
                              const int32_t* ri_d, int64_t n, const int32_t* penalty,
                              int32_t matrix_size, int32_t go, int32_t ge, int32_t* score_d,
                              int32_t* start_d, char* ops_d, int64_t out_cap, cudaStream_t stream) {
    if (qs.alphabet < 0 || qs.alphabet != rs.alphabet)
        fail(ST_EINVAL, "seqtree_b200: alignment sets must be encoded with one alphabet");
    const int A = alphabet_size(qs.alphabet);
    if (penalty && matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
    if (go < 0 || ge < 0) fail(ST_EINVAL, "seqtree: gap_open and gap_extend must be >= 0");
    if (n < 0) fail(ST_EINVAL, "seqtree_b200: negative pair count");
    if (out_cap < int64_t(qs.max_len) + rs.max_len)
        fail(ST_EINVAL, "seqtree_b200: output slots shorter than the longest query + ref");
    if (n == 0) return;
    Context& ctx = context();
    int32_t* d_pen = nullptr;
    if (penalty) {
        d_pen = ctx.table_buf.as<int32_t>(size_t(A) * A);
        h2d(d_pen, penalty, size_t(A) * A * 4, stream);
    }
    PenaltyArgs a{};
    a.qc = qs.d_bytes;
    a.qoff = qs.d_off;
    a.rc = rs.d_bytes;
    a.roff = rs.d_off;
    a.qi = qi_d;
    a.ri = ri_d;
    a.n = n;
    a.pen = d_pen;
    a.A = A;
    a.go = go;
    a.ge = ge;
    a.nmax1 = int64_t(rs.max_len) + 1;
    a.dir_cap = (int64_t(qs.max_len) + 1) * a.nmax1;
    const int64_t per = 3 * a.nmax1 * 4 + a.dir_cap;
    int64_t T = std::min<int64_t>(int64_t(ctx.num_sms) * 1024, n);
    T = std::min<int64_t>(T, std::max<int64_t>(128, (int64_t(1) << 30) / per));
    T = ceil_div(T, 128) * 128;
    a.rows = ctx.work_a.as<int32_t>(size_t(3 * a.nmax1 * T));
    a.dirs = ctx.work_c.as<uint8_t>(size_t(a.dir_cap * T));
    a.score_out = score_d;
    a.start_out = start_d;
    a.ops_out = ops_d;
    a.out_cap = out_cap;
    penalty_trace_kernel<<<unsigned(T / 128), 128, penalty ? size_t(A) * A * 4 : 0, stream>>>(a);
    STB_CUDA(cudaGetLastError());
    note_launch("penalty_trace_kernel");
}

}  // namespace stb
