// extern "C" entry points of libseqtree_b200 (declared in include/seqtree_b200.h).
//
// Host-buffer calls follow the reference's validation order exactly, so the same bad input
// fails with the same message: gap costs, alphabet, matrix size, empty shapes (no further
// checks, as in the reference), symbol encoding (queries before refs), then per-family checks.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace stb {
void gapblock_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* penalty, int32_t matrix_size,
                   int32_t go, int32_t ge, const int32_t* prior, int64_t prior_len,
                   uint32_t prior_width, int32_t* out_d, cudaStream_t stream);
void gapblock_sparse_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* penalty,
                          int32_t matrix_size, int32_t go, int32_t ge, const int32_t* prior,
                          int64_t prior_len, uint32_t prior_width, int32_t max_penalty,
                          st_hits_s& hits, cudaStream_t stream);
void align_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* similarity, int32_t matrix_size,
                int32_t mode, int32_t go, int32_t ge, int32_t dist, int32_t* out_d,
                cudaStream_t stream);
void hamming_sets(st_seqset_s& a, st_seqset_s& b, int32_t* out_d, cudaStream_t stream);
void levenshtein_sets(st_seqset_s& a, st_seqset_s& b, int32_t* out_d, cudaStream_t stream,
                      int64_t r0 = 0, int64_t r1 = -1);
void gapblock_pairs_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* qi_d, const int32_t* ri_d,
                         int64_t n, const int32_t* penalty, int32_t matrix_size, int32_t go,
                         int32_t ge, const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                         int32_t* out_d, int32_t* pos_d, cudaStream_t stream);
struct Encoder;
int64_t encoder_param_count();
Encoder* encoder_create(const float* params);
void encoder_destroy(Encoder* m);
void encoder_params(Encoder& m, float* out);
void encoder_set_precision(Encoder& m, int precision);
void gemm_bf16(bool ta, bool tb, int M, int N, int K, const float* A, int lda, const float* B,
               int ldb, float* C, int ldc, bool accumulate, cudaStream_t st, int sms);
float encoder_loss_grad(Encoder& m, const uint8_t* codes, const int32_t* lens, const int32_t* scores,
                        int S, float* grad_out);
float encoder_train_step(Encoder& m, const uint8_t* codes, const int32_t* lens, const int32_t* scores,
                         int S, float lr);
void encoder_embed(Encoder& m, const st_seqset_s& set, void* out, int layout, cudaStream_t st);
void propose_topk(const void* qemb, int64_t nq, const void* remb, int64_t nr, int k, int32_t* ids,
                  float* scores, cudaStream_t stream,
                  const int32_t* ranges = nullptr);
int64_t propose_range(const void* qemb, int64_t nq, const uint8_t* qlens, const void* remb,
                      int64_t nr, const uint8_t* rlens, const float* thr, int32_t* pq, int32_t* pr,
                      int64_t cap, cudaStream_t stream, const int32_t* ranges);
void embed_dots(const void* qemb, int64_t nq, const void* remb, int64_t nr, const int32_t* qi,
                const int32_t* ri, int64_t n, float* out, cudaStream_t stream);
void profile_scores(const int32_t* table, int32_t width, int32_t c, uint8_t gap, int32_t unreachable,
                    const st_seqset_s& set, int32_t* out_d, cudaStream_t stream);
void align_pairs_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* qi_d, const int32_t* ri_d,
                      int64_t n, const int32_t* similarity, int32_t matrix_size, int32_t mode,
                      int32_t go, int32_t ge, int64_t* score_d, int32_t* start_d, char* qa_d,
                      char* ra_d, char* ops_d, int64_t out_cap, cudaStream_t stream);
void penalty_align_pairs_sets(st_seqset_s& qs, st_seqset_s& rs, const int32_t* qi_d,
                              const int32_t* ri_d, int64_t n, const int32_t* penalty,
                              int32_t matrix_size, int32_t go, int32_t ge, int32_t* score_d,
                              int32_t* start_d, char* ops_d, int64_t out_cap, cudaStream_t stream);
void thetas_csr(const int64_t* indptr_d, const int32_t* scores_d, int64_t rows, int32_t k, int rule3,
                int32_t theta_max, int exclude_exact, int32_t* out_d, cudaStream_t stream);
int last_launches();
int64_t total_launches();
std::string tuning_table();
const char* last_kernel();
void* host_alloc(uint64_t bytes);
void host_free(void* p);
}  // namespace stb

using namespace stb;

namespace {

template <class F>
int32_t guard(st_error* err, F&& f) {
    try {
        f();
        if (err) {
            err->code = ST_OK;
            err->message[0] = 0;
        }
        return ST_OK;
    } catch (const StError& e) {
        if (err) {
            err->code = e.code;
            std::snprintf(err->message, sizeof err->message, "%s", e.what());
        }
        return e.code;
    } catch (const std::bad_alloc&) {
        if (err) {
            err->code = ST_ENOMEM;
            std::snprintf(err->message, sizeof err->message, "seqtree_b200: out of host memory");
        }
        return ST_ENOMEM;
    } catch (const std::exception& e) {
        if (err) {
            err->code = ST_ECUDA;
            std::snprintf(err->message, sizeof err->message, "%s", e.what());
        }
        return ST_ECUDA;
    }
}

int64_t count_of(const st_strings* s) { return s ? s->count : 0; }

void check_strings(const st_strings* s) {
    if (!s) fail(ST_EINVAL, "seqtree_b200: null st_strings");
    if (s->count < 0) fail(ST_EINVAL, "seqtree_b200: negative sequence count");
    if (s->count > 0 && !s->offsets) fail(ST_EINVAL, "seqtree_b200: null offsets");
}

// Transient device sets for one host call: storage borrowed from the context.
struct Transient {
    std::unique_ptr<st_seqset_s> q, r;
};

// Device -> host copy of the N*K result, then the error words written by the kernels.
void finish(Context& ctx, int32_t* out, int64_t N, int64_t K, int32_t* out_d) {
    const size_t bytes = size_t(N) * size_t(K) * sizeof(int32_t);
    STB_CUDA(cudaMemcpyAsync(out, out_d, bytes, cudaMemcpyDeviceToHost, ctx.stream));
    STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, 8 * sizeof(int64_t),
                             cudaMemcpyDeviceToHost, ctx.stream));
    STB_CUDA(cudaStreamSynchronize(ctx.stream));
}

// The result copy overlapped with the computation: `launch(r0, r1)` enqueues the kernels of rows
// [r0, r1) on the context's stream, and each block of rows is copied to `out` on a second stream
// as soon as its kernels are done, so the copy of one block runs beside the next block's
// kernels.  (With a pageable `out` the copies are synchronous and nothing overlaps.)
void finish_pipelined(Context& ctx, int32_t* out, int64_t N, int64_t K, int32_t* out_d,
                      int blocks, const std::function<void(int64_t, int64_t)>& launch) {
    constexpr int kMaxBlocks = 8;
    blocks = int(std::max<int64_t>(1, std::min<int64_t>({int64_t(blocks), int64_t(kMaxBlocks), N})));
    if (!ctx.copy_stream) {
        STB_CUDA(cudaStreamCreateWithFlags(&ctx.copy_stream, cudaStreamNonBlocking));
        for (int b = 0; b < kMaxBlocks; ++b)
            STB_CUDA(cudaEventCreateWithFlags(&ctx.block_ev[b], cudaEventDisableTiming));
    }
    for (int b = 0; b < blocks; ++b) {
        const int64_t r0 = N * b / blocks, r1 = N * (b + 1) / blocks;
        launch(r0, r1);
        STB_CUDA(cudaEventRecord(ctx.block_ev[b], ctx.stream));
        STB_CUDA(cudaStreamWaitEvent(ctx.copy_stream, ctx.block_ev[b], 0));
        STB_CUDA(cudaMemcpyAsync(out + r0 * K, out_d + r0 * K, size_t(r1 - r0) * size_t(K) * 4,
                                 cudaMemcpyDeviceToHost, ctx.copy_stream));
    }
    STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, 8 * sizeof(int64_t),
                             cudaMemcpyDeviceToHost, ctx.stream));
    STB_CUDA(cudaStreamSynchronize(ctx.stream));
    STB_CUDA(cudaStreamSynchronize(ctx.copy_stream));
}

void check_timeout(Context& ctx) {
    if (ctx.flags_h[8] != 0)
        fail(ST_ETIMEOUT, "seqtree_b200: a bounded device-side wait gave up (shared-memory staging)");
}

void clear_flags(Context& ctx) {
    STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, 8 * sizeof(int64_t), ctx.stream));
}

}  // namespace

extern "C" {

int32_t st_version(void) { return 100; }

int32_t st_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

namespace {
#include "builtin_tables.inc"
}  // namespace

int32_t st_builtin_similarity(const char* name, int32_t* out, int32_t capacity, int32_t* size,
                              st_error* err) {
    return guard(err, [&] {
        if (!name) fail(ST_EINVAL, "matrix name is NULL");
        for (size_t m = 0; m < sizeof(kBuiltinNames) / sizeof(kBuiltinNames[0]); ++m) {
            if (std::strcmp(name, kBuiltinNames[m]) != 0) continue;
            if (size) *size = 24;
            if (out) {
                if (capacity < 24 * 24) fail(ST_EINVAL, "output holds fewer than 576 entries");
                std::memcpy(out, kBuiltinSimilarity[m], sizeof(kBuiltinSimilarity[m]));
            }
            return;
        }
        fail(ST_EINVAL, std::string("unknown built-in matrix '") + name + "'");
    });
}

int32_t st_last_launch_count(void) { return last_launches(); }

int64_t st_total_launch_count(void) { return total_launches(); }

int64_t st_tuning_table(char* buf, int64_t capacity) {
    const std::string t = tuning_table();
    if (buf && capacity > 0) {
        const size_t n = std::min<size_t>(t.size(), size_t(capacity - 1));
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    }
    return int64_t(t.size());
}
const char* st_last_kernel_name(void) { return last_kernel(); }

void* st_host_alloc(uint64_t bytes) { return host_alloc(bytes); }
void st_host_free(void* ptr) { host_free(ptr); }

int64_t st_split_joined(const uint8_t* joined, int64_t size, int64_t count, uint8_t* data_out,
                        int64_t* offsets_out) {
    if (count <= 0 || size < count - 1 || !joined || !data_out || !offsets_out) return -1;
    const uint8_t* p = joined;
    const uint8_t* end = joined + size;
    int64_t w = 0;
    offsets_out[0] = 0;
    for (int64_t i = 0; i < count; ++i) {
        const uint8_t* nl =
            static_cast<const uint8_t*>(std::memchr(p, '\n', size_t(end - p)));
        const uint8_t* stop = nl ? nl : end;
        if ((i + 1 < count) != (nl != nullptr)) return -1;  // separator count != count - 1
        std::memcpy(data_out + w, p, size_t(stop - p));
        w += stop - p;
        offsets_out[i + 1] = w;
        p = nl ? nl + 1 : end;
    }
    return w;
}

int32_t st_gapblock_matrix(const st_strings* queries, const st_strings* refs, int32_t alphabet,
                           const int32_t* penalty, int32_t matrix_size, int32_t gap_open,
                           int32_t gap_extend, const int32_t* prior, int64_t prior_len,
                           uint32_t prior_width, int32_t threads, int32_t* out, st_error* err) {
    (void)threads;
    return guard(err, [&] {
        reset_launches();
        check_strings(queries);
        check_strings(refs);
        // src/gapblock.cpp:71-81
        if (gap_open < 0 || gap_extend < 0) fail(ST_EINVAL, "gap_open and gap_extend must be >= 0");
        const int A = alphabet_size(alphabet);
        if (A == 0) fail(ST_EINVAL, "unknown alphabet code " + std::to_string(alphabet));
        if (penalty && matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
        const int64_t N = count_of(queries), K = count_of(refs);
        if (N == 0 || K == 0) return;
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output buffer");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        clear_flags(ctx);
        // src/gapblock.cpp:85-94: queries are encoded before refs.  The symbol check is
        // deferred to the call's one synchronisation (words 0 and 1 of the flag area: the first
        // invalid byte of the queries, of the refs); invalid symbols compute as code 0 meanwhile
        // and the call then fails with the reference's message, queries first, as the reference
        // does.  `out` is unspecified after a failed call.
        Transient t;
        {
            Phase ph("upload+encode");
            STB_CUDA(cudaMemsetAsync(ctx.flags_d, 0xFF, 2 * sizeof(int64_t), ctx.stream));
            t.q.reset(make_seqset(queries, alphabet, ctx.stream, nullptr, nullptr, ctx.tq, 0));
            t.r.reset(make_seqset(refs, alphabet, ctx.stream, nullptr, nullptr, ctx.tr, 1));
        }
        auto check_symbols = [&] {
            for (int w = 0; w < 2; ++w) {
                const uint64_t bad = static_cast<uint64_t>(ctx.flags_h[w]);
                if (bad != ~uint64_t(0)) {
                    const st_strings* s = w == 0 ? queries : refs;
                    const char c =
                        reinterpret_cast<const char*>(s->bytes)[s->offsets[0] + int64_t(bad)];
                    fail(ST_EINVAL, std::string("symbol '") + c + "' is not in the alphabet");
                }
            }
        };
        int32_t* out_d = ctx.out_buf.as<int32_t>(size_t(N) * size_t(K));
        {
            Phase ph("plan+launch");
            try {
                gapblock_sets(*t.q, *t.r, penalty, matrix_size, gap_open, gap_extend, prior,
                              prior_len, prior_width, out_d, ctx.stream);
            } catch (...) {
                // the reference reports an invalid symbol before the prior-table errors that
                // planning finds (src/gapblock.cpp:85-102)
                STB_CUDA(cudaMemcpyAsync(ctx.flags_h, ctx.flags_d, 2 * sizeof(int64_t),
                                         cudaMemcpyDeviceToHost, ctx.stream));
                STB_CUDA(cudaStreamSynchronize(ctx.stream));
                check_symbols();
                throw;
            }
        }
        {
            Phase ph("kernel+d2h");
            STB_CUDA(cudaMemcpyAsync(ctx.flags_h, ctx.flags_d, 2 * sizeof(int64_t),
                                     cudaMemcpyDeviceToHost, ctx.stream));
            finish(ctx, out, N, K, out_d);
        }
        check_symbols();
        check_timeout(ctx);
        trace_report("st_gapblock_matrix");
    });
}

int32_t st_gapblock_sparse(const st_strings* queries, const st_strings* refs, int32_t alphabet,
                           const int32_t* penalty, int32_t matrix_size, int32_t gap_open,
                           int32_t gap_extend, const int32_t* prior, int64_t prior_len,
                           uint32_t prior_width, int32_t max_penalty, int32_t threads,
                           st_sparse* out, st_error* err) {
    (void)threads;
    return guard(err, [&] {
        reset_launches();
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output");
        *out = st_sparse{};
        check_strings(queries);
        check_strings(refs);
        if (max_penalty < 0) fail(ST_EINVAL, "max_penalty must be >= 0");
        // the dense call's checks, in its order (src/gapblock.cpp:71-81)
        if (gap_open < 0 || gap_extend < 0) fail(ST_EINVAL, "gap_open and gap_extend must be >= 0");
        const int A = alphabet_size(alphabet);
        if (A == 0) fail(ST_EINVAL, "unknown alphabet code " + std::to_string(alphabet));
        if (penalty && matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
        const int64_t N = count_of(queries), K = count_of(refs);
        st_sparse res{};
        res.rows = N;
        res.cols = K;
        auto release = [&res] {
            host_free(res.indptr);
            host_free(res.ref_ids);
            host_free(res.scores);
        };
        res.indptr = static_cast<int64_t*>(host_alloc(sizeof(int64_t) * size_t(N + 1)));
        if (!res.indptr) fail(ST_ENOMEM, "seqtree_b200: pinned host allocation failed");
        if (N == 0 || K == 0) {
            std::memset(res.indptr, 0, sizeof(int64_t) * size_t(N + 1));
            *out = res;
            return;
        }
        try {
            Context& ctx = context();
            std::lock_guard<std::mutex> lk(ctx.mu);
            clear_flags(ctx);
            Transient t;
            {
                Phase ph("upload+encode");
                t.q.reset(make_seqset(queries, alphabet, ctx.stream, nullptr, nullptr, ctx.tq));
                t.r.reset(make_seqset(refs, alphabet, ctx.stream, nullptr, nullptr, ctx.tr));
            }
            if (!ctx.tmp_hits) ctx.tmp_hits = std::make_shared<st_hits_s>();
            st_hits_s& h = *static_cast<st_hits_s*>(ctx.tmp_hits.get());
            {
                Phase ph("kernel+sort");
                gapblock_sparse_sets(*t.q, *t.r, penalty, matrix_size, gap_open, gap_extend, prior,
                                     prior_len, prior_width, max_penalty, h, ctx.stream);
            }
            Phase ph("d2h");
            res.nnz = h.nnz;
            const size_t nb = size_t(std::max<int64_t>(h.nnz, 1));
            res.ref_ids = static_cast<int32_t*>(host_alloc(sizeof(int32_t) * nb));
            res.scores = static_cast<int32_t*>(host_alloc(sizeof(int32_t) * nb));
            if (!res.ref_ids || !res.scores)
                fail(ST_ENOMEM, "seqtree_b200: pinned host allocation failed");
            STB_CUDA(cudaMemcpyAsync(res.indptr, h.indptr.ptr, sizeof(int64_t) * size_t(N + 1),
                                     cudaMemcpyDeviceToHost, ctx.stream));
            if (h.nnz > 0) {
                STB_CUDA(cudaMemcpyAsync(res.ref_ids, h.ref_ids.ptr, sizeof(int32_t) * size_t(h.nnz),
                                         cudaMemcpyDeviceToHost, ctx.stream));
                STB_CUDA(cudaMemcpyAsync(res.scores, h.scores.ptr, sizeof(int32_t) * size_t(h.nnz),
                                         cudaMemcpyDeviceToHost, ctx.stream));
            }
            STB_CUDA(cudaStreamSynchronize(ctx.stream));
        } catch (...) {
            release();
            throw;
        }
        *out = res;
        trace_report("st_gapblock_sparse");
    });
}

void st_sparse_free(st_sparse* s) {
    if (!s) return;
    host_free(s->indptr);
    host_free(s->ref_ids);
    host_free(s->scores);
    *s = st_sparse{};
}

static int32_t align_common(const st_strings* queries, const st_strings* refs,
                            const int32_t* similarity, int32_t matrix_size, int32_t alphabet,
                            int32_t mode, int32_t gap_open, int32_t gap_extend, int32_t dist,
                            int32_t* out, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_strings(queries);
        check_strings(refs);
        // src/pairwise.cpp:62-68 (check), then the empty shortcut (:281-282), then encoding.
        if (gap_open < 0 || gap_extend < 0)
            fail(ST_EINVAL, "seqtree: gap_open and gap_extend must be >= 0 (they are magnitudes, "
                            "and are subtracted)");
        const int A = alphabet_size(alphabet);
        if (A == 0) fail(ST_EINVAL, "unknown alphabet code " + std::to_string(alphabet));
        if (!similarity || matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
        if (mode != ST_MODE_GLOBAL && mode != ST_MODE_LOCAL)
            fail(ST_EINVAL, "unknown mode (use 'global' or 'local')");
        const int64_t N = count_of(queries), K = count_of(refs);
        if (N == 0 || K == 0) return;
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output buffer");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        clear_flags(ctx);
        Transient t;
        int64_t bad = -1;
        char bc = 0;
        t.q.reset(make_seqset(queries, alphabet, ctx.stream, &bad, &bc, ctx.tq));
        if (bad >= 0) fail(ST_EINVAL, std::string("invalid symbol '") + bc + "' in sequence");
        t.r.reset(make_seqset(refs, alphabet, ctx.stream, &bad, &bc, ctx.tr));
        if (bad >= 0) fail(ST_EINVAL, std::string("invalid symbol '") + bc + "' in sequence");
        int32_t* out_d = ctx.out_buf.as<int32_t>(size_t(N) * size_t(K));
        {
            Phase ph("plan+launch");
            align_sets(*t.q, *t.r, similarity, matrix_size, mode, gap_open, gap_extend, dist, out_d,
                       ctx.stream);
        }
        {
            Phase ph("kernel+d2h");
            finish(ctx, out, N, K, out_d);
        }
        trace_report(dist ? "st_align_dist_matrix" : "st_align_score_matrix");
        check_timeout(ctx);
        if (ctx.flags_h[9] != 0)
            fail(ST_EOVERFLOW, std::string("seqtree: the alignment ") + (dist ? "distance" : "score") +
                                   " does not fit in 32 bits -- the gap costs are absurdly large "
                                   "for these sequences");
    });
}

int32_t st_align_pair(const char* query, int64_t query_len, const char* ref, int64_t ref_len,
                      const int32_t* similarity, int32_t matrix_size, int32_t alphabet, int32_t mode,
                      int32_t gap_open, int32_t gap_extend, int32_t* score, char* aligned_query,
                      char* aligned_ref, char* ops, int64_t capacity, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        // src/pairwise.cpp:141-146: check(), then encode the query, then the ref.
        if (gap_open < 0 || gap_extend < 0)
            fail(ST_EINVAL, "seqtree: gap_open and gap_extend must be >= 0 (they are magnitudes, "
                            "and are subtracted)");
        const int A = alphabet_size(alphabet);
        if (A == 0) fail(ST_EINVAL, "unknown alphabet code " + std::to_string(alphabet));
        if (!similarity || matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
        if (mode != ST_MODE_GLOBAL && mode != ST_MODE_LOCAL)
            fail(ST_EINVAL, "unknown mode (use 'global' or 'local')");
        if (query_len < 0 || ref_len < 0 || (query_len && !query) || (ref_len && !ref))
            fail(ST_EINVAL, "seqtree_b200: bad sequence buffer");
        if (!score || !aligned_query || !aligned_ref || !ops || capacity < query_len + ref_len + 1)
            fail(ST_EINVAL, "seqtree_b200: output buffers need query_len + ref_len + 1 bytes");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        const int64_t qo[2] = {0, query_len}, ro[2] = {0, ref_len};
        const st_strings qs{query, qo, 1}, rs{ref, ro, 1};
        Transient t;
        int64_t bad = -1;
        char bc = 0;
        t.q.reset(make_seqset(&qs, alphabet, ctx.stream, &bad, &bc, ctx.tq));
        if (bad >= 0) fail(ST_EINVAL, std::string("invalid symbol '") + bc + "' in sequence");
        t.r.reset(make_seqset(&rs, alphabet, ctx.stream, &bad, &bc, ctx.tr));
        if (bad >= 0) fail(ST_EINVAL, std::string("invalid symbol '") + bc + "' in sequence");
        const int64_t slot = std::max<int64_t>(query_len + ref_len, 1);
        // device scratch: pair indices, score, start, three string slots
        auto* base = static_cast<uint8_t*>(ctx.work_b.get(size_t(64 + 3 * slot)));
        auto* idx = reinterpret_cast<int32_t*>(base);
        auto* sc = reinterpret_cast<int64_t*>(base + 16);
        auto* st = reinterpret_cast<int32_t*>(base + 24);
        char* strs = reinterpret_cast<char*>(base + 64);
        STB_CUDA(cudaMemsetAsync(idx, 0, 8, ctx.stream));
        align_pairs_sets(*t.q, *t.r, idx, idx + 1, 1, similarity, matrix_size, mode, gap_open,
                         gap_extend, sc, st, strs, strs + slot, strs + 2 * slot, slot, ctx.stream);
        std::vector<uint8_t> host(size_t(64 + 3 * slot));
        STB_CUDA(cudaMemcpyAsync(host.data(), base, host.size(), cudaMemcpyDeviceToHost, ctx.stream));
        STB_CUDA(cudaStreamSynchronize(ctx.stream));
        int64_t s64;
        int32_t start;
        std::memcpy(&s64, host.data() + 16, 8);
        std::memcpy(&start, host.data() + 24, 4);
        if (s64 > INT32_MAX || s64 < INT32_MIN)
            fail(ST_EOVERFLOW, "seqtree: the alignment score does not fit in 32 bits -- the gap "
                               "costs are absurdly large for these sequences");
        *score = int32_t(s64);
        std::string aq, ar, op;
        if (start < 0) {  // an empty side: raw input in global mode, nothing in local mode
            if (mode == ST_MODE_GLOBAL) {
                aq = std::string(query ? query : "", size_t(query_len)) + std::string(size_t(ref_len), '-');
                ar = std::string(size_t(query_len), '-') + std::string(ref ? ref : "", size_t(ref_len));
                op = std::string(size_t(query_len), 'D') + std::string(size_t(ref_len), 'I');
            }
        } else {
            const char* h = reinterpret_cast<const char*>(host.data() + 64);
            aq.assign(h + start, size_t(slot - start));
            ar.assign(h + slot + start, size_t(slot - start));
            op.assign(h + 2 * slot + start, size_t(slot - start));
        }
        std::memcpy(aligned_query, aq.c_str(), aq.size() + 1);
        std::memcpy(aligned_ref, ar.c_str(), ar.size() + 1);
        std::memcpy(ops, op.c_str(), op.size() + 1);
    });
}

int32_t st_penalty_align_pairs(const st_strings* queries, const st_strings* refs,
                               const int32_t* query_idx, const int32_t* ref_idx, int64_t n,
                               int32_t alphabet, const int32_t* penalty, int32_t matrix_size,
                               int32_t gap_open, int32_t gap_extend, int32_t* scores,
                               char* aligned_query, char* aligned_ref, char* ops, int64_t stride,
                               int32_t* lengths, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_strings(queries);
        check_strings(refs);
        const int A = alphabet_size(alphabet);
        if (A == 0) fail(ST_EINVAL, "unknown alphabet code " + std::to_string(alphabet));
        if (n < 0) fail(ST_EINVAL, "seqtree_b200: negative pair count");
        if (n > 0 && (!query_idx || !ref_idx || !scores || !lengths))
            fail(ST_EINVAL, "seqtree_b200: null pair list or output");
        const int64_t N = count_of(queries), K = count_of(refs);
        int64_t mq = 0, mr = 0;
        for (int64_t i = 0; i < N; ++i) mq = std::max(mq, queries->offsets[i + 1] - queries->offsets[i]);
        for (int64_t i = 0; i < K; ++i) mr = std::max(mr, refs->offsets[i + 1] - refs->offsets[i]);
        const bool strings = aligned_query || aligned_ref || ops;
        if (strings && (!aligned_query || !aligned_ref || !ops))
            fail(ST_EINVAL, "seqtree_b200: give all three string outputs or none");
        if (strings && stride < mq + mr + 1)
            fail(ST_EINVAL, "seqtree_b200: string stride shorter than the longest query + ref + 1");
        for (int64_t p = 0; p < n; ++p)
            if (query_idx[p] < 0 || query_idx[p] >= N || ref_idx[p] < 0 || ref_idx[p] >= K)
                fail(ST_EINVAL, "seqtree_b200: pair index out of range");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        clear_flags(ctx);
        // Order of the reference's checks: the refs at Index::build (src/trie.cpp:62-66), the
        // matrix against the alphabet (src/_bindings.cpp:90-95), then, in Index::align, the
        // query's symbols and the gap costs (src/index.cpp:109-114).
        Transient t;
        int64_t bad = -1;
        char bc = 0;
        t.r.reset(make_seqset(refs, alphabet, ctx.stream, &bad, &bc, ctx.tr));
        if (bad >= 0) {
            const auto& off = t.r->h_off;
            const int64_t id = int64_t(std::upper_bound(off.begin(), off.end(), bad) - off.begin()) - 1;
            fail(ST_EINVAL, std::string("invalid symbol '") + bc + "' in reference #" +
                                std::to_string(id));
        }
        if (penalty && matrix_size != A) fail(ST_EINVAL, "matrix size does not match the alphabet");
        t.q.reset(make_seqset(queries, alphabet, ctx.stream, &bad, &bc, ctx.tq));
        if (bad >= 0) fail(ST_EINVAL, std::string("invalid symbol '") + bc + "' in query");
        if (gap_open < 0 || gap_extend < 0)
            fail(ST_EINVAL, "seqtree: gap_open and gap_extend must be >= 0");
        if (n == 0) return;
        const int64_t slot = std::max<int64_t>(mq + mr, 1);
        // device: pair indices, scores, starts, op slots
        const size_t idx_b = size_t(n) * 8, sc_b = size_t(n) * 4, st_b = size_t(n) * 4;
        auto* base = static_cast<uint8_t*>(ctx.work_b.get(idx_b + sc_b + st_b + size_t(n * slot) + 64));
        auto* qi_d = reinterpret_cast<int32_t*>(base);
        auto* ri_d = qi_d + n;
        auto* sc_d = reinterpret_cast<int32_t*>(base + idx_b);
        auto* st_d = reinterpret_cast<int32_t*>(base + idx_b + sc_b);
        char* ops_d = reinterpret_cast<char*>(base + idx_b + sc_b + st_b);
        h2d(qi_d, query_idx, size_t(n) * 4, ctx.stream);
        h2d(ri_d, ref_idx, size_t(n) * 4, ctx.stream);
        penalty_align_pairs_sets(*t.q, *t.r, qi_d, ri_d, n, penalty, matrix_size, gap_open,
                                 gap_extend, sc_d, st_d, ops_d, slot, ctx.stream);
        std::vector<int32_t> starts(static_cast<size_t>(n));
        std::vector<char> opsh(strings ? static_cast<size_t>(n * slot) : 0);
        STB_CUDA(cudaMemcpyAsync(scores, sc_d, sc_b, cudaMemcpyDeviceToHost, ctx.stream));
        STB_CUDA(cudaMemcpyAsync(starts.data(), st_d, st_b, cudaMemcpyDeviceToHost, ctx.stream));
        if (strings)
            STB_CUDA(cudaMemcpyAsync(opsh.data(), ops_d, opsh.size(), cudaMemcpyDeviceToHost,
                                     ctx.stream));
        STB_CUDA(cudaStreamSynchronize(ctx.stream));
        for (int64_t p = 0; p < n; ++p) {
            if (starts[size_t(p)] < 0)
                fail(ST_EOVERFLOW, "seqtree_b200: the traceback left the matrix -- gap costs near "
                                   "2^29 overflow the reference's int32 recurrence");
            const int64_t len = slot - starts[size_t(p)];
            lengths[p] = int32_t(len);
            if (!strings) continue;
            // The aligned strings carry the caller's own characters (src/index.cpp:160-172).
            const char* op = opsh.data() + p * slot + starts[size_t(p)];
            const char* q = queries->bytes + queries->offsets[query_idx[p]];
            const char* r = refs->bytes + refs->offsets[ref_idx[p]];
            char* aq = aligned_query + p * stride;
            char* ar = aligned_ref + p * stride;
            char* oo = ops + p * stride;
            for (int64_t c = 0; c < len; ++c) {
                const char o = op[c];
                aq[c] = o == 'I' ? '-' : *q++;
                ar[c] = o == 'D' ? '-' : *r++;
                oo[c] = o;
            }
            aq[len] = ar[len] = oo[len] = 0;
        }
    });
}

int32_t st_align_score_matrix(const st_strings* queries, const st_strings* refs,
                              const int32_t* similarity, int32_t matrix_size, int32_t alphabet,
                              int32_t mode, int32_t gap_open, int32_t gap_extend,
                              int32_t threads, int32_t* out, st_error* err) {
    (void)threads;
    return align_common(queries, refs, similarity, matrix_size, alphabet, mode, gap_open,
                        gap_extend, 0, out, err);
}

int32_t st_align_dist_matrix(const st_strings* queries, const st_strings* refs,
                             const int32_t* similarity, int32_t matrix_size, int32_t alphabet,
                             int32_t mode, int32_t gap_open, int32_t gap_extend,
                             int32_t threads, int32_t* out, st_error* err) {
    (void)threads;
    return align_common(queries, refs, similarity, matrix_size, alphabet, mode, gap_open,
                        gap_extend, 1, out, err);
}

static int32_t distance_common(const st_strings* a, const st_strings* b, bool lev, int32_t* out,
                               st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_strings(a);
        check_strings(b);
        const int64_t N = count_of(a), K = count_of(b);
        if (N == 0 || K == 0) return;  // src/distance.cpp:34
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output buffer");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        clear_flags(ctx);
        Transient t;
        {
            Phase ph("upload");
            t.q.reset(make_seqset(a, -1, ctx.stream, nullptr, nullptr, ctx.tq));
            t.r.reset(make_seqset(b, -1, ctx.stream, nullptr, nullptr, ctx.tr));
        }
        int32_t* out_d = ctx.out_buf.as<int32_t>(size_t(N) * size_t(K));
        if (lev && N * K >= (int64_t(1) << 24)) {
            // Levenshtein's kernel time is of the order of its result copy: overlap the two.
            Phase ph("kernels+d2h (row blocks)");
            finish_pipelined(ctx, out, N, K, out_d, 8, [&](int64_t r0, int64_t r1) {
                levenshtein_sets(*t.q, *t.r, out_d, ctx.stream, r0, r1);
            });
        } else {
            {
                Phase ph("plan+launch");
                if (lev)
                    levenshtein_sets(*t.q, *t.r, out_d, ctx.stream);
                else
                    hamming_sets(*t.q, *t.r, out_d, ctx.stream);
            }
            Phase ph("kernel+d2h");
            finish(ctx, out, N, K, out_d);
        }
        trace_report(lev ? "st_levenshtein_matrix" : "st_hamming_matrix");
    });
}

int32_t st_hamming_matrix(const st_strings* a, const st_strings* b, int32_t threads, int32_t* out,
                          st_error* err) {
    (void)threads;
    return distance_common(a, b, false, out, err);
}

int32_t st_levenshtein_matrix(const st_strings* a, const st_strings* b, int32_t threads,
                              int32_t* out, st_error* err) {
    (void)threads;
    return distance_common(a, b, true, out, err);
}

// ------------------------------------------------------------------------- device sets ------
int32_t st_seqset_create(const st_strings* seqs, int32_t alphabet, st_seqset* out, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_strings(seqs);
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output handle");
        *out = nullptr;
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        *out = make_seqset(seqs, alphabet, ctx.stream, nullptr, nullptr, nullptr);
        STB_CUDA(cudaStreamSynchronize(ctx.stream));
    });
}

void st_seqset_destroy(st_seqset set) { delete set; }

int64_t st_seqset_count(st_seqset set) { return set ? set->count : -1; }

static void check_set(st_seqset s) {
    if (!s) fail(ST_EINVAL, "seqtree_b200: null sequence set");
    int dev = -1;
    STB_CUDA(cudaGetDevice(&dev));
    if (dev != s->device) fail(ST_EINVAL, "seqtree_b200: sequence set lives on another device");
}

int32_t st_gapblock_matrix_sets(st_seqset queries, st_seqset refs, const int32_t* penalty,
                                int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                                const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                                int32_t* out_device, void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(queries);
        check_set(refs);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        auto stream = static_cast<cudaStream_t>(cuda_stream);
        gapblock_sets(*queries, *refs, penalty, matrix_size, gap_open, gap_extend, prior, prior_len,
                      prior_width, out_device, stream);
    });
}

int32_t st_hits_create(st_hits* out, st_error* err) {
    return guard(err, [&] {
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output handle");
        *out = nullptr;
        auto h = std::make_unique<st_hits_s>();
        STB_CUDA(cudaGetDevice(&h->device));
        *out = h.release();
    });
}

void st_hits_destroy(st_hits hits) {
    if (!hits) return;
    int prev = -1;
    cudaGetDevice(&prev);
    const int home = hits->device;
    if (prev != home) cudaSetDevice(home);
    delete hits;  // frees its device buffers on their device
    if (prev >= 0 && prev != home) cudaSetDevice(prev);
}

int32_t st_hits_info(st_hits hits, int64_t* rows, int64_t* cols, int64_t* nnz,
                     const int64_t** indptr_device, const int32_t** ref_ids_device,
                     const int32_t** scores_device) {
    if (!hits) return ST_EINVAL;
    if (rows) *rows = hits->rows;
    if (cols) *cols = hits->cols;
    if (nnz) *nnz = hits->nnz;
    if (indptr_device) *indptr_device = static_cast<const int64_t*>(hits->indptr.ptr);
    if (ref_ids_device) *ref_ids_device = static_cast<const int32_t*>(hits->ref_ids.ptr);
    if (scores_device) *scores_device = static_cast<const int32_t*>(hits->scores.ptr);
    return ST_OK;
}

int32_t st_hits_download(st_hits hits, int64_t* indptr, int32_t* ref_ids, int32_t* scores,
                         st_error* err) {
    return guard(err, [&] {
        if (!hits) fail(ST_EINVAL, "seqtree_b200: null hits handle");
        int dev = -1;
        STB_CUDA(cudaGetDevice(&dev));
        if (dev != hits->device) fail(ST_EINVAL, "seqtree_b200: hits handle lives on another device");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        if (indptr && hits->indptr.ptr)
            STB_CUDA(cudaMemcpyAsync(indptr, hits->indptr.ptr, sizeof(int64_t) * size_t(hits->rows + 1),
                                     cudaMemcpyDeviceToHost, ctx.stream));
        if (hits->nnz > 0) {
            if (ref_ids)
                STB_CUDA(cudaMemcpyAsync(ref_ids, hits->ref_ids.ptr, sizeof(int32_t) * size_t(hits->nnz),
                                         cudaMemcpyDeviceToHost, ctx.stream));
            if (scores)
                STB_CUDA(cudaMemcpyAsync(scores, hits->scores.ptr, sizeof(int32_t) * size_t(hits->nnz),
                                         cudaMemcpyDeviceToHost, ctx.stream));
        }
        STB_CUDA(cudaStreamSynchronize(ctx.stream));
    });
}

int32_t st_gapblock_sparse_sets(st_seqset queries, st_seqset refs, const int32_t* penalty,
                                int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                                const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                                int32_t max_penalty, st_hits out, void* cuda_stream,
                                st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(queries);
        check_set(refs);
        if (!out) fail(ST_EINVAL, "seqtree_b200: null hits handle");
        int dev = -1;
        STB_CUDA(cudaGetDevice(&dev));
        if (dev != out->device) fail(ST_EINVAL, "seqtree_b200: hits handle lives on another device");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        gapblock_sparse_sets(*queries, *refs, penalty, matrix_size, gap_open, gap_extend, prior,
                             prior_len, prior_width, max_penalty, *out,
                             static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_gapblock_pairs_sets(st_seqset queries, st_seqset refs, const int32_t* query_idx,
                               const int32_t* ref_idx, int64_t n, const int32_t* penalty,
                               int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                               const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                               int32_t* out_device, void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(queries);
        check_set(refs);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        gapblock_pairs_sets(*queries, *refs, query_idx, ref_idx, n, penalty, matrix_size, gap_open,
                            gap_extend, prior, prior_len, prior_width, out_device, nullptr,
                            static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_gapblock_pairs_pos_sets(st_seqset queries, st_seqset refs, const int32_t* query_idx,
                                   const int32_t* ref_idx, int64_t n, const int32_t* penalty,
                                   int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                                   const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                                   int32_t* out_device, int32_t* pos_device, void* cuda_stream,
                                   st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(queries);
        check_set(refs);
        if (!pos_device) fail(ST_EINVAL, "seqtree_b200: null position output");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        gapblock_pairs_sets(*queries, *refs, query_idx, ref_idx, n, penalty, matrix_size, gap_open,
                            gap_extend, prior, prior_len, prior_width, out_device, pos_device,
                            static_cast<cudaStream_t>(cuda_stream));
    });
}

// ---------------------------------------------------------------------------- encoder -------
struct st_encoder_s {
    int device = 0;
    stb::Encoder* impl = nullptr;
};

int64_t st_encoder_param_count(void) { return encoder_param_count(); }

int32_t st_encoder_create(const float* params, st_encoder* out, st_error* err) {
    return guard(err, [&] {
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output handle");
        *out = nullptr;
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        auto h = std::make_unique<st_encoder_s>();
        h->device = ctx.device;
        h->impl = encoder_create(params);
        *out = h.release();
    });
}

void st_encoder_destroy(st_encoder enc) {
    if (!enc) return;
    int prev = -1;
    cudaGetDevice(&prev);
    const int home = enc->device;
    if (prev != home) cudaSetDevice(home);
    encoder_destroy(enc->impl);
    delete enc;
    if (prev >= 0 && prev != home) cudaSetDevice(prev);
}

static Context& encoder_ctx(st_encoder enc) {
    if (!enc || !enc->impl) fail(ST_EINVAL, "seqtree_b200: null encoder");
    int dev = -1;
    STB_CUDA(cudaGetDevice(&dev));
    if (dev != enc->device) fail(ST_EINVAL, "seqtree_b200: encoder lives on another device");
    return context();
}

int32_t st_encoder_get_params(st_encoder enc, float* out, st_error* err) {
    return guard(err, [&] {
        Context& ctx = encoder_ctx(enc);
        if (!out) fail(ST_EINVAL, "seqtree_b200: null output");
        std::lock_guard<std::mutex> lk(ctx.mu);
        encoder_params(*enc->impl, out);
    });
}

int32_t st_encoder_set_precision(st_encoder enc, int32_t precision, st_error* err) {
    return guard(err, [&] {
        Context& ctx = encoder_ctx(enc);
        std::lock_guard<std::mutex> lk(ctx.mu);
        encoder_set_precision(*enc->impl, precision);
    });
}

int32_t st_encoder_loss_grad(st_encoder enc, const uint8_t* codes, const int32_t* lens,
                             const int32_t* scores, int32_t S, float* loss, float* grad,
                             st_error* err) {
    return guard(err, [&] {
        reset_launches();
        Context& ctx = encoder_ctx(enc);
        if (!codes || !lens || !scores) fail(ST_EINVAL, "seqtree_b200: null batch");
        std::lock_guard<std::mutex> lk(ctx.mu);
        const float l = encoder_loss_grad(*enc->impl, codes, lens, scores, S, grad);
        if (loss) *loss = l;
    });
}

int32_t st_encoder_train_step(st_encoder enc, const uint8_t* codes, const int32_t* lens,
                              const int32_t* scores, int32_t S, float lr, float* loss,
                              st_error* err) {
    return guard(err, [&] {
        reset_launches();
        Context& ctx = encoder_ctx(enc);
        if (!codes || !lens || !scores) fail(ST_EINVAL, "seqtree_b200: null batch");
        std::lock_guard<std::mutex> lk(ctx.mu);
        const float l = encoder_train_step(*enc->impl, codes, lens, scores, S, lr);
        if (loss) *loss = l;
    });
}

int32_t st_encoder_embed(st_encoder enc, st_seqset set, void* out_device, int32_t layout,
                         void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        Context& ctx = encoder_ctx(enc);
        check_set(set);
        if (!out_device) fail(ST_EINVAL, "seqtree_b200: null output");
        if (layout < 0 || layout > 2) fail(ST_EINVAL, "seqtree_b200: embedding layout is 0, 1 or 2");
        std::lock_guard<std::mutex> lk(ctx.mu);
        encoder_embed(*enc->impl, *set, out_device, layout, static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_train_gemm_bf16(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K,
                           const float* A_device, int32_t lda, const float* B_device, int32_t ldb,
                           float* C_device, int32_t ldc, int32_t accumulate, void* cuda_stream,
                           st_error* err) {
    return guard(err, [&] {
        reset_launches();
        Context& ctx = context();
        if (M < 0 || N < 0 || K < 0) fail(ST_EINVAL, "seqtree_b200: negative GEMM size");
        if (ldc < std::max(N, 1) || lda < std::max(trans_a ? M : K, 1) ||
            ldb < std::max(trans_b ? K : N, 1))
            fail(ST_EINVAL, "seqtree_b200: GEMM leading dimension too small");
        if (M > 0 && N > 0 && (!C_device || (K > 0 && (!A_device || !B_device))))
            fail(ST_EINVAL, "seqtree_b200: null GEMM operand");
        std::lock_guard<std::mutex> lk(ctx.mu);
        const auto st = static_cast<cudaStream_t>(cuda_stream);
        STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, sizeof(int64_t), st));
        gemm_bf16(trans_a != 0, trans_b != 0, M, N, K, A_device, lda, B_device, ldb, C_device, ldc,
                  accumulate != 0, st, ctx.num_sms);
        STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, st));
        STB_CUDA(cudaStreamSynchronize(st));
        if (ctx.flags_h[8] != 0)
            fail(ST_ETIMEOUT, "seqtree_b200: a bounded device-side wait gave up (training GEMM)");
    });
}

int32_t st_propose_topk(const void* query_emb, int64_t nq, const void* ref_emb, int64_t nr,
                        int32_t k, int32_t* ids_device, float* scores_device, void* cuda_stream,
                        st_error* err) {
    return guard(err, [&] {
        reset_launches();
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        propose_topk(query_emb, nq, ref_emb, nr, k, ids_device, scores_device,
                     static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_propose_topk_ranges(const void* query_emb, int64_t nq, const void* ref_emb, int64_t nr,
                               int32_t k, const int32_t* tile_ranges_device, int32_t* ids_device,
                               float* scores_device, void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        if (!tile_ranges_device) fail(ST_EINVAL, "seqtree_b200: null tile ranges");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        propose_topk(query_emb, nq, ref_emb, nr, k, ids_device, scores_device,
                     static_cast<cudaStream_t>(cuda_stream), tile_ranges_device);
    });
}

int32_t st_propose_range(const void* query_emb, int64_t nq, const uint8_t* query_lens_device,
                         const void* ref_emb, int64_t nr, const uint8_t* ref_lens_device,
                         const float* thresholds, const int32_t* tile_ranges_device,
                         int32_t* pair_query_device, int32_t* pair_ref_device, int64_t capacity,
                         int64_t* count, void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        if (!count) fail(ST_EINVAL, "seqtree_b200: null count");
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        *count = propose_range(query_emb, nq, query_lens_device, ref_emb, nr, ref_lens_device,
                               thresholds, pair_query_device, pair_ref_device, capacity,
                               static_cast<cudaStream_t>(cuda_stream), tile_ranges_device);
    });
}

int32_t st_embed_dots(const void* query_emb, int64_t nq, const void* ref_emb, int64_t nr,
                      const int32_t* query_idx_device, const int32_t* ref_idx_device, int64_t n,
                      float* out_device, void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        embed_dots(query_emb, nq, ref_emb, nr, query_idx_device, ref_idx_device, n, out_device,
                   static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_thetas_csr(const int64_t* indptr_device, const int32_t* scores_device, int64_t rows,
                      int64_t n_target, int64_t m_control, double e_target, int32_t theta_max,
                      int32_t exclude_exact, int32_t* out_device, void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        if (n_target <= 0 || m_control <= 0) fail(ST_EINVAL, "n_target and m_control must be > 0");
        if (!(e_target > 0.0)) fail(ST_EINVAL, "e_target must be > 0");
        if (theta_max < 0) fail(ST_EINVAL, "theta_max must be >= 0");
        const double c_max = e_target * double(m_control) / double(n_target);
        const double kd = std::floor(c_max);
        const int32_t k = kd > 2147483647.0 ? 2147483647 : int32_t(kd);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        thetas_csr(indptr_device, scores_device, rows, k, c_max < 3.0 ? 1 : 0, theta_max,
                   exclude_exact, out_device, static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_profile_scores_sets(const int32_t* table, int32_t width, int32_t c, uint8_t gap,
                               int32_t unreachable, st_seqset set, int32_t* out_device,
                               void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(set);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        profile_scores(table, width, c, gap, unreachable, *set, out_device,
                       static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_align_pairs_sets(st_seqset queries, st_seqset refs, const int32_t* query_idx,
                            const int32_t* ref_idx, int64_t n, const int32_t* similarity,
                            int32_t matrix_size, int32_t mode, int32_t gap_open, int32_t gap_extend,
                            int64_t* score_device, int32_t* start_device, char* aligned_query_device,
                            char* aligned_ref_device, char* ops_device, int64_t slot_bytes,
                            void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(queries);
        check_set(refs);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        align_pairs_sets(*queries, *refs, query_idx, ref_idx, n, similarity, matrix_size, mode,
                         gap_open, gap_extend, score_device, start_device, aligned_query_device,
                         aligned_ref_device, ops_device, slot_bytes,
                         static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_stream_status(void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
        STB_CUDA(cudaStreamSynchronize(st));
        STB_CUDA(cudaMemcpyAsync(ctx.flags_h + 8, ctx.flags_d + 8, 8 * sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, st));
        STB_CUDA(cudaMemsetAsync(ctx.flags_d + 8, 0, 8 * sizeof(int64_t), st));
        STB_CUDA(cudaStreamSynchronize(st));
        check_timeout(ctx);
    });
}

int32_t st_align_matrix_sets(st_seqset queries, st_seqset refs, const int32_t* similarity,
                             int32_t matrix_size, int32_t mode, int32_t gap_open,
                             int32_t gap_extend, int32_t dist, int32_t* out_device,
                             void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(queries);
        check_set(refs);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        align_sets(*queries, *refs, similarity, matrix_size, mode, gap_open, gap_extend, dist,
                   out_device, static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_hamming_matrix_sets(st_seqset a, st_seqset b, int32_t* out_device, void* cuda_stream,
                               st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(a);
        check_set(b);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        hamming_sets(*a, *b, out_device, static_cast<cudaStream_t>(cuda_stream));
    });
}

int32_t st_levenshtein_matrix_sets(st_seqset a, st_seqset b, int32_t* out_device,
                                   void* cuda_stream, st_error* err) {
    return guard(err, [&] {
        reset_launches();
        check_set(a);
        check_set(b);
        Context& ctx = context();
        std::lock_guard<std::mutex> lk(ctx.mu);
        levenshtein_sets(*a, *b, out_device, static_cast<cudaStream_t>(cuda_stream));
    });
}

}  // extern "C"
