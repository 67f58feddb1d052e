/*
 * seqtree_b200 -- C ABI of the B200 (sm_100a) all-vs-all scoring library.
 *
 * Drop-in boundary for the dense matrix calls of seqtree 0.6.0.  Every entry point below names
 * the reference interface it replaces (file:line inside the seqtree project).  Plain pointers
 * and sizes only: no C++ or torch types cross this boundary, so it binds from ctypes, cffi,
 * pybind11 or any FFI.
 *
 * Conventions shared by every call
 *   - Sequences cross as one st_strings: all sequences concatenated in `bytes`, with
 *     `offsets` holding count+1 non-decreasing byte offsets (offsets[0] == 0).
 *   - Results are dense row-major int32 matrices, row i = queries[i] against every ref,
 *     exactly the reference's std::vector<int32_t> / ScoreMatrix layout.
 *   - Each call returns ST_OK (0) or an error code, and fills `err` (may be NULL) with the
 *     code and the message the reference would raise: ST_EINVAL <-> std::invalid_argument
 *     (Python ValueError), ST_EOVERFLOW <-> std::overflow_error (Python OverflowError).
 *   - `threads` is accepted for signature parity with the reference and ignored: the work
 *     runs on the current CUDA device.
 *   - There is no CPU fallback.  Without a usable CUDA device the calls return ST_ENODEV.
 *   - Calls are thread-safe; calls on the same device are serialised internally.
 */
#ifndef SEQTREE_B200_H
#define SEQTREE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ST_OK = 0,
    ST_EINVAL = 1,    /* bad argument (reference: std::invalid_argument)              */
    ST_EOVERFLOW = 2, /* a result does not fit int32 (reference: std::overflow_error) */
    ST_ECUDA = 3,     /* CUDA runtime error                                          */
    ST_ETIMEOUT = 4,  /* a bounded device-side wait gave up                          */
    ST_ENOMEM = 5,    /* device or pinned host allocation failed                     */
    ST_ENODEV = 6     /* no usable CUDA device                                        */
};

/* Alphabet codes: the reference's enum class Alphabet (include/seqtree/types.hpp:9). */
enum { ST_ALPHABET_AA = 0, ST_ALPHABET_NT = 1, ST_ALPHABET_IUPAC = 2 };

/* Alignment modes: the reference's enum class AlignMode (include/seqtree/seqtree.hpp:186). */
enum { ST_MODE_GLOBAL = 0, ST_MODE_LOCAL = 1 };

typedef struct st_strings {
    const char *bytes;      /* concatenated sequences (may be NULL when offsets[count]==0) */
    const int64_t *offsets; /* count + 1 entries                                          */
    int64_t count;
} st_strings;

typedef struct st_error {
    int32_t code;
    char message[256];
} st_error;

/* Library version, encoded as major*10000 + minor*100 + patch. */
int32_t st_version(void);

/* Number of visible CUDA devices (0 when none). */
int32_t st_device_count(void);

/*
 * Dense single-gap-block penalty matrix.
 * Replaces seqtree::gapblock_matrix (include/seqtree/seqtree.hpp:218-222,
 * src/gapblock.cpp:66-133) and its binding _core.gapblock_matrix (src/_bindings.cpp:218-233,
 * 570-576).
 *   penalty      A*A row-major penalty grid (SubstitutionMatrix::penalty, seqtree.hpp:60), or
 *                NULL for unit cost (the reference's null matrix).
 *   matrix_size  A of `penalty` (checked against the alphabet like the reference); ignored
 *                when `penalty` is NULL.
 *   prior        the [m][d][i] gap-prior cube of (prior_width+1)^3 entries, or NULL /
 *                prior_len == 0 for no prior.
 *   out          N*K int32, host memory (pinned or pageable); its contents are unspecified
 *                after a call that fails (the symbol check runs beside the kernel).
 */
int32_t st_gapblock_matrix(const st_strings *queries, const st_strings *refs, int32_t alphabet,
                           const int32_t *penalty, int32_t matrix_size, int32_t gap_open,
                           int32_t gap_extend, const int32_t *prior, int64_t prior_len,
                           uint32_t prior_width, int32_t threads, int32_t *out, st_error *err);

/*
 * Dense Gotoh Needleman-Wunsch / Smith-Waterman similarity matrix.
 * Replaces seqtree::align_score_matrix (include/seqtree/seqtree.hpp:198-201,
 * src/pairwise.cpp:338-344) and _core.align_score_matrix (src/_bindings.cpp:527-546).
 *   similarity   A*A row-major similarity grid (SubstitutionMatrix::similarity, seqtree.hpp:61).
 *   mode         ST_MODE_GLOBAL or ST_MODE_LOCAL.
 */
int32_t st_align_score_matrix(const st_strings *queries, const st_strings *refs,
                              const int32_t *similarity, int32_t matrix_size, int32_t alphabet,
                              int32_t mode, int32_t gap_open, int32_t gap_extend,
                              int32_t threads, int32_t *out, st_error *err);

/*
 * Optimal alignment of one pair with its traceback.
 * Replaces seqtree::align_pair (include/seqtree/seqtree.hpp:190-192, src/pairwise.cpp:141-267)
 * and _core.align_pair (src/_bindings.cpp:515-525).  Host buffers: aligned_query, aligned_ref and
 * ops receive NUL-terminated strings and must hold query_len + ref_len + 1 bytes; ops per
 * column: 'M' match, 'S' substitution, 'D' gap in the ref, 'I' gap in the query.  Same checks,
 * messages and tie order as the reference; ST_EOVERFLOW when the score does not fit int32.
 */
int32_t st_align_pair(const char *query, int64_t query_len, const char *ref, int64_t ref_len,
                      const int32_t *similarity, int32_t matrix_size, int32_t alphabet, int32_t mode,
                      int32_t gap_open, int32_t gap_extend, int32_t *score, char *aligned_query,
                      char *aligned_ref, char *ops, int64_t capacity, st_error *err);

/*
 * Penalty-minimising global alignment with traceback for a list of (query, ref) pairs.
 * Replaces seqtree::Index::align (src/index.cpp:105-179; Python Index.align,
 * src/_bindings.cpp:197-201,454): pair p aligns queries[query_idx[p]] to refs[ref_idx[p]] with
 * substitution cost penalty[a * matrix_size + b] (the matrix's penalty grid; NULL: unit cost
 * on codec equality, case-insensitive) and affine gaps gap_open + (L-1) * gap_extend.  Same
 * int32 arithmetic, tie order and messages as the reference: "invalid symbol 'c' in reference
 * #k", "matrix size does not match the alphabet", "invalid symbol 'c' in query", "seqtree:
 * gap_open and gap_extend must be >= 0" (checked in that order).  scores[p] and lengths[p]
 * (alignment columns) are always written; aligned_query, aligned_ref and ops (all three or
 * none) receive NUL-terminated strings at p * stride (stride >= longest query + longest ref + 1)
 * made of the caller's own characters; ops per column 'M' match, 'S' substitution, 'D' query
 * residue against a gap, 'I' ref residue against a gap.
 */
int32_t st_penalty_align_pairs(const st_strings *queries, const st_strings *refs,
                               const int32_t *query_idx, const int32_t *ref_idx, int64_t n,
                               int32_t alphabet, const int32_t *penalty, int32_t matrix_size,
                               int32_t gap_open, int32_t gap_extend, int32_t *scores,
                               char *aligned_query, char *aligned_ref, char *ops, int64_t stride,
                               int32_t *lengths, st_error *err);

/*
 * Dense sequence-level Gram distance d = s(a,a) + s(b,b) - 2 s(a,b) over Gotoh scores.
 * Replaces seqtree::align_dist_matrix (include/seqtree/seqtree.hpp:206-209,
 * src/pairwise.cpp:346-352) and _core.align_dist_matrix (src/_bindings.cpp:548-568).
 */
int32_t st_align_dist_matrix(const st_strings *queries, const st_strings *refs,
                             const int32_t *similarity, int32_t matrix_size, int32_t alphabet,
                             int32_t mode, int32_t gap_open, int32_t gap_extend,
                             int32_t threads, int32_t *out, st_error *err);

/*
 * Dense Hamming matrix over raw bytes, case-sensitive.
 * Replaces seqtree::hamming_matrix (include/seqtree/seqtree.hpp:239-240,
 * src/distance.cpp:97-102) and _core.hamming_matrix (src/_bindings.cpp:586-600).
 * Fails with ST_EINVAL when any (a[i], b[k]) pair differs in length.
 */
int32_t st_hamming_matrix(const st_strings *a, const st_strings *b, int32_t threads,
                          int32_t *out, st_error *err);

/*
 * Dense Levenshtein (unit-cost edit distance) matrix over raw bytes, case-sensitive.
 * Replaces seqtree::levenshtein_matrix (include/seqtree/seqtree.hpp:241-242,
 * src/distance.cpp:104-109) and _core.levenshtein_matrix (src/_bindings.cpp:602-615).
 */
int32_t st_levenshtein_matrix(const st_strings *a, const st_strings *b, int32_t threads,
                              int32_t *out, st_error *err);

/*
 * Thresholded sparse gap-block matrix: only the cells with score <= max_penalty, as CSR rows
 * over the queries.  Row i holds the refs k (ascending) with gapblock_matrix[i][k] <= max_penalty
 * and their scores -- exactly the dense matrix's entries that pass, for matrices too large to
 * hold densely (e.g. 1e5 x 1e6).  An addition to the reference's API: it is the dense call of
 * seqtree::gapblock_matrix (include/seqtree/seqtree.hpp:218-222) filtered the way
 * GapBlockIndex.search filters (python/seqtree/gapblock.py:611-634: keep score <= max_penalty,
 * ValueError "max_penalty must be >= 0"), without that index's |m-n| cap.  Arguments and checks
 * are st_gapblock_matrix's.  The library allocates the three arrays (pinned host memory);
 * release them with st_sparse_free.
 */
typedef struct st_sparse {
    int64_t rows, cols, nnz;
    int64_t *indptr;  /* rows + 1 */
    int32_t *ref_ids; /* nnz */
    int32_t *scores;  /* nnz */
} st_sparse;

int32_t st_gapblock_sparse(const st_strings *queries, const st_strings *refs, int32_t alphabet,
                           const int32_t *penalty, int32_t matrix_size, int32_t gap_open,
                           int32_t gap_extend, const int32_t *prior, int64_t prior_len,
                           uint32_t prior_width, int32_t max_penalty, int32_t threads,
                           st_sparse *out, st_error *err);
void st_sparse_free(st_sparse *sparse);

/* ------------------------------------------------------------------------------------------
 * Device-resident form.  For callers whose sequences stay on the GPU across many calls (and
 * for measuring the kernels alone): a sequence set is uploaded and encoded once, and the
 * *_sets calls write into DEVICE memory on the given stream without any host round trip.
 * These have no single reference counterpart; they are the same computations as the calls
 * above, split at the host/device boundary.
 * ------------------------------------------------------------------------------------------ */
typedef struct st_seqset_s *st_seqset;

/* Upload and encode a set.  alphabet = ST_ALPHABET_* for gap-block / alignment use, or -1 to
 * keep raw bytes (Hamming / Levenshtein).  Invalid symbols fail with the reference message. */
int32_t st_seqset_create(const st_strings *seqs, int32_t alphabet, st_seqset *out,
                         st_error *err);
void st_seqset_destroy(st_seqset set);
int64_t st_seqset_count(st_seqset set);

int32_t st_gapblock_matrix_sets(st_seqset queries, st_seqset refs, const int32_t *penalty,
                                int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                                const int32_t *prior, int64_t prior_len, uint32_t prior_width,
                                int32_t *out_device, void *cuda_stream, st_error *err);

/* Sparse result kept on the device (CSR over the query set; see st_gapblock_sparse).  Its
 * buffers belong to the handle and are reused by the next call that fills it. */
typedef struct st_hits_s *st_hits;
int32_t st_hits_create(st_hits *out, st_error *err);
void st_hits_destroy(st_hits hits);
int32_t st_hits_info(st_hits hits, int64_t *rows, int64_t *cols, int64_t *nnz,
                     const int64_t **indptr_device, const int32_t **ref_ids_device,
                     const int32_t **scores_device);
/* Copy a hits handle's rows into host arrays of rows + 1 / nnz / nnz entries (any may be NULL);
 * synchronous. */
int32_t st_hits_download(st_hits hits, int64_t *indptr, int32_t *ref_ids, int32_t *scores,
                         st_error *err);

/* Sparse gap-block matrix of two device sets into `out`.  Synchronises cuda_stream once (to
 * read the hit count), then enqueues the sort and the row build on it. */
int32_t st_gapblock_sparse_sets(st_seqset queries, st_seqset refs, const int32_t *penalty,
                                int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                                const int32_t *prior, int64_t prior_len, uint32_t prior_width,
                                int32_t max_penalty, st_hits out, void *cuda_stream,
                                st_error *err);

/* Gap-block scores of listed pairs: out_device[p] = score(queries[query_idx[p]], refs[ref_idx[p]])
 * (index arrays and output in device memory).  The dense call's arithmetic and checks
 * (src/gapblock.cpp:39-62, 66-81) on a pair list instead of the full product -- the exact rescore
 * of the learned proposals and the labeller of the encoder's training pairs.  No counterpart in
 * the reference. */
int32_t st_gapblock_pairs_sets(st_seqset queries, st_seqset refs, const int32_t *query_idx,
                               const int32_t *ref_idx, int64_t n, const int32_t *penalty,
                               int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                               const int32_t *prior, int64_t prior_len, uint32_t prior_width,
                               int32_t *out_device, void *cuda_stream, st_error *err);

/* The same pair scores plus, in pos_device[p], the position of the gap block that attains the
 * minimum (the smallest such position, counted in residues of the shorter sequence; 0 for equal
 * lengths): the (block_length, block_position) report of GapBlockIndex.search
 * (python/seqtree/gapblock.py:607-661), where block_length is |m - n|. */
int32_t st_gapblock_pairs_pos_sets(st_seqset queries, st_seqset refs, const int32_t *query_idx,
                                   const int32_t *ref_idx, int64_t n, const int32_t *penalty,
                                   int32_t matrix_size, int32_t gap_open, int32_t gap_extend,
                                   const int32_t *prior, int64_t prior_len, uint32_t prior_width,
                                   int32_t *out_device, int32_t *pos_device, void *cuda_stream,
                                   st_error *err);

/* ------------------------------------------------------------------------------------------
 * Sequence encoder of the learned-proposal path (no counterpart in the reference).  One-hot
 * amino-acid codes padded to 32 positions -> 2 conv layers -> 2 attention layers (width 128) ->
 * mean pool -> 64-d unit vector; trained so that |z_a - z_b|^2 tracks the exact gap-block score.
 * Parameters are a flat fp32 array of st_encoder_param_count() values.
 * ------------------------------------------------------------------------------------------ */
typedef struct st_encoder_s *st_encoder;
int64_t st_encoder_param_count(void);
/* params: host array of st_encoder_param_count() floats (NULL: all zero). */
int32_t st_encoder_create(const float *params, st_encoder *out, st_error *err);
void st_encoder_destroy(st_encoder enc);
int32_t st_encoder_get_params(st_encoder enc, float *out, st_error *err);
/* Precision of the training products (forward and backward of loss_grad / train_step):
 * 1 (the default) bf16 tensor cores with fp32 accumulation, 0 fp32 on CUDA cores.  Weights,
 * activations, gradients and the Adam state are fp32 either way. */
int32_t st_encoder_set_precision(st_encoder enc, int32_t precision, st_error *err);
/* A batch is S sequences (S even; pairs are (2i, 2i+1)) as host arrays: codes [S][32] (0..23,
 * zero beyond the length), lens [S] (1..32), scores [S/2] (exact gap-block scores).  loss_grad
 * returns the mean pair loss and, when grad is not NULL, its gradient; train_step also applies
 * one Adam step with learning rate lr. */
int32_t st_encoder_loss_grad(st_encoder enc, const uint8_t *codes, const int32_t *lens,
                             const int32_t *scores, int32_t S, float *loss, float *grad,
                             st_error *err);
int32_t st_encoder_train_step(st_encoder enc, const uint8_t *codes, const int32_t *lens,
                              const int32_t *scores, int32_t S, float lr, float *loss,
                              st_error *err);
/* Embeddings of a device set (amino acids, lengths 1..32) into out_device.
 *   layout 0: fp32 [n][64] from the fp32 forward (the training kernels' numbers);
 *   layout 1: bf16 [n][64] from the bf16 tensor-core inference kernels, the 16-byte chunks of
 *             row r stored at chunk ^ (r & 7) (the operand layout of st_propose_topk);
 *   layout 2: the fp32 forward stored in layout 1's format. */
int32_t st_encoder_embed(st_encoder enc, st_seqset set, void *out_device, int32_t layout,
                         void *cuda_stream, st_error *err);

/* The encoder's bf16 training GEMM (no counterpart in the reference), exported so it can be
 * checked on its own: C = op(A) op(B) (C += when accumulate), op(A) [M x K] = A or, when trans_a,
 * the transpose of A [K x M]; op(B) [K x N] = B or, when trans_b, the transpose of B [N x K]; all
 * fp32 row-major device arrays with leading dimensions lda / ldb / ldc.  Operands are rounded to
 * bf16 (nearest even) and the products accumulated in fp32 on the tensor cores.  Synchronous:
 * returns when C is written. */
int32_t st_train_gemm_bf16(int32_t trans_a, int32_t trans_b, int32_t M, int32_t N, int32_t K,
                           const float *A_device, int32_t lda, const float *B_device, int32_t ldb,
                           float *C_device, int32_t ldc, int32_t accumulate, void *cuda_stream,
                           st_error *err);

/* Learned candidate proposal (no counterpart in the reference): for every query, the k refs with
 * the largest embedding dot product, computed on the tensor cores without materialising the
 * nq x nr similarity matrix.  query_emb / ref_emb are device arrays of st_encoder_embed layout 1
 * (bf16 [n][64], 16-byte aligned).  ids_device[q*k + i] (and scores_device, which may be NULL)
 * receive the i-th best ref of query q, best first (score descending, ties by ascending ref
 * id); slots beyond nr refs hold -1 / -inf.  k is 1..256.  Asynchronous on cuda_stream; a
 * bounded device wait that gave up is reported by st_stream_status. */
int32_t st_propose_topk(const void *query_emb, int64_t nq, const void *ref_emb, int64_t nr,
                        int32_t k, int32_t *ids_device, float *scores_device, void *cuda_stream,
                        st_error *err);

/* st_propose_topk with each tile of 256 queries (rows 256t .. 256t+255) scanning only the ref
 * tiles of 128 refs [tile_ranges_device[2t], tile_ranges_device[2t + 1]) (device int32, two per
 * query tile; clamped into the ref tiles that exist).  With queries and refs sorted by length,
 * this restricts each query's candidates to refs of nearby length.  The result is the exact
 * top-k of the scanned refs.  No counterpart in the reference. */
int32_t st_propose_topk_ranges(const void *query_emb, int64_t nq, const void *ref_emb, int64_t nr,
                               int32_t k, const int32_t *tile_ranges_device, int32_t *ids_device,
                               float *scores_device, void *cuda_stream, st_error *err);

/* Learned candidate proposal by threshold (no counterpart in the reference): every (query, ref)
 * pair whose embedding dot product is >= thresholds[query_len * 33 + ref_len], where the lengths
 * come from query_lens_device[q] / ref_lens_device[r] (device uint8; lengths above 32 use row or
 * column 32) and thresholds is a host float [33][33] table (+inf switches a length cell off).
 * Embeddings as for st_propose_topk.  tile_ranges_device may be NULL (every ref tile) or limit
 * each tile of 256 queries to ref tiles of 128 refs as st_propose_topk_ranges does.  The pairs
 * found first (in no particular order) are written to pair_query_device / pair_ref_device (device
 * int32, capacity entries each); *count receives how many pairs pass in all, so a count above
 * capacity means the call should be repeated with room for that many.  Synchronous: returns when
 * the pairs are written.  The candidate pairs are meant to be rescored by the exact gap-block
 * kernel (st_gapblock_pairs_sets). */
int32_t st_propose_range(const void *query_emb, int64_t nq, const uint8_t *query_lens_device,
                         const void *ref_emb, int64_t nr, const uint8_t *ref_lens_device,
                         const float *thresholds, const int32_t *tile_ranges_device,
                         int32_t *pair_query_device, int32_t *pair_ref_device, int64_t capacity,
                         int64_t *count, void *cuda_stream, st_error *err);

/* Dot products of listed pairs of layout-1 embeddings (no counterpart in the reference):
 * out_device[i] = <query_emb[query_idx_device[i]], ref_emb[ref_idx_device[i]]> in fp32, NaN for
 * an index outside [0, nq) / [0, nr).  Used to calibrate st_propose_range's thresholds on known
 * hits.  Asynchronous on cuda_stream. */
int32_t st_embed_dots(const void *query_emb, int64_t nq, const void *ref_emb, int64_t nr,
                      const int32_t *query_idx_device, const int32_t *ref_idx_device, int64_t n,
                      float *out_device, void *cuda_stream, st_error *err);

/* Per-row score cutoffs for a target E-value: thetas_from_scores of seqtree's
 * python/seqtree/evalue.py:102-143 (with _theta, :86-99) over CSR rows of control hit scores in
 * device memory (indptr_device rows + 1 int64, scores_device int32; row order within a row is
 * free, e.g. the rows of st_gapblock_sparse_sets).  out_device[row] is the largest cutoff in
 * [0, theta_max] whose control count stays <= floor(e_target * m_control / n_target), or -1
 * (the reference's rules).  Errors as the reference: "n_target and m_control must be > 0",
 * "e_target must be > 0", "theta_max must be >= 0" (ST_EINVAL). */
int32_t st_thetas_csr(const int64_t *indptr_device, const int32_t *scores_device, int64_t rows,
                      int64_t n_target, int64_t m_control, double e_target, int32_t theta_max,
                      int32_t exclude_exact, int32_t *out_device, void *cuda_stream, st_error *err);

/* IslandProfile.score_batch (seqtree python/seqtree/gapblock.py:365-377): the penalty of every
 * sequence of a raw-byte device set (alphabet -1) in a profile's frame.  table is host
 * int32 [width][256]: column j's penalty for each byte (the profile's cap for bytes it does not
 * list); c is the frame column of the gap block and gap the gap byte.  A sequence longer than
 * width, or shorter than c, scores `unreachable`.  out_device: int32 per sequence. */
int32_t st_profile_scores_sets(const int32_t *table, int32_t width, int32_t c, uint8_t gap,
                               int32_t unreachable, st_seqset set, int32_t *out_device,
                               void *cuda_stream, st_error *err);

/* Alignments with traceback of listed pairs: seqtree::align_pair (include/seqtree/seqtree.hpp:
 * 190-192, src/pairwise.cpp:141-267) for pair p = (queries[query_idx[p]], refs[ref_idx[p]]),
 * e.g. the top hits of a sparse search.  All outputs are device memory: score_device[p] (int64;
 * the reference refuses a score beyond int32 with std::overflow_error, which the caller
 * reports), and in slot p of slot_bytes bytes (>= longest query + longest ref) of each of
 * aligned_query_device / aligned_ref_device / ops_device the alignment, occupying
 * [start_device[p], slot_bytes).  start_device[p] == -1 marks a pair with an empty side, whose
 * strings are the raw inputs (global mode) or empty (local mode) as in the reference.  Ops:
 * 'M' match, 'S' substitution, 'D' gap in the ref, 'I' gap in the query.  Exact for any gap
 * cost (int64 cells); ties resolve as the reference. */
int32_t st_align_pairs_sets(st_seqset queries, st_seqset refs, const int32_t *query_idx,
                            const int32_t *ref_idx, int64_t n, const int32_t *similarity,
                            int32_t matrix_size, int32_t mode, int32_t gap_open, int32_t gap_extend,
                            int64_t *score_device, int32_t *start_device, char *aligned_query_device,
                            char *aligned_ref_device, char *ops_device, int64_t slot_bytes,
                            void *cuda_stream, st_error *err);

/* Synchronises cuda_stream and reports (then clears) the device error words written by the
 * asynchronous *_sets and proposal calls since the last check: ST_ETIMEOUT when a bounded
 * device-side wait gave up. */
int32_t st_stream_status(void *cuda_stream, st_error *err);

int32_t st_align_matrix_sets(st_seqset queries, st_seqset refs, const int32_t *similarity,
                             int32_t matrix_size, int32_t mode, int32_t gap_open,
                             int32_t gap_extend, int32_t dist, int32_t *out_device,
                             void *cuda_stream, st_error *err);

int32_t st_hamming_matrix_sets(st_seqset a, st_seqset b, int32_t *out_device, void *cuda_stream,
                               st_error *err);

int32_t st_levenshtein_matrix_sets(st_seqset a, st_seqset b, int32_t *out_device,
                                   void *cuda_stream, st_error *err);

/*
 * Levenshtein matrix that allocates nothing, for callers that cannot let a library allocate
 * device memory (their device memory is owned by their own allocator or reserved to a fixed
 * budget, or an allocation's latency or failure is unacceptable on their path).  No counterpart
 * in the reference.  All pointers are DEVICE memory owned by the caller: the concatenated raw
 * bytes and count+1 int64 offsets of each side, and the a_count*b_count int32 row-major output.
 * Same results as st_levenshtein_matrix.  The kernel's scratch is a fixed 32 MiB array inside
 * the library (held by every GPU that loads it); inputs whose DP row (shorter length + 1 words)
 * does not fit it for 256 threads are rejected with ST_EINVAL.  The first call on a device looks
 * up the array's address (make it before any stream capture).  The call synchronises
 * cuda_stream once (to size the launch, under a per-device host lock) and returns with the matrix
 * kernel enqueued on it.  Calls share the array: calls whose kernels overlap on the GPU (several
 * streams) race on its DP rows and may return wrong distances; the kernel never writes outside the
 * array, and a pair whose row would not fit its launch's share of it gets -1.
 */
int32_t st_levenshtein_matrix_noalloc(const char *a_bytes, const int64_t *a_offsets,
                                      int64_t a_count, const char *b_bytes,
                                      const int64_t *b_offsets, int64_t b_count, int32_t *out,
                                      void *cuda_stream, st_error *err);

/*
 * Peak issue rate of one instruction on the current device, measured by a register-only (or, for
 * ST_PEAK_LDS32, conflict-free shared-memory) probe: the denominators of the scoring kernels'
 * rooflines (the gap-block sweep of src/gapblock.cpp:119-125 is LDS.32 + __viaddmin_s16x2 per
 * cell pair; the Gotoh cell update of src/pairwise.cpp:106-117 is DPX add-max; the Levenshtein
 * bit-vector step replacing src/distance.cpp:78-95 is LOP3/IADD3).  No counterpart in the
 * reference.  all_sms = 0 runs one 1,024-thread block (one SM), otherwise two per SM.  Allocates
 * and frees a few bytes of device memory; about 10 ms per call.
 */
enum {
    ST_PEAK_LOP3 = 0,
    ST_PEAK_IADD3 = 1,
    ST_PEAK_IMAD = 2,
    ST_PEAK_VIADDMIN_S16X2 = 3,
    ST_PEAK_VIADDMAX_S32 = 4,
    ST_PEAK_VIMAX3_S32 = 5,
    ST_PEAK_LDS32 = 6
};

typedef struct st_peak {
    double lane_ops_per_s;      /* lane operations (one thread's op, or one 4-byte load) per s */
    double lane_ops_per_sm_clk; /* per SM per SM clock cycle (clock64 span of the longest block) */
    double ms;                  /* duration of the fastest of three launches */
    int32_t sms;                /* SMs the launch covered */
    int32_t threads;            /* threads launched */
} st_peak;

int32_t st_measure_peak(int32_t op, int32_t all_sms, st_peak *out, st_error *err);

/*
 * The raw similarity grid of a built-in amino-acid matrix ("blosum62", "blosum45", "blosum80",
 * "pam250", "pam100", "structural"), row-major 24*24 in the AminoAcid codec order, the numbers
 * behind seqtree::SubstitutionMatrix::blosum62() etc. (include/seqtree/seqtree.hpp:48-53,
 * src/substitution_matrix.cpp:52-74).  Writes *size = 24 and, when `out` is not NULL, the 576
 * entries (capacity must be >= 576).  Host-only: needs no GPU.
 */
int32_t st_builtin_similarity(const char *name, int32_t *out, int32_t capacity, int32_t *size,
                              st_error *err);

/* Launch statistics of the last *_sets / host call on this thread: how many kernels of this
 * library it launched and the name of the main kernel variant it chose. */
int32_t st_last_launch_count(void);
/* Kernels of this library launched by the whole process so far (all threads, all calls). */
int64_t st_total_launch_count(void);
/* The launch autotuner's decisions so far, one line per shape key ("device|key -> choice
 * (variant:time ...)"), written NUL-terminated into buf (truncated to capacity); returns the full
 * length.  Shapes are tuned on first use unless SEQTREE_B200_TUNE=0 is set in the environment. */
int64_t st_tuning_table(char *buf, int64_t capacity);
const char *st_last_kernel_name(void);

/* Pinned host buffers from a per-device cache.  A result written into one of these travels
 * device->host at full PCIe rate.  st_host_free returns the block to the cache. */
void *st_host_alloc(uint64_t bytes);
void st_host_free(void *ptr);

/* Host helper for bindings that hold sequences as one buffer of `count` sequences joined by
 * '\n' (no trailing separator): writes the sequences' bytes back to back into data_out
 * (size - (count - 1) bytes) and their count + 1 offsets into offsets_out, the st_strings
 * layout.  Returns the number of bytes written, or -1 when the buffer does not hold exactly
 * count - 1 separators (a sequence containing '\n'). */
int64_t st_split_joined(const uint8_t *joined, int64_t size, int64_t count, uint8_t *data_out,
                        int64_t *offsets_out);

#ifdef __cplusplus
}
#endif

#endif /* SEQTREE_B200_H */
