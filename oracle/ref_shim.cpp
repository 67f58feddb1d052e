// C entry points over the REFERENCE seqtree C++ API -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file together with the reference's own hot-path sources
// (src/codec.cpp, src/substitution_matrix.cpp, src/gapblock.cpp, src/pairwise.cpp,
// src/distance.cpp of seqtree 0.6.0, and the index sources Index::align needs) into
// oracle/_ref/libseqtree_ref.so.  The tests use it to
// generate and re-check golden vectors, and the benchmark's reference arm times it as the CPU
// baseline.  Nothing here is part of the product.
//
// Strings cross as packed bytes plus int64 offsets (count+1 entries).  Every function returns
// 0 on success, 1 for std::invalid_argument, 2 for std::overflow_error, 3 for anything else,
// and copies the exception text into `err`.
#include "seqtree/seqtree.hpp"

#include <algorithm>
#include <cstdint>
#include <utility>
#include <cstring>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

using namespace seqtree;

namespace {

std::vector<std::string> unpack(const char* bytes, const int64_t* off, int64_t n) {
    std::vector<std::string> v;
    v.reserve(size_t(n));
    for (int64_t i = 0; i < n; ++i) v.emplace_back(bytes + off[i], size_t(off[i + 1] - off[i]));
    return v;
}

void put_err(char* err, int errlen, const char* what) {
    if (!err || errlen <= 0) return;
    std::strncpy(err, what, size_t(errlen) - 1);
    err[errlen - 1] = 0;
}

// matrix_id: 0 blosum62, 1 blosum45, 2 blosum80, 3 pam250, 4 pam100, 5 structural,
// 6 unit(size), 7 custom from `sim` (size x size).
std::optional<SubstitutionMatrix> make(int matrix_id, const int32_t* sim, int size) {
    switch (matrix_id) {
        case 0: return SubstitutionMatrix::blosum62();
        case 1: return SubstitutionMatrix::blosum45();
        case 2: return SubstitutionMatrix::blosum80();
        case 3: return SubstitutionMatrix::pam250();
        case 4: return SubstitutionMatrix::pam100();
        case 5: return SubstitutionMatrix::structural();
        case 6: return SubstitutionMatrix::unit(uint8_t(size));
        case 7: return SubstitutionMatrix::from_similarity(uint8_t(size), sim);
        default: return std::nullopt;
    }
}

template <class F>
int guard(char* err, int errlen, F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        put_err(err, errlen, e.what());
        return 1;
    } catch (const std::overflow_error& e) {
        put_err(err, errlen, e.what());
        return 2;
    } catch (const std::exception& e) {
        put_err(err, errlen, e.what());
        return 3;
    }
}

}  // namespace

extern "C" {

// Similarity and penalty grids, size and scale() of a reference matrix.
int ref_matrix_tables(int matrix_id, const int32_t* sim_in, int size_in, int32_t* sim_out,
                      int32_t* pen_out, int* size_out, int32_t* scale_out) {
    auto m = make(matrix_id, sim_in, size_in);
    if (!m) return 1;
    const int A = m->size();
    *size_out = A;
    *scale_out = m->scale();
    for (int a = 0; a < A; ++a)
        for (int b = 0; b < A; ++b) {
            sim_out[a * A + b] = m->similarity(uint8_t(a), uint8_t(b));
            pen_out[a * A + b] = m->penalty(uint8_t(a), uint8_t(b));
        }
    return 0;
}

// seqtree::gapblock_matrix (include/seqtree/seqtree.hpp:218-222).  matrix_id < 0 = unit cost
// (null matrix).
int ref_gapblock_matrix(const char* qb, const int64_t* qo, int64_t nq, const char* rb,
                        const int64_t* ro, int64_t nr, int alphabet, int matrix_id,
                        const int32_t* sim, int size, int32_t gap_open, int32_t gap_extend,
                        const int32_t* prior, int64_t prior_len, uint32_t prior_width,
                        int threads, int32_t* out, char* err, int errlen) {
    return guard(err, errlen, [&] {
        auto q = unpack(qb, qo, nq), r = unpack(rb, ro, nr);
        auto m = matrix_id >= 0 ? make(matrix_id, sim, size) : std::nullopt;
        std::vector<int32_t> p(prior, prior + prior_len);
        auto res = gapblock_matrix(q, r, Alphabet(alphabet), m ? &*m : nullptr, gap_open,
                                   gap_extend, p, prior_width, threads);
        std::memcpy(out, res.data(), res.size() * sizeof(int32_t));
    });
}

// seqtree::align_score_matrix / align_dist_matrix (seqtree.hpp:198-209).
int ref_align_matrix(const char* qb, const int64_t* qo, int64_t nq, const char* rb,
                     const int64_t* ro, int64_t nr, int alphabet, int matrix_id,
                     const int32_t* sim, int size, int local, int32_t gap_open,
                     int32_t gap_extend, int dist, int threads, int32_t* out, char* err,
                     int errlen) {
    return guard(err, errlen, [&] {
        auto q = unpack(qb, qo, nq), r = unpack(rb, ro, nr);
        auto m = make(matrix_id, sim, size);
        if (!m) throw std::invalid_argument("bad matrix id");
        const AlignMode md = local ? AlignMode::Local : AlignMode::Global;
        auto res = dist ? align_dist_matrix(q, r, *m, Alphabet(alphabet), md, gap_open,
                                            gap_extend, threads)
                        : align_score_matrix(q, r, *m, Alphabet(alphabet), md, gap_open,
                                             gap_extend, threads);
        std::memcpy(out, res.data(), res.size() * sizeof(int32_t));
    });
}

// seqtree::align_score (seqtree.hpp:187-188).
int ref_align_score(const char* q, int64_t m, const char* r, int64_t n, int alphabet,
                    int matrix_id, const int32_t* sim, int size, int local, int32_t gap_open,
                    int32_t gap_extend, int32_t* out, char* err, int errlen) {
    return guard(err, errlen, [&] {
        auto mat = make(matrix_id, sim, size);
        if (!mat) throw std::invalid_argument("bad matrix id");
        *out = align_score(std::string_view(q, size_t(m)), std::string_view(r, size_t(n)), *mat,
                           Alphabet(alphabet), local ? AlignMode::Local : AlignMode::Global,
                           gap_open, gap_extend);
    });
}

// seqtree::align_pair (seqtree.hpp:190-192, src/pairwise.cpp:141-267): score plus the aligned
// strings and ops, each written NUL-terminated into a caller buffer of `cap` bytes.
int ref_align_pair(const char* q, int64_t m, const char* r, int64_t n, int alphabet, int matrix_id,
                   const int32_t* sim, int size, int local, int32_t gap_open, int32_t gap_extend,
                   int32_t* score, char* aq, char* ar, char* ops, int64_t cap, char* err,
                   int errlen) {
    return guard(err, errlen, [&] {
        auto mat = make(matrix_id, sim, size);
        if (!mat) throw std::invalid_argument("bad matrix id");
        const Alignment al = align_pair(std::string_view(q, size_t(m)), std::string_view(r, size_t(n)),
                                        *mat, Alphabet(alphabet),
                                        local ? AlignMode::Local : AlignMode::Global, gap_open,
                                        gap_extend);
        *score = al.score;
        for (auto [dst, src] : {std::pair<char*, const std::string*>{aq, &al.aligned_query},
                                {ar, &al.aligned_ref}, {ops, &al.ops}}) {
            const size_t len = std::min(src->size(), size_t(cap - 1));
            std::memcpy(dst, src->data(), len);
            dst[len] = 0;
        }
    });
}

// seqtree::Index::align (src/index.cpp:105-179): builds an Index over the packed refs, then
// aligns `q` to reference `ref_id`.  matrix_id < 0 is unit cost (a null matrix); the strings go
// NUL-terminated into caller buffers of `cap` bytes.
int ref_index_align(const char* rb, const int64_t* ro, int64_t nr, int alphabet, int64_t ref_id,
                    const char* q, int64_t m, int matrix_id, const int32_t* sim, int size,
                    int32_t gap_open, int32_t gap_extend, int32_t* score, char* aq, char* ar,
                    char* ops, int64_t cap, char* err, int errlen) {
    return guard(err, errlen, [&] {
        auto idx = Index::build(unpack(rb, ro, nr), Alphabet(alphabet));
        std::optional<SubstitutionMatrix> mat;
        if (matrix_id >= 0) {
            mat = make(matrix_id, sim, size);
            if (!mat) throw std::invalid_argument("bad matrix id");
        }
        SearchParams p;
        p.gap_open = gap_open;
        p.gap_extend = gap_extend;
        p.matrix = mat ? &*mat : nullptr;
        const Alignment al = idx->align(std::string_view(q, size_t(m)), uint32_t(ref_id), p);
        *score = al.score;
        for (auto [dst, src] : {std::pair<char*, const std::string*>{aq, &al.aligned_query},
                                {ar, &al.aligned_ref}, {ops, &al.ops}}) {
            const size_t len = std::min(src->size(), size_t(cap - 1));
            std::memcpy(dst, src->data(), len);
            dst[len] = 0;
        }
    });
}

// seqtree::hamming_matrix / levenshtein_matrix (seqtree.hpp:234-242).
int ref_distance_matrix(const char* ab, const int64_t* ao, int64_t na, const char* bb,
                        const int64_t* bo, int64_t nb, int levenshtein, int threads,
                        int32_t* out, char* err, int errlen) {
    return guard(err, errlen, [&] {
        auto a = unpack(ab, ao, na), b = unpack(bb, bo, nb);
        auto res = levenshtein ? levenshtein_matrix(a, b, threads) : hamming_matrix(a, b, threads);
        std::memcpy(out, res.data(), res.size() * sizeof(int32_t));
    });
}

}  // extern "C"
