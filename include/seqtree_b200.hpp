// seqtree_b200.hpp -- C++ form of the all-vs-all scoring calls, header-only over the C ABI.
//
// Mirrors the dense-matrix part of seqtree 0.6.0's public C++ API
// (include/seqtree/seqtree.hpp:186-242 and include/seqtree/types.hpp:9) with the same names,
// argument order, defaults, result layout and exception types, in namespace seqtree_b200.  A
// C++ caller switches by changing the include and the namespace:
//
//     #include <seqtree/seqtree.hpp>        ->  #include "seqtree_b200.hpp"
//     seqtree::gapblock_matrix(...)         ->  seqtree_b200::gapblock_matrix(...)
//
// and links libseqtree_b200.so.  The work runs on the current CUDA device; `threads` is kept
// for signature parity and ignored.  Errors: std::invalid_argument (bad input, same messages
// as the reference), std::overflow_error (a score does not fit int32), std::bad_alloc (device or
// pinned memory exhausted), std::runtime_error (CUDA errors, no device).
#ifndef SEQTREE_B200_HPP
#define SEQTREE_B200_HPP

#include <algorithm>
#include <cstdint>
#include <new>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "seqtree_b200.h"

namespace seqtree_b200 {

// seqtree::Alphabet (include/seqtree/types.hpp:9); the values are the C ABI's ST_ALPHABET_*.
enum class Alphabet : uint8_t { AminoAcid, Nucleotide, NucleotideIUPAC };

// seqtree::AlignMode (include/seqtree/seqtree.hpp:186); the values are ST_MODE_*.
enum class AlignMode { Global, Local };

namespace detail {

inline void check(int32_t rc, const st_error& err) {
    if (rc == ST_OK) return;
    if (rc == ST_EINVAL) throw std::invalid_argument(err.message);
    if (rc == ST_EOVERFLOW) throw std::overflow_error(err.message);
    if (rc == ST_ENOMEM) throw std::bad_alloc();
    throw std::runtime_error(err.message);
}

// One st_strings view over a list of strings (bytes concatenated, count+1 offsets).
struct Packed {
    std::string bytes;
    std::vector<int64_t> offsets;
    st_strings view{};

    template <class Seq>
    explicit Packed(const Seq& seqs) {
        size_t total = 0;
        for (const auto& s : seqs) total += std::string_view(s).size();
        bytes.reserve(total);
        offsets.reserve(seqs.size() + 1);
        offsets.push_back(0);
        for (const auto& s : seqs) {
            bytes.append(std::string_view(s));
            offsets.push_back(static_cast<int64_t>(bytes.size()));
        }
        view = st_strings{bytes.data(), offsets.data(), static_cast<int64_t>(seqs.size())};
    }
};

}  // namespace detail

// seqtree::SubstitutionMatrix (include/seqtree/seqtree.hpp:43-82): a penalty view (>= 0, zero
// diagonal; what the gap-block matrix minimises) and the raw similarity (what Needleman-Wunsch
// and Smith-Waterman maximise).  Built-ins come from the library's copy of the same grids.
class SubstitutionMatrix {
public:
    // 0 for a match, 1 for a mismatch; similarity +1 on the diagonal, 0 elsewhere.
    static SubstitutionMatrix unit(uint8_t size) {
        SubstitutionMatrix m;
        m.size_ = size;
        m.pen_.assign(size_t(size) * size, 1);
        m.sim_.assign(size_t(size) * size, 0);
        for (uint8_t i = 0; i < size; ++i) {
            m.pen_[size_t(i) * size + i] = 0;
            m.sim_[size_t(i) * size + i] = 1;
        }
        return m;
    }
    static SubstitutionMatrix blosum62() { return builtin("blosum62"); }
    static SubstitutionMatrix blosum45() { return builtin("blosum45"); }
    static SubstitutionMatrix blosum80() { return builtin("blosum80"); }
    static SubstitutionMatrix pam250() { return builtin("pam250"); }
    static SubstitutionMatrix pam100() { return builtin("pam100"); }
    static SubstitutionMatrix structural() { return builtin("structural"); }

    // Penalty by the Gram / squared-distance transform, clamped at zero:
    // pen(a,b) = max(0, sim(a,a) + sim(b,b) - 2 sim(a,b)).  The similarity is kept as given.
    static SubstitutionMatrix from_similarity(uint8_t size, const int32_t* sim) {
        SubstitutionMatrix m;
        m.size_ = size;
        m.sim_.assign(sim, sim + size_t(size) * size);
        m.pen_.resize(size_t(size) * size);
        for (size_t a = 0; a < size; ++a)
            for (size_t b = 0; b < size; ++b) {
                int32_t p = sim[a * size + a] + sim[b * size + b] - 2 * sim[a * size + b];
                m.pen_[a * size + b] = p < 0 ? 0 : p;
            }
        return m;
    }

    uint8_t size() const { return size_; }
    int32_t penalty(uint8_t a, uint8_t b) const { return pen_[size_t(a) * size_ + b]; }
    int32_t similarity(uint8_t a, uint8_t b) const { return sim_[size_t(a) * size_ + b]; }
    // Median off-diagonal penalty (the upper median of the size*(size-1) values).
    int32_t scale() const {
        if (size_ < 2) return 0;
        std::vector<int32_t> off;
        off.reserve(size_t(size_) * (size_ - 1));
        for (size_t a = 0; a < size_; ++a)
            for (size_t b = 0; b < size_; ++b)
                if (a != b) off.push_back(pen_[a * size_ + b]);
        auto mid = off.begin() + off.size() / 2;
        std::nth_element(off.begin(), mid, off.end());
        return *mid;
    }

    const int32_t* penalty_data() const { return pen_.data(); }
    const int32_t* similarity_data() const { return sim_.data(); }

private:
    static SubstitutionMatrix builtin(const char* name) {
        std::vector<int32_t> sim(24 * 24);
        int32_t size = 0;
        st_error err{};
        detail::check(st_builtin_similarity(name, sim.data(), int32_t(sim.size()), &size, &err),
                      err);
        return from_similarity(static_cast<uint8_t>(size), sim.data());
    }

    uint8_t size_ = 0;
    std::vector<int32_t> pen_;
    std::vector<int32_t> sim_;
};

// Dense N*K similarity matrix, row-major.  seqtree::align_score_matrix
// (include/seqtree/seqtree.hpp:198-201).
inline std::vector<int32_t> align_score_matrix(const std::vector<std::string>& queries,
                                               const std::vector<std::string>& refs,
                                               const SubstitutionMatrix& m, Alphabet alphabet,
                                               AlignMode mode, int32_t gap_open,
                                               int32_t gap_extend, int threads = 0) {
    detail::Packed q(queries), r(refs);
    std::vector<int32_t> out(queries.size() * refs.size());
    st_error err{};
    detail::check(st_align_score_matrix(&q.view, &r.view, m.similarity_data(), m.size(),
                                        int32_t(alphabet), int32_t(mode), gap_open, gap_extend,
                                        threads, out.data(), &err),
                  err);
    return out;
}

// Dense N*K distance s(a,a) + s(b,b) - 2 s(a,b).  seqtree::align_dist_matrix
// (include/seqtree/seqtree.hpp:206-209).
inline std::vector<int32_t> align_dist_matrix(const std::vector<std::string>& queries,
                                              const std::vector<std::string>& refs,
                                              const SubstitutionMatrix& m, Alphabet alphabet,
                                              AlignMode mode, int32_t gap_open,
                                              int32_t gap_extend, int threads = 0) {
    detail::Packed q(queries), r(refs);
    std::vector<int32_t> out(queries.size() * refs.size());
    st_error err{};
    detail::check(st_align_dist_matrix(&q.view, &r.view, m.similarity_data(), m.size(),
                                       int32_t(alphabet), int32_t(mode), gap_open, gap_extend,
                                       threads, out.data(), &err),
                  err);
    return out;
}

// Optimal score of one pair.  seqtree::align_score (include/seqtree/seqtree.hpp:189-190); one
// 1x1 matrix launch, so batch pairs with align_score_matrix where possible.
inline int32_t align_score(std::string_view query, std::string_view ref,
                           const SubstitutionMatrix& m, Alphabet alphabet, AlignMode mode,
                           int32_t gap_open, int32_t gap_extend) {
    return align_score_matrix({std::string(query)}, {std::string(ref)}, m, alphabet, mode,
                              gap_open, gap_extend)[0];
}

// An alignment with its traceback.  seqtree::Alignment (include/seqtree/types.hpp:67-72).
struct Alignment {
    std::string aligned_query;
    std::string aligned_ref;
    std::string ops;  // per column: 'M' match, 'S' substitution, 'I' insertion, 'D' deletion
    int32_t score = 0;
};

// Optimal score plus the aligned strings and ops.  seqtree::align_pair
// (include/seqtree/seqtree.hpp:190-192): one traceback launch on the GPU; for many pairs use
// the batched st_align_pairs_sets.
inline Alignment align_pair(std::string_view query, std::string_view ref, const SubstitutionMatrix& m,
                            Alphabet alphabet, AlignMode mode, int32_t gap_open, int32_t gap_extend) {
    const size_t cap = query.size() + ref.size() + 1;
    std::string aq(cap, '\0'), ar(cap, '\0'), ops(cap, '\0');
    Alignment al;
    st_error err{};
    detail::check(st_align_pair(query.data(), int64_t(query.size()), ref.data(),
                                int64_t(ref.size()), m.similarity_data(), m.size(), int32_t(alphabet),
                                int32_t(mode), gap_open, gap_extend, &al.score, aq.data(),
                                ar.data(), ops.data(), int64_t(cap), &err),
                  err);
    al.aligned_query = aq.c_str();
    al.aligned_ref = ar.c_str();
    al.ops = ops.c_str();
    return al;
}

// Penalty-minimising global alignments of the pairs (queries[query_idx[p]], refs[ref_idx[p]]),
// one GPU launch for the batch.  seqtree::Index::align (include/seqtree/seqtree.hpp, Index;
// src/index.cpp:105-179) with `refs` as the index's references: `matrix` null means unit cost,
// gaps cost gap_open + (L-1) * gap_extend, and the aligned strings keep the callers' characters.
inline std::vector<Alignment> penalty_align_pairs(const std::vector<std::string>& queries,
                                                  const std::vector<std::string>& refs,
                                                  const std::vector<int32_t>& query_idx,
                                                  const std::vector<int32_t>& ref_idx,
                                                  Alphabet alphabet, const SubstitutionMatrix* matrix,
                                                  int32_t gap_open, int32_t gap_extend) {
    if (query_idx.size() != ref_idx.size())
        throw std::invalid_argument("query_idx and ref_idx must have the same length");
    detail::Packed q(queries), r(refs);
    size_t mq = 0, mr = 0;
    for (const auto& s : queries) mq = std::max(mq, s.size());
    for (const auto& s : refs) mr = std::max(mr, s.size());
    const size_t n = query_idx.size(), stride = mq + mr + 1;
    std::vector<int32_t> scores(n), lengths(n);
    std::string aq(std::max<size_t>(n * stride, 1), '\0'), ar(aq.size(), '\0'), ops(aq.size(), '\0');
    st_error err{};
    detail::check(st_penalty_align_pairs(&q.view, &r.view, query_idx.data(), ref_idx.data(),
                                         int64_t(n), int32_t(alphabet),
                                         matrix ? matrix->penalty_data() : nullptr,
                                         matrix ? matrix->size() : 0, gap_open, gap_extend,
                                         scores.data(), aq.data(), ar.data(), ops.data(),
                                         int64_t(stride), lengths.data(), &err),
                  err);
    std::vector<Alignment> out(n);
    for (size_t p = 0; p < n; ++p) {
        const size_t at = p * stride, len = size_t(lengths[p]);
        out[p].aligned_query.assign(aq, at, len);
        out[p].aligned_ref.assign(ar, at, len);
        out[p].ops.assign(ops, at, len);
        out[p].score = scores[p];
    }
    return out;
}

// One pair of penalty_align_pairs: Index::align(query, ref_id, params) for ref = ref_seq(ref_id).
inline Alignment penalty_align(std::string_view query, std::string_view ref,
                               const SubstitutionMatrix* matrix, Alphabet alphabet,
                               int32_t gap_open, int32_t gap_extend) {
    return penalty_align_pairs({std::string(query)}, {std::string(ref)}, {0}, {0}, alphabet,
                               matrix, gap_open, gap_extend)[0];
}

// Dense N*K single-gap-block penalty matrix.  seqtree::gapblock_matrix
// (include/seqtree/seqtree.hpp:215-222).  `matrix` null means unit cost; `prior` is the
// [m][d][i] cube with stride prior_width + 1, or empty for none.
inline std::vector<int32_t> gapblock_matrix(const std::vector<std::string>& queries,
                                            const std::vector<std::string>& refs,
                                            Alphabet alphabet, const SubstitutionMatrix* matrix,
                                            int32_t gap_open, int32_t gap_extend,
                                            const std::vector<int32_t>& prior,
                                            uint32_t prior_width, int threads = 0) {
    detail::Packed q(queries), r(refs);
    std::vector<int32_t> out(queries.size() * refs.size());
    st_error err{};
    detail::check(st_gapblock_matrix(&q.view, &r.view, int32_t(alphabet),
                                     matrix ? matrix->penalty_data() : nullptr,
                                     matrix ? matrix->size() : 0, gap_open, gap_extend,
                                     prior.empty() ? nullptr : prior.data(),
                                     int64_t(prior.size()), prior_width, threads, out.data(),
                                     &err),
                  err);
    return out;
}

// Dense N*K Hamming matrix (raw bytes, case-sensitive; throws on a length mismatch).
// seqtree::hamming_matrix (include/seqtree/seqtree.hpp:239-240).
inline std::vector<int32_t> hamming_matrix(const std::vector<std::string>& a,
                                           const std::vector<std::string>& b, int threads = 0) {
    detail::Packed pa(a), pb(b);
    std::vector<int32_t> out(a.size() * b.size());
    st_error err{};
    detail::check(st_hamming_matrix(&pa.view, &pb.view, threads, out.data(), &err), err);
    return out;
}

// Dense N*K Levenshtein matrix (raw bytes, unit costs).  seqtree::levenshtein_matrix
// (include/seqtree/seqtree.hpp:241-242).
inline std::vector<int32_t> levenshtein_matrix(const std::vector<std::string>& a,
                                               const std::vector<std::string>& b,
                                               int threads = 0) {
    detail::Packed pa(a), pb(b);
    std::vector<int32_t> out(a.size() * b.size());
    st_error err{};
    detail::check(st_levenshtein_matrix(&pa.view, &pb.view, threads, out.data(), &err), err);
    return out;
}

// One pair each (seqtree::hamming / seqtree::levenshtein, include/seqtree/seqtree.hpp:234-235);
// a 1x1 matrix launch.
inline int hamming(std::string_view a, std::string_view b) {
    return hamming_matrix({std::string(a)}, {std::string(b)})[0];
}
inline int levenshtein(std::string_view a, std::string_view b) {
    return levenshtein_matrix({std::string(a)}, {std::string(b)})[0];
}

}  // namespace seqtree_b200

#endif  // SEQTREE_B200_HPP
