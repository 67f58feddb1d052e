// Exercises the C++ API (include/seqtree_b200.hpp) the way a seqtree C++ caller would.
//
//   api_check tables   prints every built-in matrix (name, size, scale, penalty grid,
//                      similarity grid); needs no GPU.
//   api_check run      reads sets from stdin and prints each matrix call's result:
//                        Q n / n lines     queries (amino acids)
//                        R k / k lines     refs (amino acids)
//                        H h / h lines     equal-length strings for the Hamming call
//                        P width len / one line of len ints   the gap-prior cube
//                      output lines are "<call> v0 v1 ..." or "<call> !<exception>: <what>".
#include <algorithm>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "seqtree_b200.hpp"

namespace st = seqtree_b200;

static void emit(const std::string& name, const std::vector<int32_t>& v) {
    std::cout << name;
    for (int32_t x : v) std::cout << ' ' << x;
    std::cout << '\n';
}

template <class F>
static void call(const std::string& name, F&& f) {
    try {
        emit(name, f());
    } catch (const std::invalid_argument& e) {
        std::cout << name << " !invalid_argument: " << e.what() << '\n';
    } catch (const std::overflow_error& e) {
        std::cout << name << " !overflow_error: " << e.what() << '\n';
    } catch (const std::exception& e) {
        std::cout << name << " !other: " << e.what() << '\n';
    }
}

static std::vector<std::string> read_set(std::istream& in, char tag) {
    std::string line;
    std::getline(in, line);
    std::istringstream head(line);
    char t = 0;
    size_t n = 0;
    head >> t >> n;
    if (t != tag) throw std::runtime_error(std::string("expected set ") + tag);
    std::vector<std::string> v(n);
    for (auto& s : v) std::getline(in, s);
    return v;
}

int main(int argc, char** argv) {
    std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "tables") {
        const std::pair<const char*, st::SubstitutionMatrix (*)()> all[] = {
            {"blosum62", st::SubstitutionMatrix::blosum62},
            {"blosum45", st::SubstitutionMatrix::blosum45},
            {"blosum80", st::SubstitutionMatrix::blosum80},
            {"pam250", st::SubstitutionMatrix::pam250},
            {"pam100", st::SubstitutionMatrix::pam100},
            {"structural", st::SubstitutionMatrix::structural}};
        for (auto& [name, make] : all) {
            st::SubstitutionMatrix m = make();
            std::vector<int32_t> v{m.size(), m.scale()};
            for (int a = 0; a < m.size(); ++a)
                for (int b = 0; b < m.size(); ++b) v.push_back(m.penalty(a, b));
            for (int a = 0; a < m.size(); ++a)
                for (int b = 0; b < m.size(); ++b) v.push_back(m.similarity(a, b));
            emit(name, v);
        }
        st::SubstitutionMatrix u = st::SubstitutionMatrix::unit(4);
        emit("unit4", {u.size(), u.scale(), u.penalty(0, 1), u.penalty(2, 2), u.similarity(1, 1),
                       u.similarity(1, 2)});
        return 0;
    }
    if (mode != "run") {
        std::cerr << "usage: api_check tables|run\n";
        return 2;
    }
    auto q = read_set(std::cin, 'Q');
    auto r = read_set(std::cin, 'R');
    auto h = read_set(std::cin, 'H');
    std::string line;
    std::getline(std::cin, line);
    std::istringstream ph(line);
    char t = 0;
    uint32_t width = 0;
    size_t len = 0;
    ph >> t >> width >> len;
    std::vector<int32_t> prior(len);
    for (auto& x : prior) std::cin >> x;

    const st::SubstitutionMatrix b62 = st::SubstitutionMatrix::blosum62();
    const auto AA = st::Alphabet::AminoAcid;
    call("gapblock_b62_prior", [&] { return st::gapblock_matrix(q, r, AA, &b62, 8, 1, prior, width); });
    call("gapblock_unit", [&] { return st::gapblock_matrix(q, r, AA, nullptr, 1, 1, {}, 0); });
    call("align_score_global", [&] {
        return st::align_score_matrix(q, r, b62, AA, st::AlignMode::Global, 11, 1);
    });
    call("align_dist_local", [&] {
        return st::align_dist_matrix(q, r, b62, AA, st::AlignMode::Local, 11, 1);
    });
    call("align_score_one", [&] {
        return std::vector<int32_t>{
            st::align_score(q[0], r[0], b62, AA, st::AlignMode::Global, 11, 1)};
    });
    call("levenshtein", [&] { return st::levenshtein_matrix(q, r); });
    call("levenshtein_one", [&] { return std::vector<int32_t>{st::levenshtein(q[0], r[0])}; });
    call("hamming", [&] { return st::hamming_matrix(h, h); });
    call("hamming_one", [&] { return std::vector<int32_t>{st::hamming(h[0], h[1])}; });
    call("hamming_ragged", [&] { return st::hamming_matrix({"ABC"}, {"ABCD"}); });
    call("gapblock_bad_symbol", [&] {
        return st::gapblock_matrix({"CASJ"}, r, AA, &b62, 8, 1, {}, 0);
    });
    call("align_overflow", [&] {
        return st::align_score_matrix({"AAAA"}, {"AAAAAAAA"}, b62, AA, st::AlignMode::Global,
                                      1500000000, 1500000000);
    });
    // align_pair: "alignpair <i> <mode> <score> <aligned_query> <aligned_ref> <ops>" (strings
    // never hold spaces; an empty one prints as "~")
    auto show = [](const std::string& s) { return s.empty() ? std::string("~") : s; };
    for (size_t i = 0; i < std::min<size_t>(q.size(), r.size()); ++i)
        for (int md = 0; md < 2; ++md) {
            try {
                const st::Alignment al = st::align_pair(q[i], r[i], b62, AA, md ? st::AlignMode::Local
                                                                             : st::AlignMode::Global,
                                                        11, 1);
                std::cout << "alignpair " << i << ' ' << md << ' ' << al.score << ' '
                          << show(al.aligned_query) << ' ' << show(al.aligned_ref) << ' '
                          << show(al.ops) << '\n';
            } catch (const std::exception& e) {
                std::cout << "alignpair " << i << ' ' << md << " !" << e.what() << '\n';
            }
        }
    // Index::align: "penalign <i> <score> <aligned_query> <aligned_ref> <ops>", BLOSUM62 for
    // even i, unit cost for odd i
    for (size_t i = 0; i < std::min<size_t>(q.size(), r.size()); ++i) {
        const st::Alignment al = st::penalty_align_pairs(q, r, {int32_t(i)}, {int32_t(i)}, AA,
                                                         (i & 1) ? nullptr : &b62, 11, 1)[0];
        std::cout << "penalign " << i << ' ' << al.score << ' ' << show(al.aligned_query) << ' '
                  << show(al.aligned_ref) << ' ' << show(al.ops) << '\n';
    }
    call("penalty_align_bad_symbol", [&] {
        return std::vector<int32_t>{st::penalty_align("CASJ", "CASS", nullptr, AA, 1, 1).score};
    });
    call("align_pair_bad_symbol", [&] {
        return std::vector<int32_t>{st::align_pair("CASJ", "CASS", b62, AA, st::AlignMode::Global,
                                                   11, 1).score};
    });
    return 0;
}
