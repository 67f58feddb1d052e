"""Host-side logic of the Python mirror: priors and the prior cube, matrices, the result
buffer, argument parsing and packing.  No device needed."""
from __future__ import annotations

import numpy as np
import pytest

from seqtree_b200 import _lib
from seqtree_b200.gapblock import (UNREACHABLE, central_prior, frame_prior, gap_cost,
                                   positions_prior, prior_cube, profile_prior)
from seqtree_b200.matrix import (ScoreMatrix, SubstitutionMatrix, alphabet_symbols, amino_acids,
                                 parse_align_mode, parse_alphabet)


def test_alphabet_and_mode_names():
    assert [parse_alphabet(a) for a in ("aa", "AMINO", "protein", "nt", "dna", "nucleotide",
                                        "iupac", "nt_iupac")] == [0, 0, 0, 1, 1, 1, 2, 2]
    with pytest.raises(ValueError, match="unknown alphabet"):
        parse_alphabet("rna")
    assert [parse_align_mode(m) for m in ("global", "NW", "needleman-wunsch", "local", "sw",
                                          "Smith-Waterman")] == [0, 0, 0, 1, 1, 1]
    with pytest.raises(ValueError, match="mode"):
        parse_align_mode("semiglobal")
    assert amino_acids() == "ARNDCQEGHILKMFPSTWYVBZX*" and alphabet_symbols("nt") == "ACGT"


def test_prior_cube_layout_and_checks():
    cp = central_prior(21)
    cube = prior_cube(cp, 6)
    w1 = 7
    for m in range(w1):
        for d in range(1, m + 1):
            for i in range(m - d + 1):
                assert cube[(m * w1 + d) * w1 + i] == cp(i, d, m)
    assert all(cube[(m * w1) * w1 + i] == 0 for m in range(w1) for i in range(w1))
    with pytest.raises(ValueError, match="negative"):
        prior_cube(lambda i, d, m: -1, 3)
    with pytest.raises(ValueError):
        central_prior(-1)
    with pytest.raises(ValueError):
        frame_prior(1, -1)
    with pytest.raises(ValueError):
        positions_prior(())
    assert profile_prior(10, [0.5] * 8)(1, 2, 8) == 10
    assert positions_prior((2,))(0, 1, 5) == UNREACHABLE
    assert gap_cost(2, 8, 1) == 9


def test_priors_vanish_without_a_gap():
    for p in (central_prior(20), frame_prior(21, 5), positions_prior((3, 4, -4, -3)),
              profile_prior(21, lambda j, m: 1.0)):
        for m in range(1, 12):
            assert p(0, 0, m) == 0


def test_substitution_matrix_views_and_errors():
    m = SubstitutionMatrix.blosum62()
    assert m.size() == 24 and m.similarity("A", "K") < 0 < m.penalty("A", "K")
    assert m.penalty("W", "W") == m.penalty("C", "C") == 0
    with pytest.raises(ValueError):
        m.penalty("AA", "A")
    with pytest.raises(ValueError, match="unknown amino acid"):
        m.penalty("J", "A")
    small = SubstitutionMatrix.unit(4)
    with pytest.raises(ValueError, match="out of range"):
        small.similarity("C", "G")  # index 4 in the amino-acid order
    with pytest.raises(ValueError, match="square"):
        SubstitutionMatrix.from_similarity([[1, 2], [3]])
    with pytest.raises(ValueError):
        SubstitutionMatrix.from_similarity([])
    c = SubstitutionMatrix.from_similarity([[5, -1], [-1, 3]])
    assert c.penalty_grid.tolist() == [[0, 10], [10, 0]]
    assert SubstitutionMatrix.unit(1).scale() == 0


def test_score_matrix_buffer_protocol_and_indexing():
    a = np.arange(6, dtype=np.int32).reshape(2, 3)
    sm = ScoreMatrix(a)
    mv = memoryview(sm)
    assert mv.format == "i" and mv.shape == (2, 3) and mv.c_contiguous and mv.readonly
    assert np.asarray(sm).tolist() == a.tolist()
    assert sm.shape == (2, 3) and len(sm) == 2 and sm[1, 2] == 5 and sm.row(0) == [0, 1, 2]
    with pytest.raises(IndexError):
        sm.row(2)
    with pytest.raises(IndexError):
        sm[2, 0]
    with pytest.raises(IndexError):
        sm[0, 3]
    assert repr(sm) == "ScoreMatrix(2, 3)"
    # the reference binds row(size_t) and __getitem__(pair<size_t, size_t>): pybind11 turns an
    # argument it cannot convert (negative, float, not a pair) into TypeError, and accepts any
    # integer-like value or a two-element list
    assert sm.row(np.int64(1)) == [3, 4, 5] and sm[[1, 2]] == 5 and sm[np.int32(1), 2] == 5
    for bad in (lambda: sm.row(-1), lambda: sm.row(1.0), lambda: sm[-1, 0], lambda: sm[0],
                lambda: sm[0, 1, 2], lambda: sm[1.0, 0], lambda: sm["ab"]):
        with pytest.raises(TypeError):
            bad()


def test_packing_offsets_and_utf8():
    p = _lib.Packed(["CASS", "", "AB"])
    assert p.offsets.tolist() == [0, 4, 4, 6] and bytes(p.data[:6]) == b"CASSAB"
    p = _lib.Packed(["é", "ab"])  # byte lengths, as the reference's std::string sees them
    assert p.offsets.tolist() == [0, 2, 4]
    with pytest.raises(TypeError):
        _lib.Packed([1, 2])


@pytest.mark.parametrize("seqs", [["CASS", "", "AB"], [""], ["", ""], ["ACDEFGHIKLMNPQRSTVWY"] * 3,
                                  ["A\nB", "C"], ["\n"], ["A", "B\n"], [b"AC", "D"], ["é", "a"]])
def test_joined_packing_matches_the_general_path(seqs):
    """The newline-joined fast path (``st_split_joined``, host code) and the per-string path give
    the same bytes and offsets; strings with a newline, bytes items and non-ASCII text take the
    general path."""
    fast = _lib._pack_ascii(list(seqs))
    enc = [s if isinstance(s, bytes) else s.encode() for s in seqs]
    want_off = np.concatenate([[0], np.cumsum([len(e) for e in enc])])
    if fast is None:
        assert any(b"\n" in e for e in enc) or any(isinstance(s, bytes) for s in seqs) or \
            any(not s.isascii() for s in seqs if isinstance(s, str))
    else:
        assert fast[1].tolist() == want_off.tolist()
        assert bytes(fast[0][:want_off[-1]]) == b"".join(enc)
    p = _lib.pack(seqs)
    assert p.offsets.tolist() == want_off.tolist() and _lib.pack(p) is p
    assert p.max_len == max(len(e) for e in enc)


@pytest.mark.parametrize("seqs", [["CASS", "", "AB"], [""], [], ["ACDEFGHIKLMNPQRSTVWY"] * 3,
                                  ["A\nB", "C"], ["\n"], [b"AC", "D"], ["é", "a"], [1, "A"]])
def test_list_packer_extension_matches_the_general_path(seqs):
    """seqtree_b200._pack (csrc/pack_py.c) packs lists of ASCII str in one pass -- newlines
    included -- into the bytes and offsets of the per-string path, and declines (None) anything
    else, which then takes the general path."""
    from seqtree_b200 import _pack
    got = _pack.pack(list(seqs))
    if any(not isinstance(s, str) or not s.isascii() for s in seqs):
        assert got is None
        return
    enc = [s.encode() for s in seqs]
    want_off = np.concatenate([[0], np.cumsum([len(e) for e in enc])]).astype(np.int64)
    data, off = np.frombuffer(got[0], np.uint8), np.frombuffer(got[1], np.int64)
    assert off.tolist() == want_off.tolist() and bytes(data[:want_off[-1]]) == b"".join(enc)
    assert data.size >= 1
    assert _pack.pack(tuple(seqs)) is None  # lists only; other sequences are listed first


def test_builtin_prior_cubes_are_memoised_read_only():
    cp = central_prior(7)
    a, b = prior_cube(cp, 9), prior_cube(cp, 9)
    assert a is b and not a.flags.writeable and a.dtype == np.int32
    assert prior_cube(cp, 4) is not a and prior_cube(central_prior(7), 9) is not a
    assert (a == prior_cube(central_prior(7), 9)).all()


def test_pinned_results_are_plain_int32_arrays():
    a = _lib.pinned_int32(3, 4)
    assert a.shape == (3, 4) and a.dtype == np.int32 and a.flags.c_contiguous
    a[:] = 7
    v = a[1:]
    del a
    assert int(v.sum()) == 7 * 8


def test_penalty_alignment_matrix_argument_like_search_params():
    """``penalty_align``'s matrix argument follows seqtree's SearchParams (src/_bindings.cpp:
    67-119): None or '' is unit cost, built-in names are case-insensitive, 'identity' is the unit
    grid of the alphabet, the others need amino acids, anything else is refused -- all checked
    on the host before the library is called."""
    from seqtree_b200.pairwise import _penalty_grid
    assert _penalty_grid(None, "aa") is None and _penalty_grid("", "aa") is None
    b62 = SubstitutionMatrix.blosum62().penalty_grid
    assert np.array_equal(_penalty_grid("BLOSUM62", "aa"), b62)
    assert np.array_equal(_penalty_grid(SubstitutionMatrix.blosum62(), "aa"), b62)
    assert np.array_equal(_penalty_grid("identity", "nt"), 1 - np.eye(4, dtype=np.int32))
    with pytest.raises(ValueError, match="unknown matrix 'BLOSUM99'"):
        _penalty_grid("BLOSUM99", "aa")
    with pytest.raises(ValueError, match="requires the amino-acid alphabet"):
        _penalty_grid("pam250", "nt")
    with pytest.raises(TypeError, match="name string or a SubstitutionMatrix"):
        _penalty_grid(3, "aa")


def test_integer_arguments_convert_like_the_reference_binding():
    """int32_t / uint32_t arguments of the reference binding reject floats, strings, None and
    out-of-range values with TypeError (pybind11 never truncates or parses); the checks run on
    the host before the library computes anything."""
    from seqtree_b200 import _core
    b62 = SubstitutionMatrix.blosum62()
    calls = [lambda: _core.gapblock_matrix(["A"], ["A"], gap_open=1.5),
             lambda: _core.gapblock_matrix(["A"], ["A"], gap_extend=2 ** 31),
             lambda: _core.gapblock_matrix(["A"], ["A"], prior_width=-1),
             lambda: _core.gapblock_matrix(["A"], ["A"], threads=0.5),
             lambda: _core.align_score_matrix(["A"], ["A"], b62, gap_open="11"),
             lambda: _core.align_dist_matrix(["A"], ["A"], b62, threads=None),
             lambda: _core.hamming_matrix(["A"], ["A"], threads=1.0),
             lambda: _core.levenshtein_matrix(["A"], ["A"], threads="0")]
    for call in calls:
        with pytest.raises(TypeError):
            call()
    assert _core._i32("gap_open", np.int64(8)) == 8 and _core._u32("w", np.uint8(25)) == 25


def test_threshold_tile_ranges_cover_every_cell_that_is_on():
    """range_tile_ranges: a 256-query tile scans the 128-ref tiles holding every ref length with a
    finite threshold for one of the tile's query lengths, and nothing for a tile without one."""
    from seqtree_b200.learned import range_tile_ranges
    rng = np.random.default_rng(3)
    q = np.sort(rng.integers(8, 26, size=1000))
    r = np.sort(rng.integers(8, 26, size=5000))
    thr = np.full((33, 33), np.inf, np.float32)
    for a in range(33):
        thr[a, max(0, a - 1):a + 2] = 0.5  # lengths within one residue
    thr[8:11, :] = np.inf                  # short queries: no proposals
    out = range_tile_ranges(q, r, thr)
    assert out.shape == (4, 2) and out.dtype == np.int32
    for t in range(4):
        blk = q[256 * t:256 * (t + 1)]
        on = np.isfinite(thr[blk.min():blk.max() + 1]).any(axis=0)
        need = np.flatnonzero(on[r])
        if need.size == 0:
            assert out[t, 0] == out[t, 1]
            continue
        assert out[t, 0] * 128 <= need.min() and need.max() < out[t, 1] * 128
        assert out[t, 1] * 128 - need.max() <= 128 and need.min() - out[t, 0] * 128 < 128
    assert (range_tile_ranges(q, r, np.full((33, 33), np.inf)) == 0).all()


def test_recall_allocation_prefers_cheap_proposals_and_falls_back_where_they_are_dear():
    """allocate_recall: a cell whose proposals recover hits cheaply gets them, a query length
    whose cells would need more candidates than exhaustive scoring costs falls back, and the
    estimated recall reaches the target."""
    from seqtree_b200.learned import allocate_recall
    S, LV = 4, 3
    wq = np.array([0, 100, 100, 0], float)
    wr = np.array([0, 1000, 1000, 0], float)
    E = np.zeros((S, S))
    E[1, 1], E[1, 2], E[2, 2] = 500, 400, 50      # short queries (length 1) carry most hits
    FL = np.zeros((S, S, LV))
    CL = np.zeros((S, S, LV))
    FL[1, 1], CL[1, 1] = [250, 400, 490], [5e4, 8e4, 1e5]   # dear: half of all pairs
    FL[1, 2], CL[1, 2] = [200, 300, 390], [5e4, 8e4, 1e5]
    FL[2, 2], CL[2, 2] = [40, 48, 50], [10, 30, 100]        # cheap
    costs = {"exhaustive": 1e-9, "scan": 1e-11, "candidate": 1e-8}
    level, qf, rf, rec, est = allocate_recall(E, FL, CL, wq, wr, costs, 0.99)
    assert qf == [1] and rf == []
    assert level[2, 2] >= 1 and (level[1] == -1).all()
    assert rec >= 0.99 and est > 0
    # with free candidates nothing falls back and every cell with hits gets proposals
    cheap = dict(costs, candidate=0.0)
    level, qf, rf, rec, _ = allocate_recall(E, FL, CL, wq, wr, cheap, 0.95)
    assert qf == [] and rf == [] and rec >= 0.95 and (level[E > 0] >= 0).all()


def test_long_indel_share_of_near_neighbour_pairs():
    """training_pairs_codes: the default pairs are unchanged by the long-block option, and with
    long_share > 0 that share of the near-neighbour pairs differs in length by 4..long_max
    residues (insertions capped at 32 residues)."""
    from seqtree_b200 import learned as L
    c0, l0 = L.training_pairs_codes(11, 4000)
    c1, l1 = L.training_pairs_codes(11, 4000, 0.0)
    assert np.array_equal(c0, c1) and np.array_equal(l0, l1)
    c, ln = L.training_pairs_codes(11, 20000, 0.5, 12)
    d = np.abs(ln[0::2] - ln[1::2])[:10000]  # the near-neighbour half
    assert d.max() == 12 and 0.3 < np.mean(d >= 4) < 0.55
    assert ln.min() >= 1 and ln.max() <= 32
    assert ((c[np.arange(32)[None, :] >= ln[:, None]]) == 0).all()


def test_gather_rows_of_a_packed_set():
    """learned.gather_rows: the listed rows' bytes and offsets, in the listed order (empty rows and
    repeats included), as concatenating the strings would give."""
    from seqtree_b200.learned import gather_rows
    seqs = ["CASSLF", "", "CAW", "CASSPGQAYEQYF", "A"]
    p = _lib.Packed(seqs)
    from seqtree_b200 import _lib as lib
    ext = lib._pack
    try:
        for use_ext in (True, False):  # the extension's copy and the numpy fallback
            lib._pack = ext if use_ext else None
            for rows in ([4, 0, 3], [1, 1, 2], [], list(range(5))[::-1]):
                data, off = gather_rows(p.data, p.offsets, np.array(rows, np.int64))
                want = [seqs[i] for i in rows]
                assert off.tolist() == np.concatenate(
                    [[0], np.cumsum([len(x) for x in want])]).tolist()
                assert bytes(data[:off[-1]]) == "".join(want).encode()
    finally:
        lib._pack = ext
    with pytest.raises(IndexError):
        gather_rows(p.data, p.offsets, np.array([5], np.int64))
