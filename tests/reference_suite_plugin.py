"""pytest plugin that runs the reference's own hot-path test files against this library.

Loaded with ``-p reference_suite_plugin`` before collection, it installs ``seqtree``,
``seqtree.gapblock``, ``seqtree.pairwise``, ``seqtree.distance`` and ``seqtree.evalue`` as this
library's modules, so a
reference test's ``import seqtree`` / ``from seqtree.gapblock import ...`` binds the drop-in's
names, defaults, exceptions and buffers unchanged.  The test files themselves are not part of this
repository: ``tests/test_reference_suite_gpu.py`` points pytest at a copy of the reference's
``tests/python`` directory.

Tests that exercise what the drop-in does not replace -- the trie ``Index`` and its
``SearchParams`` engines -- are skipped by name below, each with its reason.  BioPython-based
comparisons skip themselves (``pytest.importorskip``) where BioPython is not installed.
"""
from __future__ import annotations

import sys
import types

import pytest

OUT_OF_SCOPE = "uses the trie Index / SearchParams engines, which the drop-in does not replace"
SKIP = {
    "test_pairwise.py::test_named_matrices_reach_the_search_path_too": OUT_OF_SCOPE,
    "test_matrix.py::test_named_matrix_exact_match_is_zero": OUT_OF_SCOPE,
    "test_matrix.py::test_named_matrix_seqtm_score": OUT_OF_SCOPE,
    "test_matrix.py::test_identity_is_edit_cost": OUT_OF_SCOPE,
    "test_matrix.py::test_aa_matrix_rejects_nt_alphabet": OUT_OF_SCOPE,
    "test_matrix.py::test_unknown_matrix_name_rejected": OUT_OF_SCOPE,
    "test_matrix.py::test_custom_matrix_matches_builtin": OUT_OF_SCOPE,
    "test_matrix.py::test_matrix_size_mismatch_raises": OUT_OF_SCOPE,
    "test_matrix.py::test_collisions_only_with_indels": OUT_OF_SCOPE,
    "test_gapblock.py::test_index_handles_an_empty_auxiliary_level":
        "inspects the reference index's private per-deletion-level trie indexes (_var); the "
        "search it then checks is covered by the other GapBlockIndex tests",
}


def _install() -> None:
    import seqtree_b200 as lib
    from seqtree_b200 import distance, evalue, gapblock, matrix, pairwise
    pkg = types.ModuleType("seqtree")
    pkg.__path__ = []  # a package: submodules come from sys.modules below
    for name in ("SubstitutionMatrix", "ScoreMatrix", "alphabet_symbols", "amino_acids"):
        setattr(pkg, name, getattr(matrix, name))
    for name in ("GapBlockIndex", "IslandProfile", "central_prior", "embed_in_frame",
                 "frame_prior", "gapblock_score", "positions_prior", "profile_prior",
                 "score_matrix"):
        setattr(pkg, name, getattr(gapblock, name))
    pkg.gapblock, pkg.pairwise, pkg.distance, pkg.evalue = gapblock, pairwise, distance, evalue
    for name in ("thetas_from_scores", "evalues", "threshold_for_evalue"):
        if hasattr(evalue, name):
            setattr(pkg, name, getattr(evalue, name))
    pkg.__version__ = lib.__version__
    sys.modules["seqtree"] = pkg
    sys.modules["seqtree.gapblock"] = gapblock
    sys.modules["seqtree.pairwise"] = pairwise
    sys.modules["seqtree.distance"] = distance
    sys.modules["seqtree.evalue"] = evalue


_install()


def pytest_collection_modifyitems(config, items):
    for item in items:
        key = f"{item.path.name}::{item.originalname}"
        if key in SKIP:
            item.add_marker(pytest.mark.skip(reason=SKIP[key]))
