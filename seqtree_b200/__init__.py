"""seqtree_b200: B200-native (sm_100a) all-vs-all sequence scoring, a drop-in for seqtree's
dense matrix calls.

* :mod:`seqtree_b200.gapblock` -- single-gap-block penalty matrix (``score_matrix``) and priors;
* :mod:`seqtree_b200.pairwise` -- Gotoh Needleman-Wunsch / Smith-Waterman scores and distances;
* :mod:`seqtree_b200.distance` -- Hamming and Levenshtein matrices;
* :mod:`seqtree_b200.device` -- the same computations on device-resident sequence sets;
* :mod:`seqtree_b200.learned` -- learned candidate proposal + exact rescore for 1e6 x 1e6 searches;
* ``GapBlockIndex`` -- thresholded gap-block search (the reference's index, on the GPU).

Everything runs on the current CUDA device through ``libseqtree_b200.so``; there is no CPU
fallback.  Results are bit-identical to seqtree 0.6.0's C++ on the same inputs.  The compiled
library is loaded on first use of a module that needs it, so ``python -m seqtree_b200.build``
works before it exists.
"""
import importlib

from .matrix import ScoreMatrix, SubstitutionMatrix, alphabet_symbols, amino_acids

__version__ = "0.1.0"

_MODULES = {"distance", "gapblock", "pairwise", "device", "shard", "learned", "evalue", "_core",
            "_lib"}
_FROM_GAPBLOCK = {"score_matrix", "score_sparse", "central_prior", "frame_prior",
                  "positions_prior", "profile_prior", "GapBlockIndex", "IslandProfile",
                  "embed_in_frame", "gapblock_score", "UNREACHABLE"}

__all__ = ["distance", "gapblock", "pairwise", "score_matrix", "score_sparse", "gapblock_score",
           "central_prior",
           "frame_prior", "positions_prior", "profile_prior", "GapBlockIndex", "IslandProfile",
           "embed_in_frame", "UNREACHABLE", "evalue", "ScoreMatrix",
           "SubstitutionMatrix", "alphabet_symbols", "amino_acids"]


def __getattr__(name):
    if name in _MODULES:
        return importlib.import_module(f".{name}", __name__)
    if name in _FROM_GAPBLOCK:
        return getattr(importlib.import_module(".gapblock", __name__), name)
    raise AttributeError(f"module 'seqtree_b200' has no attribute '{name}'")
