"""seqtree_b200: B200-native (sm_100a) all-vs-all sequence scoring, a drop-in for seqtree's
dense matrix calls.

* :mod:`seqtree_b200.gapblock` -- single-gap-block penalty matrix (``score_matrix``) and priors;
* :mod:`seqtree_b200.pairwise` -- Gotoh Needleman-Wunsch / Smith-Waterman scores and distances;
* :mod:`seqtree_b200.distance` -- Hamming and Levenshtein matrices;
* :mod:`seqtree_b200.device` -- the same computations on device-resident sequence sets.

Everything runs on the current CUDA device through ``libseqtree_b200.so``; there is no CPU
fallback.  Results are bit-identical to seqtree 0.6.0's C++ on the same inputs.
"""
from . import _core, distance, gapblock, pairwise
from .gapblock import central_prior, frame_prior, positions_prior, profile_prior, score_matrix
from .matrix import ScoreMatrix, SubstitutionMatrix, alphabet_symbols, amino_acids

__version__ = "0.1.0"

__all__ = ["distance", "gapblock", "pairwise", "score_matrix", "central_prior", "frame_prior",
           "positions_prior", "profile_prior", "ScoreMatrix", "SubstitutionMatrix",
           "alphabet_symbols", "amino_acids"]
