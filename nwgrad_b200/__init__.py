"""nwgrad_b200: the SeqPairBatch alignment path of michalsta/nwgrad on one B200.

Global / local Needleman-Wunsch / Smith-Waterman with linear and affine gaps; hard
(Viterbi path counts) and soft (forward-backward expected counts) gradients with respect to
the substitution matrices and gap costs; K parameter sets with per-residue tracks.  The
host API mirrors the reference's (AlignParams, SubstMatrix, Alphabet, SeqPair,
SeqPairBatch, SeqPairBatchDouble); every alignment runs in hand-written sm_100a CUDA
kernels behind the C ABI in include/nwgrad_b200.h (libnwgrad_b200.so).
"""
from .params import (AA20, AlignParams, Alphabet, DNA, DNA_N, IUPAC_DNA, NCBI_PROTEIN, PROTEIN,
                     PROTEIN_UO, PROTEIN_UOX, PROTEIN_X, RNA, RNA_N, SubstMatrix)
from .batch import BatchResult, SeqPair, SeqPairBatch, SeqPairBatchDouble, SeqPairDouble, guide_j_from_aligned

__all__ = ["AA20", "AlignParams", "Alphabet", "DNA", "DNA_N", "IUPAC_DNA", "NCBI_PROTEIN", "PROTEIN",
           "PROTEIN_UO", "PROTEIN_UOX", "PROTEIN_X", "RNA", "RNA_N", "SubstMatrix", "SeqPair",
           "SeqPairBatch", "SeqPairBatchDouble", "SeqPairDouble", "BatchResult", "guide_j_from_aligned"]
__version__ = "0.1.0"


def load_library():
    """Load libnwgrad_b200.so (building it if stale) and return the ctypes handle."""
    from . import _capi
    return _capi.lib()
