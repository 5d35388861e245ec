"""B200-native ADGA ladder hot path.

chi0 bubble, density/magnetic Bethe-Salpeter solve (FP64 or mixed
FP32/BF16x3 with FP64 refinement), chi_d/m(q, omega) frequency sums and the
EOM self-energy, as hand-written sm_100a CUDA behind the C ABI of
``include/adga.h`` (``libadga_b200.so``).  ``Ladder`` mirrors the reference's
hot-path routines for Python callers; ``synth`` builds seeded inputs.
"""
from .ladder import (AdgaError, Ladder, create_u, generate_q_vol, index_kq, inverse_matrix,
                     run_ladder)
from ._lib import ADGA_FP64, ADGA_MIXED, EXPORTS, LIB_PATH

__all__ = ["AdgaError", "Ladder", "create_u", "generate_q_vol", "index_kq", "inverse_matrix",
           "run_ladder", "ADGA_FP64", "ADGA_MIXED", "EXPORTS", "LIB_PATH"]
