"""B200-native single-chain-in-mean-field polymer Monte Carlo engine.

Host mirror (Python) of libscmf.so, whose hot path is hand-written sm_100a
CUDA: smart-MC bead moves on an odd/even checkerboard with a counter-based
Philox stream, integer per-type density gridding, and the fused SCMF0 field
update with energy and acceptance reductions.
"""
from ._lib import FIELD_EVERY, FIELD_REFERENCE, HAM_LITERAL, HAM_SCMF0, ScmfError, lib
from .spec import Arch, SystemSpec
from .system import Batch, System, checkpoint_info, read_coords_file, vtk_convert

__all__ = ["Arch", "SystemSpec", "System", "Batch", "ScmfError", "lib", "read_coords_file", "vtk_convert", "checkpoint_info",
           "FIELD_EVERY", "FIELD_REFERENCE", "HAM_SCMF0", "HAM_LITERAL"]
