"""ml_prec_b200: B200-native (sm_100a) PCG with the multi-split / Chebyshev
multilevel preconditioners of ml_prec, behind the reference's host interface.

The compute path is the CUDA library ml_prec_b200/lib/libmlp_b200.so (C ABI in
include/mlp_b200.h); this package is its Python binding.
"""
from .api import (ChebSolver, Config, ConfigError, ConfigFile, CSRMatrix, MultiSplitPrec, PCGSolver,  # noqa: F401
                  Prec, PrecBase, SolverStats, SymPrec, generate_x0, msplit_params)
from ._capi import MlpError, LIB_PATH  # noqa: F401
