"""oxiblas_b200 -- B200-native (sm_100a) engine for OxiBLAS.jl's dense LU hot path.

The package directory is ``oxiblas.jl_b200/``; it is imported under the module
name ``oxiblas_b200`` (see ``load_package`` in the repository's
``__graft_entry__.py``).  The compute lives in ``liboxiblas_b200.so`` (C ABI in
``include/oxiblas_b200.h``); this Python layer mirrors the reference's public
API for the path.
"""
from ._lib import (ArgumentError, DimensionMismatch, ExtensionMissing, Handle, SingularException,
                   exported_symbols, load)
from .lu import (LU, colmajor_copy, det, gemm_update, ldiv, ldiv_, ldiv_into, logabsdet, lu, lu_,
                 options)
from .mixed import equilibrate, gemm_update_lowp, mixed_solve, mixed_solve_device
from .adjoint import lu_adjoint, solve
from .expert import expert_solve, factorize, inv, inverse_norm_estimate, refine_solve
from .cholesky import Cholesky, PosDefException, cholesky, cholesky_
from .batched import BatchedLU, autotune as batched_autotune, set_tuning as batched_set_tuning, \
    tuning as batched_tuning
from . import synthetic

__all__ = [
    "LU", "lu", "lu_", "ldiv", "ldiv_", "ldiv_into", "det", "logabsdet", "gemm_update", "options",
    "colmajor_copy", "SingularException", "DimensionMismatch", "ArgumentError", "ExtensionMissing",
    "Handle", "load", "exported_symbols", "mixed_solve", "mixed_solve_device", "gemm_update_lowp",
    "equilibrate", "expert_solve", "refine_solve", "inverse_norm_estimate", "inv", "factorize",
    "Cholesky", "PosDefException", "cholesky", "cholesky_",
    "lu_adjoint", "solve", "BatchedLU", "batched_autotune", "batched_tuning", "batched_set_tuning",
]
