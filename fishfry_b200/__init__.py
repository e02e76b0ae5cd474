"""fishfry_b200: the Fish Fry periodic Poisson solve (lap phi = f by FFT
spectral filtering) as hand-written sm_100a kernels behind a C ABI.

Native pieces: lib/libfishfry.so (C ABI, include/fishfry.h) and bin/fishfry
(the benchmark driver with the reference's arguments and printout).
"""
from ._lib import (EXPORTS, FF_ERR_BYTES, FF_ERR_CUDA, FF_ERR_INVALID, FF_ERR_NOMEM, FF_ERR_TASKS, FF_ERR_TIMEOUT,
                   FF_ERR_UNSUPPORTED, FF_FP32,
                   FF_FP64, FF_MAX_AXIS, FF_MAX_PHASES, FF_OK, FFError, LIB_PATH, lib)
from .api import (Batch, ParisPencil, Server, Plan, alias_free_kaxis, error_sums, init_field, modes_generate, phase_names,
                  reference_domain, rel_norms)

__all__ = [
    "EXPORTS", "FF_ERR_BYTES", "FF_ERR_CUDA", "FF_ERR_INVALID", "FF_ERR_NOMEM", "FF_ERR_TASKS", "FF_ERR_TIMEOUT",
    "FF_ERR_UNSUPPORTED", "FF_FP32",
    "FF_FP64", "FF_MAX_AXIS", "FF_MAX_PHASES", "FF_OK", "FFError", "LIB_PATH", "lib", "Batch", "ParisPencil", "Plan", "Server",
    "alias_free_kaxis", "error_sums", "init_field", "modes_generate", "phase_names", "reference_domain",
    "rel_norms",
]
