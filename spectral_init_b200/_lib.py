"""ctypes binding of ``libspectral_init_b200.so`` (declarations mirror
``include/spectral_init_gpu.h``).  Loading fails loudly when the library has
not been built: there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libspectral_init_b200.so"
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "spectral_init_gpu.h"

SI_OK = 0
SI_CONVERGENCE_FAILURE = 1
SI_INVALID_GRAPH = 2
SI_TOO_FEW_NODES = 3
SI_CUDA_ERROR = 4
SI_ITERATION_CAP = 5
SI_INVALID_ARGUMENT = 6
SI_OUT_OF_MEMORY = 7

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)


class SiConfig(C.Structure):
    _fields_ = [
        ("compute_mode", C.c_int32), ("precision", C.c_int32), ("warm_start", C.c_int32),
        ("block_size", C.c_int32), ("dense_threshold", C.c_int32), ("force_level", C.c_int32),
        ("rsvd_oversampling", C.c_int32), ("rsvd_nbiter", C.c_int32), ("max_iterations", C.c_int32),
        ("learned_filter", C.c_int32), ("tol", C.c_double), ("mixed_switch_tol", C.c_double),
    ]


class SiReport(C.Structure):
    _fields_ = [
        ("level", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
        ("n_components_graph", C.c_int32), ("fp32_iterations", C.c_int32), ("spmm_calls", C.c_int32),
        ("learned_start", C.c_int32), ("reserved1", C.c_int32),
        ("max_residual", C.c_double), ("solve_ms", C.c_double), ("eigenvalues", C.c_double * 16),
    ]


class SiCsrF32(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("indptr", C.c_void_p), ("indices", C.c_void_p),
                ("data", C.c_void_p)]


class SiCsrF64(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("indptr", C.c_void_p), ("indices", C.c_void_p),
                ("data", C.c_void_p)]


class SiOperator(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("indptr", C.c_void_p), ("indices", C.c_void_p),
                ("values", C.c_void_p), ("values_f32", C.c_void_p), ("diag", C.c_double)]


vp = C.c_void_p
_SIGNATURES = {
    "si_config_default": (None, [C.POINTER(SiConfig)]),
    "si_abi_version": (C.c_int32, []),
    "si_kernel_launches": (C.c_uint64, []),
    "si_ctx_create": (C.c_int, [C.c_int32, C.POINTER(vp)]),
    "si_ctx_destroy": (None, [vp]),
    "si_last_error": (C.c_char_p, [vp]),
    "si_ctx_synchronize": (C.c_int, [vp]),
    "si_ctx_stream": (vp, [vp]),
    "si_spectral_init": (C.c_int, [vp, C.POINTER(SiCsrF32), C.c_uint32, C.c_uint64, vp, C.c_uint64,
                                   C.POINTER(SiConfig), vp, C.POINTER(SiReport)]),
    "si_spectral_init_device": (C.c_int, [vp, C.POINTER(SiCsrF32), C.c_uint32, C.c_uint64, vp, C.c_uint64,
                                          C.POINTER(SiConfig), vp, C.POINTER(SiReport)]),
    "si_compute_degrees": (C.c_int, [vp, C.POINTER(SiCsrF32), C.c_int32, vp, vp]),
    "si_build_laplacian": (C.c_int, [vp, C.POINTER(SiCsrF32), vp, vp, vp]),
    "si_build_laplacian_csr": (C.c_int, [vp, C.POINTER(SiCsrF32), vp, vp, vp, vp, u64p]),
    "si_find_components": (C.c_int, [vp, C.POINTER(SiCsrF32), vp, u64p]),
    "si_fuzzy_graph": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32, C.c_uint32, vp, vp, vp, vp, vp, vp, vp,
                                 C.c_uint64, u64p]),
    "si_spmm": (C.c_int, [vp, C.POINTER(SiOperator), vp, vp, C.c_uint32]),
    "si_spmm_f32": (C.c_int, [vp, C.POINTER(SiOperator), vp, vp, C.c_uint32]),
    "si_operator_plan_create": (C.c_int, [vp, C.POINTER(SiOperator), C.POINTER(vp)]),
    "si_operator_plan_destroy": (None, [vp]),
    "si_spmm_planned": (C.c_int, [vp, vp, vp, vp, C.c_uint32]),
    "si_spmm_planned_f32": (C.c_int, [vp, vp, vp, vp, C.c_uint32]),
    "si_solve_eigenproblem": (C.c_int, [vp, C.POINTER(SiOperator), C.c_uint32, C.c_uint64, vp,
                                        C.POINTER(SiConfig), vp, vp, i32p, C.POINTER(SiReport)]),
    "si_solve_eigenproblem_host": (C.c_int, [vp, C.POINTER(SiCsrF64), C.c_uint32, C.c_uint64,
                                             C.POINTER(SiConfig), vp, vp, i32p, C.POINTER(SiReport)]),
    "si_lobpcg_solve_host": (C.c_int, [vp, C.POINTER(SiCsrF64), C.c_uint32, C.c_uint64, C.c_int32, vp,
                                       C.POINTER(SiConfig), vp, vp, i32p, C.POINTER(SiReport)]),
    "si_rsvd_solve_host": (C.c_int, [vp, C.POINTER(SiCsrF64), C.c_uint32, C.c_uint64, C.c_int32, C.c_int32,
                                     vp, vp]),
    "si_dense_evd_host": (C.c_int, [vp, C.POINTER(SiCsrF64), C.c_uint32, vp, vp]),
    "si_normalize_signs": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32]),
    "si_normalize_signs_noalloc": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32]),
    "si_scale_and_add_noise": (C.c_int, [vp, vp, C.c_uint64, C.c_uint32, C.c_uint64, vp]),
    "si_model_param_count": (C.c_uint64, []),
    "si_model_create": (C.c_int, [vp, C.c_uint64, C.POINTER(vp)]),
    "si_model_destroy": (None, [vp]),
    "si_model_set_params": (C.c_int, [vp, vp, vp]),
    "si_model_get_params": (C.c_int, [vp, vp, vp]),
    "si_model_train_step": (C.c_int, [vp, vp, C.POINTER(SiOperator), vp, vp, C.c_uint32, C.c_uint64, C.c_float,
                                      C.POINTER(C.c_double)]),
    "si_model_gradient": (C.c_int, [vp, vp, C.POINTER(SiOperator), vp, vp, vp, C.c_uint32, C.c_uint64,
                                    C.POINTER(C.c_double), vp]),
    "si_model_predict": (C.c_int, [vp, vp, C.POINTER(SiOperator), vp, vp, C.c_uint64, vp]),
    "si_ctx_set_model": (C.c_int, [vp, vp]),
    "si_gemm_bf16_nt": (C.c_int, [vp, C.c_uint64, C.c_uint32, C.c_uint64, vp, C.c_uint64, vp, C.c_uint64, vp,
                                  C.c_uint64, C.c_uint32]),
}

_lib = None


def header_symbols() -> list[str]:
    """Function names declared in the public header."""
    text = HEADER_PATH.read_text()
    return sorted(set(re.findall(r"\b(si_[a-z0-9_]+)\s*\(", text)))


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the library (once).  Raises RuntimeError if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build the CUDA library first (python -m spectral_init_b200.build); "
            "spectral_init_b200 has no CPU fallback")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
