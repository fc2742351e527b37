"""spectral_init_b200: the spectral-init eigensolve path on NVIDIA B200 (sm_100a).

The numerical work lives in ``libspectral_init_b200.so`` (C ABI declared in
``include/spectral_init_gpu.h``); this package is its Python mirror of the
crate's public API.
"""
from .api import (  # noqa: F401
    fuzzy_graph,
    ComputeMode,
    Context,
    ConvergenceFailure,
    CsrOperator,
    CudaError,
    InvalidArgument,
    InvalidGraph,
    IterationCap,
    OutOfMemory,
    Precision,
    Report,
    SpectralError,
    SpectralInitConfig,
    TooFewNodes,
    WarmStart,
    as_csr_f32,
    build_laplacian_values,
    build_normalized_laplacian,
    compute_degrees,
    dense_evd,
    find_components,
    get_context,
    lobpcg_solve,
    normalize_signs,
    rsvd_solve,
    scale_and_add_noise,
    select_eigenvectors,
    solve_eigenproblem_pub,
    spectral_init,
)

__all__ = [n for n in dir() if not n.startswith("_")]
