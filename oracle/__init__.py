"""CPU oracle for the spectral-init eigensolve path.

TEST INFRASTRUCTURE ONLY.  Nothing under ``oracle/`` is part of the product:
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import it, and only as the checker (or as the timed CPU
restatement of the reference).  The product path lives in
``spectral_init_b200`` and calls the CUDA library; it never routes through
this package.

Contents
--------
``spectral_oracle``  numpy/scipy restatement of the reference crate's path
                     (degrees, Laplacian, components, SpMM, Chebyshev filter,
                     LOBPCG with warm restarts, Rayleigh-Ritz, rSVD, dense EVD,
                     selection, sign convention, scaling, multi-component).
``graphgen``         seeded synthetic UMAP fuzzy-kNN graphs (Gaussian mixtures,
                     exact kNN, smooth-kNN sigma/rho search, fuzzy union, prune).
``csr_cpu.c``        C kernels (f32 column-scatter degrees, OpenMP CSR SpMM with
                     an AVX2 gather inner loop) used to time the CPU baseline.

Parity pinning: the restatement is checked against the reference's own golden
fixtures (``tests/golden``: degrees bit-exact, Laplacian 1e-14, components,
eigenvalues vs. ARPACK/eigh, selection, scaling).  The LOBPCG iteration of the
reference lives in the un-vendored ``linfa-linalg 0.2`` crate; it is restated
from the published algorithm (Knyazev 2001, SIAM J. Sci. Comput. 23(2)) and is
pinned at the eigenpair level only (eigenvalues, residuals, subspaces), never
at the iterate level.
"""
