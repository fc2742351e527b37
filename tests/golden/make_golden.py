"""Copy the reference crate's golden fixtures into ``tests/golden``.

The spectral-init crate ships Python-generated golden vectors (UMAP 0.5.11 /
scipy stage outputs) under ``tests/fixtures/<dataset>/``.  The GPU test box has
no copy of the reference, so the subset the parity tests need is committed
here, byte-for-byte.  Re-run with the reference checkout path as argument:

    python tests/golden/make_golden.py /path/to/spectral-init
"""
import shutil
import sys
from pathlib import Path

DATASETS = [
    "blobs_50", "blobs_500", "blobs_5000", "moons_200", "circles_300",
    "near_dupes_100", "disconnected_200", "blobs_connected_200", "blobs_connected_2000",
]
FILES = [
    "meta.json", "step5a_pruned.npz", "step5a_pruned_exact.npz",
    "comp_a_degrees.npz", "comp_b_laplacian.npz", "comp_c_components.npz",
    "comp_d_eigensolver.npz", "comp_e_selection.npz", "comp_f_scaling.npz",
]
# inputs of the fuzzy-kNN construction stages, for the graph generator checks
GEN_FILES = [
    "step0_raw_data.npz", "step1_knn_exact.npz", "step2_smooth_knn_exact.npz",
    "step3_membership_exact.npz", "step4_symmetrized_exact.npz",
]
GEN_DATASETS = ["blobs_connected_200", "moons_200", "near_dupes_100"]


def main(ref_root: str) -> None:
    src = Path(ref_root) / "tests" / "fixtures"
    dst = Path(__file__).resolve().parent
    for ds in DATASETS:
        (dst / ds).mkdir(parents=True, exist_ok=True)
        names = FILES + (GEN_FILES if ds in GEN_DATASETS else [])
        for f in names:
            shutil.copyfile(src / ds / f, dst / ds / f)
    shutil.copyfile(src / "manifest.json", dst / "manifest.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the spectral-init checkout>")
    main(sys.argv[1])
