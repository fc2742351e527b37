import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"

ALL_DATASETS = ["blobs_50", "blobs_500", "blobs_5000", "moons_200", "circles_300", "near_dupes_100",
                "disconnected_200", "blobs_connected_200", "blobs_connected_2000"]
CONNECTED = ["blobs_connected_200", "blobs_connected_2000", "moons_200", "circles_300", "near_dupes_100"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_npz(dataset, name):
    return np.load(GOLDEN / dataset / name, allow_pickle=False)


def load_csr(dataset, name):
    z = load_npz(dataset, name)
    return sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))


def load_graph(dataset, exact=False):
    """Pruned fuzzy graph (the crate's spectral_init input), f32 weights."""
    g = load_csr(dataset, "step5a_pruned_exact.npz" if exact else "step5a_pruned.npz")
    g = sp.csr_matrix(g, dtype=np.float32)
    g.sort_indices()
    return g


@pytest.fixture(scope="session")
def gpu_ctx():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from spectral_init_b200 import get_context
    return get_context(0)
