import gzip
import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_idx(tmp_path_factory):
    """Path of the reference-built small index (tests/golden/small_index.idx.gz)."""
    p = tmp_path_factory.mktemp("golden") / "small.idx"
    with gzip.open(os.path.join(GOLDEN, "small_index.idx.gz"), "rb") as g, open(p, "wb") as f:
        shutil.copyfileobj(g, f)
    return str(p)


@pytest.fixture(scope="session")
def golden_search():
    return dict(np.load(os.path.join(GOLDEN, "small_search.npz")))


@pytest.fixture(scope="session")
def golden_refine():
    return dict(np.load(os.path.join(GOLDEN, "small_pre_refine.npz")))


@pytest.fixture(scope="session")
def golden_l2():
    return dict(np.load(os.path.join(GOLDEN, "l2_pairs.npz")))


def golden_results(gs, i):
    off, lab = gs[f"off_{i}"], gs[f"lab_{i}"]
    return [lab[off[q]:off[q + 1]] for q in range(len(off) - 1)]


def have_ref():
    from oracle import ref
    return ref.available()
