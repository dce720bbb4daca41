import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libgbfk.so")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
            return {k: z[k] for k in z.files}

    return load


@pytest.fixture(scope="session")
def gbfk_lib():
    """libgbfk.so, built in-tree if needed; a GPU test fails loudly without it."""
    from gliomasolver_b200 import _lib
    from gliomasolver_b200.build import build_library

    build_library()
    return _lib.load()
