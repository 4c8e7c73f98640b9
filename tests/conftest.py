import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and librr_ri.so")


def golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def ref_lib():
    """The reference compiled from its own sources (oracle/_ref); skipped where it is not built."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/librrref.so not built (make -C oracle needs the reference tree)")
    ref.set_threads(4)
    return ref
