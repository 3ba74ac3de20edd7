import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

BB_P = 0x78000001
GL_P = 0xFFFFFFFF00000001


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O


def rand_field(field: int, shape, seed: int) -> np.ndarray:
    """Seeded uniform field elements (canonical)."""
    rng = np.random.default_rng(seed)
    if field == 0:
        return rng.integers(0, BB_P, size=shape, dtype=np.uint32)
    return rng.integers(0, GL_P, size=shape, dtype=np.uint64)
