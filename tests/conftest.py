import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def splitmix_u32(n: int, seed: int) -> np.ndarray:
    """Seeded uniform u32 values in [0, 2^31) (the oracle's generator)."""
    import oracle
    return oracle.fill_uniform_u32(n, seed)


@pytest.fixture(scope="session")
def cuda_ready():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mdiscriminator_b200 as mdx
    mdx.lib()  # raises if the library is missing: no silent fallback
    return torch
