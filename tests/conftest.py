import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "dwave-samplers_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
GOLDEN = sorted(os.path.splitext(os.path.basename(p))[0]
                for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def load_golden(name):
    with np.load(os.path.join(GOLDEN_DIR, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def bits(x):
    """float64 array viewed as raw bits, for exact comparison (NaN-safe)."""
    return np.ascontiguousarray(x, dtype=np.float64).view(np.uint64)


@pytest.fixture(scope="session")
def gpu_available():
    import torch
    return torch.cuda.is_available()
