import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

os.environ.setdefault("HIPARTI_B200_QUIET", "1")

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Orc, ensure_built
    ensure_built(ref=False)
    return Orc()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref, ensure_built
    try:
        ensure_built(ref=True)
    except Exception:
        pass
    if not Ref.available():
        pytest.skip("reference library not built here")
    return Ref()


@pytest.fixture(scope="session")
def lib():
    from hiparti_b200 import build
    build.build()
    from hiparti_b200 import lib as _lib
    return _lib()


@pytest.fixture(scope="session")
def cuda(lib):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch.device("cuda:0")


def load_golden(name):
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
