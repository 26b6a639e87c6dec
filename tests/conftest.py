import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))

for var in ("OMP_NUM_THREADS", "MKL_NUM_THREADS", "OPENBLAS_NUM_THREADS"):
    os.environ.setdefault(var, str(min(8, os.cpu_count() or 1)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def demo():
    return _load("demo")


@pytest.fixture(scope="session")
def synth():
    return _load("synth")


@pytest.fixture(scope="session")
def edge():
    return _load("edge")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def solvers_golden():
    return _load("solvers")


@pytest.fixture(scope="session")
def demo_gpu():
    return _load("demo_gpu")


@pytest.fixture(scope="session")
def cv_proj():
    return _load("cv_proj")


@pytest.fixture(scope="session")
def align_golden():
    return _load("align")


@pytest.fixture(scope="session")
def supervised_golden():
    return _load("supervised")
