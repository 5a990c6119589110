import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def oracle():
    import py_oracle
    return py_oracle.Oracle()


@pytest.fixture(scope="session")
def ref_kyber():
    import py_oracle
    if not py_oracle.RefKyber.available():
        pytest.skip("reference C build (oracle/_ref) not available on this machine")
    return py_oracle.RefKyber(3)


@pytest.fixture(scope="session")
def tk():
    import tensorkyber_b200
    tensorkyber_b200.lib()
    return tensorkyber_b200


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def golden():
    """The committed golden vectors (outputs of the reference's own C)."""
    import numpy as np
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_vectors.npz")
    return dict(np.load(path))


def rng(seed):
    return np.random.default_rng(seed)
