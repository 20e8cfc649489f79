import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests proper")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built():
    """Builds the library and the oracle once per session if they are missing."""
    import subprocess
    lib = os.path.join(ROOT, "ngap_b200", "libngap_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "ngap_b200", "csrc")],
                       check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"],
                       check=True)
    return True


@pytest.fixture(scope="session")
def engine(built):
    if not gpu_available():
        pytest.skip("no CUDA device")
    import ngap_b200 as nb
    return nb.Engine(0)
