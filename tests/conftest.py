import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs the CUDA library)")


@pytest.fixture(scope="session")
def port_lib():
    """The C restatement oracle (oracle/_build/liboracle.so), built on first use if a compiler is at hand."""
    from oracle import oracle
    if not oracle.port_available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True, capture_output=True)
    assert oracle.port_available()
    return oracle.PORT_LIB


@pytest.fixture(scope="session")
def ref_lib():
    """The reference compiled from its sources (oracle/_ref); skipped where it was not built."""
    from oracle import oracle
    if not oracle.ref_available("parity"):
        pytest.skip("the compiled reference (oracle/_ref) is not present")
    return oracle.REF_LIBS["parity"]


def golden(name):
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz")))
