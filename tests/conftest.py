import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the in-tree libuph.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_port_built():
    """The CPU restatement is test infrastructure; build it if it is missing."""
    from oracle import oracle as O
    if not os.path.exists(os.path.join(O.REF_DIR, "libuph_oracle.so")):
        O.build(reference=False)
