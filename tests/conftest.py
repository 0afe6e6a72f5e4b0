"""Test configuration: the `gpu` marker and import paths.

CPU tests (-m "not gpu") check the oracle against the reference's own test
expectations, the host packing against the oracle's packing, and that the C
ABI library loads and exports every declared symbol. GPU tests (-m gpu) are
the parity tests proper: they call the CUDA tracer through the C ABI and
compare it with the CPU oracle on the same inputs.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200) and runs the CUDA tracer")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def hdcx_lib():
    from hdcodex_b200 import build as B
    B.build()
    import hdcodex_b200
    return hdcodex_b200
