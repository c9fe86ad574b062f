"""pytest configuration: the `gpu` marker and the oracle on sys.path.

GPU tests (marked `gpu`) call libchaoslab_b200 through its C ABI on a B200 and compare against the CPU oracle
(oracle/); everything else runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA kernels)")
    # the files tests write (the run store's chunk files) stay inside the checkout, in a folder pytest clears
    if not config.option.basetemp:
        config.option.basetemp = os.path.join(ROOT, ".pytest_tmp")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O   # oracle/oracle.py (test infrastructure)
    O.lib()
    return O
