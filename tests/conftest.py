"""Shared test set-up: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs here without a GPU: the oracle against the golden vectors,
host logic, and the C ABI's exports.  ``-m gpu`` holds the parity tests proper, which
call the CUDA path through the C ABI and compare with the oracle.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(REPO, "tests", "golden")
