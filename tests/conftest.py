"""Shared fixtures. GPU tests carry the ``gpu`` marker; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def fp():
    return ge.load_package()


@pytest.fixture(scope="session")
def O():
    return ge.load_oracle()


@pytest.fixture(scope="session")
def ctx(fp):
    c = fp._capi.Context(0)
    yield c
    c.close()


def freestream(aoa_deg=4.2, mag=1.0):
    a = np.deg2rad(aoa_deg)
    return mag * np.array([np.cos(a), 0.0, np.sin(a)])
