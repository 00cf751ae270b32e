"""Shared test setup: the `gpu` marker and handles on the package/oracle."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_NAME = "hornofusion-full3d_b200"


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA GPU (B200); runs through libeafcg.so")


def pkg():
    return importlib.import_module(PKG_NAME)


def gen():
    return importlib.import_module(PKG_NAME + ".eafgen")


@pytest.fixture(scope="session")
def eaf():
    return pkg()


@pytest.fixture(scope="session")
def eafgen():
    return gen()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
