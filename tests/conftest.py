"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""

import importlib
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def sf():
    return importlib.import_module("stable-fluids_b200")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def lib(sf):
    return sf.load_library()


@pytest.fixture(scope="session")
def ref_lib(sf):
    from oracle import oracle

    if not oracle.REF_LIB_PATH.exists():
        pytest.skip("reference library not built (oracle/_ref)")
    return sf.load_library(oracle.REF_LIB_PATH)
