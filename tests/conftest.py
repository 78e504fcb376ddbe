import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import LIB_ORACLE, Oracle, build
    if not LIB_ORACLE.exists():
        build(ref=False)
    return Oracle("oracle")


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle.oracle import LIB_REF, Oracle
    if not LIB_REF.exists():
        pytest.skip("the reference make_rhs.H build (oracle/_ref) is not present")
    return Oracle("ref")


@pytest.fixture(scope="session")
def parity_oracle():
    """The parity authority for GPU comparisons: the reference's own
    make_rhs.H under the oracle's driver (oracle/_ref) where it was built,
    else the restatement (liboracle)."""
    from oracle.oracle import LIB_ORACLE, LIB_REF, Oracle, build
    if LIB_REF.exists():
        return Oracle("ref")
    if not LIB_ORACLE.exists():
        build(ref=False)
    return Oracle("oracle")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from zoomy_amrex_b200.build import build
    build()
    return torch.device("cuda:0")
