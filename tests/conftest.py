"""Shared test setup: the `gpu` marker, build of the native library and the oracle,
and helpers to reach the golden fixtures."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
INPUTS = os.path.join(GOLDEN, "inputs")
REF = os.path.join(GOLDEN, "ref")
EXAMPLES = os.path.join(GOLDEN, "examples")
SMALL_FIXTURES = ["sq16_pbc", "sq12_open_vac", "graphene_8x4", "cubic6", "chain_z2",
                  "sq20_charge", "general40", "general_spin"]
ORACLE_FIXTURES = ["sq16_pbc", "sq12_open_vac", "graphene_8x4", "cubic6", "chain_z2"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than ~20 s")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (C restatement) and the native library once per session."""
    import oracle
    oracle.build(ref=None)
    from gpuqt_b200 import build
    build.build()
    yield


def fixture_dir(name: str) -> str:
    return os.path.join(INPUTS, name)


def ref_moments(name: str, which: str = "moments"):
    p = os.path.join(REF, name, which + ".txt")
    a = np.loadtxt(p, ndmin=2)
    return a[:, 0].copy(), a[:, 1].copy()


def ref_npz(name: str, which: str):
    return np.load(os.path.join(REF, name, which + ".npz"))


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
