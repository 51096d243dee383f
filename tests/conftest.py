"""Shared pytest setup: marker registration and import paths.

GPU tests are marked ``gpu``; the CPU suite runs with ``-m "not gpu"``.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "gpu-powerflow_b200", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


def max_dv_vs_oracle(oracle, g, S, V0, V) -> np.ndarray:
    """Per scenario: max |V - V_oracle|, the oracle (FP64 CPU restatement)
    solving every scenario to ||F||inf <= 1e-12 from the same start, on all
    host cores."""
    import os

    ref = oracle.solve_many(g, S, V0, tol=1e-12, max_iter=30, threads=os.cpu_count() or 1)
    assert (ref["final_mismatch"] <= 1e-12).all()
    return np.abs(np.asarray(V) - ref["V"]).max(axis=1)
