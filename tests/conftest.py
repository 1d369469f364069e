"""Test configuration: builds libintspmv.so and the oracle once per session;
GPU tests are marked `gpu` (run on a B200 with `-m gpu`)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from int_spmv_b200 import build as B
    try:
        B.build()
    except RuntimeError as e:  # nvcc missing: the prebuilt library must be there
        if not B.LIB.exists():
            raise
        print(f"note: keeping prebuilt {B.LIB} ({e})")
    import oracle
    oracle.build()


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_ok():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
