import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    if not o.ORACLE_SO.exists():
        o.build()
    return o.Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import oracle as o

    if not o.REF_SO.exists():
        pytest.skip("reference library oracle/_ref/libtqref.so not built here")
    return o.Reference()


def golden_cases():
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "tables")


def load_golden(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        d = {k: z[k] for k in z.files}
    dim, bits, tq, k, n_calib = (int(v) for v in d["meta"])
    d.update(dim=dim, bits=bits, tq=bool(tq), k=k, n_calib=n_calib)
    if tq:
        d["calib"] = d["db"][:n_calib]
    return d


@pytest.fixture(scope="session")
def tables():
    with np.load(GOLDEN / "tables.npz") as z:
        return {k: z[k] for k in z.files}
