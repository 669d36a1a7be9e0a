import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def pytest_collection_modifyitems(config, items):
    """Every GPU test ends within 5 minutes (pytest-timeout): a host-side hang fails the
    test instead of holding the device."""
    for item in items:
        if item.get_closest_marker("gpu") and not item.get_closest_marker("timeout"):
            item.add_marker(pytest.mark.timeout(300))


def golden_cases():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    from tomogpi_b200.config import ConfigCT

    cfg = ConfigCT(**json.loads((GOLDEN / f"{name}.json").read_text()))
    data = dict(np.load(GOLDEN / f"{name}.npz"))
    return cfg, data


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def rel_l2_per_view(a, b):
    """Relative L2 error of every projection (view) of a [phi][v][u] sinogram; views whose
    reference is all zero report the absolute norm of the difference."""
    return [rel_l2(a[p], b[p]) for p in range(b.shape[0])]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle
