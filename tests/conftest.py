"""Shared test configuration: the `gpu` marker and import paths."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np

    d = np.load(os.path.join(ROOT, "tests", "golden", "lenia_golden.npz"))
    manifest = json.loads(d["manifest"].tobytes())
    for c in manifest:
        if "organism" in c["params"]:
            c["params"]["organism"] = os.path.join(ROOT, "tests", "golden", c["params"]["organism"])
    return d, {c["name"]: c for c in manifest}
