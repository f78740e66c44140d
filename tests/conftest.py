"""Shared test configuration: the `gpu` marker and import paths."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# The reference tree, where a test needs its files directly (most read the
# committed fixtures under tests/golden instead): LENIA_REFERENCE_DIR, unset
# = absent.
REFERENCE_DIR = os.environ.get("LENIA_REFERENCE_DIR") or None


def reference_preset(name):
    """(params, resolution) of a reference preset's Lenia module, from the
    fixture tests/golden/make_presets.py wrote (an "organism" path is relative
    to tests/golden)."""
    import json

    d = json.load(open(os.path.join(GOLDEN, "reference_presets.json")))[name]
    return dict(d["params"]), d["resolution"]


def orbium_organism():
    """The organism the Orbium preset stamps (tests/golden/orbium.json)."""
    import json

    return json.load(open(os.path.join(GOLDEN, "orbium.json")))


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
