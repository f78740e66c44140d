"""Writes the reference preset fixtures the tests read where the reference
tree is absent (the GPU box, a checkout without it).

Copies, from the reference tree, the Lenia module's params block of three
presets (Presets/lenia_basic.json, Presets/lenia_multikernel.json,
Presets/lenia_orbium.json) into tests/golden/reference_presets.json, and the
organism the Orbium preset stamps (Presets/organisms/orbium.json, decoded
from the Chakazul/Lenia catalogue) into tests/golden/orbium.json; the Orbium
preset's "organism" path is rewritten to that file's name.

Run from the repository root:
    LENIA_REFERENCE_DIR=<reference tree> python tests/golden/make_presets.py
(the reference tree defaults to /root/reference).
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PRESETS = ("lenia_basic", "lenia_multikernel", "lenia_orbium")


def main():
    ref = os.environ.get("LENIA_REFERENCE_DIR", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "Presets")):
        sys.exit(f"no reference tree at {ref}")
    out = {}
    for name in PRESETS:
        doc = json.load(open(os.path.join(ref, "Presets", name + ".json")))
        mod = next(m for m in doc["modules"] if m.get("type") == "Lenia")
        params = dict(mod["params"])
        if "organism" in params:
            org = json.load(open(os.path.join(ref, params["organism"])))
            with open(os.path.join(HERE, "orbium.json"), "w") as f:
                json.dump(org, f, ensure_ascii=False)
            params["organism"] = "orbium.json"
        out[name] = {"resolution": doc.get("resolution"), "params": params}
    with open(os.path.join(HERE, "reference_presets.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote reference_presets.json and orbium.json")


if __name__ == "__main__":
    main()
