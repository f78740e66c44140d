"""Generates tests/golden/lenia_golden.npz from the reference itself.

Runs the reference's own Lenia module (Modules/FieldModules/Lenia.cpp) and
Metal kernels (Shaders/Field/Lenia.metal, Shaders/Common/FFT.metal) compiled
for the CPU -- oracle/_ref/libleniaref.so, built by ``make -C oracle ref``
from the reference tree -- on small seeded cases, and stores every field it
produced. The tests check the project's CPU oracle against these fields bit
for bit, so parity stays pinned where the reference tree is absent.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.lenia_oracle import RefLenia  # noqa: E402

ORGANISM = os.path.join(HERE, "organism_synthetic.json")

BASIC = {  # the lenia_basic preset's params block, colour map omitted
    "radius": 13, "dt": 0.35, "growthMu": 0.15, "growthSigma": 0.017, "kernelShellMu": 0.5,
    "kernelShellSigma": 0.15, "initCoverage": 0.42, "initScale": 26.0, "noiseAmount": 0.0,
    "muJitter": 0.0, "injectAmount": 0.22, "injectCount": 4, "growthMode": 1,
}
MULTI = {  # the lenia_multikernel preset's params block at a reduced sim size
    "radius": 24, "dt": 0.35, "growthMode": 1, "growthMu": 0.15, "growthSigma": 0.017,
    "kernelShellMu": 0.5, "kernelShellSigma": 0.15, "initCoverage": 0.42, "initScale": 26.0,
    "noiseAmount": 0.0, "muJitter": 0.0, "simWidth": 128, "simHeight": 64, "convMode": "fft",
    "kernels": [
        {"radiusScale": 1.0, "mu": 0.15, "sigma": 0.017, "weight": 1.0, "betas": [1.0]},
        {"radiusScale": 0.55, "mu": 0.30, "sigma": 0.035, "weight": 0.6, "betas": [1.0, 0.6]},
        {"radiusScale": 0.3, "mu": 0.22, "sigma": 0.028, "weight": 0.4, "betas": [1.0]},
    ],
    "injectAmount": 0.2, "injectCount": 4,
}


def cases():
    """(name, params, scene_w, scene_h, seed, [(frame, substeps, audio_frame)], base overrides)."""
    extras = dict(BASIC, radius=9, growthMode=0, noiseAmount=0.3, muJitter=0.7,
                  injectAmount=0.4, injectCount=5)
    implicit = {"convMode": "fft", "radius": 7, "growthMode": 0, "dt": 0.2, "growthMu": 0.14,
                "growthSigma": 0.02, "initScale": 10.0, "initCoverage": 0.5}
    fallback = dict(MULTI, simWidth=96, simHeight=60)
    stamp = {"radius": 6, "dt": 0.0, "initMode": "stamp", "organism": ORGANISM, "stampCount": 7,
             "stampRotate": True, "useOrganismParams": False, "growthMode": 0,
             "growthMu": 0.16, "growthSigma": 0.02}
    noise = {"radius": 5, "dt": 0.0, "initScale": 9.5, "initCoverage": 0.55}
    small_field = dict(BASIC, radius=13, injectAmount=0.0)
    return [
        ("direct_basic", BASIC, 96, 80, 7777, [(0, 2, 0), (1, 2, 1), (2, 2, 2)]),
        ("direct_extras", extras, 64, 48, 1234, [(f, 1, 3 * f + 1) for f in range(4)]),
        ("fft_multi", MULTI, 200, 100, 7777, [(f, 1, f) for f in range(3)]),
        ("fft_implicit", implicit, 64, 64, 99, [(f, 1, f) for f in range(3)]),
        ("fft_fallback_nonpow2", fallback, 96, 60, 5, [(0, 1, 0), (1, 1, 1)]),
        ("stamp_init", stamp, 80, 64, 42, [(0, 1, 0)]),
        ("noise_init", noise, 100, 70, 3, [(0, 1, 0)]),
        ("small_field_wrap", small_field, 20, 18, 11, [(0, 1, 0), (1, 1, 1)]),
    ]


def write_organism():
    rng = np.random.default_rng(20240611)
    cells = rng.random((10, 12)) * (rng.random((10, 12)) > 0.3)
    doc = {"name": "synthetic", "R": 9, "T": 8, "mu": 0.16, "sigma": 0.02,
           "width": 12, "height": 10, "cells": [[round(float(v), 6) for v in row] for row in cells]}
    with open(ORGANISM, "w") as f:
        json.dump(doc, f)


def main():
    if not RefLenia.available():
        sys.exit("oracle/_ref/libleniaref.so is missing (make -C oracle ref)")
    write_organism()
    out = {}
    manifest = []
    for name, params, w, h, seed, frames in cases():
        r = RefLenia(params, w, h)
        r.reset(seed)
        fields = []
        for (f, sub, af) in frames:
            fields.append(r.encode(f, sub, af).copy())
        out[name + "/fields"] = np.stack(fields)
        lut = r.upload(".kernel")
        if lut.size:
            out[name + "/lut"] = lut
        img = r.upload(".kernelImageUpload")
        if img.size:
            out[name + "/last_kernel_image"] = img.reshape(r.h, r.w)
        p = dict(params)
        if "organism" in p:
            p["organism"] = os.path.basename(p["organism"])
        manifest.append({"name": name, "params": p, "scene": [w, h], "seed": seed,
                         "frames": frames, "sim": [r.w, r.h], "passes": r.pass_count()})
    # PCG hash and rand01 samples (Random.metal:5-19).
    v = np.array([0, 1, 2, 3, 0xFFFFFFFF, 0x4C454E31, 123456789, 2891336453], np.uint64)
    L = RefLenia.lib()
    out["pcg/in"] = v.astype(np.uint32)
    out["pcg/out"] = np.array([L.ref_pcg(int(x)) for x in v], np.uint32)
    rs = np.array([[x, y, t, s] for x, y, t, s in [(0, 0, 0, 0), (5, 7, 401, 99), (1919, 1079, 503, 7),
                                                    (3, 0, 811, 12345), (0, 3, 823, 12345)]], np.uint32)
    out["rand/in"] = rs
    out["rand/out"] = np.array([L.ref_rand(*map(int, r)) for r in rs], np.float32)
    out["manifest"] = np.frombuffer(json.dumps(manifest).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "lenia_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "lenia_golden.npz"), len(manifest), "cases")


if __name__ == "__main__":
    main()
