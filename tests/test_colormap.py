"""The colour map's palette configuration (the reference Lenia module's
defaults and the "colorMap" block) and the CPU-compiled reference kernels it
is checked against. No GPU."""
import numpy as np
import pytest

import life_simulation_b200 as lb
from oracle.lenia_oracle import RefLenia, ref_colormap


def test_lenia_default_palette():
    cm = lb.colormap_from_params({"convMode": "direct"}).as_dict()
    assert cm["a"] == [0.5] * 3 and cm["b"] == [0.5] * 3 and cm["c"] == [1.0] * 3
    assert np.allclose(cm["d"], [0.60, 0.45, 0.30], rtol=0, atol=1e-7)
    assert cm["channel"] == 0 and cm["inputScale"] == 1.0 and cm["inputBias"] == 0.0 and cm["exposure"] == 1.0


def test_colormap_block():
    cm = lb.colormap_from_params({"colorMap": {"palette": "mono"}}).as_dict()
    assert cm["a"] == cm["b"] == cm["c"] == cm["d"] == [0.5] * 3
    cm = lb.colormap_from_params({"colorMap": {"palette": "mono", "d": [0.1, 0.2, 0.3], "inputScale": 3,
                                               "inputBias": -0.25, "exposure": 1.5, "channel": 2,
                                               "a": [1, 2]}}).as_dict()
    assert cm["a"] == [0.5] * 3  # fewer than 3 numbers: ignored
    assert np.allclose(cm["d"], [0.1, 0.2, 0.3]) and cm["inputScale"] == 3.0 and cm["channel"] == 2
    assert cm["inputBias"] == -0.25 and cm["exposure"] == 1.5


@pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built")
def test_reference_kernel_is_the_palette_formula():
    """The CPU-compiled reference kernel against the formula in numpy
    (checks the shim's vector and sampler stand-ins)."""
    rng = np.random.default_rng(0)
    f = rng.random((24, 40)).astype(np.float32)
    cm = {"a": [0.5, 0.4, 0.3], "b": [0.5, 0.6, 0.2], "c": [1.0, 0.7, 2.0], "d": [0.6, 0.45, 0.3],
          "inputScale": 1.3, "inputBias": -0.1, "exposure": 1.2, "channel": 0}
    out = ref_colormap(f, cm, 40, 24)
    t = np.clip(f.astype(np.float64) * 1.3 - 0.1, 0, 1)
    for i in range(3):
        rgb = np.maximum(cm["a"][i] + cm["b"][i] * np.cos(2 * np.pi * (cm["c"][i] * t + cm["d"][i])), 0) * 1.2
        assert np.abs(out[..., i] - rgb).max() < 1e-5
    assert np.abs(out[..., 3] - t).max() < 1e-6
    # Scaled, at exact 2x: output pixel centres fall between texel centres.
    up = ref_colormap(f, dict(cm, inputScale=1.0, inputBias=0.0), 80, 48)
    v = up[..., 3]
    assert abs(v[1, 1] - (0.75 * (0.75 * f[0, 0] + 0.25 * f[0, 1]) + 0.25 * (0.75 * f[1, 0] + 0.25 * f[1, 1]))) < 1e-6
