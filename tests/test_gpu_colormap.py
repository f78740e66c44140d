"""The colour layer (RGBA16F) against the reference's colorMapField /
colorMapFieldScaled compiled for the CPU, on a stepped field: same size and
rescaled (up, down, non-integer ratios), several palettes and channels."""
import numpy as np
import pytest
import torch

import life_simulation_b200 as lb
from life_simulation_b200 import workloads as wl
from oracle.lenia_oracle import RefLenia, ref_colormap

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built")]

PALETTES = [
    {},
    {"colorMap": {"palette": "mono"}},
    {"colorMap": {"a": [0.2, 0.3, 0.4], "b": [0.8, 0.5, 0.3], "c": [2.0, 1.0, 0.5], "d": [0.0, 0.33, 0.67],
                  "inputScale": 2.5, "inputBias": -0.2, "exposure": 1.4}},
    {"colorMap": {"channel": 3}},
    {"colorMap": {"channel": 1, "inputBias": 0.3}},
]


def half_ulps(a: np.ndarray, b: np.ndarray) -> int:
    ia = a.astype(np.float16).view(np.int16).astype(np.int32)
    ib = b.astype(np.float16).view(np.int16).astype(np.int32)
    return int(np.abs(ia - ib).max())


@pytest.mark.parametrize("pal", range(len(PALETTES)))
@pytest.mark.parametrize("size", [(128, 96), (256, 192), (64, 48), (200, 150)])
def test_colour_layer_matches_reference(pal, size):
    params, w, h, init = wl.workload("single_256")
    params = dict(params, **PALETTES[pal])
    m = lb.LeniaModule(params, w, h)
    m.reset(1)
    m.upload(init)
    for f in range(3):
        m.encode(f, 1)
    field = m.field()
    ow, oh = size
    out = torch.empty((oh, ow, 4), dtype=torch.float16, device="cuda")
    m.render_device(out.data_ptr(), ow, oh)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    ref = ref_colormap(field, m.colormap().as_dict(), ow, oh)
    # cosf (CUDA) and the host's cosf may differ in the last float bit,
    # which can move a half by one unit; alpha has no cosine: exact.
    assert half_ulps(got[..., :3], ref[..., :3]) <= 1
    assert np.array_equal(got[..., 3], ref[..., 3].astype(np.float16))
    m.close()


def test_render_same_size_on_the_fft_path_and_profile():
    params, w, h, init = wl.workload("fft3_1024x512")
    m = lb.LeniaModule(params, w, h)
    m.upload(init)
    m.encode(0, 1)
    out = torch.empty((h, w, 4), dtype=torch.float16, device="cuda")
    m.profile(True)
    m.render_device(out.data_ptr(), w, h)
    prof = m.profile_read()
    assert prof["colormap"]["count"] == 1
    ref = ref_colormap(m.field(), m.colormap().as_dict(), w, h)
    assert half_ulps(out.cpu().numpy()[..., :3], ref[..., :3]) <= 1
    m.close()


@pytest.mark.parametrize("pal", [0, 2, 3])
@pytest.mark.parametrize("case", ["fft3_1080p", "fft_128x64", "direct_64x48", "fft_rescaled"])
def test_fused_step_render_equals_step_then_render(pal, case):
    """lenia_step_render (the colour pass fused into the last substep's row
    pass where it can be) gives the same field and the same texels as
    lenia_step followed by lenia_render_rgba16f."""
    if case == "fft3_1080p":
        params, w, h, init = wl.workload("fft3_1080p")
        ow, oh = w, h
    elif case == "fft_128x64":
        w, h = 128, 64
        params, init = wl.fft3_params(w, h), wl.patches(w, h, 6, 24, seed=5)
        params["radius"] = 12
        ow, oh = w, h
    elif case == "direct_64x48":
        w, h = 64, 48
        params, init = {"radius": 8}, wl.patches(w, h, 4, 16, seed=6)
        ow, oh = w, h
    else:
        w, h = 128, 64
        params, init = wl.fft3_params(w, h), wl.patches(w, h, 6, 24, seed=5)
        params["radius"] = 12
        ow, oh = 200, 90
    params = dict(params, noiseAmount=0.05, **PALETTES[pal])
    a, b = lb.LeniaModule(params, w, h), lb.LeniaModule(params, w, h)
    out_a = torch.zeros((oh, ow, 4), dtype=torch.float16, device="cuda")
    out_b = torch.ones((oh, ow, 4), dtype=torch.float16, device="cuda")
    for m in (a, b):
        m.reset(4)
        m.upload(init)
    for f in range(2):  # two frames in a row: the fused texels follow each step
        fa, fb = a.frame_params(f), b.frame_params(f)
        a.step_render(fa, 2, out_a.data_ptr(), ow, oh)
        b.step(fb, 2)
        b.render_device(out_b.data_ptr(), ow, oh)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(a.field(), b.field())
        assert torch.equal(out_a.view(torch.int16), out_b.view(torch.int16)), (case, pal, f)
    a.close()
    b.close()
