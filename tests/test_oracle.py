"""The CPU oracle against the reference's own outputs (CPU only).

* Bit-exact: the FP32 restatement ("ref32") against fields the compiled
  reference produced (tests/golden, made by tests/golden/make_golden.py), and
  against the compiled reference live where oracle/_ref was built.
* FP64 oracle vs FP32 restatement: close (the restatement's rounding only).
* FP64 convolution two ways (numpy FFT vs tap-by-tap C): 1e-12.
* The reference's stated checks: its FFT round trip, direct vs FFT after one
  step, and the Orbium preset surviving 400 frames.
"""
import json
import os

import numpy as np
import pytest

from oracle import lenia_oracle as lo
from oracle.lenia_oracle import OracleLenia, RefLenia
from tests.conftest import orbium_organism, reference_preset


def _organism_for(params):
    import json
    if "organism" not in params:
        return None
    d = json.load(open(params["organism"]))
    return lo.Organism(np.asarray(d["cells"], np.float32), d["R"], d["T"], d["mu"], d["sigma"])


CASES = ["direct_basic", "direct_extras", "fft_multi", "fft_implicit", "fft_fallback_nonpow2",
         "stamp_init", "noise_init", "small_field_wrap"]


@pytest.mark.parametrize("name", CASES)
def test_ref32_matches_reference_golden_bit_exact(golden, name):
    d, man = golden
    c = man[name]
    w, h = c["scene"]
    o = OracleLenia(c["params"], w, h, "ref32", organism=_organism_for(c["params"]))
    assert [o.w, o.h] == c["sim"]
    o.reset(c["seed"])
    want = d[name + "/fields"]
    for i, (f, sub, af) in enumerate(c["frames"]):
        got = o.encode(f, sub, af)
        np.testing.assert_array_equal(got, want[i], err_msg=f"{name} frame {f}")
    if name + "/lut" in d.files and not (o.use_fft or o.direct_multi):
        np.testing.assert_array_equal(o.lut.ravel(), d[name + "/lut"])
    if name + "/last_kernel_image" in d.files:
        np.testing.assert_array_equal(o.kimg[-1], d[name + "/last_kernel_image"])


def test_fallback_warnings_match_reference(golden):
    _, man = golden
    c = man["fft_fallback_nonpow2"]
    o = OracleLenia(c["params"], *c["scene"], precision="ref32")
    assert not o.use_fft
    assert any("power-of-two" in w for w in o.warnings)
    assert any("kernels[0]" in w for w in o.warnings)


def test_pcg_and_rand01_golden(golden):
    d, _ = golden
    got = np.array([lo.pcg_hash(int(v)) for v in d["pcg/in"]], np.uint32)
    np.testing.assert_array_equal(got, d["pcg/out"])
    got_np = lo.pcg_hash_np(d["pcg/in"])
    np.testing.assert_array_equal(got_np, d["pcg/out"])
    r = np.array([lo.rand01(*map(int, x)) for x in d["rand/in"]], np.float32)
    np.testing.assert_array_equal(r, d["rand/out"])


@pytest.mark.parametrize("name", ["direct_basic", "direct_extras", "fft_multi", "fft_implicit"])
def test_f64_oracle_close_to_ref32(golden, name):
    d, man = golden
    c = man[name]
    w, h = c["scene"]
    o64 = OracleLenia(c["params"], w, h, "f64")
    o64.reset(c["seed"])
    want = d[name + "/fields"]
    for i, (f, sub, af) in enumerate(c["frames"]):
        got = o64.encode(f, sub, af)
        # Only the FP32 rounding of the reference separates the two; the
        # dynamics amplify it a little per step (tolerance per frame).
        assert np.abs(got - want[i]).max() < 5e-5, (name, f)


def test_fft_conv_equals_direct_conv_f64():
    rng = np.random.default_rng(0)
    a = rng.random((48, 40))
    k = lo.ring_image(40, 48, 9.5, 0.15, [1.0, 0.6], lo.CORE_GAUSS_SHELL)
    k2 = lo.ring_image(40, 48, 13.0, 0.15, [1.0], lo.CORE_EXP)
    for kimg in (k, k2):
        np.testing.assert_allclose(lo.conv_circular_f64(a, kimg), lo.conv_direct_f64(a, kimg),
                                   rtol=0, atol=1e-12)


def test_kernel_images_normalised_and_symmetric():
    for core in (lo.CORE_GAUSS_SHELL, lo.CORE_EXP):
        img = lo.ring_image(120, 90, 24.0, 0.15, [1.0, 0.667, 0.333], core)
        assert abs(img.astype(np.float64).sum() - 1.0) < 1e-5
        # even in x and in y on the torus
        np.testing.assert_array_equal(img, np.roll(img[:, ::-1], 1, axis=1))
        np.testing.assert_array_equal(img, np.roll(img[::-1, :], 1, axis=0))
    lut = lo.direct_lut(13, core=lo.CORE_EXP)
    assert abs(lut.astype(np.float64).sum() - 1.0) < 1e-5
    assert np.count_nonzero(lut) == 516  # 0 < d^2 < 169


def test_exp_core_direct_equals_ring_image_single_peak():
    # With one peak the exponential ring kernel equals the direct LUT (both
    # exp(4 - 1/(r(1-r))) over 0 < r < 1, normalised in FP64).
    R = 13
    img = lo.ring_image(64, 64, float(R), 0.15, [1.0], lo.CORE_EXP)
    lut = lo.direct_lut(R, core=lo.CORE_EXP)
    win = np.zeros_like(lut)
    for dy in range(-R, R + 1):
        for dx in range(-R, R + 1):
            win[dy + R, dx + R] = img[dy % 64, dx % 64]
    np.testing.assert_allclose(win, lut, rtol=1e-6, atol=0)


@pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built (reference tree absent)")
def test_ref32_matches_compiled_reference_live():
    rng = np.random.default_rng(7)
    for trial in range(3):
        params = {"radius": int(rng.integers(3, 11)), "dt": float(rng.uniform(0.05, 0.4)),
                  "growthMu": float(rng.uniform(0.1, 0.3)), "growthSigma": float(rng.uniform(0.01, 0.05)),
                  "growthMode": int(trial % 2), "noiseAmount": 0.2, "muJitter": 0.5,
                  "injectAmount": 0.3, "injectCount": 2, "initScale": 12.0}
        w, h = int(rng.integers(20, 60)), int(rng.integers(20, 60))
        r = RefLenia(params, w, h)
        o = OracleLenia(params, w, h, "ref32")
        r.reset(trial)
        o.reset(trial)
        for f in range(3):
            np.testing.assert_array_equal(o.encode(f, 2, f + 5), r.encode(f, 2, f + 5))


def test_reference_fft_roundtrip_within_its_stated_bound():
    # The reference's own FFT check: a random 256x128 real field, forward
    # then inverse, max abs error < 1e-4 (Shaders/Common/FFT.metal:29-34,
    # docs/specs/phase9_lenia_fft.md:155-158). The forward transform is the
    # unscaled DFT with exp(-i...) (numpy's convention).
    rng = np.random.default_rng(11)
    re = rng.random((128, 256)).astype(np.float32)
    im = np.zeros_like(re)
    fr, fi = lo.fft2d_ref_f32(re, im, +1)
    want = np.fft.fft2(re.astype(np.float64))
    scale = np.abs(want).max()
    assert np.abs(fr - want.real).max() / scale < 1e-5
    assert np.abs(fi - want.imag).max() / scale < 1e-5
    rr, ri = lo.fft2d_ref_f32(fr, fi, -1)
    assert np.abs(rr - re).max() < 1e-4
    assert np.abs(ri).max() < 1e-4


def test_reference_direct_and_fft_agree_after_one_step():
    # The reference's convolution check: the same init and kernel (R=13) one
    # step by convMode direct and by fft at 256x256, max abs difference
    # < 1e-3 (docs/specs/phase9_lenia_fft.md:159-162); here on the FP32
    # restatement of both paths.
    rng = np.random.default_rng(5)
    init = np.zeros((256, 256), np.float32)
    init[96:160, 96:160] = rng.random((64, 64)).astype(np.float32)
    out = {}
    for conv in ("direct", "fft"):
        o = OracleLenia({"radius": 13, "convMode": conv}, 256, 256, "ref32")
        assert o.use_fft == (conv == "fft")
        o.reset(1)
        o.set_initial_field(init)
        out[conv] = o.encode(0, 1)
    d = np.abs(out["direct"].astype(np.float64) - out["fft"]).max()
    assert 0.0 < d < 1e-3, d
    assert np.abs(out["direct"] - init).max() > 1e-3  # the step changed the field


def test_orbium_glides_and_survives_400_frames():
    # The reference's qualitative known answer: the Orbium preset
    # (Presets/lenia_orbium.json, stamp init of Presets/organisms/orbium.json
    # with its own R, T, mu, sigma) survives 400 frames as a glider
    # (docs/specs/phase11_organisms.md:74-81). One stamp on a 96x96 torus,
    # FP32 restatement: the mass holds and the pattern moves.
    params = reference_preset("lenia_orbium")[0]
    d = orbium_organism()
    org = lo.Organism(np.asarray(d["cells"], np.float32), d["R"], d["T"], d["mu"], d["sigma"])
    p = dict(params, simWidth=96, simHeight=96, stampCount=1, stampRotate=False)
    o = OracleLenia(p, 96, 96, "ref32", organism=org)
    o.reset(7777)
    first = o.encode(0, 1)
    m0 = float(first.sum())
    assert m0 > 10.0
    for fr in range(1, 400):
        f = o.encode(fr, 1)
        if fr % 50 == 49:
            assert 0.8 * m0 < float(f.sum()) < 1.2 * m0, (fr, float(f.sum()), m0)
            assert f.max() > 0.5
    body0, body = first > 0.1, f > 0.1
    assert (body0 & body).sum() < 0.25 * body0.sum()  # it has moved off its start
