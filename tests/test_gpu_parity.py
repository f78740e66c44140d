"""Parity of the CUDA path (called through the C ABI) with the reference.

Anchors, in order of strength:
* the reference's own outputs (tests/golden, produced by the reference's
  Lenia.cpp and Metal kernels compiled for the CPU);
* the FP32 restatement of the reference ("ref32", bit-exact with those);
* the FP64 oracle (same update in double precision, exact convolution).
Tolerances: integer hashing and the init passes are compared bit for bit;
float fields within the bounds stated per test (the GPU sums taps in a
different order and contracts multiply-adds, the FFT path rounds in a
different pattern; the FP64 oracle is the accuracy reference).
"""
import json
import os

import numpy as np
import pytest

import life_simulation_b200 as lb
from life_simulation_b200 import workloads as wl
from oracle import lenia_oracle as lo
from oracle.lenia_oracle import OracleLenia

pytestmark = pytest.mark.gpu


def organism_for(params):
    if "organism" not in params:
        return None
    d = json.load(open(params["organism"]))
    return lo.Organism(np.asarray(d["cells"], np.float32), d["R"], d["T"], d["mu"], d["sigma"])


GOLDEN_TOL = {  # max |gpu - reference| per frame
    "direct_basic": 2e-5, "direct_extras": 5e-5, "fft_multi": 2e-5, "fft_implicit": 2e-5,
    "fft_fallback_nonpow2": 2e-5, "small_field_wrap": 2e-5,
}


@pytest.mark.parametrize("name", sorted(GOLDEN_TOL))
def test_gpu_matches_reference_golden(golden, name):
    d, man = golden
    c = man[name]
    m = lb.LeniaModule(c["params"], *c["scene"])
    assert [m.width, m.height] == c["sim"]
    m.reset(c["seed"])
    want = d[name + "/fields"]
    for i, (f, sub, af) in enumerate(c["frames"]):
        m.encode(f, sub, af)
        err = np.abs(m.field() - want[i]).max()
        assert err <= GOLDEN_TOL[name], (name, f, err)


@pytest.mark.parametrize("name", ["stamp_init", "noise_init"])
def test_gpu_init_bit_exact(golden, name):
    d, man = golden
    c = man[name]
    m = lb.LeniaModule(c["params"], *c["scene"])
    m.reset(c["seed"])
    f, sub, af = c["frames"][0]
    m.encode(f, sub, af)  # dt = 0: the field after the frame is the init
    np.testing.assert_array_equal(m.field(), d[name + "/fields"][0])


def run_pair(params, w, h, init, steps, precision="f64", substeps=1, seed=3, frame0=0):
    """Steps the GPU module and the oracle from the same field; yields both."""
    m = lb.LeniaModule(params, w, h)
    o = OracleLenia(params, w, h, precision)
    m.reset(seed)
    o.reset(seed)
    if init is not None:
        m.upload(init)
        o.set_initial_field(init)
    for s in range(steps):
        m.encode(frame0 + s, substeps)
        yield m.field(), o.encode(frame0 + s, substeps)


def test_noise_and_injection_hash_patterns():
    # Growth switched off (dt = 0): the step adds only the hashed noise and
    # blends in the hashed blobs, so any hash difference shows at O(1e-2).
    p = {"radius": 5, "dt": 0.0, "noiseAmount": 1.0, "injectAmount": 0.8, "injectCount": 6,
         "growthMode": 0}
    init = np.full((70, 90), 0.5, np.float32)
    for g, o in run_pair(p, 90, 70, init, 3, "ref32"):
        assert np.abs(g - o).max() < 1e-6


def test_mu_jitter_uses_audio_frame():
    p = {"radius": 6, "dt": 0.3, "muJitter": 1.0, "growthMode": 0, "growthSigma": 0.05}
    rng = np.random.default_rng(1)
    init = rng.random((64, 64)).astype(np.float32)
    m = lb.LeniaModule(p, 64, 64)
    o = OracleLenia(p, 64, 64, "f64")
    for x in (m, o):
        x.reset(9)
    m.upload(init)
    o.set_initial_field(init)
    m.encode(4, 1, 77)
    want = o.encode(4, 1, 77)
    assert np.abs(m.field() - want).max() < 1e-5


def local_errors(params, w, h, init, steps):
    """Per-step error: every step, GPU and FP64 oracle both start from the
    GPU's current state; returns max |gpu - fp64| per step."""
    m = lb.LeniaModule(params, w, h)
    o = OracleLenia(params, w, h, "f64")
    m.reset(3)
    o.reset(3)
    m.upload(init)
    o.set_initial_field(init)
    o.encode(0)  # builds kernels; state replaced below
    errs, a = [], np.asarray(init, np.float32)
    fp = m.frame_params(0)
    for s in range(steps):
        fp.frame_index = fp.audio_frame = s
        m.upload(a)
        m.step(fp, 1)
        g = m.field()
        o.state = a.astype(np.float64)
        o.step_once(o.frame_params(), lo.pcg_hash(o.seed_ ^ (s * 197)), s, s)
        errs.append(float(np.abs(g - o.state).max()))
        a = g
    return np.array(errs)


def test_direct_single_256_100_steps_vs_fp64():
    # Per-step error over the whole 100-step run of the 256x256 direct workload ...
    params, w, h, init = wl.workload("single_256")
    errs = local_errors(params, w, h, init, 100)
    assert errs.max() <= 1e-5, errs.max()
    # ... and the free-running trajectory while it is not yet chaotic: the
    # reference's own FP32 arithmetic drifts from FP64 by ~1e-5 after 10
    # steps and by O(0.1) after 100 (error doubling every ~5 steps), so the
    # GPU is held to the same early bound rather than a 100-step one.
    worst = 0.0
    for s, (g, o) in enumerate(run_pair(params, w, h, init, 10)):
        worst = max(worst, float(np.abs(g - o).max()))
    assert worst <= 1e-4, worst


def test_fft_1080p_per_step_vs_fp64():
    params, w, h, init = wl.workload("fft3_1080p")
    errs = local_errors(params, w, h, init, 12)
    assert errs.max() <= 1e-5, errs.max()


def test_fft_1080p_100_steps_vs_fp64_unsynced():
    """The 1080p workload stepped 100 times on the GPU (FP32) and by the FP64
    oracle from the same field, never re-synchronised: the accumulated
    difference stays within 1e-5. (Its seeded patches die out after a few
    dozen steps in both; the live phase is checked at steps 1, 10 and 25.)"""
    params, w, h, init = wl.workload("fft3_1080p")
    worst = {}
    for s, (g, o) in enumerate(run_pair(params, w, h, init, 100), start=1):
        if s in (1, 10, 25, 50, 100):
            worst[s] = float(np.abs(g - o).max())
            if s == 10:
                assert float(o.max()) > 0.1  # alive
    assert max(worst.values()) <= 1e-5, worst


@pytest.mark.parametrize("w,h,mode", [(128, 64, 1), (120, 90, 0), (96, 60, 0), (64, 48, 1)])
def test_fft_vs_fp64_oracle(w, h, mode):
    p = wl.fft3_params(w, h)
    p["growthMode"] = mode
    p["radius"] = 12
    init = wl.patches(w, h, 6, 24, seed=5)
    worst = 0.0
    for g, o in run_pair(p, w, h, init, 20):
        worst = max(worst, float(np.abs(g - o).max()))
    assert worst <= 1e-5, worst


def test_fft_extras_vs_ref32():
    # injection, noise and jitter through the FFT path's growth epilogue
    p = {"convMode": "fft", "radius": 9, "dt": 0.2, "growthMode": 1, "noiseAmount": 0.4,
         "muJitter": 0.6, "injectAmount": 0.5, "injectCount": 3,
         "kernels": [{"mu": 0.15, "sigma": 0.02, "weight": 0.7, "betas": [1.0]},
                     {"radiusScale": 0.6, "mu": 0.25, "sigma": 0.04, "weight": 0.3, "betas": [1.0, 0.5]}]}
    rng = np.random.default_rng(2)
    init = (rng.random((64, 128)) * 0.6).astype(np.float32)
    for g, o in run_pair(p, 128, 64, init, 5, "ref32"):
        assert np.abs(g - o).max() < 2e-5


@pytest.mark.parametrize("w,h", [(256, 256), (120, 90), (384, 216), (1920, 1080)])
def test_direct_and_fft_agree_per_step(w, h):
    pf = wl.fft3_params(w, h)
    pd = wl.fft3_params(w, h, conv="directMulti")
    init = wl.patches(w, h, 8, 40, seed=4)
    mf, md = lb.LeniaModule(pf, w, h), lb.LeniaModule(pd, w, h)
    for m in (mf, md):
        m.reset(1)
    a = init
    worst = 0.0
    for s in range(10):
        mf.upload(a)
        md.upload(a)
        mf.encode(s)
        md.encode(s)
        f, d = mf.field(), md.field()
        worst = max(worst, float(np.abs(f - d).max()))
        a = f
    assert worst <= 1e-5, worst


def test_determinism_same_seed_same_bits():
    p = wl.fft3_params(240, 120)
    p["noiseAmount"] = 0.2
    runs = []
    for _ in range(2):
        m = lb.LeniaModule(p, 240, 120)
        m.reset(1234)
        for f in range(5):
            m.encode(f, 2)
        runs.append(m.field())
    np.testing.assert_array_equal(runs[0], runs[1])


@pytest.mark.parametrize("w,h", [(1920, 1080), (512, 512)])
def test_every_launch_shape_gives_the_same_bits(w, h):
    """Rows and columns are transformed independently with one plan, so the
    field must not depend on the rows/columns per CTA the autotuner picks."""
    p = wl.fft3_params(w, h)
    p["noiseAmount"] = 0.1
    init = wl.patches(w, h, 8, 64, seed=6)
    m = lb.LeniaModule(p, w, h)
    cols, rows = m.tuning()
    assert cols in (8, 4, 2, 4 | lb.COLS_HALF_THREADS) and rows & ~lb.ROWS_PIPELINED in (4, 2, 1)
    ref = None
    shapes = [(c, r | f) for c in (8, 4, 2, 4 | lb.COLS_HALF_THREADS) for r in (4, 2, 1)
              for f in (0, lb.ROWS_PIPELINED)]
    ran = 0
    for c, r in shapes:
        try:
            m.set_tuning(c, r)
        except lb.LeniaError:
            continue  # a shape over the thread or shared-memory limit
        assert m.tuning() == (c, r)
        m.reset(1)
        m.upload(init)
        for f in range(3):
            m.encode(f, 2)
        out = m.field()
        if ref is None:
            ref = out
        np.testing.assert_array_equal(out, ref, err_msg=f"{c} columns, {r:#x} rows per CTA")
        ran += 1
    assert ran >= 6
    for bad in ((3, 2), (4, 3), (4, 8), (16, 1), (4, 2 | 0x200), (8 | lb.COLS_HALF_THREADS, 2),
                (4, 2 | lb.COLS_HALF_THREADS)):
        with pytest.raises(lb.LeniaError, match="unsupported launch shape"):
            m.set_tuning(*bad)
    m.close()
    d = lb.LeniaModule(wl.fft3_params(w, h, conv="directMulti"), w, h)
    assert d.tuning() == (0, 0)
    with pytest.raises(lb.LeniaError):
        d.set_tuning(4, 2)
    d.close()


def test_upload_download_roundtrip_and_device_copy():
    m = lb.LeniaModule({"radius": 4}, 37, 23)
    a = np.random.default_rng(3).random((23, 37)).astype(np.float32)
    m.upload(a)
    np.testing.assert_array_equal(m.field(), a)
    assert m.field_device_ptr() != 0
    with pytest.raises(ValueError):
        m.upload(np.zeros(10, np.float32))


def test_params_table_and_overrides():
    p = {"radius": 7, "dt": 0.25, "growthMu": 0.2, "growthMode": 0}
    m = lb.LeniaModule(p, 48, 48)
    fp = m.frame_params(3)
    assert abs(fp.dt - 0.25) < 1e-7 and fp.growth_mode == 0 and fp.inject_count == 3
    m.set_override("dt", 0.5)
    assert abs(m.frame_params(3).dt - 0.5) < 1e-7
    m.clear_override("dt")
    m.set_param("growthSigma", 0.03)
    fp = m.frame_params(3)
    assert abs(fp.growth_sigma - 0.03) < 1e-7 and abs(fp.dt - 0.25) < 1e-7


def test_fft_falls_back_to_direct_like_reference(golden):
    d, man = golden
    c = man["fft_fallback_nonpow2"]
    m = lb.LeniaModule(c["params"], *c["scene"])
    assert "powers of two" in m.warning and m.info()["conv_mode"] == lb.CONV_DIRECT


def test_radius_beyond_direct_limit_is_an_error():
    with pytest.raises(lb.LeniaError):
        lb.LeniaModule({"radius": 40}, 128, 128)


def test_zero_radius_and_tiny_fields():
    for p, w, h in [({"radius": 0, "growthMode": 0}, 16, 16), ({"radius": 13}, 7, 5),
                    ({"convMode": "fft", "radius": 3}, 8, 4)]:
        init = np.random.default_rng(w).random((h, w)).astype(np.float32)
        for g, o in run_pair(p, w, h, init, 3, "ref32"):
            assert np.abs(g - o).max() < 2e-5, (p, w, h)


@pytest.mark.parametrize("w,h,radius", [(256, 256, 13), (512, 320, 32), (200, 120, 7)])
def test_direct_tma_halo_tiles_equal_element_loads(monkeypatch, w, h, radius):
    """The direct path's interior halo tiles arrive by one TMA box load each
    (edge tiles, whose halo wraps around the torus, by element loads): the
    field is bit-identical to staging every tile by element loads."""
    params = {"radius": radius, "noiseAmount": 0.05, "muJitter": 0.2}
    init = wl.patches(w, h, 8, 40, seed=9)
    out = []
    for env in ("1", "0"):
        monkeypatch.setenv("LENIA_DIRECT_TMA", env)
        m = lb.LeniaModule(params, w, h)
        assert m.info()["direct_tma"] == (env == "1")
        m.reset(5)
        m.upload(init)
        for f in range(4):
            m.encode(f, 2)
        m.sync()
        out.append(m.field())
        m.close()
    np.testing.assert_array_equal(out[0], out[1])


def test_direct_split_for_small_fields():
    """Small fields split each tile's kernel rows over several thread groups
    (a size rule: the same configuration always sums in the same order)."""
    small = lb.LeniaModule(wl.workload("single_256")[0], 256, 256)
    assert small.info()["direct_split"] == 8
    assert small.info()["direct_taps"] == 516  # exp core, R=13: 0 < d^2 < 169
    big = lb.LeniaModule({"radius": 13}, 1920, 1080)
    assert big.info()["direct_split"] == 1
    small.close()
    big.close()


def test_direct_outputs_per_thread_give_the_same_bits(monkeypatch):
    """Large direct fields (64x32 tiles) may run 16 outputs per thread instead
    of 8; every output's sum runs in the same order, so the field is the same
    bit for bit."""
    w, h = 1920, 1080
    p = wl.fft3_params(w, h, conv="directMulti")
    p["noiseAmount"] = 0.05
    init = wl.patches(w, h, 12, 96, seed=8)
    out = []
    for ox in ("8", "16"):
        monkeypatch.setenv("LENIA_DIRECT_OX", ox)
        m = lb.LeniaModule(p, w, h)
        assert m.info()["direct_outputs_per_thread"] == int(ox)
        m.reset(3)
        m.upload(init)
        for f in range(2):
            m.encode(f, 2)
        out.append(m.field())
        m.close()
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("w,h,conv,radius", [(1920, 1080, "directMulti", 24), (1280, 720, "direct", 32),
                                             (1920, 1080, "direct", 13), (1024, 512, "direct", 7)])
def test_direct_two_rows_per_thread_same_bits(monkeypatch, w, h, conv, radius):
    """Two output rows per thread (each staged input chunk feeding two kernel
    rows) against one row per thread, for both outputs-per-thread widths
    where the tile allows them: the same bits (every output sums its taps in
    the same order; the union of two rows' chunk spans adds exact zeros)."""
    p = wl.fft3_params(w, h, conv=conv) if conv == "directMulti" else {"radius": radius, "dt": 0.2,
                                                                       "growthMode": 0}
    p["radius"] = radius
    p["noiseAmount"] = 0.05
    init = wl.patches(w, h, 12, 96, seed=8)
    out = {}
    for ox in ("8", "16"):
        for oy in ("1", "2"):
            monkeypatch.setenv("LENIA_DIRECT_OX", ox)
            monkeypatch.setenv("LENIA_DIRECT_OY", oy)
            m = lb.LeniaModule(p, w, h)
            info = m.info()
            if (info["direct_outputs_per_thread"], info["direct_rows_per_thread"]) != (int(ox), int(oy)):
                m.close()
                continue  # the tile this size gets has no such variant
            m.reset(3)
            m.upload(init)
            for f in range(2):
                m.encode(f, 2)
            out[(ox, oy)] = m.field()
            m.close()
    assert ("8", "2") in out, "two rows per thread never ran"
    ref = out[("8", "1")]
    for k, v in out.items():
        np.testing.assert_array_equal(v, ref, err_msg=str(k))


def test_direct_tma_off_for_unaligned_widths():
    m = lb.LeniaModule({"radius": 5}, 37, 23)  # row stride not a multiple of 16 bytes
    assert m.info()["direct_tma"] is False
    m.close()


_CHAIN_SNIPPET = r"""
import hashlib, sys
sys.path.insert(0, {root!r})
import life_simulation_b200 as lb
from life_simulation_b200 import workloads as wl
w, h = 384, 216
p = wl.fft3_params(w, h)
p["noiseAmount"] = 0.05
m = lb.LeniaModule(p, w, h)
m.reset(11)
m.upload(wl.patches(w, h, 6, 40, seed=3))
for f in range(4):
    m.encode(f, 3)
print(hashlib.sha256(m.field().tobytes()).hexdigest())
"""


def test_chained_launches_change_no_bits():
    """Consecutive spectral passes launched with programmatic dependent
    launch (the default) and in plain stream order (LENIA_CHAINED_LAUNCH=0,
    read once per process, so each setting runs in its own process) give the
    same field bit for bit."""
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = _CHAIN_SNIPPET.format(root=root)
    out = {}
    for env in ("1", "0"):
        e = dict(os.environ, LENIA_CHAINED_LAUNCH=env)
        r = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[env] = r.stdout.strip().splitlines()[-1]
    assert out["1"] == out["0"]
