"""The parameter bus and scene loader against the reference's own
ParameterBus.cpp / Scene.cpp (compiled for the CPU in oracle/_ref): the same
mappings, bases, overrides and per-frame inputs give bit-identical values.
Host code only; no GPU."""
import json

import numpy as np
import pytest

import life_simulation_b200 as lb
from oracle.lenia_oracle import REF_ENV_CHANNELS, REF_ENV_PARTS, REF_LANES, REF_SCALARS, RefBus, RefLenia

pytestmark = pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built")

SOURCES = (
    ["kick", "snare.raw", "hihat.peak", "perc.trigger", "beat.hold", "kick.smoothed", "snare.bogus"]
    + ["rms", "low", "mid", "high", "centroid", "flux", "time", "low.raw"]
    + ["lane." + n for n in REF_LANES] + ["lane.unknown"]
    + ["section.energy", "section.progress", "section.changed", "section.index", "section.is:peak",
       "section.n:2", "section.bogus"]
    + ["event:freeze", "event:freeze.active", "event:freeze.started", "event:freeze.ended",
       "event:freeze.progress", "event:freeze.cutoff", "event:warp.cutoff", "event:warp.progress"]
    + ["time.sin:2.5", "time.tri:1.7@0.25", "time.ramp:0.9", "time.noise:0.6", "time.noise:1.3@0.1",
       "time.sin:0.01"]
    + ["bogus"]
)
TARGETS = ["lenia0.growthMu", "lenia0.growthSigma", "lenia0.dt", "lenia0.noiseAmount", "rd0.feed"]


def random_mappings(rng, n):
    out = []
    for _ in range(n):
        lo, hi = sorted(rng.uniform(-1.0, 2.0, 2))
        norm = rng.random() < 0.4
        out.append(dict(source=str(rng.choice(SOURCES)), target=str(rng.choice(TARGETS)),
                        in_min=float(lo) if norm else 0.0, in_max=float(hi) if norm else 0.0,
                        scale=float(rng.uniform(-2, 2)), offset=float(rng.uniform(-0.5, 0.5)),
                        smoothing=float(rng.choice([0.0, 0.0, 0.05, 0.5, 2.0])),
                        mode=str(rng.choice(["add", "set", "mul", "multiply"]))))
    return out


def frame_inputs(rng):
    feats = {}
    for ch in REF_ENV_CHANNELS:
        for part in REF_ENV_PARTS:
            feats[f"{ch}.{part}"] = float(np.float32(rng.random()))
    for n in REF_SCALARS:
        feats[n] = float(np.float32(rng.random() * 3))
    for n in REF_LANES:
        feats["lane." + n] = float(np.float32(rng.random()))
    feats["section.energy"] = float(np.float32(rng.random()))
    feats["section.progress"] = float(np.float32(rng.random()))
    feats["section.changed"] = float(rng.random() < 0.2)
    role = str(rng.choice(["peak", "coda", "build"]))
    index = int(rng.integers(-1, 4))
    events = []
    if rng.random() < 0.6:
        events.append(dict(type="freeze", progress=float(np.float32(rng.random())), started=bool(rng.random() < 0.3),
                           ended=bool(rng.random() < 0.3),
                           curve="cutoff" if rng.random() < 0.7 else "",
                           curve_value=float(np.float32(rng.random() * 1000))))
    return feats, role, index, events


def feed(bus: lb.ParamBus, feats, role, index, events):
    bus.clear_features()
    for k, v in feats.items():
        bus.set_feature(k, v)
    bus.set_section(role, index)
    for e in events:
        t = "event:" + e["type"]
        bus.set_feature(t + ".active", 1.0)
        bus.set_feature(t + ".started", float(e["started"]))
        bus.set_feature(t + ".ended", float(e["ended"]))
        bus.set_feature(t + ".progress", e["progress"])
        if e.get("curve"):
            bus.set_feature(t + "." + e["curve"], e["curve_value"])


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_bus_matches_reference_bit_for_bit(seed):
    rng = np.random.default_rng(seed)
    mine, ref = lb.ParamBus(seed=77 + seed), RefBus(seed=77 + seed)
    for m in random_mappings(rng, 40):
        mine.add_mapping(**m)
        ref.add_mapping(**m)
    for t in TARGETS[:3]:
        v = float(np.float32(rng.random()))
        mine.set_base(t, v)
        ref.set_base(t, v)
    for frame in range(240):
        if frame == 100:
            mine.set_override("lenia0.dt", 0.05)
            ref.set_override("lenia0.dt", 0.05)
        if frame == 150:
            mine.clear_override("lenia0.dt")
            ref.clear_override("lenia0.dt")
        feats, role, index, events = frame_inputs(rng)
        dt = float(np.float32(1.0 / 60.0 + rng.uniform(-2e-3, 2e-3)))
        feed(mine, feats, role, index, events)
        mine.update(dt)
        ref.update(feats, dt, role, index, events)
        for t in TARGETS + ["lenia0.unmapped"]:
            for fb in (0.0, 0.25):
                a, b = mine.value(t, fb), ref.value(t, fb)
                assert a == b or (np.isnan(a) and np.isnan(b)), (frame, t, fb, a, b)


def test_long_run_clock_and_time_sources():
    """8 hours of 1/60 s frames: the double clock keeps the time sources'
    phase (the reference's point of keeping it in double)."""
    mine, ref = lb.ParamBus(seed=5), RefBus(seed=5)
    for src in ("time.sin:600", "time.tri:1080@0.3", "time.ramp:37", "time.noise:90"):
        mine.add_mapping(src, "x." + src, mode="set")
        ref.add_mapping(src, "x." + src, mode="set")
    dt = float(np.float32(1.0 / 60.0))
    for frame in range(8 * 3600 * 60):
        mine.update(dt)
        ref.update({}, dt)
        if frame % 86400 == 0 or frame > 8 * 3600 * 60 - 3:
            for src in ("time.sin:600", "time.tri:1080@0.3", "time.ramp:37", "time.noise:90"):
                assert mine.value("x." + src) == ref.value("x." + src)


SCENE = {
    "seed": 4242,
    "resolution": [256, 128],
    "modules": [
        {"type": "Lenia", "name": "lenia0",
         "params": {"convMode": "fft", "radius": 10, "dt": 0.1, "growthMu": 0.15, "growthSigma": 0.017,
                    "muJitter": 0.5, "fftAnySize": True, "injectAmount": 0, "palette": [1, 2, 3]}},
        {"type": "ReactionDiffusion", "name": "rd0", "params": {"feed": 0.037, "kill": 0.06, "wrap": False}},
    ],
    "audioMappings": [
        {"source": "kick", "target": "lenia0.growthMu", "scale": 0.02, "smoothing": 0.2},
        {"source": "rms", "target": "rd0.feed", "mode": "mul", "offset": 1.0},
    ],
    "musicMappings": [
        {"source": "section.energy", "target": "lenia0.growthSigma", "mode": "set", "inMin": 0.2, "inMax": 0.8,
         "scale": 0.01, "offset": 0.012},
        {"source": "event:freeze.cutoff", "target": "lenia0.dt", "mode": "set", "inMin": 200, "inMax": 2000,
         "scale": 0.1},
    ],
    "automation": [
        {"source": "time.noise:3@0.5", "target": "lenia0.muJitter", "scale": 0.3},
        {"source": "time.sin:5", "target": "rd0.kill", "scale": 0.01},
    ],
}


def test_scene_load_matches_reference():
    mine, ref = lb.ParamBus(), RefBus()
    info = mine.load_scene(SCENE)
    ref.load_scene(SCENE)
    assert info == {"seed": 4242, "width": 256, "height": 128, "num_modules": 2, "num_mappings": 6}
    keys = ["lenia0.growthMu", "lenia0.growthSigma", "lenia0.dt", "lenia0.muJitter", "lenia0.radius",
            "lenia0.fftAnySize", "rd0.feed", "rd0.kill", "rd0.wrap", "lenia0.palette"]
    rng = np.random.default_rng(9)
    for frame in range(120):
        feats, role, index, events = frame_inputs(rng)
        feed(mine, feats, role, index, events)
        mine.update(1.0 / 60.0)
        ref.update(feats, 1.0 / 60.0, role, index, events)
        for k in keys:
            assert mine.value(k, -1.0) == ref.value(k, -1.0), (frame, k)


@pytest.mark.parametrize("bad", ["time.sin:-1", "time.sin:0", "time.foo:1", "time.sin", "time.tri:abc",
                                 "time.ramp:2@x"])
def test_malformed_time_sources_fail_like_the_reference(bad):
    scene = json.loads(json.dumps(SCENE))
    scene["automation"].append({"source": bad, "target": "lenia0.dt"})
    with pytest.raises(ValueError):
        RefBus().load_scene(scene)
    with pytest.raises(lb.LeniaError, match="time source"):
        lb.ParamBus().load_scene(scene)
    with pytest.raises(lb.LeniaError, match="time source"):
        lb.ParamBus().add_mapping(bad, "lenia0.dt")


def test_scene_structure_errors():
    for scene in ({"modules": [{"name": "x"}]},
                  {"audioMappings": [{"source": "kick"}]},
                  {"musicMappings": [{"target": "a.b"}]}):
        with pytest.raises(ValueError):
            RefBus().load_scene(scene)
        with pytest.raises(lb.LeniaError):
            lb.ParamBus().load_scene(scene)
