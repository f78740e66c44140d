"""A Lenia module built from a scene document and driven through a shared
parameter bus (audio, section and time-source mappings) against the
reference's own module and bus compiled for the CPU, fed the same inputs."""
import numpy as np
import pytest

import life_simulation_b200 as lb
from oracle.lenia_oracle import RefBus, RefLenia

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built")]

SCENE = {
    "seed": 99,
    "resolution": [128, 128],
    "modules": [
        {"type": "Lenia", "name": "lenia0",
         "params": {"convMode": "direct", "radius": 9, "dt": 0.1, "growthMu": 0.15,
                    "growthSigma": 0.017, "growthMode": 0, "initCoverage": 0.5, "initScale": 20}},
        {"type": "ReactionDiffusion", "name": "rd0", "params": {"feed": 0.03}},
    ],
    "audioMappings": [
        {"source": "kick", "target": "lenia0.growthMu", "scale": 0.02, "smoothing": 0.1},
        {"source": "rms", "target": "lenia0.growthSigma", "mode": "mul", "scale": 0.2, "offset": 0.9},
    ],
    "musicMappings": [
        {"source": "section.is:peak", "target": "lenia0.noiseAmount", "scale": 0.5},
    ],
    "automation": [
        {"source": "time.sin:0.5", "target": "lenia0.dt", "scale": 0.03},
        {"source": "time.noise:0.2", "target": "lenia0.muJitter", "scale": 0.4, "offset": 0.4},
    ],
}


def test_scene_module_with_shared_bus_matches_reference():
    bus = lb.ParamBus()
    bus.load_scene(SCENE)
    m = lb.scene_module(SCENE, "lenia0", bus)
    assert (m.width, m.height) == (128, 128)
    ref = RefLenia(SCENE["modules"][0]["params"], 128, 128, "lenia0")
    rbus = RefBus(session=ref)
    rbus.load_scene(SCENE)
    m.reset(7)
    ref.reset(7)
    rng = np.random.default_rng(1)
    for frame in range(12):
        feats = {"kick.smoothed": float(np.float32(rng.random())), "rms": float(np.float32(rng.random()))}
        role = "peak" if frame % 4 == 1 else "build"
        bus.clear_features()
        for k, v in feats.items():
            bus.set_feature(k, v)
        bus.set_section(role, frame // 4)
        bus.update(1.0 / 60.0)
        rbus.update(feats, 1.0 / 60.0, role, frame // 4)
        for key in ("lenia0.dt", "lenia0.growthMu", "lenia0.growthSigma", "lenia0.noiseAmount", "lenia0.muJitter"):
            assert bus.value(key) == rbus.value(key), (frame, key)
        m.encode(frame, 1, audio_frame=frame)
        g = ref.encode(frame, 1, frame)
        err = float(np.abs(m.field() - g).max())
        # The direct path's bar against the reference (noise and jitter on).
        assert err <= 5e-5, (frame, err)
    m.close()


def test_scene_module_errors_and_own_bus():
    with pytest.raises(lb.LeniaError, match="ReactionDiffusion"):
        lb.scene_module(SCENE, "rd0")
    with pytest.raises(lb.LeniaError, match="no module named"):
        lb.scene_module(SCENE, "nope")
    # Without a shared bus the context loads the scene into its own bus.
    m = lb.scene_module(SCENE)
    fp = m.frame_params(0)
    assert abs(fp.growth_mu - 0.15) < 1e-7 and abs(fp.dt - 0.1) < 1e-7
    m.set_override("growthMu", 0.2)
    assert abs(m.frame_params(0).growth_mu - 0.2) < 1e-7
    m.close()
