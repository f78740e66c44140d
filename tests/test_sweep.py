"""Sweep files and variant enumeration (the reference's LifePresetLab
semantics, Apps/LifePresetLab/main.cpp:103-324). No GPU."""
import pytest

from life_simulation_b200.sweep import (SweepError, apply_overrides, build_variants, cartesian_indices, is_alive,
                                        load_sweep, scene_world)


def test_per_axis_with_seeds_and_range():
    cfg = load_sweep({"mode": "per-axis", "seeds": [11, 22],
                      "axes": [{"target": "lenia0.growthMu", "values": [0.13, 0.15, 0.17]},
                               {"target": "lenia0.growthSigma", "range": [0.014, 0.022], "steps": 3}]})
    assert cfg.axes[1].values == [0.014, 0.014 + 0.5 * (0.022 - 0.014), 0.022]
    vs = build_variants(cfg, base_seed=5)
    assert len(vs) == 12 and [v.id for v in vs[:3]] == ["v0000", "v0001", "v0002"]
    assert [(v.seed, v.overrides) for v in vs[:4]] == [
        (11, [("lenia0.growthMu", 0.13)]), (11, [("lenia0.growthMu", 0.15)]),
        (11, [("lenia0.growthMu", 0.17)]), (11, [("lenia0.growthSigma", 0.014)])]
    assert vs[6].seed == 22 and vs[6].overrides == [("lenia0.growthMu", 0.13)]


def test_cartesian_odometer_last_axis_fastest():
    cfg = load_sweep({"axes": [{"target": "a.x", "values": [1, 2]}, {"target": "a.y", "values": [3, 4, 5]},
                               {"target": "b.z", "range": [0, 1], "steps": 1}]})
    assert cfg.mode == "cartesian" and cfg.axes[2].values == [0.0]
    assert cartesian_indices(cfg.axes) == [(0, 0, 0), (0, 1, 0), (0, 2, 0), (1, 0, 0), (1, 1, 0), (1, 2, 0)]
    vs = build_variants(cfg, base_seed=9)
    assert len(vs) == 6 and all(v.seed == 9 for v in vs)
    assert vs[4].overrides == [("a.x", 2), ("a.y", 4), ("b.z", 0.0)]
    assert build_variants(load_sweep({}), 3)[0].overrides == []  # a pure seed sweep


@pytest.mark.parametrize("bad", [
    {"mode": "grid"}, {"seeds": 5}, {"axes": {}}, {"axes": [{"values": [1]}]},
    {"axes": [{"target": "nodot", "values": [1]}]}, {"axes": [{"target": "a.b", "values": []}]},
    {"axes": [{"target": "a.b", "range": [0]}]}, {"axes": [{"target": "a.b", "range": [0, 1], "steps": 0}]},
    {"axes": [{"target": "a.b"}]},
])
def test_sweep_errors(bad):
    with pytest.raises(SweepError):
        load_sweep(bad)


def test_overrides_and_world():
    scene = {"seed": 1, "resolution": [64, 64],
             "modules": [{"type": "Lenia", "name": "lenia0", "params": {"radius": 9, "growthMu": 0.15}}]}
    v = build_variants(load_sweep({"seeds": [42], "axes": [{"target": "lenia0.growthMu", "values": [0.2]}]}), 1)[0]
    s2 = apply_overrides(scene, v)
    assert s2["seed"] == 42 and s2["modules"][0]["params"]["growthMu"] == 0.2 and scene["seed"] == 1
    w, cov, scale, _ = scene_world(s2, "lenia0")
    assert (w.width, w.height, w.radius, w.seed, w.growth_mode) == (64, 64, 9, 42, 1)
    assert abs(w.mu - 0.2) < 1e-7 and abs(w.sigma - 0.017) < 1e-7 and (cov, scale) == (0.4, 24.0)
    with pytest.raises(SweepError, match="unknown module"):
        apply_overrides(scene, build_variants(load_sweep({"axes": [{"target": "x.y", "values": [1]}]}), 1)[0])
    bad = {**scene, "modules": [{"type": "Lenia", "name": "lenia0", "params": {"noiseAmount": 0.1}}]}
    with pytest.raises(SweepError, match="noiseAmount"):
        scene_world(bad, "lenia0")
    mapped = {**scene, "automation": [{"source": "time.sin:3", "target": "lenia0.growthMu"}]}
    with pytest.raises(SweepError, match="automation"):
        scene_world(mapped, "lenia0")


def test_alive_rule():
    assert is_alive(0.2, 0.05) and not is_alive(0.005, 0.05) and not is_alive(0.8, 0.05)
    assert not is_alive(0.2, 0.01) and is_alive(0.01, 0.02) and is_alive(0.7, 0.02)
