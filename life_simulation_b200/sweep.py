"""Parameter sweeps over the batched form (the reference's LifePresetLab).

The reference explores a scene's parameters one variant at a time: each
variant is a copy of the scene with some module params overridden, run in its
own SceneRunner for a number of frames, and rated by the activity of its
colour layer (Apps/LifePresetLab/main.cpp). This module keeps that
vocabulary -- the sweep file, the variant enumeration, the overrides, the
luma activity and the "alive" rule -- and runs all variants at once as the
worlds of one LeniaBatch.

Sweep file (main.cpp:103-190)::

    {"mode": "cartesian" | "per-axis",          # default "cartesian"
     "seeds": [7777, 1234],                      # default: the scene's seed
     "axes": [{"target": "lenia0.growthMu", "values": [0.13, 0.15]},
              {"target": "lenia0.growthSigma", "range": [0.014, 0.022], "steps": 3}]}

cartesian: every combination, last axis fastest, for each seed; per-axis:
one axis at a time from the base scene, for each seed. Variant ids "v0000".
"""
from __future__ import annotations

import copy
import json
from dataclasses import dataclass, field
from typing import Any, List, Optional, Sequence, Tuple

import numpy as np

from . import BATCH_AUTO, CORE_EXP, CORE_GAUSS_SHELL, LeniaBatch, colormap_from_params, make_world


class SweepError(ValueError):
    pass


@dataclass
class AxisSpec:
    target: str
    values: List[Any]


@dataclass
class SweepConfig:
    mode: str = "cartesian"
    seeds: List[int] = field(default_factory=list)
    axes: List[AxisSpec] = field(default_factory=list)


@dataclass
class Variant:
    id: str
    seed: int
    overrides: List[Tuple[str, Any]]


def resolve_axis(a: dict) -> AxisSpec:
    """An axis with its value list (main.cpp:109-151): "values" verbatim, or
    "range": [lo, hi] with "steps" points, both ends included."""
    target = a.get("target", "")
    if not target:
        raise SweepError('sweep axis missing "target"')
    if "." not in target:
        raise SweepError(f'sweep axis target "{target}" must be "module.param"')
    if "values" in a:
        vals = a["values"]
        if not isinstance(vals, list) or not vals:
            raise SweepError(f'axis "{target}": "values" must be a non-empty array')
        return AxisSpec(target, list(vals))
    if "range" in a:
        r = a["range"]
        if (not isinstance(r, list) or len(r) != 2
                or not all(isinstance(x, (int, float)) and not isinstance(x, bool) for x in r)):
            raise SweepError(f'axis "{target}": "range" must be [lo, hi]')
        lo, hi = float(r[0]), float(r[1])
        steps = a.get("steps", 0)
        if not isinstance(steps, int) or steps < 1:
            raise SweepError(f'axis "{target}": "steps" must be >= 1')
        if steps == 1:
            return AxisSpec(target, [lo])
        return AxisSpec(target, [lo + (i / (steps - 1)) * (hi - lo) for i in range(steps)])
    raise SweepError(f'axis "{target}": need "values" or "range"+"steps"')


def load_sweep(j) -> SweepConfig:
    """A sweep document (dict or JSON text), validated as main.cpp:153-190."""
    if isinstance(j, str):
        j = json.loads(j)
    mode = j.get("mode", "cartesian")
    if mode not in ("cartesian", "per-axis"):
        raise SweepError(f'sweep "mode" must be "cartesian" or "per-axis" (got "{mode}")')
    cfg = SweepConfig(mode=mode)
    if "seeds" in j:
        if not isinstance(j["seeds"], list):
            raise SweepError('sweep "seeds" must be an array')
        cfg.seeds = [int(s) for s in j["seeds"]]
    if "axes" in j:
        if not isinstance(j["axes"], list):
            raise SweepError('sweep "axes" must be an array')
        cfg.axes = [resolve_axis(a) for a in j["axes"]]
    return cfg


def cartesian_indices(axes: Sequence[AxisSpec]) -> List[Tuple[int, ...]]:
    """Every combination of value indices, last axis fastest (an odometer);
    no axes: one empty combination."""
    if not axes:
        return [()]
    if any(not ax.values for ax in axes):
        return []
    counter = [0] * len(axes)
    out = []
    while True:
        out.append(tuple(counter))
        a = len(axes) - 1
        while a >= 0:
            counter[a] += 1
            if counter[a] < len(axes[a].values):
                break
            counter[a] = 0
            a -= 1
        if a < 0:
            return out


def build_variants(sweep: SweepConfig, base_seed: int) -> List[Variant]:
    """The variant list (main.cpp:233-270)."""
    seeds = sweep.seeds or [base_seed]
    raw: List[Tuple[int, List[Tuple[str, Any]]]] = []
    if sweep.mode == "cartesian":
        combos = cartesian_indices(sweep.axes)
        for seed in seeds:
            for combo in combos:
                raw.append((seed, [(ax.target, ax.values[i]) for ax, i in zip(sweep.axes, combo)]))
    else:
        for seed in seeds:
            for ax in sweep.axes:
                for v in ax.values:
                    raw.append((seed, [(ax.target, v)]))
    return [Variant(f"v{i:04d}", seed, ov) for i, (seed, ov) in enumerate(raw)]


def apply_overrides(scene: dict, variant: Variant) -> dict:
    """The variant's scene: its seed, and each override written into the
    named module's params (main.cpp:303-324)."""
    s = copy.deepcopy(scene)
    s["seed"] = variant.seed
    for target, value in variant.overrides:
        mod, key = target.split(".", 1)
        found = next((m for m in s.get("modules", []) if m.get("name", m.get("type")) == mod), None)
        if found is None:
            raise SweepError(f'unknown module "{mod}" (target "{target}")')
        found.setdefault("params", {})[key] = value
    return s


def is_alive(mean: float, stddev: float) -> bool:
    """main.cpp:84-86: visible but not saturated, and not uniform."""
    return 0.01 <= mean <= 0.7 and stddev >= 0.02


# Per-frame params the batched form evolves with (single-ring Lenia worlds);
# the others must keep the reference module's neutral defaults.
_NEUTRAL = {"noiseAmount": 0.0, "muJitter": 0.0, "injectAmount": 0.0}


def scene_world(scene: dict, module: str):
    """(lenia_world, initCoverage, initScale, params) of a scene's Lenia module, with
    the reference module's defaults (Lenia.h:77-105, Lenia.cpp:336-356)."""
    mod = next((m for m in scene.get("modules", []) if m.get("name", m.get("type")) == module), None)
    if mod is None or mod.get("type") != "Lenia":
        raise SweepError(f'scene has no Lenia module named "{module}"')
    p = mod.get("params", {})
    res = scene.get("resolution", [1920, 1080])
    w, h = int(p.get("simWidth", 0)) or int(res[0]), int(p.get("simHeight", 0)) or int(res[1])
    if (w, h) != (int(res[0]), int(res[1])):
        raise SweepError("the batched sweep needs the sim size equal to the scene resolution")
    if "kernels" in p or p.get("initMode", "noise") != "noise" or "organism" in p:
        raise SweepError('the batched sweep runs single-ring worlds with the noise init ("kernels", '
                         '"organism" and stamp inits are not supported)')
    for key in ("audioMappings", "musicMappings", "automation"):
        if any(str(m.get("target", "")).startswith(module + ".") for m in scene.get(key, [])):
            raise SweepError(f'the batched sweep does not run "{key}" mappings of the swept module')
    for k, v in _NEUTRAL.items():
        if float(p.get(k, v)) != v:
            raise SweepError(f'the batched sweep does not support "{k}" (got {p[k]})')
    core = CORE_EXP if p.get("kernelCore", "gaussShell") == "exp" else CORE_GAUSS_SHELL
    world = make_world(w, h, int(round(float(p.get("radius", 13)))), float(p.get("growthMu", 0.15)),
                       float(p.get("growthSigma", 0.017)), float(p.get("dt", 0.1)),
                       growth_mode=int(float(p.get("growthMode", 1)) + 0.5), kernel_core=core,
                       shell_mu=float(p.get("kernelShellMu", 0.5)),
                       shell_sigma=float(p.get("kernelShellSigma", 0.15)), seed=int(scene.get("seed", 1234)))
    return world, float(p.get("initCoverage", 0.4)), float(p.get("initScale", 24.0)), p


def run_sweep(scene: dict, sweep, frames: int = 240, substeps: int = 1, module: str = "lenia0",
              policy: int = BATCH_AUTO, rank: int = 0, world_size: int = 1, group=None) -> dict:
    """Every variant of `sweep` on `scene`, run together for `frames` frames
    of `substeps` substeps; activity measured on the last frame (the lab's
    default thumbnail). Returns {"mode", "frames", "variants": [{"id", "seed",
    "overrides", "activity": {"meanLuma", "stddevLuma", "alive"}}],
    "aliveCount"}.

    With world_size > 1 (one process per GPU, torch.distributed initialised)
    every rank runs its cost-balanced share of the variants
    (life_simulation_b200.shard.partition) as its own batch and the per-
    variant records are gathered afterwards: every rank returns the same
    result as one GPU would."""
    from .shard import gather_records, partition, world_cost

    cfg = sweep if isinstance(sweep, SweepConfig) else load_sweep(sweep)
    if frames < 1:
        raise SweepError("frames must be >= 1")
    variants = build_variants(cfg, int(scene.get("seed", 1234)))
    worlds, inits, cmap = [], [], None
    for v in variants:
        vs = apply_overrides(scene, v)
        world, cov, scale, params = scene_world(vs, module)
        worlds.append(world)
        inits.append((v.seed, cov, scale))
        cm = colormap_from_params(params)
        if cmap is None:
            cmap = cm
        elif bytes(cm) != bytes(cmap):
            raise SweepError("all variants must share one colour map")
    mine = list(range(len(variants)))
    if world_size > 1:
        costs = [world_cost(w.width, w.height, w.radius) for w in worlds]
        mine = partition(costs, world_size)[rank]
    records = []
    if mine:
        batch = LeniaBatch([worlds[i] for i in mine], policy)
        for j, i in enumerate(mine):
            batch.init_noise(j, *inits[i])
        batch.step(frames * max(1, substeps))
        mean, std = batch.activity(cmap)
        paths = [batch.path(j) for j in range(len(mine))]
        batch.close()
        for j, i in enumerate(mine):
            v = variants[i]
            records.append({"world": i, "id": v.id, "seed": v.seed,
                            "overrides": {t: val for t, val in v.overrides},
                            "activity": {"meanLuma": float(mean[j]), "stddevLuma": float(std[j]),
                                         "alive": is_alive(float(mean[j]), float(std[j]))},
                            "path": "fft" if paths[j] == 1 else "direct"})
    if world_size > 1:
        records = gather_records(records, group)
    out = [{k: r[k] for k in ("id", "seed", "overrides", "activity", "path")} for r in records]
    return {"mode": cfg.mode, "frames": frames, "substeps": substeps, "variants": out,
            "aliveCount": sum(1 for e in out if e["activity"]["alive"])}
