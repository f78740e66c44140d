"""The batched sweep: per-world luma activity against the reference's colour
map kernels and luma statistic, and a sweep run as one batch against the
reference's one-variant-at-a-time loop (a context per variant)."""
import numpy as np
import pytest
import torch

import life_simulation_b200 as lb
from life_simulation_b200.sweep import apply_overrides, build_variants, is_alive, load_sweep, run_sweep
from oracle.lenia_oracle import RefLenia, ref_colormap

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not RefLenia.available(), reason="oracle/_ref not built")]

SCENE = {"seed": 3, "resolution": [128, 96],
         "modules": [{"type": "Lenia", "name": "lenia0",
                      "params": {"radius": 10, "growthMu": 0.15, "growthSigma": 0.017, "dt": 0.1,
                                 "initCoverage": 0.5, "initScale": 20}}]}
SWEEP = {"mode": "cartesian", "seeds": [7, 8],
         "axes": [{"target": "lenia0.growthMu", "values": [0.12, 0.15, 0.3]},
                  {"target": "lenia0.growthSigma", "range": [0.015, 0.03], "steps": 2}]}


def luma_stats(rgba16f: np.ndarray):
    """computeLumaStats (Apps/LifePresetLab/main.cpp:66-82) on RGBA halves."""
    px = rgba16f.astype(np.float32).astype(np.float64)
    l = 0.2126 * px[..., 0] + 0.7152 * px[..., 1] + 0.0722 * px[..., 2]
    mean = l.sum() / l.size
    var = max(0.0, (l * l).sum() / l.size - mean * mean)
    return mean, np.sqrt(var)


def test_batch_activity_matches_reference_colour_map():
    worlds = [lb.make_world(128, 96, 10, mu, 0.017, 0.1, growth_mode=1, seed=5) for mu in (0.13, 0.15, 0.2)]
    b = lb.LeniaBatch(worlds, lb.BATCH_DIRECT)
    for i in range(len(worlds)):
        b.init_noise(i, 11 + i, 0.5, 20.0)
    b.step(6)
    cm = lb.colormap_from_params({})
    mean, std = b.activity(cm)
    for i in range(len(worlds)):
        ref = ref_colormap(b.field(i), cm.as_dict(), 128, 96).astype(np.float16)
        m, s = luma_stats(ref)
        assert abs(mean[i] - m) <= 1e-6 * max(m, 1e-3) and abs(std[i] - s) <= 1e-6 * max(s, 1e-3), (i, mean[i], m)
    b.close()


def test_sweep_matches_one_variant_at_a_time():
    frames = 8
    res = run_sweep(SCENE, SWEEP, frames=frames, policy=lb.BATCH_DIRECT)
    variants = build_variants(load_sweep(SWEEP), SCENE["seed"])
    assert [v["id"] for v in res["variants"]] == [v.id for v in variants]
    alive = 0
    for v, out in zip(variants, res["variants"]):
        scene = apply_overrides(SCENE, v)
        m = lb.scene_module(scene, "lenia0")
        m.reset(v.seed)
        for f in range(frames):
            m.encode(f, 1)
        img = torch.empty((96, 128, 4), dtype=torch.float16, device="cuda")
        m.render_device(img.data_ptr(), 128, 96)
        torch.cuda.synchronize()
        mean, std = luma_stats(img.cpu().numpy())
        m.close()
        act = out["activity"]
        assert abs(act["meanLuma"] - mean) < 1e-4 and abs(act["stddevLuma"] - std) < 1e-4, (v.id, act, mean, std)
        assert act["alive"] == is_alive(mean, std) or min(abs(mean - 0.01), abs(mean - 0.7), abs(std - 0.02)) < 1e-4
        alive += act["alive"]
    assert res["aliveCount"] == alive


def _sharded_rank(rank, world_size, port, out):
    import os

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        out[rank] = run_sweep(SCENE, SWEEP, frames=8, policy=lb.BATCH_DIRECT, rank=rank, world_size=world_size)
    finally:
        dist.destroy_process_group()


def test_sweep_sharded_over_two_processes_equals_one():
    """Two ranks (here both on the one GPU, each with its own independent
    batch; only the per-variant records cross, on the host) give the same
    result as the whole sweep in one process."""
    import socket

    import torch.multiprocessing as mp

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.spawn(_sharded_rank, args=(2, port, out), nprocs=2, join=True)
    whole = run_sweep(SCENE, SWEEP, frames=8, policy=lb.BATCH_DIRECT)
    for r in range(2):
        got = out[r]
        assert [v["id"] for v in got["variants"]] == [v["id"] for v in whole["variants"]]
        for a, b in zip(got["variants"], whole["variants"]):
            # Same fields; the FP64 luma sums may add in another order
            # (atomics over a differently sized grid).
            for k in ("meanLuma", "stddevLuma"):
                assert a["activity"][k] == pytest.approx(b["activity"][k], rel=1e-12, abs=1e-15), (a["id"], k)
            assert a["activity"]["alive"] == b["activity"]["alive"]
        assert got["aliveCount"] == whole["aliveCount"]
