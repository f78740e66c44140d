"""The batched form: every world of a batch evolves exactly as the same world
stepped alone through a single-world context (direct or spectral path), for
all three path policies, over worlds of uneven sizes and parameters; and the
per-world activity statistics match numpy on the downloaded fields."""
import numpy as np
import pytest

import life_simulation_b200 as lb

pytestmark = pytest.mark.gpu


def mixed_worlds():
    rng = np.random.default_rng(3)
    sizes = [(128, 128), (256, 256), (384, 216), (96, 80), (512, 512), (128, 128)]
    out = []
    for i, (w, h) in enumerate(sizes):
        out.append(lb.make_world(w, h, radius=int(rng.integers(8, 33)), mu=float(rng.uniform(0.10, 0.35)),
                                 sigma=float(rng.uniform(0.01, 0.05)), dt=float(rng.uniform(0.05, 0.2)),
                                 growth_mode=0, seed=100 + i))
    return out


def central_square(w, h, seed):
    a = np.zeros((h, w), np.float32)
    s = min(w, h) // 4
    y0, x0 = (h - s) // 2, (w - s) // 2
    a[y0:y0 + s, x0:x0 + s] = np.random.default_rng(seed).random((s, s))
    return a


@pytest.mark.parametrize("policy", [lb.BATCH_AUTO, lb.BATCH_DIRECT, lb.BATCH_FFT])
def test_batch_worlds_match_single_world_contexts(policy):
    worlds = mixed_worlds()
    if policy == lb.BATCH_FFT:  # 96x80 has no compile-time spectral plan
        worlds = [w for w in worlds if (w.width, w.height) != (96, 80)]
    b = lb.LeniaBatch(worlds, policy)
    inits = [central_square(w.width, w.height, i) for i, w in enumerate(worlds)]
    for i, a in enumerate(inits):
        b.upload(i, a)
    steps = 5
    b.step(2)
    b.step(steps - 2)  # two graph replays of different lengths and parities
    for i, w in enumerate(worlds):
        path = b.path(i)
        conv = "fft" if path == lb.CONV_FFT else "direct"
        m = lb.LeniaModule(lb.single_world_params(w, conv), w.width, w.height)
        m.reset(w.seed)
        m.upload(inits[i])
        for f in range(steps):
            m.encode(f, 1)
        # The same kernels' arithmetic; different instantiations may contract
        # a multiply-add differently (one rounding), which 5 chaotic steps
        # can grow to ~1e-6.
        err = float(np.abs(b.field(i) - m.field()).max())
        assert err <= 2e-5, (policy, i, path, err)
        m.close()
    mean, var = b.stats()
    for i in range(len(worlds)):
        f = b.field(i).astype(np.float64)
        assert abs(mean[i] - f.mean()) < 1e-9 and abs(var[i] - f.var()) < 1e-9
    b.close()


def test_batch_auto_prefers_direct_for_small_radius():
    worlds = [lb.make_world(512, 512, radius=3, mu=0.15, sigma=0.02, dt=0.1),
              lb.make_world(512, 512, radius=32, mu=0.15, sigma=0.02, dt=0.1)]
    b = lb.LeniaBatch(worlds, lb.BATCH_AUTO)
    assert b.path(0) == lb.CONV_DIRECT
    assert b.path(1) == lb.CONV_FFT
    b.close()


def test_sweep_batch_worlds_vs_fp64_oracle():
    """The benchmarked 512-world sweep batch (the autotuner's path choice per
    world): one world of each size class compared with the FP64 oracle
    directly. Every step the sampled worlds are set to a state, the whole
    batch steps once, and each sampled world must be within 1e-5 of one FP64
    step of the oracle from the same state (the plain path's per-step bound);
    the states are the batch's own trajectory."""
    from life_simulation_b200 import workloads as wl
    from oracle.lenia_oracle import OracleLenia

    params, inits = wl.sweep512()
    worlds = [lb.make_world(**p) for p in params]
    b = lb.LeniaBatch(worlds, lb.BATCH_AUTO)
    for i, a in enumerate(inits):
        b.upload(i, a)
    sample = []
    for size in [(128, 128), (256, 256), (384, 216), (512, 512)]:
        sample.append(next(i for i, w in enumerate(worlds) if (w.width, w.height) == size))
    oracles = {}
    for i in sample:
        w = worlds[i]
        conv = "fft" if b.path(i) == lb.CONV_FFT else "direct"
        o = OracleLenia(lb.single_world_params(w, conv), w.width, w.height, "f64")
        o.reset(w.seed)
        o.set_initial_field(inits[i])
        o.encode(0)  # builds the kernels; the state is replaced below
        oracles[i] = o
    b.step(3)  # into the live phase
    worst = {i: 0.0 for i in sample}
    for s in range(8):
        states = {i: b.field(i) for i in sample}
        b.step(1)
        for i in sample:
            o = oracles[i]
            o.state = states[i].astype(np.float64)
            o.step_once(o.frame_params(), 0, 3 + s, 3 + s)
            worst[i] = max(worst[i], float(np.abs(b.field(i) - o.state).max()))
    assert max(worst.values()) <= 1e-5, {(worlds[i].width, worlds[i].height, b.path(i)): e for i, e in worst.items()}
    b.close()
