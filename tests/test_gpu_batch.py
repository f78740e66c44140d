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
