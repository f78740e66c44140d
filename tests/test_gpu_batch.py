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


@pytest.mark.parametrize("policy", [lb.BATCH_AUTO, lb.BATCH_DIRECT, lb.BATCH_FFT])
def test_persistent_form_equals_per_size_form(policy):
    """One persistent launch per substep (a work list of every world's column
    groups, direct tiles and row groups) gives the same bits as the per-size
    launches: the same plans, twiddles and per-pixel arithmetic, only grouped
    differently over CTAs."""
    worlds = mixed_worlds()
    if policy == lb.BATCH_FFT:
        worlds = [w for w in worlds if (w.width, w.height) != (96, 80)]
    inits = [central_square(w.width, w.height, i) for i, w in enumerate(worlds)]
    fields = {}
    for form in (lb.BATCH_FORM_PER_SIZE, lb.BATCH_FORM_PERSISTENT):
        b = lb.LeniaBatch(worlds, policy)
        b.set_launch_form(form)
        assert b.launch_form() == form
        for i, a in enumerate(inits):
            b.upload(i, a)
        b.step(2)
        b.step(3)  # two graph replays of different lengths and parities
        b.sync()
        fields[form] = [b.field(i) for i in range(len(worlds))]
        b.close()
    for i, w in enumerate(worlds):
        a, p = fields[lb.BATCH_FORM_PER_SIZE][i], fields[lb.BATCH_FORM_PERSISTENT][i]
        assert np.array_equal(a, p), (policy, i, w.width, w.height, float(np.abs(a - p).max()))
        assert p.max() > 0.0  # alive, so the comparison is not of zeros


def test_persistent_form_replays_match_single_world_contexts():
    """Graph replays of odd and even lengths in the persistent form (the
    launches alternate the parity tables and counter sets) leave each world
    where the same world stepped alone through a single-world context is."""
    worlds = mixed_worlds()[:3]
    b = lb.LeniaBatch(worlds, lb.BATCH_FFT)
    b.set_launch_form(lb.BATCH_FORM_PERSISTENT)
    inits = [central_square(w.width, w.height, 10 + i) for i, w in enumerate(worlds)]
    for i, a in enumerate(inits):
        b.upload(i, a)
    for k in (1, 2, 3, 1):
        b.step(k)
    b.sync()
    for i, w in enumerate(worlds):
        m = lb.LeniaModule(lb.single_world_params(w, "fft"), w.width, w.height)
        m.reset(w.seed)
        m.upload(inits[i])
        for f in range(7):
            m.encode(f, 1)
        err = float(np.abs(b.field(i) - m.field()).max())
        assert err <= 2e-5, (i, err)
        m.close()
    b.close()


def test_sweep_batch_persistent_form_vs_fp64_oracle():
    """The 512-world sweep in the persistent form: one world of each size
    class stepped once from the batch's own states, within 1e-5 of one FP64
    oracle step (as test_sweep_batch_worlds_vs_fp64_oracle does for the form
    the autotuner picks)."""
    from life_simulation_b200 import workloads as wl
    from oracle.lenia_oracle import OracleLenia

    params, inits = wl.sweep512()
    worlds = [lb.make_world(**p) for p in params]
    b = lb.LeniaBatch(worlds, lb.BATCH_AUTO)
    b.set_launch_form(lb.BATCH_FORM_PERSISTENT)
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
        o.encode(0)
        oracles[i] = o
    b.step(3)
    worst = {i: 0.0 for i in sample}
    for s in range(6):
        states = {i: b.field(i) for i in sample}
        b.step(1)
        for i in sample:
            o = oracles[i]
            o.state = states[i].astype(np.float64)
            o.step_once(o.frame_params(), 0, 3 + s, 3 + s)
            worst[i] = max(worst[i], float(np.abs(b.field(i) - o.state).max()))
    b.sync()
    assert max(worst.values()) <= 1e-5, {(worlds[i].width, worlds[i].height): e for i, e in worst.items()}
    b.close()


@pytest.mark.parametrize("form", [lb.BATCH_FORM_PER_SIZE, lb.BATCH_FORM_PERSISTENT])
def test_odd_sized_world_before_spectral_worlds(form):
    """A direct world of odd size (97 x 81) ahead of spectral worlds: every
    field still starts 16-byte aligned for the row passes' asynchronous
    copies, and each world matches its single-world context."""
    worlds = [lb.make_world(97, 81, radius=9, mu=0.15, sigma=0.02, dt=0.1, seed=7),
              lb.make_world(128, 128, radius=20, mu=0.2, sigma=0.03, dt=0.1, seed=8),
              lb.make_world(256, 256, radius=24, mu=0.25, sigma=0.04, dt=0.1, seed=9)]
    b = lb.LeniaBatch(worlds, lb.BATCH_AUTO)
    b.set_launch_form(form)
    assert b.path(0) == lb.CONV_DIRECT
    inits = [central_square(w.width, w.height, 20 + i) for i, w in enumerate(worlds)]
    for i, a in enumerate(inits):
        b.upload(i, a)
    b.step(4)
    b.sync()
    for i, w in enumerate(worlds):
        conv = "fft" if b.path(i) == lb.CONV_FFT else "direct"
        m = lb.LeniaModule(lb.single_world_params(w, conv), w.width, w.height)
        m.reset(w.seed)
        m.upload(inits[i])
        for f in range(4):
            m.encode(f, 1)
        err = float(np.abs(b.field(i) - m.field()).max())
        assert err <= 2e-5, (form, i, conv, err)
        m.close()
    b.close()
