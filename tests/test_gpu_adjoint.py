"""The adjoint form on the GPU: gradients of a T-step rollout through the
C ABI against the FP64 oracle's adjoint and against central finite
differences (eps = 1e-3, FP64 forward), checkpoint invariance, the
torch.autograd binding, and the full-size batch (32 worlds of 512x512)."""
import numpy as np
import pytest
import torch

import life_simulation_b200 as lb
from life_simulation_b200.adjoint import RolloutParams, rollout
from oracle import lenia_adjoint_oracle as O

pytestmark = pytest.mark.gpu

KERNELS = [{"mu": 0.15, "sigma": 0.03, "weight": 0.6, "betas": [1.0]},
           {"mu": 0.25, "sigma": 0.05, "weight": 0.4, "betas": [0.5, 1.0]}]


def oracle_params(kernels, radius, dt, mode, core, shell_sigma=0.15):
    return O.AdjParams([O.AdjKernel(k["mu"], k["sigma"], k.get("weight", 1.0), list(k["betas"]),
                                    k.get("radiusScale", 1.0)) for k in kernels],
                       radius=radius, dt=dt, growth_mode=mode, core=core, shell_sigma=shell_sigma)


def fields(batch, h, w, seed, lo=0.25, hi=0.75):
    rng = np.random.default_rng(seed)
    a = np.zeros((batch, h, w), np.float32)
    y0, y1, x0, x1 = int(h * lo), int(h * hi), int(w * lo), int(w * hi)
    a[:, y0:y1, x0:x1] = rng.random((batch, y1 - y0, x1 - x0))
    return a


def run_engine(eng, a0, target):
    """(A_T, dL/dA_0, parameter gradients) for the batch MSE loss."""
    s = torch.cuda.current_stream().cuda_stream
    a = torch.from_numpy(a0).cuda()
    out = torch.empty_like(a)
    eng.forward(a.data_ptr(), out.data_ptr(), s)
    t = torch.from_numpy(target).cuda()
    g = 2.0 * (out - t) / out.numel()
    ga0 = torch.empty_like(a)
    gp = torch.zeros(lb.ADJOINT_NUM_PARAMS, dtype=torch.float64, device="cuda")
    eng.backward(g.data_ptr(), ga0.data_ptr(), gp.data_ptr(), s)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ga0.cpu().numpy(), gp.cpu().numpy()


def oracle_vector(g, p):
    from life_simulation_b200.adjoint import pack_param_grads
    return pack_param_grads(g.mu, g.sigma, g.weight, g.betas, g.dt).numpy()


@pytest.mark.parametrize("mode,core,ckpt", [(0, lb.CORE_EXP, 4), (1, lb.CORE_EXP, 3),
                                            (0, lb.CORE_GAUSS_SHELL, 10)])
def test_adjoint_matches_fp64_oracle(mode, core, ckpt):
    w, h, batch, steps, radius = 128, 128, 3, 10, 12
    eng = lb.LeniaAdjoint(w, h, batch, KERNELS, radius, steps, checkpoint_every=ckpt, dt=0.1,
                          growth_mode=mode, kernel_core=core)
    a0 = fields(batch, h, w, seed=4)
    target = fields(batch, h, w, seed=5) * 0.5
    aT, ga0, gp = run_engine(eng, a0, target)
    p = oracle_params(KERNELS, radius, 0.1, mode, core)
    _, g = O.loss_and_grads(a0.astype(np.float64), target.astype(np.float64), p, steps)
    finals = np.stack([O.forward(a, p, steps)[-1] for a in a0.astype(np.float64)])
    # FP32 spectral steps vs FP64: the chaotic dynamics grow the rounding.
    assert np.abs(aT - finals).max() <= 2e-4
    # Gradients: relative to the largest entry (FP32 accumulation and the
    # FP32 trajectory both enter).
    gf = g.field
    assert np.abs(ga0 - gf).max() <= 2e-3 * np.abs(gf).max(), np.abs(ga0 - gf).max() / np.abs(gf).max()
    ref = oracle_vector(g, p)
    for i, v in enumerate(ref):
        assert abs(gp[i] - v) <= 2e-3 * abs(v) + 1e-7 * np.abs(ref).max(), (i, gp[i], v)
    eng.close()


def test_adjoint_matches_central_differences():
    """eps = 1e-3 central differences of the FP64 forward on 16 sampled A_0
    pixels and on every scalar parameter."""
    w, h, batch, steps, radius = 128, 64, 2, 8, 8
    eng = lb.LeniaAdjoint(w, h, batch, KERNELS, radius, steps, checkpoint_every=4, dt=0.1)
    a0 = fields(batch, h, w, seed=11)
    target = fields(batch, h, w, seed=12) * 0.5
    _, ga0, gp = run_engine(eng, a0, target)
    p = oracle_params(KERNELS, radius, 0.1, 0, lb.CORE_EXP)
    a64, t64 = a0.astype(np.float64), target.astype(np.float64)
    eps = 1e-3
    rng = np.random.default_rng(13)
    for _ in range(16):
        b, y, x = rng.integers(0, batch), rng.integers(16, 48), rng.integers(32, 96)
        ap, am = a64.copy(), a64.copy()
        ap[b, y, x] += eps
        am[b, y, x] -= eps
        fd = (O.loss(ap, t64, p, steps) - O.loss(am, t64, p, steps)) / (2 * eps)
        assert abs(ga0[b, y, x] - fd) <= 2e-3 * abs(fd) + 2e-3 * np.abs(ga0).max() * 1e-2, (b, y, x, ga0[b, y, x], fd)
    per = lb.ADJOINT_PARAMS_PER_KERNEL
    slots = {"mu": 0, "sigma": 1, "weight": 2}
    for name, k, j in O.param_vector(p):
        lp = O.loss(a64, t64, O.perturbed(p, name, k, j, eps), steps)
        lm = O.loss(a64, t64, O.perturbed(p, name, k, j, -eps), steps)
        fd = (lp - lm) / (2 * eps)
        i = lb.ADJOINT_NUM_PARAMS - 1 if name == "dt" else k * per + (3 + j if name == "beta" else slots[name])
        # Central differences at eps = 1e-3 carry an O(eps^2) error of up
        # to ~1e-2 relative on the steep bells (the oracle's own test).
        assert abs(gp[i] - fd) <= 3e-2 * abs(fd) + 1e-7, (name, k, j, gp[i], fd)
    eng.close()


def test_checkpoint_interval_does_not_change_the_gradient():
    w, h, batch, steps, radius = 128, 128, 2, 9, 10
    a0 = fields(batch, h, w, seed=21)
    target = fields(batch, h, w, seed=22) * 0.5
    res = []
    for ckpt in (1, 4, 9):
        eng = lb.LeniaAdjoint(w, h, batch, KERNELS, radius, steps, checkpoint_every=ckpt)
        res.append(run_engine(eng, a0, target))
        eng.close()
    for aT, ga0, gp in res[1:]:
        # Recomputed segments are bit-identical; only the order of the FP64
        # atomic sums of the parameter gradients may differ.
        assert np.array_equal(aT, res[0][0])
        assert np.array_equal(ga0, res[0][1])
        np.testing.assert_allclose(gp, res[0][2], rtol=1e-9, atol=1e-15)


def test_autograd_binding_and_gradient_descent():
    w, h, batch, steps, radius = 128, 128, 2, 6, 10
    model = RolloutParams(w, h, batch, KERNELS, radius, steps, checkpoint_every=3)
    a0 = torch.from_numpy(fields(batch, h, w, seed=31)).cuda().requires_grad_(True)
    target = torch.from_numpy(fields(batch, h, w, seed=32) * 0.5).cuda()
    out = model(a0)
    loss = torch.mean((out - target) ** 2)
    loss.backward()
    # The same numbers through the raw engine.
    eng = lb.LeniaAdjoint(w, h, batch, KERNELS, radius, steps, checkpoint_every=3)
    aT, ga0, gp = run_engine(eng, a0.detach().cpu().numpy(), target.cpu().numpy())
    eng.close()
    np.testing.assert_array_equal(out.detach().cpu().numpy(), aT)
    # torch's MSE backward rounds 2 (A_T - target) / N in another order.
    np.testing.assert_allclose(a0.grad.cpu().numpy(), ga0, rtol=1e-5, atol=1e-6 * np.abs(ga0).max())
    per = lb.ADJOINT_PARAMS_PER_KERNEL
    np.testing.assert_allclose(model.mu.grad.numpy(), gp[[0, per]], rtol=1e-5)
    np.testing.assert_allclose(model.betas.grad[1, :2].numpy(), gp[per + 3:per + 5], rtol=1e-5, atol=1e-12)
    assert float(model.betas.grad[0].abs().sum()) == 0.0 and float(model.betas.grad[1, 2:].abs().sum()) == 0.0
    # A few steps of gradient descent on the initial fields lower the loss.
    x = a0.detach().clone().requires_grad_(True)
    opt = torch.optim.Adam([x], lr=0.02)
    losses = []
    for _ in range(8):
        opt.zero_grad()
        l = torch.mean((model(x) - target) ** 2)
        l.backward()
        opt.step()
        with torch.no_grad():
            x.clamp_(0.0, 1.0)
        losses.append(float(l.detach()))
    assert losses[-1] < losses[0]
    # Parameter updates rebuild the kernels; the next forward uses them.
    with torch.no_grad():
        model.mu += 0.01
    out2 = model(a0.detach())
    assert not torch.equal(out2, out.detach())


def test_full_size_batch_512():
    """32 worlds of 512x512, K=2, R=16, T=64, checkpoints every 8: finite
    gradients, and the checkpointed backward equals the stored-everything
    one. With these parameters (sigma 0.015 / 0.03 at dt 0.1) random fields
    die out within ~30 steps, so the T=64 gradient is zero; the values are
    checked against the FP64 oracle at T=16, while the worlds are alive."""
    kernels = [{"mu": 0.15, "sigma": 0.015, "weight": 0.5, "betas": [1.0]},
               {"mu": 0.25, "sigma": 0.03, "weight": 0.5, "betas": [0.5, 1.0]}]
    w = h = 512
    batch, steps = 32, 64
    a0 = fields(batch, h, w, seed=4, lo=0.0, hi=1.0)
    target = fields(batch, h, w, seed=5, lo=0.0, hi=1.0) * 0.5
    eng = lb.LeniaAdjoint(w, h, batch, kernels, 16, steps, checkpoint_every=8)
    aT, ga0, gp = run_engine(eng, a0, target)
    eng.close()
    assert np.isfinite(ga0).all() and np.isfinite(gp).all()
    eng = lb.LeniaAdjoint(w, h, batch, kernels, 16, steps, checkpoint_every=steps)
    aT2, ga02, gp2 = run_engine(eng, a0, target)
    eng.close()
    assert np.array_equal(aT, aT2) and np.array_equal(ga0, ga02)
    np.testing.assert_allclose(gp, gp2, rtol=1e-9, atol=1e-15)
    # Two worlds, 16 steps, against the FP64 oracle.
    eng = lb.LeniaAdjoint(w, h, 2, kernels, 16, 16, checkpoint_every=8)
    aT1, ga01, gp1 = run_engine(eng, a0[:2], target[:2])
    eng.close()
    p = oracle_params(kernels, 16, 0.1, 0, lb.CORE_EXP)
    _, g = O.loss_and_grads(a0[:2].astype(np.float64), target[:2].astype(np.float64), p, 16)
    assert np.abs(g.field).max() > 0.0
    assert np.abs(ga01 - g.field).max() <= 2e-3 * np.abs(g.field).max()
    ref = oracle_vector(g, p)
    for i, v in enumerate(ref):
        assert abs(gp1[i] - v) <= 2e-3 * abs(v) + 1e-6 * np.abs(ref).max(), (i, gp1[i], v)


def test_benchmark_workload_against_fp64_oracle():
    """The benchmarked adjoint workload itself (growth mode 1, seeded
    uniform[0,1) fields, targets from a forward run of other seeds, T=64,
    checkpoints every 8) for two of its 32 worlds: live, non-zero gradients
    that agree with the FP64 oracle's adjoint."""
    from life_simulation_b200 import workloads as wl
    c = wl.ADJOINT_512
    w, h, steps = c["width"], c["height"], c["steps"]
    eng = lb.LeniaAdjoint(w, h, 2, wl.ADJOINT_KERNELS, c["radius"], steps, c["checkpoint_every"], c["dt"],
                          c["growth_mode"], lb.CORE_EXP)
    a0 = wl.adjoint_fields(4000, 2, w, h).astype(np.float32)
    s = torch.cuda.current_stream().cuda_stream
    t0 = torch.from_numpy(wl.adjoint_fields(5000, 2, w, h).astype(np.float32)).cuda()
    tgt = torch.empty_like(t0)
    eng.forward(t0.data_ptr(), tgt.data_ptr(), s)
    target = tgt.cpu().numpy()
    aT, ga0, gp = run_engine(eng, a0, target)
    eng.close()
    assert ((aT > 0) & (aT < 1)).all()
    p = oracle_params(wl.ADJOINT_KERNELS, c["radius"], c["dt"], c["growth_mode"], lb.CORE_EXP)
    states = O.forward(a0[0].astype(np.float64), p, steps)
    assert np.abs(aT[0] - states[-1]).max() < 1e-4
    _, g = O.loss_and_grads(a0.astype(np.float64), target.astype(np.float64), p, steps)
    assert np.abs(g.field).max() > 0.0
    assert np.abs(ga0 - g.field).max() <= 2e-3 * np.abs(g.field).max()
    ref = oracle_vector(g, p)
    assert np.abs(ref).max() > 0.0
    for i, v in enumerate(ref):
        assert abs(gp[i] - v) <= 2e-3 * abs(v) + 1e-6 * np.abs(ref).max(), (i, gp[i], v)


def test_invalid_configs_are_rejected():
    with pytest.raises(lb.LeniaError, match="no compile-time FFT plan"):
        lb.LeniaAdjoint(100, 100, 1, KERNELS, 8, 4)
    with pytest.raises(lb.LeniaError):
        lb.LeniaAdjoint(128, 128, 1, KERNELS, 8, 4, checkpoint_every=5)
    eng = lb.LeniaAdjoint(128, 128, 1, KERNELS, 8, 4)
    g = torch.zeros(1, 128, 128, device="cuda")
    with pytest.raises(lb.LeniaError, match="backward needs a forward"):
        eng.backward(g.data_ptr(), g.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    with pytest.raises(lb.LeniaError, match="num_betas"):
        eng.set_params([KERNELS[0], dict(KERNELS[1], betas=[1.0])], 0.1)
    eng.close()
