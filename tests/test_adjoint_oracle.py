"""The FP64 adjoint oracle, pinned against central finite differences of its
own forward, and the multi-rank gradient reduction of the adjoint form
(world sharding + one all-reduce of the parameter gradients) on gloo ranks.
No GPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import lenia_adjoint_oracle as O


def small_case(mode, core=O.EXP, seed=0, w=32, h=32, batch=2):
    rng = np.random.default_rng(seed)
    p = O.AdjParams([O.AdjKernel(0.15, 0.03, 0.6, [1.0]), O.AdjKernel(0.25, 0.05, 0.4, [0.5, 1.0])],
                    radius=6, dt=0.1, growth_mode=mode, core=core)
    a0 = np.zeros((batch, h, w))
    a0[:, h // 4:3 * h // 4, w // 4:3 * w // 4] = rng.random((batch, h // 2, w // 2))
    target = rng.random((batch, h, w)) * 0.3
    return p, a0, target


def fd_param(a0, target, p, steps, name, k, j, eps):
    lp = O.loss(a0, target, O.perturbed(p, name, k, j, eps), steps)
    lm = O.loss(a0, target, O.perturbed(p, name, k, j, -eps), steps)
    return (lp - lm) / (2 * eps)


@pytest.mark.parametrize("mode,core", [(0, O.EXP), (1, O.EXP), (0, O.GAUSS_SHELL)])
def test_oracle_gradient_matches_central_differences(mode, core):
    p, a0, target = small_case(mode, core)
    steps = 6
    _, g = O.loss_and_grads(a0, target, p, steps)
    # eps = 1e-5: truncation error ~eps^2, so the match is tight; eps = 1e-3
    # (the check the gradient form is specified with) leaves the O(eps^2)
    # term, up to ~1e-2 relative for the steep bells (sigma 0.03).
    for name, k, j in O.param_vector(p):
        an = O.grad_of(g, name, k, j)
        fd5 = fd_param(a0, target, p, steps, name, k, j, 1e-5)
        fd3 = fd_param(a0, target, p, steps, name, k, j, 1e-3)
        scale = max(abs(fd5), 1e-9)
        assert abs(an - fd5) <= 1e-5 * scale + 1e-12, (name, k, j, an, fd5)
        assert abs(an - fd3) <= 2e-2 * scale + 1e-9, (name, k, j, an, fd3)
    rng = np.random.default_rng(7)
    for _ in range(16):
        b, y, x = rng.integers(0, a0.shape[0]), rng.integers(8, 24), rng.integers(8, 24)
        ap, am = a0.copy(), a0.copy()
        ap[b, y, x] += 1e-3
        am[b, y, x] -= 1e-3
        fd = (O.loss(ap, target, p, steps) - O.loss(am, target, p, steps)) / 2e-3
        assert abs(g.field[b, y, x] - fd) <= 1e-4 * abs(fd) + 1e-10, (b, y, x, g.field[b, y, x], fd)


def test_beta_gradient_identities():
    p, a0, target = small_case(0)
    _, g = O.loss_and_grads(a0, target, p, 5)
    # One ring: the normalisation cancels beta exactly.
    assert g.betas[0][0] == 0.0
    # Scale invariance: sum_i beta_i dL/dbeta_i = 0.
    s = float(np.dot(p.kernels[1].betas, g.betas[1]))
    assert abs(s) <= 1e-12 * float(np.abs(g.betas[1]).max())
    assert float(np.abs(g.betas[1]).max()) > 0.0


def test_mode1_zero_weights_has_zero_parameter_gradient():
    p, a0, target = small_case(1)
    for k in p.kernels:
        k.weight = 0.0
    _, g = O.loss_and_grads(a0, target, p, 4)
    assert np.all(g.mu == 0) and np.all(g.sigma == 0) and np.all(g.weight == 0) and g.dt == 0.0
    # pre = A: the field gradient passes through the clip mask unchanged.
    assert np.abs(g.field).max() > 0.0


def test_saturated_pixels_block_the_gradient():
    p, a0, target = small_case(0)
    a0[:] = 0.0  # growth -dt everywhere: every pixel stays clipped at 0
    _, g = O.loss_and_grads(a0, target, p, 3)
    assert np.abs(g.field).max() == 0.0 and g.dt == 0.0


# ------------------------------------------------------- multi-rank reduce

def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world_size, port, out):
    from life_simulation_b200.adjoint import allreduce_param_grads, pack_param_grads, shard_worlds
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        p, a0, target = small_case(0, batch=5, w=24, h=24)
        steps = 4
        ids = list(shard_worlds(a0.shape[0], world_size, rank))
        # The loss is the mean over the whole batch: each rank's share of it.
        runs = [O.forward(a0[i], p, steps) for i in ids]
        finals = np.stack([r[-1] for r in runs])
        d = finals - target[ids]
        gfin = 2.0 * d / (a0.shape[0] * a0[0].size)
        gs = [O.backward(r, gf, p) for r, gf in zip(runs, gfin)]
        gp = sum(pack_param_grads(g.mu, g.sigma, g.weight, g.betas, g.dt) for g in gs)
        allreduce_param_grads(gp)
        out[rank] = gp.numpy().tolist()
    finally:
        dist.destroy_process_group()


def test_sharded_parameter_gradients_allreduce_to_full_batch():
    from life_simulation_b200.adjoint import pack_param_grads, shard_worlds
    assert [list(shard_worlds(5, 2, r)) for r in range(2)] == [[0, 1, 2], [3, 4]]
    assert sum(len(shard_worlds(32, 3, r)) for r in range(3)) == 32
    world_size = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world_size, _free_port(), out), nprocs=world_size, join=True)
    p, a0, target = small_case(0, batch=5, w=24, h=24)
    _, g = O.loss_and_grads(a0, target, p, 4)
    full = pack_param_grads(g.mu, g.sigma, g.weight, g.betas, g.dt).numpy()
    for r in range(world_size):
        np.testing.assert_allclose(np.array(out[r]), full, rtol=1e-12, atol=1e-15)
