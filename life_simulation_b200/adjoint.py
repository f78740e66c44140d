"""Gradients of Lenia rollouts for PyTorch (the adjoint form).

``rollout(engine, a0, mu, sigma, weight, betas, dt)`` maps a batch of initial
fields ``a0`` (batch x height x width, float32, CUDA) to the fields after
``engine.steps`` spectral steps; it is a ``torch.autograd.Function`` whose
backward is the library's hand-written adjoint (``lenia_adjoint_backward``)
with checkpointed recomputation. Gradients flow to ``a0`` and to the shared
parameters: ``mu``, ``sigma``, ``weight`` (K values each), ``betas``
(K x 8, entries past a kernel's ring count get zero gradient) and ``dt``.

The parameters are read on the host at every forward (they define the kernel
spectra, which are rebuilt in FP64 when they change); keep them on the CPU,
as ``RolloutParams`` does. The reference has no gradient form; its forward
is the multi-kernel spectral step of Shaders/Field/Lenia.metal:188-231
without noise, mu jitter or injection.

Several GPUs: the worlds are independent, so ``shard_worlds`` splits them
over ranks and ``allreduce_param_grads`` sums the scalar parameter gradients
(one all-reduce of a few dozen doubles); the field gradients stay local.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import torch
import torch.distributed as dist

from . import (ADJOINT_NUM_PARAMS, ADJOINT_PARAMS_PER_KERNEL, CORE_EXP, LeniaAdjoint)

MAX_BETAS = 8


def _kernels_from(mu, sigma, weight, betas, num_betas) -> List[dict]:
    mu, sigma, weight = mu.tolist(), sigma.tolist(), weight.tolist()
    bt = betas.tolist()
    return [{"mu": mu[k], "sigma": sigma[k], "weight": weight[k], "betas": bt[k][:num_betas[k]]}
            for k in range(len(num_betas))]


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, engine: LeniaAdjoint, a0, mu, sigma, weight, betas, dt, group):
        if not a0.is_cuda or a0.dtype != torch.float32:
            raise TypeError("a0 must be a float32 CUDA tensor")
        if tuple(a0.shape) != (engine.batch, engine.height, engine.width):
            raise ValueError(f"a0 must have shape {(engine.batch, engine.height, engine.width)}")
        a0 = a0.contiguous()
        values = (mu.tolist(), sigma.tolist(), weight.tolist(), betas.tolist(), float(dt))
        if getattr(engine, "_values", None) != values:
            engine.set_params(_kernels_from(mu, sigma, weight, betas, engine.num_betas), float(dt))
            engine._values = values
        out = torch.empty_like(a0)
        stream = torch.cuda.current_stream(a0.device).cuda_stream
        engine.forward(a0.data_ptr(), out.data_ptr(), stream)
        ctx.engine = engine
        ctx.values = values
        ctx.count = engine.forward_count
        ctx.group = group
        ctx.param_meta = [(t.device, t.dtype, t.shape) for t in (mu, sigma, weight, betas, dt)]
        ctx.save_for_backward(a0)
        return out

    @staticmethod
    def backward(ctx, g):
        engine: LeniaAdjoint = ctx.engine
        (a0,) = ctx.saved_tensors
        stream = torch.cuda.current_stream(a0.device).cuda_stream
        if engine.forward_count != ctx.count or getattr(engine, "_values", None) != ctx.values:
            # Another rollout ran on this engine since: redo this one's forward.
            mu, sigma, weight, betas, dt = ctx.values
            engine.set_params([{"mu": mu[k], "sigma": sigma[k], "weight": weight[k],
                                "betas": betas[k][:engine.num_betas[k]]} for k in range(engine.num_kernels)], dt)
            engine._values = ctx.values
            scratch = torch.empty_like(a0)
            engine.forward(a0.data_ptr(), scratch.data_ptr(), stream)
        g = g.contiguous().to(torch.float32)
        ga0 = torch.empty_like(g)
        gp = torch.empty(ADJOINT_NUM_PARAMS, dtype=torch.float64, device=a0.device)
        engine.backward(g.data_ptr(), ga0.data_ptr(), gp.data_ptr(), stream)
        if ctx.group is not None:
            allreduce_param_grads(gp, ctx.group)
        K, per = engine.num_kernels, ADJOINT_PARAMS_PER_KERNEL
        blk = gp[: K * per].view(K, per)
        gbetas = torch.zeros(K, MAX_BETAS, dtype=torch.float64, device=a0.device)
        gbetas[:, :per - 3] = blk[:, 3:]
        grads = [blk[:, 0], blk[:, 1], blk[:, 2], gbetas, gp[ADJOINT_NUM_PARAMS - 1]]
        out = []
        for gr, (dev, dtype, shape) in zip(grads, ctx.param_meta):
            out.append(gr.to(device=dev, dtype=dtype).reshape(shape))
        return (None, ga0, *out, None)


def rollout(engine: LeniaAdjoint, a0: torch.Tensor, mu: torch.Tensor, sigma: torch.Tensor,
            weight: torch.Tensor, betas: torch.Tensor, dt: torch.Tensor, group=None) -> torch.Tensor:
    """A_T of every world, differentiable in a0 and the parameters. With a
    process group, the parameter gradients are summed over its ranks."""
    return _Rollout.apply(engine, a0, mu, sigma, weight, betas, dt, group)


class RolloutParams(torch.nn.Module):
    """Learnable Lenia parameters (CPU, float64) for gradient search, and
    the engine they drive."""

    def __init__(self, width: int, height: int, batch: int, kernels: Sequence[dict], radius: int,
                 steps: int, checkpoint_every: Optional[int] = None, dt: float = 0.1, growth_mode: int = 0,
                 kernel_core: int = CORE_EXP, shell_sigma: float = 0.15):
        super().__init__()
        self.engine = LeniaAdjoint(width, height, batch, kernels, radius, steps, checkpoint_every, dt,
                                   growth_mode, kernel_core, shell_sigma)
        f64 = torch.float64
        self.mu = torch.nn.Parameter(torch.tensor([k["mu"] for k in kernels], dtype=f64))
        self.sigma = torch.nn.Parameter(torch.tensor([k["sigma"] for k in kernels], dtype=f64))
        self.weight = torch.nn.Parameter(torch.tensor([k.get("weight", 1.0) for k in kernels], dtype=f64))
        bt = torch.zeros(len(kernels), MAX_BETAS, dtype=f64)
        for i, k in enumerate(kernels):
            b = list(k.get("betas", [1.0]))
            bt[i, :len(b)] = torch.tensor(b, dtype=f64)
        self.betas = torch.nn.Parameter(bt)
        self.dt = torch.nn.Parameter(torch.tensor(dt, dtype=f64))

    def forward(self, a0: torch.Tensor, group=None) -> torch.Tensor:
        return rollout(self.engine, a0, self.mu, self.sigma, self.weight, self.betas, self.dt, group)


def shard_worlds(n: int, world_size: int, rank: int) -> range:
    """Contiguous share of n worlds for a rank (sizes differ by at most one)."""
    base, extra = divmod(n, world_size)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def allreduce_param_grads(gp: torch.Tensor, group=None) -> torch.Tensor:
    """Sum of the parameter-gradient vectors of every rank, in place."""
    dist.all_reduce(gp, op=dist.ReduceOp.SUM, group=group)
    return gp


def pack_param_grads(mu, sigma, weight, betas, dt, dtype=torch.float64) -> torch.Tensor:
    """The LENIA_ADJOINT_NUM_PARAMS layout from per-kernel gradients."""
    gp = torch.zeros(ADJOINT_NUM_PARAMS, dtype=dtype)
    per = ADJOINT_PARAMS_PER_KERNEL
    for k in range(len(mu)):
        gp[k * per] = float(mu[k])
        gp[k * per + 1] = float(sigma[k])
        gp[k * per + 2] = float(weight[k])
        for j, b in enumerate(betas[k]):
            gp[k * per + 3 + j] = float(b)
    gp[ADJOINT_NUM_PARAMS - 1] = float(dt)
    return gp
