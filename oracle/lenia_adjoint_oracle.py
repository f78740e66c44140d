"""FP64 oracle of the spectral Lenia step's adjoint (test infrastructure).

Only tests, the smoke entry and the benchmark's CPU baseline use this module,
as the reference the CUDA adjoint is compared against; the product never
calls it.

The reference has no adjoint. The forward it differentiates is the reference's
multi-kernel spectral step without noise, mu jitter or injection:
  U_k  = K_k (*) A                       circular convolution (Lenia.metal:
                                           166-186, leniaGrowthMulti's inputs)
  pre  = A + dt * sum_k h_k (2 bell_k - 1)          growth mode 0
       = A + dt * (sum_k h_k bell_k / sum h - A)    growth mode 1 (sum h > 1e-6)
  A'   = clamp(pre, 0, 1)                (Lenia.metal:188-231)
bell_k = exp(-0.5 ((U_k - mu_k) / sigma_k)^2) (Lenia.metal:156-159), and the
kernel K_k = sum_i beta_i R_i / sum_i beta_i s_i, R_i the image of ring i
with peak 1 and s_i its sum (buildRingKernelImage, Lenia.cpp:95-125, here
evaluated in FP64 throughout).

The backward is the exact derivative of that map, with the clamp's
subgradient taken as 1 strictly inside (0, 1) and 0 on or outside the
bounds. Because every K_k is even, the adjoint of U_k = K_k (*) A is again a
convolution with K_k. The beta gradients come from the ring potentials
E_i = (R_i / Z) (*) A, Z = sum_j beta_j s_j:
  dL/dbeta_i = sum_x q_k(x) (E_i(x) - (s_i / Z) U_k(x)),
  q_k = dL/dpre * dpre/dU_k.
Parity of this oracle is pinned against central finite differences of its
own forward (eps = 1e-3, FP64), not against the reference (which has no
gradient).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

GAUSS_SHELL, EXP = 0, 1


def exp_core(r: np.ndarray) -> np.ndarray:
    """exp(4 - 1/(r(1-r))) on (0, 1), 0 elsewhere (the exponential core)."""
    r = np.asarray(r, np.float64)
    out = np.zeros_like(r)
    m = (r > 0.0) & (r < 1.0)
    rr = r[m]
    out[m] = np.exp(4.0 - 1.0 / (rr * (1.0 - rr)))
    return out


def shell_images(w: int, h: int, radius_k: float, nshell: int, core: int,
                 shell_sigma: float) -> List[np.ndarray]:
    """Unnormalised ring images (peak 1 each) on an h x w torus, centred at
    (0, 0): the terms of buildRingKernelImage (Lenia.cpp:95-125) by ring."""
    dy = np.arange(h)
    dy = np.where(dy > h // 2, dy - h, dy).astype(np.float64)
    dx = np.arange(w)
    dx = np.where(dx > w // 2, dx - w, dx).astype(np.float64)
    r = np.sqrt(dx[None, :] ** 2 + dy[:, None] ** 2)
    inside = (r > 0.0) & (r <= radius_k)
    u = r / radius_k * nshell
    idx = np.minimum(np.floor(u), nshell - 1).astype(np.int64)
    if core == EXP:
        val = exp_core(u - idx)
    else:
        t = (u - idx - 0.5) / (shell_sigma * nshell)
        val = np.exp(-0.5 * t * t)
    return [np.where(inside & (idx == i), val, 0.0) for i in range(nshell)]


@dataclass
class AdjKernel:
    mu: float
    sigma: float
    weight: float
    betas: List[float]
    radius_scale: float = 1.0


@dataclass
class AdjParams:
    kernels: List[AdjKernel]
    radius: float
    dt: float = 0.1
    growth_mode: int = 0
    core: int = EXP
    shell_sigma: float = 0.15

    def copy(self) -> "AdjParams":
        return AdjParams([AdjKernel(k.mu, k.sigma, k.weight, list(k.betas), k.radius_scale) for k in self.kernels],
                         self.radius, self.dt, self.growth_mode, self.core, self.shell_sigma)


@dataclass
class AdjGrads:
    mu: np.ndarray
    sigma: np.ndarray
    weight: np.ndarray
    betas: List[np.ndarray]
    dt: float = 0.0
    field: Optional[np.ndarray] = None


class _Kernels:
    """Per-kernel FP64 spectra of K_k and of the normalised rings."""

    def __init__(self, p: AdjParams, w: int, h: int):
        self.khat, self.ehat, self.c = [], [], []
        for k in p.kernels:
            rings = shell_images(w, h, p.radius * k.radius_scale, len(k.betas), p.core, p.shell_sigma)
            s = np.array([r.sum() for r in rings])
            z = float(np.dot(k.betas, s))
            kimg = sum(b * r for b, r in zip(k.betas, rings)) / z
            self.khat.append(np.fft.rfft2(kimg))
            self.ehat.append([np.fft.rfft2(r / z) for r in rings])
            self.c.append(s / z)


def _conv(fa: np.ndarray, khat: np.ndarray, shape) -> np.ndarray:
    return np.fft.irfft2(fa * khat, s=shape)


def _growth(a: np.ndarray, p: AdjParams, ks: _Kernels):
    fa = np.fft.rfft2(a)
    us = [_conv(fa, kh, a.shape) for kh in ks.khat]
    bells = [np.exp(-0.5 * ((u - k.mu) / k.sigma) ** 2) for u, k in zip(us, p.kernels)]
    if p.growth_mode == 1:
        sw = sum(k.weight for k in p.kernels)
        if sw > 1e-6:
            g = sum(k.weight * b for k, b in zip(p.kernels, bells)) / sw
            pre = a + p.dt * (g - a)
        else:
            g = None
            pre = a.copy()
    else:
        g = sum(k.weight * (2.0 * b - 1.0) for k, b in zip(p.kernels, bells))
        pre = a + p.dt * g
    return fa, us, bells, g, pre


def step(a: np.ndarray, p: AdjParams, ks: Optional[_Kernels] = None) -> np.ndarray:
    ks = ks or _Kernels(p, a.shape[1], a.shape[0])
    return np.clip(_growth(a, p, ks)[4], 0.0, 1.0)


def forward(a0: np.ndarray, p: AdjParams, steps: int) -> List[np.ndarray]:
    """States A_0..A_T (FP64)."""
    ks = _Kernels(p, a0.shape[1], a0.shape[0])
    out = [np.asarray(a0, np.float64)]
    for _ in range(steps):
        out.append(step(out[-1], p, ks))
    return out


def backward(states: List[np.ndarray], g_final: np.ndarray, p: AdjParams) -> AdjGrads:
    """Gradients of L given dL/dA_T = g_final, by reverse sweep over the
    stored states."""
    h, w = states[0].shape
    ks = _Kernels(p, w, h)
    nk = len(p.kernels)
    gr = AdjGrads(np.zeros(nk), np.zeros(nk), np.zeros(nk), [np.zeros(len(k.betas)) for k in p.kernels])
    ga = np.asarray(g_final, np.float64)
    sw = sum(k.weight for k in p.kernels)
    for t in range(len(states) - 2, -1, -1):
        a = states[t]
        fa, us, bells, gsum, pre = _growth(a, p, ks)
        g = ga * ((pre > 0.0) & (pre < 1.0))
        if p.growth_mode == 1:
            if sw > 1e-6:
                ca = 1.0 - p.dt
                dpdu = [p.dt * k.weight * b * (k.mu - u) / (k.sigma ** 2) / sw
                        for k, b, u in zip(p.kernels, bells, us)]
                for i, b in enumerate(bells):
                    gr.weight[i] += np.sum(g * p.dt * (b - gsum) / sw)
                gr.dt += np.sum(g * (gsum - a))
            else:
                ca = 1.0
                dpdu = [np.zeros_like(a) for _ in p.kernels]
        else:
            ca = 1.0
            dpdu = [2.0 * p.dt * k.weight * b * (k.mu - u) / (k.sigma ** 2)
                    for k, b, u in zip(p.kernels, bells, us)]
            for i, b in enumerate(bells):
                gr.weight[i] += np.sum(g * p.dt * (2.0 * b - 1.0))
            gr.dt += np.sum(g * gsum)
        new = ca * g
        for i, k in enumerate(p.kernels):
            q = g * dpdu[i]
            gr.mu[i] += -np.sum(q)
            gr.sigma[i] += np.sum(q * (k.mu - us[i]) / k.sigma)
            new = new + _conv(np.fft.rfft2(q), ks.khat[i], a.shape)
            if len(k.betas) > 1:
                for j in range(len(k.betas)):
                    e = _conv(fa, ks.ehat[i][j], a.shape)
                    gr.betas[i][j] += np.sum(q * (e - ks.c[i][j] * us[i]))
        ga = new
    gr.field = ga
    return gr


def mse_loss_grad(fields: np.ndarray, targets: np.ndarray):
    """Mean squared error over every world and pixel, and its gradient."""
    d = np.asarray(fields, np.float64) - np.asarray(targets, np.float64)
    return float(np.mean(d * d)), 2.0 * d / d.size


def loss(a0s: np.ndarray, targets: np.ndarray, p: AdjParams, steps: int) -> float:
    """MSE of the T-step states of a batch of worlds (shared parameters)."""
    finals = np.stack([forward(a, p, steps)[-1] for a in a0s])
    return mse_loss_grad(finals, targets)[0]


def loss_and_grads(a0s: np.ndarray, targets: np.ndarray, p: AdjParams, steps: int):
    """(loss, AdjGrads summed over the batch with `field` = dL/dA_0 per world)."""
    runs = [forward(a, p, steps) for a in a0s]
    finals = np.stack([r[-1] for r in runs])
    value, gfin = mse_loss_grad(finals, targets)
    total = None
    fields = []
    for r, gf in zip(runs, gfin):
        g = backward(r, gf, p)
        fields.append(g.field)
        if total is None:
            total = g
        else:
            total.mu += g.mu
            total.sigma += g.sigma
            total.weight += g.weight
            total.dt += g.dt
            for x, y in zip(total.betas, g.betas):
                x += y
    total.field = np.stack(fields)
    return value, total


def param_vector(p: AdjParams) -> List[tuple]:
    """Every scalar parameter as (name, kernel, index) for finite differences."""
    out = []
    for i, k in enumerate(p.kernels):
        out += [("mu", i, 0), ("sigma", i, 0), ("weight", i, 0)]
        out += [("beta", i, j) for j in range(len(k.betas))]
    out.append(("dt", -1, 0))
    return out


def perturbed(p: AdjParams, name: str, k: int, j: int, delta: float) -> AdjParams:
    q = p.copy()
    if name == "dt":
        q.dt += delta
    elif name == "beta":
        q.kernels[k].betas[j] += delta
    else:
        setattr(q.kernels[k], name, getattr(q.kernels[k], name) + delta)
    return q


def grad_of(g: AdjGrads, name: str, k: int, j: int) -> float:
    if name == "dt":
        return float(g.dt)
    if name == "beta":
        return float(g.betas[k][j])
    return float(getattr(g, name)[k])
