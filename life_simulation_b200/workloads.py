"""Seeded synthetic Lenia workloads (the benchmark and test inputs).

The reference measures on no public dataset; every input here is generated
from a seed by SplitMix64 (the algorithm of LifeCore/Math/Random.h:11-31,
``nextFloat01`` = top 24 bits / 2^24), vectorised with numpy.

* ``single_256``: a 256x256 torus, direct convolution, R=13, exponential
  kernel core, growth mode 0 (mu 0.15, sigma 0.015, dt 0.1); uniform[0,1)
  in the central 64x64 square (seed 1), zeros elsewhere.
* ``adjoint_512`` (the gradient form): 32 worlds of 512x512, two kernels
  R=16, peaks [1] and [0.5, 1], mu {0.15, 0.25}, sigma {0.015, 0.03},
  weights {0.5, 0.5}, dt 0.1, growth mode 1 (asymptotic: A += dt (G - A)),
  exponential core, T=64 steps with checkpoints every 8; world b starts from
  uniform[0,1) over the whole field (SplitMix64 seed 4000 + b) and its target
  is the T-step state from seed 5000 + b; loss = mean squared error over
  every world and pixel. Under growth mode 0 these kernels take every
  seeded start (whole field, central square or patches, any amplitude)
  to the all-zero field within ~25 steps, where the clip mask makes the
  T=64 gradient identically zero; growth mode 1 keeps every pixel strictly
  inside (0, 1), so every term of the backward pass is live.
* ``fft3_1080p`` / ``fft3_1024x512``: three kernels of radius 24, peaks
  [1], [0.5, 1], [1, 0.667, 0.333], mu {0.156, 0.193, 0.342}, sigma
  {0.0118, 0.049, 0.0891}, weights {0.5, 0.3, 0.2}, dt 0.1, growth mode 0,
  exponential core; uniform[0,1) in 20 patches of 96x96 at seeded positions
  (seed 2, toroidally wrapped, later patches overwrite earlier ones).
"""
from __future__ import annotations

import copy

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Outputs start..start+n-1 of SplitMix64(seed) (Random.h:14-21)."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + GOLDEN + i * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, n: int, start: int = 0) -> np.ndarray:
    """nextFloat01 (Random.h:24-26): float32 in [0, 1)."""
    return (splitmix64(seed, n, start) >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def central_square(w: int, h: int, side: int, seed: int) -> np.ndarray:
    a = np.zeros((h, w), np.float32)
    y0, x0 = (h - side) // 2, (w - side) // 2
    a[y0:y0 + side, x0:x0 + side] = uniform01(seed, side * side).reshape(side, side)
    return a


def patches(w: int, h: int, count: int, side: int, seed: int) -> np.ndarray:
    a = np.zeros((h, w), np.float32)
    pos = uniform01(seed, 2 * count)
    vals = uniform01(seed, count * side * side, start=2 * count).reshape(count, side, side)
    for p in range(count):
        x0 = int(pos[2 * p] * w)
        y0 = int(pos[2 * p + 1] * h)
        ys = (y0 + np.arange(side)) % h
        xs = (x0 + np.arange(side)) % w
        a[np.ix_(ys, xs)] = vals[p]
    return a


SINGLE_256 = {
    "convMode": "direct", "radius": 13, "kernelCore": "exp",
    "growthMode": 0, "growthMu": 0.15, "growthSigma": 0.015, "dt": 0.1,
    "noiseAmount": 0.0, "muJitter": 0.0, "injectAmount": 0.0,
}

FFT3_KERNELS = [
    {"radiusScale": 1.0, "mu": 0.156, "sigma": 0.0118, "weight": 0.5, "betas": [1.0]},
    {"radiusScale": 1.0, "mu": 0.193, "sigma": 0.049, "weight": 0.3, "betas": [0.5, 1.0]},
    {"radiusScale": 1.0, "mu": 0.342, "sigma": 0.0891, "weight": 0.2, "betas": [1.0, 0.667, 0.333]},
]


def fft3_params(w: int, h: int, conv: str = "fft") -> dict:
    return {
        "convMode": conv, "fftAnySize": True, "simWidth": w, "simHeight": h, "radius": 24,
        "kernelCore": "exp", "growthMode": 0, "dt": 0.1, "noiseAmount": 0.0, "muJitter": 0.0,
        "injectAmount": 0.0, "kernels": copy.deepcopy(FFT3_KERNELS),
    }


ADJOINT_KERNELS = [
    {"mu": 0.15, "sigma": 0.015, "weight": 0.5, "betas": [1.0]},
    {"mu": 0.25, "sigma": 0.03, "weight": 0.5, "betas": [0.5, 1.0]},
]
ADJOINT_512 = {"width": 512, "height": 512, "batch": 32, "radius": 16, "steps": 64,
               "checkpoint_every": 8, "dt": 0.1, "growth_mode": 1}


def adjoint_fields(seed_base: int, batch: int = 32, w: int = 512, h: int = 512) -> np.ndarray:
    """batch x h x w uniform[0,1) fields, world b from SplitMix64(seed_base + b)."""
    return np.stack([uniform01(seed_base + b, w * h).reshape(h, w) for b in range(batch)])


def sweep512(count_per_size: int = 128):
    """The 512-world sweep: 128 worlds each of 128x128, 256x256, 384x216 and
    512x512; per world (seed 3 + world id, SplitMix64) radius uniform in
    8..32, mu in U[0.10, 0.35], sigma in U[0.01, 0.05], dt in U[0.05, 0.2];
    single Gaussian-shell ring (shell sigma 0.15), growth mode 0; init
    uniform[0,1) in a central square of side min(W, H)/4.
    Returns (list of world parameter dicts, list of initial fields)."""
    sizes = [(128, 128), (256, 256), (384, 216), (512, 512)]
    worlds, inits = [], []
    wid = 0
    for (w, h) in sizes:
        for _ in range(count_per_size):
            u = uniform01(3 + wid, 5)
            worlds.append({"width": w, "height": h, "radius": 8 + min(24, int(u[0] * 25)),
                           "mu": 0.10 + 0.25 * float(u[1]), "sigma": 0.01 + 0.04 * float(u[2]),
                           "dt": 0.05 + 0.15 * float(u[3]), "seed": 3 + wid})
            side = min(w, h) // 4
            a = np.zeros((h, w), np.float32)
            y0, x0 = (h - side) // 2, (w - side) // 2
            a[y0:y0 + side, x0:x0 + side] = uniform01(10_000 + wid, side * side).reshape(side, side)
            inits.append(a)
            wid += 1
    return worlds, inits


def workload(name: str):
    """(params, width, height, initial field) of a named workload."""
    if name == "single_256":
        return dict(SINGLE_256), 256, 256, central_square(256, 256, 64, seed=1)
    if name == "fft3_1080p":
        return fft3_params(1920, 1080), 1920, 1080, patches(1920, 1080, 20, 96, seed=2)
    if name == "fft3_1024x512":
        return fft3_params(1024, 512), 1024, 512, patches(1024, 512, 20, 96, seed=2)
    if name == "direct_720p_r32":  # the reference's published direct configuration (one kernel, R=32)
        return {"radius": 32, "convMode": "direct"}, 1280, 720, patches(1280, 720, 12, 96, seed=2)
    raise KeyError(name)
