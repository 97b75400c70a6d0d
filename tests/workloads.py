"""Seeded synthetic inputs of the benchmark workloads.

Test and benchmark infrastructure: `bench.py`, the full-size parity tests and
the CPU baseline draw their inputs from here, so that the GPU path, the
oracle and the reference arm all see identical values.  Every generator runs
on the host with numpy's seeded generator (device independent); callers copy
the arrays to the GPU themselves.  The recipes follow the workload
descriptions (no public dataset is involved):

* `smooth`: sin(0.10x) cos(0.13y) sin(0.07z) + N(0, 1e-3), x the fastest axis;
  at 64^3 float32 this is the launch-bound plain single array.
* `spiky_f64`: the same field x 1e3 as float64, 10% of its 4x4x4 blocks set
  to exactly zero and 1% of its values replaced by +-10^U(-30, 30).
* `grf_f32`: a 2-D Gaussian random field with power spectrum ~ k^-3.
* `random_walk_i32`: a 1-D random walk with steps U{-100..100}.
* `uniform_i64`: values uniform in [-2^40, 2^40].
"""

from __future__ import annotations

import numpy as np


def smooth(shape, seed=0, dtype=np.float32, scale=1.0):
    """sin(0.10x) cos(0.13y) sin(0.07z) + N(0, 1e-3) over a C-order `shape`
    (1-3 axes, x the last), times `scale`, as `dtype`."""
    rng = np.random.default_rng(seed)
    dims = len(shape)
    freqs, funcs = [0.10, 0.13, 0.07], [np.sin, np.cos, np.sin]
    f = np.ones(shape, dtype=np.float64)
    for ax in range(dims):  # zfp axis ax is numpy axis dims - 1 - ax
        c = np.arange(shape[dims - 1 - ax], dtype=np.float64)
        view = [1] * dims
        view[dims - 1 - ax] = -1
        f = f * funcs[ax](freqs[ax] * c).reshape(view)
    f = f + rng.normal(0.0, 1e-3, size=shape)
    if scale != 1.0:
        f *= scale
    return f.astype(dtype, copy=False)


def spiky_f64(n, seed=0):
    """The n^3 float64 field of the variable-rate workload."""
    f = smooth((n, n, n), seed=seed, dtype=np.float64, scale=1e3)
    rng = np.random.default_rng(seed + 1)
    nb = n // 4
    zero = rng.random((nb, nb, nb)) < 0.10
    v = f[: 4 * nb, : 4 * nb, : 4 * nb].reshape(nb, 4, nb, 4, nb, 4)
    v[zero[:, None, :, None, :, None].repeat(4, 1).repeat(4, 3).repeat(4, 5)] = 0.0
    spikes = np.flatnonzero(rng.random(f.size) < 0.01)
    sign = np.where(rng.random(spikes.size) < 0.5, -1.0, 1.0)
    f.reshape(-1)[spikes] = sign * 10.0 ** rng.uniform(-30.0, 30.0, size=spikes.size)
    return f


def grf_f32(n, seed=1):
    """An n x n float32 Gaussian random field, power spectrum ~ k^-3 (the
    amplitude of white noise scaled by k^-1.5 in Fourier space), unit
    standard deviation."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n, n), dtype=np.float32)
    W = np.fft.rfft2(w)
    del w
    ky = np.fft.fftfreq(n)[:, None]
    kx = np.fft.rfftfreq(n)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = np.inf
    W *= k ** -1.5
    f = np.fft.irfft2(W, s=(n, n))
    f /= f.std()
    return f.astype(np.float32)


def random_walk_i32(count, seed=2):
    """A random walk of `count` int32 values with steps U{-100..100}."""
    rng = np.random.default_rng(seed)
    steps = rng.integers(-100, 101, size=count, dtype=np.int32)
    return np.cumsum(steps, dtype=np.int64).astype(np.int32)


def uniform_i64(shape, seed=3):
    """int64 values uniform in [-2^40, 2^40]."""
    rng = np.random.default_rng(seed)
    return rng.integers(-(1 << 40), (1 << 40) + 1, size=shape, dtype=np.int64)


def batched_specs(Z, n_arrays, max_elems, seed=0):
    """Shapes, types and configs of the batched workload: 60% float32, 30%
    float64, 10% int32; 1-D/2-D/3-D; element counts log-uniform from 64 to
    max_elems, no side a multiple of 4; per array fixed-rate 2-32,
    fixed-precision 8-48 or fixed-accuracy 1e-2..1e-9 (int32: the first two)
    and a random rounding.  Array i's values are `batched_array(spec, i)`."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_arrays):
        u = rng.random()
        dtype = np.float32 if u < 0.6 else (np.float64 if u < 0.9 else np.int32)
        dims = int(rng.integers(1, 4))
        n = float(np.exp(rng.uniform(np.log(64), np.log(max_elems))))
        base = n ** (1.0 / dims)
        shape = []
        for _ in range(dims):
            side = max(1, int(round(base * rng.uniform(0.8, 1.25))))
            if side % 4 == 0:
                side += 1
            shape.append(side)
        kinds = 3 if dtype != np.int32 else 2
        k = int(rng.integers(0, kinds))
        if k == 0:
            cfg = Z.ZfpConfig.fixed_rate(float(rng.integers(2, 33)), dtype, dims)
        elif k == 1:
            cfg = Z.ZfpConfig.fixed_precision(int(rng.integers(8, 49)))
        else:
            cfg = Z.ZfpConfig.fixed_accuracy(float(10.0 ** -rng.uniform(2, 9)))
        cfg = cfg.with_rounding(["never", "first", "last"][int(rng.integers(0, 3))], bool(rng.integers(0, 2)))
        specs.append((tuple(shape), dtype, cfg))
    return specs


def batched_array(spec, i, device, seed=0):
    """Array i of the batched workload on `device` (a torch tensor): the
    smooth recipe with seed i (int32: scaled by 2^20 and rounded)."""
    import torch

    shape, dtype, _ = spec
    dims = len(shape)
    g = torch.Generator(device=device)
    g.manual_seed(seed * 100003 + i)
    freqs, funcs = [0.10, 0.13, 0.07], [torch.sin, torch.cos, torch.sin]
    f = torch.ones(shape, device=device, dtype=torch.float64)
    for ax in range(dims):
        c = torch.arange(shape[dims - 1 - ax], device=device, dtype=torch.float64)
        view = [1] * dims
        view[dims - 1 - ax] = -1
        f = f * funcs[ax](freqs[ax] * c).view(view)
    f = f + 1e-3 * torch.randn(shape, generator=g, device=device, dtype=torch.float64)
    if dtype == np.int32:
        return torch.round(f * 2 ** 20).to(torch.int32)
    return f.to(torch.float32 if dtype == np.float32 else torch.float64)
