"""Seeded synthetic inputs of the benchmark configurations (point clouds, kernels, RHS).

The reference publishes no dataset for this path; its examples generate their inputs
(examples/examples.h:35-110, examples/c-cylinder.c:238-239).  These generators produce the
configurations' shapes and value distributions from fixed seeds:

  cylinder  radius 1, height 4, regular angle x height grid; point q = j * n_theta + i is
            (cos 2 pi i / n_theta, sin 2 pi i / n_theta, 4 j / (n_z - 1))
  cube      uniform points in [0, 1]^3 (numpy default_rng(seed).random((n, 3)))
  rhs       x[:, q] ~ N(0, 1) from numpy default_rng(seed), column by column; complex
            right-hand sides are (a + i b) / sqrt(2)
"""
from __future__ import annotations

import math

import numpy as np

LAPLACE_REG = 0
EXP_COV = 1
HELMHOLTZ_REG = 2


def cylinder(n_theta: int, n_z: int, radius: float = 1.0, height: float = 4.0) -> np.ndarray:
    th = 2.0 * np.pi * np.arange(n_theta) / n_theta
    z = height * np.arange(n_z) / (n_z - 1)
    p = np.empty((n_z, n_theta, 3))
    p[:, :, 0] = radius * np.cos(th)[None, :]
    p[:, :, 1] = radius * np.sin(th)[None, :]
    p[:, :, 2] = z[:, None]
    return p.reshape(-1, 3)


def cube(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).random((n, 3))


def rhs(n: int, nrhs: int, seed: int, complex_: bool = False) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if not complex_:
        return np.asfortranarray(np.stack([rng.standard_normal(n) for _ in range(nrhs)], axis=1))
    cols = [(rng.standard_normal(n) + 1j * rng.standard_normal(n)) / math.sqrt(2.0) for _ in range(nrhs)]
    return np.asfortranarray(np.stack(cols, axis=1))


def helmholtz_wavenumber(n: int, radius: float = 1.0) -> float:
    """Ten points per wavelength with the reference example's spacing rule
    step = 1.75 pi r / sqrt(N) (examples/c-cylinder.c:238-239)."""
    step = 1.75 * math.pi * radius / math.sqrt(n)
    return 2.0 * math.pi / (10.0 * step)


def config(name: str) -> dict:
    """Parameters of one named configuration."""
    if name == "cfg0":  # plain FP64, N = 8,000
        return dict(points=cylinder(80, 100), kind=LAPLACE_REG, delta=0.01, leaf=64, eta=2.0, eps=1e-4, nrhs=1,
                    seed=0, complex=False)
    if name == "cfg1":  # N = 100,000, 16 RHS
        return dict(points=cylinder(250, 400), kind=LAPLACE_REG, delta=0.01, leaf=64, eta=2.0, eps=1e-6, nrhs=16,
                    seed=1, complex=False)
    if name == "cfg3":  # complex Helmholtz, N = 200,000
        n = 400 * 500
        return dict(points=cylinder(400, 500), kind=HELMHOLTZ_REG, delta=0.01, wavenumber=helmholtz_wavenumber(n),
                    leaf=128, eta=3.0, eps=1e-4, nrhs=4, seed=0, complex=True)
    if name == "cfg4":  # adjoint, N = 50,000 cube, exp covariance l = 0.3
        return dict(points=cube(50000, 2), kind=EXP_COV, ell=0.3, nugget=1e-6, leaf=64, eta=2.0, eps=1e-6, nrhs=1,
                    seed=2, complex=False)
    raise KeyError(name)


def batch_config(count: int = 64, seed: int = 0) -> list:
    """The uneven batch: N log-uniform in [2,000, 50,000], uniform cube points (seed per
    matrix), exp covariance with l ~ U(0.1, 0.5) and 1e-6 on the diagonal, leaf 64, eta 2,
    epsilon 1e-5."""
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(math.log(2000), math.log(50000), size=count))).astype(int)
    ells = rng.uniform(0.1, 0.5, size=count)
    return [dict(points=cube(int(n), 1000 + i), kind=EXP_COV, ell=float(l), nugget=1e-6, leaf=64, eta=2.0,
                 eps=1e-5, nrhs=1, seed=2000 + i, complex=False) for i, (n, l) in enumerate(zip(ns, ells))]
