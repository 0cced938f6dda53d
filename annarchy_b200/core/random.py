"""Random distributions for initial values and weights.

Same names and parameters as the reference (ANNarchy/core/Random.py). Unlike
the reference, which draws from an unseeded generator unless ``rng=`` is
given (Random.py:88-92), a distribution without ``rng`` draws from the
owning network's generator, seeded by ``Network(seed=...)``, so runs repeat.
"""
from __future__ import annotations

import numpy as np


class RandomDistribution:
    def __init__(self, rng=None):
        self.rng = rng

    def _gen(self, rng):
        return self.rng if self.rng is not None else (rng if rng is not None
                                                      else np.random.default_rng())

    def get_values(self, shape, rng=None):
        raise NotImplementedError


class Uniform(RandomDistribution):
    def __init__(self, min: float, max: float, rng=None):
        super().__init__(rng)
        self.min, self.max = float(min), float(max)

    def get_values(self, shape, rng=None):
        return self._gen(rng).uniform(self.min, self.max, shape)


class DiscreteUniform(RandomDistribution):
    def __init__(self, min: int, max: int, rng=None):
        super().__init__(rng)
        self.min, self.max = int(min), int(max)

    def get_values(self, shape, rng=None):
        return self._gen(rng).integers(self.min, self.max + 1, shape)


class Normal(RandomDistribution):
    def __init__(self, mu: float, sigma: float, min: float | None = None, max: float | None = None,
                 rng=None):
        super().__init__(rng)
        self.mu, self.sigma, self.min, self.max = float(mu), float(sigma), min, max

    def get_values(self, shape, rng=None):
        v = self._gen(rng).normal(self.mu, self.sigma, shape)
        if self.min is not None or self.max is not None:
            v = np.clip(v, self.min, self.max)
        return v


class LogNormal(RandomDistribution):
    def __init__(self, mu: float, sigma: float, min: float | None = None, max: float | None = None,
                 rng=None):
        super().__init__(rng)
        self.mu, self.sigma, self.min, self.max = float(mu), float(sigma), min, max

    def get_values(self, shape, rng=None):
        v = self._gen(rng).lognormal(self.mu, self.sigma, shape)
        if self.min is not None or self.max is not None:
            v = np.clip(v, self.min, self.max)
        return v


class Exponential(RandomDistribution):
    def __init__(self, Lambda: float, min: float | None = None, max: float | None = None, rng=None):
        super().__init__(rng)
        self.Lambda, self.min, self.max = float(Lambda), min, max

    def get_values(self, shape, rng=None):
        v = self._gen(rng).exponential(1.0 / self.Lambda, shape)
        if self.min is not None or self.max is not None:
            v = np.clip(v, self.min, self.max)
        return v


def values(spec, shape, rng, dtype=np.float64):
    """A scalar, array or RandomDistribution -> ndarray of `shape`."""
    if isinstance(spec, RandomDistribution):
        return np.asarray(spec.get_values(shape, rng), dtype=dtype)
    arr = np.asarray(spec, dtype=dtype)
    if arr.ndim == 0:
        return np.full(shape, arr, dtype=dtype)
    if arr.shape != tuple(np.atleast_1d(shape)) and arr.size == int(np.prod(shape)):
        arr = arr.reshape(shape)
    if arr.shape != tuple(np.atleast_1d(shape)):
        raise ValueError(f"expected shape {shape}, got {arr.shape}")
    return arr.copy()
