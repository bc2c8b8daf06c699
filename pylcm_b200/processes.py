"""Discretised stochastic processes usable as states.

Same classes, fields and discretisation formulas as the reference's
``src/_lcm/processes/ar1.py:37-201``, ``iid.py:20-200`` and ``base.py:16-159``.
Each process is a *node* axis of the value function: the solve indexes it by
node, and the expectation over next period's node is a contraction with the
process's transition matrix (row = current node).

Grid points and transition matrices are computed on the host in float64 from
the process parameters (fixed at construction or supplied at runtime under
``params[regime][state_name]``); they are part of the flat parameter vector
that the kernels read.
"""

from __future__ import annotations

import dataclasses
from math import comb
from typing import ClassVar

import numpy as np
from scipy.special import ndtr

from pylcm_b200.exceptions import GridInitializationError
from pylcm_b200.grids import Grid


def gauss_hermite_normal(n_points: int, mu: float, sigma: float) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Hermite nodes/weights for N(mu, sigma^2) (``processes/base.py:16-32``)."""
    raw_nodes, raw_weights = np.polynomial.hermite.hermgauss(n_points)
    nodes = mu + sigma * np.sqrt(2) * raw_nodes
    weights = raw_weights / np.sqrt(np.pi)
    return nodes, weights


def _validate_gh(n_points: int, gauss_hermite: bool, n_std) -> None:
    """``processes/base.py:143-159``: odd node count, GH excludes n_std."""
    if gauss_hermite and n_points % 2 == 0:
        raise GridInitializationError(
            f"n_points must be odd (got {n_points}). Odd n guarantees a quadrature node at the mean."
        )
    if gauss_hermite and n_std is not None:
        raise GridInitializationError("gauss_hermite=True and n_std are mutually exclusive.")


@dataclasses.dataclass(frozen=True, kw_only=True)
class _Process(Grid):
    n_points: int
    batch_size: int = 0
    distributed: bool = False

    _NON_PARAM_FIELDS: ClassVar[frozenset] = frozenset({"n_points", "batch_size", "distributed"})
    is_ar1: ClassVar[bool] = False

    @property
    def param_field_names(self) -> tuple[str, ...]:
        return tuple(
            f.name for f in dataclasses.fields(self) if f.name not in self._NON_PARAM_FIELDS
        )

    @property
    def fixed_params(self) -> dict:
        return {n: getattr(self, n) for n in self.param_field_names if getattr(self, n) is not None}

    @property
    def runtime_param_names(self) -> tuple[str, ...]:
        return tuple(n for n in self.param_field_names if getattr(self, n) is None)

    def __len__(self) -> int:
        return int(self.n_points)

    def to_numpy(self) -> np.ndarray:
        if self.runtime_param_names:
            return np.full(self.n_points, np.nan)
        return self.compute_gridpoints(**self.fixed_params)

    def compute_gridpoints(self, **kw) -> np.ndarray:  # pragma: no cover
        raise NotImplementedError

    def compute_transition_probs(self, **kw) -> np.ndarray:  # pragma: no cover
        raise NotImplementedError


@dataclasses.dataclass(frozen=True, kw_only=True)
class TauchenAR1Process(_Process):
    """AR(1) y' = mu + rho y + eps, Tauchen (1986) (``ar1.py:37-132``)."""

    gauss_hermite: bool
    rho: float | None = None
    sigma: float | None = None
    mu: float | None = None
    n_std: float | None = None
    is_ar1: ClassVar[bool] = True

    def __post_init__(self) -> None:
        _validate_gh(self.n_points, self.gauss_hermite, self.n_std)

    @property
    def param_field_names(self) -> tuple[str, ...]:
        ex = {"gauss_hermite"} | ({"n_std"} if self.gauss_hermite else set())
        return tuple(n for n in super().param_field_names if n not in ex)

    def compute_gridpoints(self, **kw) -> np.ndarray:
        rho, sigma, mu = float(kw["rho"]), float(kw["sigma"]), float(kw["mu"])
        std_y = np.sqrt(sigma**2 / (1 - rho**2))
        if self.gauss_hermite:
            return gauss_hermite_normal(self.n_points, mu / (1 - rho), std_y)[0]
        x_max = float(kw["n_std"]) * std_y
        return np.linspace(-x_max, x_max, self.n_points) + mu / (1 - rho)

    def compute_transition_probs(self, **kw) -> np.ndarray:
        rho, sigma = float(kw["rho"]), float(kw["sigma"])
        std_y = np.sqrt(sigma**2 / (1 - rho**2))
        if self.gauss_hermite:
            nodes, _ = gauss_hermite_normal(self.n_points, 0.0, std_y)
        else:
            x_max = float(kw["n_std"]) * std_y
            nodes = np.linspace(-x_max, x_max, self.n_points)
        mid = (nodes[:-1] + nodes[1:]) / 2
        # conditional y'|y has std sigma (``ar1.py:113-115``)
        c = ndtr((mid[None, :] - rho * nodes[:, None]) / sigma)
        return np.concatenate([c[:, :1], np.diff(c, axis=1), 1 - c[:, -1:]], axis=1)


@dataclasses.dataclass(frozen=True, kw_only=True)
class RouwenhorstAR1Process(_Process):
    """AR(1) discretised by Rouwenhorst (1995) (``ar1.py:137-201``)."""

    rho: float | None = None
    sigma: float | None = None
    mu: float | None = None
    is_ar1: ClassVar[bool] = True

    def compute_gridpoints(self, **kw) -> np.ndarray:
        rho, sigma, mu = float(kw["rho"]), float(kw["sigma"]), float(kw["mu"])
        n = self.n_points
        nu = np.sqrt((n - 1) / (1 - rho**2)) * sigma
        lrm = mu / (1.0 - rho)
        return np.linspace(lrm - nu, lrm + nu, n)

    def compute_transition_probs(self, **kw) -> np.ndarray:
        rho = float(kw["rho"])
        n = self.n_points
        q = (rho + 1) / 2
        P = np.zeros((n, n))
        for i in range(n):
            for j in range(n):
                s = 0.0
                for k in range(max(0, i + j - n + 1), min(i, j) + 1):
                    s += (
                        comb(i, k)
                        * comb(n - 1 - i, j - k)
                        * q ** (n - 1 - i - j + 2 * k)
                        * (1 - q) ** (i + j - 2 * k)
                    )
                P[i, j] = s
        return P


@dataclasses.dataclass(frozen=True, kw_only=True)
class UniformIIDProcess(_Process):
    """IID U(start, stop) on equally spaced nodes (``iid.py:35-67``)."""

    start: float | None = None
    stop: float | None = None

    def compute_gridpoints(self, **kw) -> np.ndarray:
        return np.linspace(float(kw["start"]), float(kw["stop"]), self.n_points)

    def compute_transition_probs(self, **kw) -> np.ndarray:
        n = self.n_points
        return np.full((n, n), 1 / n)


def _equal_spaced_normal_probs(mu: float, sigma: float, n_std: float, n: int) -> np.ndarray:
    x_min, x_max = mu - n_std * sigma, mu + n_std * sigma
    x, h = np.linspace(x_min, x_max, n, retstep=True)
    P = np.zeros(n)
    P[1:] = np.diff(ndtr((x + 0.5 * h - mu) / sigma))
    P[0] = ndtr((x_min + 0.5 * h - mu) / sigma)
    P[-1] = 1 - ndtr((x_max - 0.5 * h - mu) / sigma)
    return np.broadcast_to(P, (n, n)).copy()


@dataclasses.dataclass(frozen=True, kw_only=True)
class NormalIIDProcess(_Process):
    """IID N(mu, sigma^2) (``iid.py:70-140``)."""

    gauss_hermite: bool
    mu: float | None = None
    sigma: float | None = None
    n_std: float | None = None

    def __post_init__(self) -> None:
        _validate_gh(self.n_points, self.gauss_hermite, self.n_std)

    @property
    def param_field_names(self) -> tuple[str, ...]:
        ex = {"gauss_hermite"} | ({"n_std"} if self.gauss_hermite else set())
        return tuple(n for n in super().param_field_names if n not in ex)

    def compute_gridpoints(self, **kw) -> np.ndarray:
        mu, sigma = float(kw["mu"]), float(kw["sigma"])
        if self.gauss_hermite:
            return gauss_hermite_normal(self.n_points, mu, sigma)[0]
        n_std = float(kw["n_std"])
        return np.linspace(mu - n_std * sigma, mu + n_std * sigma, self.n_points)

    def compute_transition_probs(self, **kw) -> np.ndarray:
        mu, sigma = float(kw["mu"]), float(kw["sigma"])
        n = self.n_points
        if self.gauss_hermite:
            _, w = gauss_hermite_normal(n, mu, sigma)
            return np.broadcast_to(w, (n, n)).copy()
        return _equal_spaced_normal_probs(mu, sigma, float(kw["n_std"]), n)


@dataclasses.dataclass(frozen=True, kw_only=True)
class LogNormalIIDProcess(_Process):
    """IID log X ~ N(mu, sigma^2) (``iid.py:145-200``)."""

    gauss_hermite: bool
    mu: float | None = None
    sigma: float | None = None
    n_std: float | None = None

    def __post_init__(self) -> None:
        _validate_gh(self.n_points, self.gauss_hermite, self.n_std)

    @property
    def param_field_names(self) -> tuple[str, ...]:
        ex = {"gauss_hermite"} | ({"n_std"} if self.gauss_hermite else set())
        return tuple(n for n in super().param_field_names if n not in ex)

    def compute_gridpoints(self, **kw) -> np.ndarray:
        mu, sigma = float(kw["mu"]), float(kw["sigma"])
        if self.gauss_hermite:
            return np.exp(gauss_hermite_normal(self.n_points, mu, sigma)[0])
        n_std = float(kw["n_std"])
        return np.exp(np.linspace(mu - n_std * sigma, mu + n_std * sigma, self.n_points))

    def compute_transition_probs(self, **kw) -> np.ndarray:
        mu, sigma = float(kw["mu"]), float(kw["sigma"])
        n = self.n_points
        if self.gauss_hermite:
            _, w = gauss_hermite_normal(n, mu, sigma)
            return np.broadcast_to(w, (n, n)).copy()
        return _equal_spaced_normal_probs(mu, sigma, float(kw["n_std"]), n)


def _mixture_cdf(x, p1: float, mu1: float, sigma1: float, mu2: float, sigma2: float) -> np.ndarray:
    """CDF of the two-component normal mixture p1 N(mu1, sigma1^2) + (1 - p1) N(mu2, sigma2^2)."""
    return p1 * ndtr((x - mu1) / sigma1) + (1.0 - p1) * ndtr((x - mu2) / sigma2)


def _mixture_moments(p1: float, mu1: float, sigma1: float, mu2: float, sigma2: float) -> tuple[float, float]:
    """Mean and variance of the two-component normal mixture."""
    mean = p1 * mu1 + (1.0 - p1) * mu2
    var = p1 * (sigma1**2 + mu1**2) + (1.0 - p1) * (sigma2**2 + mu2**2) - mean**2
    return mean, var


_MIX_FIELDS = ("p1", "mu1", "sigma1", "mu2", "sigma2")


@dataclasses.dataclass(frozen=True, kw_only=True)
class TauchenNormalMixtureAR1Process(_Process):
    """AR(1) y' = mu + rho y + eps with eps a two-component normal mixture,
    discretised by Tauchen's binning with the mixture CDF (Fella, Gallipoli &
    Pan 2019, eq. 21; ``ar1.py:206-320``): equally spaced nodes around the
    long-run mean (mu + E[eps]) / (1 - rho), n_std unconditional standard
    deviations wide; row i bins the innovation x_j - mu - rho x_i over
    half-steps, the outer bins open-ended."""

    rho: float | None = None
    mu: float | None = None
    n_std: float | None = None
    p1: float | None = None
    mu1: float | None = None
    sigma1: float | None = None
    mu2: float | None = None
    sigma2: float | None = None
    is_ar1: ClassVar[bool] = True

    def _nodes(self, kw) -> tuple[np.ndarray, float]:
        rho, mu, n_std = float(kw["rho"]), float(kw["mu"]), float(kw["n_std"])
        mean, var = _mixture_moments(*(float(kw[f]) for f in _MIX_FIELDS))
        std_y = np.sqrt(var / (1 - rho**2))
        lrm = (mu + mean) / (1 - rho)
        x_max = n_std * std_y
        x = np.linspace(lrm - x_max, lrm + x_max, self.n_points)
        return x, (2 * x_max) / (self.n_points - 1)

    def compute_gridpoints(self, **kw) -> np.ndarray:
        return self._nodes(kw)[0]

    def compute_transition_probs(self, **kw) -> np.ndarray:
        x, step = self._nodes(kw)
        rho, mu = float(kw["rho"]), float(kw["mu"])
        mix = [float(kw[f]) for f in _MIX_FIELDS]
        z = x[None, :] - mu - rho * x[:, None]
        upper = _mixture_cdf(z + 0.5 * step, *mix)
        lower = _mixture_cdf(z - 0.5 * step, *mix)
        P = upper - lower
        P[:, 0] = upper[:, 0]
        P[:, -1] = 1 - lower[:, -1]
        return P


@dataclasses.dataclass(frozen=True, kw_only=True)
class NormalMixtureIIDProcess(_Process):
    """IID draws from a two-component normal mixture (``iid.py:211-300``):
    equally spaced nodes n_std mixture standard deviations around the mixture
    mean, bin probabilities from the mixture CDF over half-steps (the outer
    bins open-ended), the same row for every current node."""

    n_std: float | None = None
    p1: float | None = None
    mu1: float | None = None
    sigma1: float | None = None
    mu2: float | None = None
    sigma2: float | None = None

    def _nodes(self, kw) -> tuple[np.ndarray, float]:
        n_std = float(kw["n_std"])
        mean, var = _mixture_moments(*(float(kw[f]) for f in _MIX_FIELDS))
        std = np.sqrt(var)
        x = np.linspace(mean - n_std * std, mean + n_std * std, self.n_points)
        return x, (2 * n_std * std) / (self.n_points - 1)

    def compute_gridpoints(self, **kw) -> np.ndarray:
        return self._nodes(kw)[0]

    def compute_transition_probs(self, **kw) -> np.ndarray:
        x, step = self._nodes(kw)
        mix = [float(kw[f]) for f in _MIX_FIELDS]
        upper = _mixture_cdf(x + 0.5 * step, *mix)
        lower = _mixture_cdf(x - 0.5 * step, *mix)
        w = upper - lower
        w[0] = upper[0]
        w[-1] = 1 - lower[-1]
        return np.broadcast_to(w, (self.n_points, self.n_points)).copy()


def is_process(grid: object) -> bool:
    return isinstance(grid, _Process)
