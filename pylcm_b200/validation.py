"""Host-side checks of transition probabilities before solve / simulate.

Restates the reference's ``validate_transitions``
(``src/_lcm/transition_checks.py:51-76``, called from ``src/lcm/model.py:502``
before every solve and simulate):

- regime transitions (``:138-370``): for every period but the last and every
  active non-terminal regime, the regime-transition probabilities over the
  grid product of the variables the transition function reads must be finite,
  within [0, 1], sum to one within 16 float64 epsilons (``:628-647``), and be
  zero toward regimes that are inactive in the next period;
- stochastic state transitions (``:414-625``): every ``MarkovTransition`` law
  must return an outcome axis of the state's size, values within [0, 1] and
  rows summing to one within 1e-6.

The log level sets the policy, as in the reference: ``"off"`` skips the
checks, ``"warning"`` / ``"progress"`` warn for each failure and continue,
``"debug"`` raises the first failure.  A model that skips the checks still
gets NaN where the continuation mass is not one (the kernels' mass check).

The functions are evaluated on the host with NumPy, through the same
``jnp`` namespace the tracer uses (plain arrays are forwarded to NumPy).
"""

from __future__ import annotations

import inspect
import warnings
from typing import Any

import numpy as np

from pylcm_b200.exceptions import (
    InvalidRegimeTransitionProbabilitiesError,
    InvalidStateTransitionProbabilitiesError,
)
from pylcm_b200.regime import MarkovTransition
from pylcm_b200.spec import ParamResolver, RegimeSpec, _rebind_numpy_namespace

_EPS64 = float(np.finfo(np.float64).eps)


def _leaf_deps(spec: RegimeSpec, name: str, seen: set | None = None) -> list[str]:
    """States / actions / period / age that function `name` reads, directly
    or through the functions it calls (dags resolution by argument name)."""
    seen = set() if seen is None else seen
    fn = spec.functions[name]
    target = fn.func if isinstance(fn, MarkovTransition) else fn
    leaves = [a.name for a in spec.states] + [a.name for a in spec.actions] + ["period", "age"]
    out: list[str] = []
    for p in inspect.signature(target).parameters:
        if p in spec.functions and p not in seen:
            seen.add(p)
            out += [d for d in _leaf_deps(spec, p, seen) if d not in out]
        elif p in leaves and p not in out:
            out.append(p)
    return out


class _HostEval:
    """Evaluates a regime's functions on NumPy arrays by argument name."""

    def __init__(self, spec: RegimeSpec, resolver: ParamResolver, env: dict) -> None:
        self.spec, self.resolver, self.env = spec, resolver, env
        self.cache: dict[str, Any] = {}

    def value(self, name: str) -> Any:
        if name in self.cache:
            return self.cache[name]
        fn = self.spec.functions[name]
        target = _rebind_numpy_namespace(fn.func if isinstance(fn, MarkovTransition) else fn)
        kwargs = {}
        for p in inspect.signature(target).parameters.values():
            if p.name in self.spec.functions:
                kwargs[p.name] = self.value(p.name)
            elif p.name in self.env:
                kwargs[p.name] = self.env[p.name]
            else:
                ok, v = self.resolver.find(self.spec.name, name, p.name)
                if ok:
                    kwargs[p.name] = np.asarray(v)
                elif p.default is not inspect.Parameter.empty:
                    kwargs[p.name] = p.default
                else:
                    raise KeyError(p.name)
        with np.errstate(all="ignore"):
            out = target(**kwargs)
        self.cache[name] = out
        return out


def _axis_values(spec: RegimeSpec, resolver: ParamResolver, name: str) -> np.ndarray:
    for ax in spec.states + spec.actions:
        if ax.name != name:
            continue
        if ax.kind == "process":
            pp = resolver.process_params(spec.name, ax.name, ax.grid)
            return np.asarray(ax.grid.compute_gridpoints(**pp), dtype=np.float64)
        if ax.kind == "discrete":
            return np.arange(ax.size, dtype=np.int64)
        return np.asarray(ax.grid.to_numpy(), dtype=np.float64)
    raise KeyError(name)


def _evaluate(spec, resolver, fname, period, age):
    """(values of `fname` with the point axis first, points, names) over the
    grid product of its leaf inputs; the reference vmaps the function over
    that product (``transition_checks.py:240-275``)."""
    deps = [d for d in _leaf_deps(spec, fname) if d not in ("period", "age")]
    grids = [_axis_values(spec, resolver, d) for d in deps]
    mesh = [m.ravel() for m in np.meshgrid(*grids, indexing="ij")] if grids else []
    n_pts = mesh[0].size if mesh else 1
    env = {"period": np.int64(period), "age": age, **dict(zip(deps, mesh))}
    out = _HostEval(spec, resolver, env).value(fname)
    return out, n_pts, dict(zip(deps, mesh))


def _point_major(out: Any, n_pts: int, n_out: int) -> np.ndarray | None:
    """Values as (points, outcomes); None when the orientation is ambiguous."""
    if isinstance(out, (list, tuple)):
        out = np.stack([np.broadcast_to(np.asarray(x, dtype=np.float64), (n_pts,)) for x in out], axis=1)
        return out
    a = np.asarray(out, dtype=np.float64)
    if a.ndim == 1 and a.size == n_out:
        return np.broadcast_to(a, (n_pts, n_out))
    if a.ndim == 2:
        if a.shape == (n_pts, n_out) and (n_pts != n_out):
            return a
        if a.shape == (n_out, n_pts) and (n_pts != n_out):
            return a.T
        if a.shape == (n_out, n_pts) == (n_pts, n_out):
            return None
        if a.shape[0] == n_out and a.shape[1] == 1:
            return np.broadcast_to(a[:, 0], (n_pts, n_out))
    return a.reshape(n_pts, -1) if a.size % max(n_pts, 1) == 0 else a.reshape(1, -1)


def _pointwise(spec, resolver, fname, period, age):
    """The function evaluated point by point (as the reference's vmap):
    (values with the point axis first, points)."""
    deps = [d for d in _leaf_deps(spec, fname) if d not in ("period", "age")]
    grids = [_axis_values(spec, resolver, d) for d in deps]
    mesh = [m.ravel() for m in np.meshgrid(*grids, indexing="ij")] if grids else []
    n_pts = mesh[0].size if mesh else 1
    rows = []
    for k in range(n_pts):
        env = {"period": np.int64(period), "age": age, **{d: m[k] for d, m in zip(deps, mesh)}}
        rows.append(np.asarray(_HostEval(spec, resolver, env).value(fname), dtype=np.float64).reshape(-1))
    return np.stack(rows), dict(zip(deps, mesh))


def _regime_probs(spec, specs, resolver, period, age):
    n_reg = len(specs)
    if isinstance(spec.user.transition, MarkovTransition):
        try:
            out, n_pts, point = _evaluate(spec, resolver, "next_regime", period, age)
            P = _point_major(out, n_pts, n_reg)
        except (ValueError, TypeError, IndexError):
            # the function mixes per-point arrays and scalars in a way only a
            # point-by-point call accepts (the reference vmaps it)
            P = None
        if P is None:
            P, point = _pointwise(spec, resolver, "next_regime", period, age)
        return P, point
    out, n_pts, point = _evaluate(spec, resolver, "next_regime", period, age)
    rid = np.broadcast_to(np.asarray(out), (n_pts,)).astype(np.int64)
    P = np.zeros((n_pts, n_reg))
    ok = (rid >= 0) & (rid < n_reg)
    P[np.flatnonzero(ok), rid[ok]] = 1.0
    P[~ok] = np.nan  # a regime id outside the regime set is not a distribution
    return P, point


def _check_regime(spec, specs, resolver, period, ages) -> None:
    age, next_age = float(ages.values[period]), float(ages.values[period + 1])
    P, point = _regime_probs(spec, specs, resolver, period, age)
    if not np.isfinite(P).all():
        raise InvalidRegimeTransitionProbabilitiesError(
            f"Non-finite values in regime transition probabilities from '{spec.name}' between ages "
            f"{age} and {next_age}. Check the 'next_regime' function of the '{spec.name}' regime."
        )
    if (P < 0).any() or (P > 1).any():
        raise InvalidRegimeTransitionProbabilitiesError(
            f"Regime transition probabilities from '{spec.name}' between ages {age} and {next_age} "
            f"contain values outside [0, 1]. Check the 'next_regime' function of the '{spec.name}' regime."
        )
    total = P.sum(axis=1)
    bad = np.abs(total - 1.0) > 16.0 * _EPS64
    if bad.any():
        idx = np.flatnonzero(bad)[:5]
        detail = ", ".join(
            "{" + ", ".join(f"{k}={float(v[i]):g}" for k, v in point.items()) + f"}}: sum {total[i]!r}"
            for i in idx
        )
        raise InvalidRegimeTransitionProbabilitiesError(
            f"Regime transition probabilities from '{spec.name}' between ages {age} and {next_age} do not "
            f"sum to 1.0. {int(bad.sum())} of {total.size} probability vectors do not sum to 1.0; first: "
            f"{detail}. Check the 'next_regime' function of the '{spec.name}' regime."
        )
    active_next = {s.name for s in specs if (period + 1) in s.active_periods}
    for s in specs:
        if s.name not in active_next and (P[:, s.rid] > 0).any():
            raise InvalidRegimeTransitionProbabilitiesError(
                f"Regime '{s.name}' is inactive at age {next_age} but has positive transition probability "
                f"from '{spec.name}' between ages {age} and {next_age} in period {period}. Its mass is not "
                "represented in the continuation, so the solve returns NaN. Either make "
                f"'{s.name}' active at that age or give it probability 0 there."
            )


def _check_states(spec, specs, resolver, period, ages) -> None:
    age = float(ages.values[period])
    by_name = {s.name: s for s in specs}
    for fname, fn in spec.functions.items():
        if not (isinstance(fn, MarkovTransition) and fname.startswith("next_") and fname != "next_regime"):
            continue
        state = fname[len("next_"):]
        size = next((a.size for s in [spec, *by_name.values()] for a in s.states if a.name == state), None)
        if size is None:
            continue
        label = f"state '{state}'"
        try:
            out, n_pts, _ = _evaluate(spec, resolver, fname, period, age)
            a = _point_major(out, n_pts, size)
        except (ValueError, TypeError, IndexError):
            a = None
        if a is None:
            a, _ = _pointwise(spec, resolver, fname, period, age)
        if a.shape[-1] != size:
            raise InvalidStateTransitionProbabilitiesError(
                f"MarkovTransition for {label} in regime '{spec.name}' at age {age} returned an outcome "
                f"axis of size {a.shape[-1]}; expected {size} from the state's DiscreteGrid."
            )
        if (a < 0).any() or (a > 1).any():
            raise InvalidStateTransitionProbabilitiesError(
                f"MarkovTransition for {label} in regime '{spec.name}' at age {age} returned values outside [0, 1]."
            )
        if not np.allclose(a.sum(axis=-1), 1.0, atol=1e-6):
            raise InvalidStateTransitionProbabilitiesError(
                f"MarkovTransition for {label} in regime '{spec.name}' at age {age} returned rows that do "
                "not sum to 1 along the outcome axis."
            )


def validate_transitions(model, params, log_level: str) -> None:
    """Check regime and stochastic state transitions for every period.

    ``"off"`` skips; ``"debug"`` raises the first failure; other levels warn
    for every failure and continue."""
    if log_level == "off":
        return
    raise_ = log_level == "debug"

    def report(err: Exception) -> None:
        if raise_:
            raise err
        warnings.warn(str(err), stacklevel=4)

    specs = model.regime_specs
    resolver = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    ages = model.ages
    last = model.n_periods - 1
    for s in specs:
        if not s.terminal and last in s.active_periods:
            report(InvalidRegimeTransitionProbabilitiesError(
                f"Non-terminal regime(s) ['{s.name}'] are active at the last period (age "
                f"{float(ages.values[last])})."
            ))
    for period in range(last):
        for s in specs:
            if s.terminal or period not in s.active_periods:
                continue
            for check in (_check_regime, _check_states):
                try:
                    check(s, specs, resolver, period, ages)
                except (InvalidRegimeTransitionProbabilitiesError, InvalidStateTransitionProbabilitiesError) as e:
                    report(e)
