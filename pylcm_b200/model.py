"""The user-facing ``Model`` (``src/lcm/model.py:102-848``).

``Model(ages=..., regimes=..., regime_id_class=..., fixed_params=...)`` builds
the canonical regime specs; ``model.solve(params=...)`` runs backward
induction on the GPU and returns ``{period: {regime_name: V}}`` like the
reference; ``model.simulate(...)`` runs forward simulation on the GPU.
"""

from __future__ import annotations

import dataclasses
import threading
from types import MappingProxyType
from typing import Any, Mapping

import numpy as np

from pylcm_b200.ages import AgeGrid
from pylcm_b200.exceptions import InvalidValueFunctionError, ModelInitializationError
from pylcm_b200.spec import build_regime_specs


class Model:
    """A finite-horizon model made of regimes."""

    def __init__(
        self,
        *,
        ages: AgeGrid,
        regimes: Mapping[str, Any],
        regime_id_class: type,
        description: str = "",
        fixed_params: Mapping = MappingProxyType({}),
        enable_jit: bool = True,
        n_subjects: int | None = None,
    ) -> None:
        self.description = description
        self.ages = ages
        self.n_periods = ages.n_periods
        self.fixed_params = dict(fixed_params)
        self.enable_jit = enable_jit
        self.n_subjects = n_subjects
        self.user_regimes = MappingProxyType(dict(regimes))
        self.regime_specs = build_regime_specs(regimes, regime_id_class, ages)
        self.regime_names_to_ids = MappingProxyType({s.name: s.rid for s in self.regime_specs})
        self.regime_id_class = regime_id_class
        last = self.n_periods - 1
        for s in self.regime_specs:
            if not s.terminal and last in s.active_periods:
                raise ModelInitializationError(
                    f"non-terminal regime {s.name!r} is active in the last period"
                )
        self._lock = threading.Lock()
        self._engines: dict = {}

    def __repr__(self) -> str:
        return f"Model(regimes={list(self.regime_names_to_ids)}, n_periods={self.n_periods})"

    # ------------------------------------------------------------------ solve
    def engine(self, precision: str = "fp64"):
        from pylcm_b200.engine import SolveEngine

        with self._lock:
            eng = self._engines.get(precision)
            if eng is None:
                eng = SolveEngine(self, precision=precision)
                self._engines[precision] = eng
            return eng

    def solve(
        self,
        *,
        params: Mapping,
        log_level: str = "progress",
        max_compilation_workers: int | None = None,
        log_path: Any = None,
        log_keep_n_latest: int = 3,
        return_simulation_policy: bool = False,
        precision: str = "fp64",
        return_policy: bool = False,
        return_device: bool = False,
    ):
        """Backward induction; returns ``{period: {regime: V}}``.

        The keywords up to ``return_simulation_policy`` are the reference's
        (``src/lcm/model.py:440-519``):

        - ``log_level``: ``"off"`` skips the transition checks and the NaN
          check; ``"warning"`` / ``"progress"`` warn; ``"debug"`` raises.
        - ``max_compilation_workers``: accepted for compatibility (kernels are
          compiled once per model structure by NVRTC and cached).
        - ``log_path`` / ``log_keep_n_latest``: the reference writes diagnostic
          snapshots there; this solver writes none and warns when a path is
          given.
        - ``return_simulation_policy``: also return, as
          ``(V, {period: {regime: EGMSimPolicy}})``, the refined rows every
          DC-EGM regime publishes per period (regimes solved by grid search
          publish none, as in the reference).

        Added here: ``precision="fp64"`` is the plain path; ``"fp32"``
        searches in single precision and re-evaluates the chosen action in
        double precision.  With ``return_policy=True`` a mapping of flat argmax
        action indices follows V in the returned tuple.  Unknown keywords raise
        ``TypeError``.
        """
        _check_compat_kwargs(max_compilation_workers, log_path, log_keep_n_latest)
        from pylcm_b200.validation import validate_transitions

        validate_transitions(self, params, log_level)
        eng = self.engine(precision)
        if return_simulation_policy:
            V, pol, carries = eng.solve(params, collect_carries=True)
        else:
            (V, pol), carries = eng.solve(params), {}
        if log_level != "off":
            _check_nan(V, raise_=(log_level == "debug"))
        if not return_device:
            V = {p: {r: v.cpu().numpy() for r, v in d.items()} for p, d in V.items()}
            pol = {p: {r: v.cpu().numpy() for r, v in d.items()} for p, d in pol.items()}
        V = MappingProxyType({p: MappingProxyType(d) for p, d in V.items()})
        out = [V]
        if return_policy:
            out.append(MappingProxyType({p: MappingProxyType(d) for p, d in pol.items()}))
        if return_simulation_policy:
            out.append(_sim_policies(self, carries, return_device))
        return out[0] if len(out) == 1 else tuple(out)

    # --------------------------------------------------------------- simulate
    def simulate(
        self,
        *,
        params: Mapping,
        initial_conditions: Mapping,
        period_to_regime_to_V_arr=None,
        log_level: str = "progress",
        seed: int | None = None,
        subject_batch_size: int = 0,
        log_path: Any = None,
        log_keep_n_latest: int = 3,
        max_compilation_workers: int | None = None,
        precision: str = "fp64",
        rng: str = "jax",
    ):
        """Forward simulation (``src/lcm/model.py:648-848``), solving first
        when ``period_to_regime_to_V_arr`` is None.

        ``rng="jax"`` (default) draws from the reference's random stream (JAX's
        Threefry-2x32 with its key threading: the same seed gives the
        reference's draws); ``"philox"`` from a counter stream keyed by
        (seed, subject, period, stream), the serving loop's.

        ``subject_batch_size`` only partitions the subject axis in the
        reference and leaves results unchanged; every subject is simulated in
        one pass here, so it is validated and otherwise has no effect."""
        _check_compat_kwargs(max_compilation_workers, log_path, log_keep_n_latest)
        if not isinstance(subject_batch_size, (int, np.integer)) or subject_batch_size < 0:
            raise ValueError("subject_batch_size must be a non-negative integer")
        from pylcm_b200.simulate import simulate as _simulate
        from pylcm_b200.validation import validate_transitions

        validate_transitions(self, params, log_level)
        return _simulate(
            self,
            params=params,
            initial_conditions=initial_conditions,
            V_arr=period_to_regime_to_V_arr,
            seed=0 if seed is None else int(seed),
            precision=precision,
            log_level=log_level,
            rng=rng,
        )


@dataclasses.dataclass(frozen=True)
class EGMSimPolicy:
    """Refined rows a DC-EGM regime publishes for one period
    (``src/_lcm/egm/published_policy.py:76-120``).

    Leading axes are the regime's discrete states then discrete actions (in
    canonical order); the trailing axis is the refined-row length, NaN-padded
    after each row's kept points."""

    endog_grid: Any
    policy: Any
    value: Any
    marginal_utility: Any


def _sim_policies(model: "Model", carries: dict, on_device: bool):
    from pylcm_b200.egm import is_egm

    specs = {s.name: s for s in model.regime_specs}
    # every period has an entry, empty where no regime publishes rows (the
    # reference's backward_induction.py:245-253)
    out = {p: MappingProxyType({}) for p in range(model.n_periods)}
    for period, regs in carries.items():
        d = {}
        for name, c in regs.items():
            s = specs[name]
            lead = tuple(a.size for a in s.states if a.kind != "continuous")
            lead += tuple(a.size for a in s.actions if a.kind != "continuous")
            assert is_egm(s)

            def conv(t, lead=lead):
                t = t[0].reshape(*lead, t.shape[-1])
                return t if on_device else t.cpu().numpy()

            d[name] = EGMSimPolicy(endog_grid=conv(c["rg"]), policy=conv(c["rc"]), value=conv(c["rv"]),
                                   marginal_utility=conv(c["mu"]))
        out[period] = MappingProxyType(d)
    return MappingProxyType(dict(sorted(out.items())))


def _check_compat_kwargs(max_compilation_workers, log_path, log_keep_n_latest) -> None:
    import warnings

    if max_compilation_workers is not None and (
        not isinstance(max_compilation_workers, (int, np.integer)) or max_compilation_workers < 1
    ):
        raise ValueError("max_compilation_workers must be a positive integer or None")
    if not isinstance(log_keep_n_latest, (int, np.integer)) or log_keep_n_latest < 0:
        raise ValueError("log_keep_n_latest must be a non-negative integer")
    if log_path is not None:
        warnings.warn("log_path: this solver writes no diagnostic snapshots", stacklevel=3)


def _check_nan(V, raise_: bool) -> None:
    import warnings

    for p, d in V.items():
        for r, v in d.items():
            a = v if isinstance(v, np.ndarray) else None
            bad = bool(np.isnan(a).any()) if a is not None else bool(v.isnan().any().item())
            if bad:
                msg = f"value function of regime {r!r} in period {p} contains NaN"
                if raise_:
                    raise InvalidValueFunctionError(msg)
                warnings.warn(msg, stacklevel=3)
