"""The user-facing ``Model`` (``src/lcm/model.py:102-848``).

``Model(ages=..., regimes=..., regime_id_class=..., fixed_params=...)`` builds
the canonical regime specs; ``model.solve(params=...)`` runs backward
induction on the GPU and returns ``{period: {regime_name: V}}`` like the
reference; ``model.simulate(...)`` runs forward simulation on the GPU.
"""

from __future__ import annotations

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
        precision: str = "fp64",
        return_policy: bool = False,
        return_device: bool = False,
        **_ignored: Any,
    ):
        """Backward induction; returns ``{period: {regime: V}}``.

        ``precision="fp64"`` is the plain path; ``"fp32"`` searches in single
        precision and re-evaluates the chosen action in double precision.
        With ``return_policy=True`` a second mapping of flat argmax action
        indices is returned as well.
        """
        eng = self.engine(precision)
        V, pol = eng.solve(params)
        if log_level != "off":
            _check_nan(V, raise_=(log_level == "debug"))
        if not return_device:
            V = {p: {r: v.cpu().numpy() for r, v in d.items()} for p, d in V.items()}
            pol = {p: {r: v.cpu().numpy() for r, v in d.items()} for p, d in pol.items()}
        V = MappingProxyType({p: MappingProxyType(d) for p, d in V.items()})
        if return_policy:
            return V, MappingProxyType({p: MappingProxyType(d) for p, d in pol.items()})
        return V

    # --------------------------------------------------------------- simulate
    def simulate(
        self,
        *,
        params: Mapping,
        initial_conditions: Mapping,
        period_to_regime_to_V_arr=None,
        log_level: str = "progress",
        seed: int | None = None,
        precision: str = "fp64",
        **_ignored: Any,
    ):
        from pylcm_b200.simulate import simulate as _simulate

        return _simulate(
            self,
            params=params,
            initial_conditions=initial_conditions,
            V_arr=period_to_regime_to_V_arr,
            seed=0 if seed is None else int(seed),
            precision=precision,
            log_level=log_level,
        )


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
