"""User-facing regime declarations.

Same fields and meaning as the reference's ``Regime`` (``src/lcm/regime.py:41-186``),
``MarkovTransition`` (``src/lcm/transition.py:44-86``), ``ExtremeValueTasteShocks``
(``src/lcm/taste_shocks.py:12``) and ``ConsumptionSavingsRegime`` /
``LiquidMargin`` (``src/lcm/consumption_savings_regime.py``).  Phases,
age-specialised grids, per-target transition dicts and non-linear certainty
equivalents are not part of this solver's scope and are rejected.
"""

from __future__ import annotations

import dataclasses
from types import MappingProxyType
from typing import Any, Callable, Mapping

from pylcm_b200 import solvers as _solvers
from pylcm_b200.exceptions import RegimeInitializationError
from pylcm_b200.grids import Grid


@dataclasses.dataclass(frozen=True)
class MarkovTransition:
    """Wraps a function returning a probability vector over the target's grid
    (a state transition) or over all regimes (a regime transition)."""

    func: Callable

    def __call__(self, *args: Any, **kwargs: Any) -> Any:
        return self.func(*args, **kwargs)


@dataclasses.dataclass(frozen=True, kw_only=True)
class ExtremeValueTasteShocks:
    """IID EV1 taste shocks on the regime's discrete-action combinations.

    The scale is the runtime parameter ``params[regime]["taste_shocks"]["scale"]``.
    """


def _frozen(m: Mapping | None) -> MappingProxyType:
    return MappingProxyType(dict(m or {}))


@dataclasses.dataclass(frozen=True, kw_only=True)
class Regime:
    """A regime: states, actions, functions, constraints and transitions.

    ``transition=None`` marks a terminal regime.
    """

    transition: Any
    active: Callable = lambda _age: True
    states: Mapping[str, Grid] = dataclasses.field(default_factory=dict)
    state_transitions: Mapping[str, Any] = dataclasses.field(default_factory=dict)
    actions: Mapping[str, Grid] = dataclasses.field(default_factory=dict)
    functions: Mapping[str, Callable] = dataclasses.field(default_factory=dict)
    constraints: Mapping[str, Callable] = dataclasses.field(default_factory=dict)
    solver: Any = dataclasses.field(default_factory=lambda: _solvers.GridSearch())
    taste_shocks: ExtremeValueTasteShocks | None = None
    description: str = ""

    def __post_init__(self) -> None:
        for name in ("states", "state_transitions", "actions", "functions", "constraints"):
            object.__setattr__(self, name, _frozen(getattr(self, name)))
        if isinstance(self.transition, Mapping):
            raise RegimeInitializationError(
                "per-target regime-transition dicts are not supported; use a bare "
                "callable or MarkovTransition"
            )
        if not self.terminal and "utility" not in self.functions:
            raise RegimeInitializationError("a regime needs a 'utility' function")
        if self.terminal and "utility" not in self.functions:
            raise RegimeInitializationError("a terminal regime needs a 'utility' function")
        overlap = set(self.states) & set(self.actions)
        if overlap:
            raise RegimeInitializationError(f"names used as both state and action: {sorted(overlap)}")
        if isinstance(self.solver, (_solvers.EGM, _solvers.NEGM)):
            raise NotImplementedError(
                f"{type(self.solver).__name__} is not implemented on the GPU path; GridSearch and DCEGM are "
                "(DCEGM solves the one-asset problem without discrete choices too)"
            )
        if not isinstance(self.solver, (_solvers.GridSearch, _solvers.DCEGM)):
            raise RegimeInitializationError(
                f"unknown solver {type(self.solver).__name__}: use GridSearch or DCEGM"
            )
        if not isinstance(self, ConsumptionSavingsRegime) and isinstance(self.solver, _solvers.DCEGM):
            raise RegimeInitializationError(
                "EGM-family solvers require regime-owned margin declarations: use "
                "ConsumptionSavingsRegime for DCEGM."
            )
        if self.taste_shocks is not None and not any(
            type(g).__name__ == "DiscreteGrid" for g in self.actions.values()
        ):
            raise RegimeInitializationError("taste shocks require at least one discrete action")

    @property
    def terminal(self) -> bool:
        return self.transition is None

    @property
    def stochastic_regime_transition(self) -> bool:
        return isinstance(self.transition, MarkovTransition)

    def replace(self, **kwargs: Any) -> "Regime":
        try:
            return dataclasses.replace(self, **kwargs)
        except TypeError as e:
            raise RegimeInitializationError(f"Failed to replace attributes of the regime: {e}") from e


@dataclasses.dataclass(frozen=True, kw_only=True)
class LiquidMargin:
    """Names of the liquid Euler margin of an EGM regime."""

    state: str
    action: str
    resources: str
    post_decision_state: str


@dataclasses.dataclass(frozen=True, kw_only=True)
class ConsumptionSavingsRegime(Regime):
    """A regime solvable by ``DCEGM``: one Euler state, one continuous action."""

    liquid: LiquidMargin | None = None

    def __post_init__(self) -> None:
        super().__post_init__()
        if isinstance(self.solver, _solvers.DCEGM) and self.liquid is None:
            raise RegimeInitializationError("DCEGM needs a LiquidMargin declaration")
