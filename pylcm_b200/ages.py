"""Age grid (``src/lcm/ages.py``): ages indexed by period."""

from __future__ import annotations

import re
from fractions import Fraction
from typing import Callable, Iterable

import numpy as np

from pylcm_b200.exceptions import GridInitializationError

_STEP_RE = re.compile(r"^(\d+)?([YQM])$")


def _parse_step(step: str) -> Fraction:
    m = _STEP_RE.match(step)
    if not m:
        raise GridInitializationError(f"invalid age step {step!r}; expected e.g. 'Y', '2Y', '6M'")
    mult = int(m.group(1) or 1)
    unit = {"Y": Fraction(1), "Q": Fraction(1, 4), "M": Fraction(1, 12)}[m.group(2)]
    return mult * unit


class AgeGrid:
    """Ages from `start` to `stop` inclusive by `step`, or explicit `exact_values`."""

    def __init__(self, *, start=None, stop=None, step: str | None = None, exact_values: Iterable | None = None) -> None:
        if start is not None and stop is not None and step is not None:
            st = _parse_step(step)
            n_steps = int((Fraction(stop) - Fraction(start)) // st) + 1
            if Fraction(start) + (n_steps - 1) * st != Fraction(stop):
                raise GridInitializationError("step must divide the age range evenly")
            vals = tuple(Fraction(start) + i * st for i in range(n_steps))
        elif exact_values is not None:
            vals = tuple(Fraction(v) for v in exact_values)
            if any(b <= a for a, b in zip(vals, vals[1:])):
                raise GridInitializationError("exact_values must be strictly increasing")
        else:
            raise GridInitializationError("Must specify 'start/stop/step' or 'exact_values'.")
        self._is_integer = all(v.denominator == 1 for v in vals)
        self._exact_values = tuple(int(v) if self._is_integer else v for v in vals)
        self._values = np.array([float(v) for v in vals])

    @property
    def is_integer(self) -> bool:
        return self._is_integer

    @property
    def values(self) -> np.ndarray:
        return self._values

    @property
    def exact_values(self) -> tuple:
        return self._exact_values

    @property
    def n_periods(self) -> int:
        return len(self._exact_values)

    def period_to_age(self, period: int):
        if period < 0 or period >= self.n_periods:
            raise IndexError(f"Period {period} out of bounds for grid with {self.n_periods} periods.")
        v = self._exact_values[period]
        return int(v) if self._is_integer else float(v)

    def get_periods_where(self, predicate: Callable) -> tuple[int, ...]:
        return tuple(p for p in range(self.n_periods) if bool(predicate(self.period_to_age(p))))
