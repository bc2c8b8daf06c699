"""Solver configuration objects (``src/lcm/solvers.py``, ``src/_lcm/solution/dcegm.py:71-255``)."""

from __future__ import annotations

import dataclasses
from typing import Any


@dataclasses.dataclass(frozen=True, kw_only=True)
class GridSearch:
    """Brute-force grid search over the full state-action product (the default)."""


@dataclasses.dataclass(frozen=True, kw_only=True)
class ExactEnvelope:
    """Certified segment-envelope configuration (``dcegm.py:71-88``); not
    implemented on the GPU path (``DCEGM`` refuses it)."""

    max_runs: int = 24
    cell_batch_size: int | None = None

    def __post_init__(self) -> None:
        if int(self.max_runs) < 2:
            raise ValueError("max_runs must be >= 2")
        if self.cell_batch_size is not None and int(self.cell_batch_size) < 1:
            raise ValueError("cell_batch_size must be a positive integer or None")


@dataclasses.dataclass(frozen=True, kw_only=True)
class FUESEnvelope:
    """Fast Upper-Envelope Scan (``dcegm.py:93-110``)."""

    jump_thresh: float = 2.0
    n_points_to_scan: int | None = None
    scan_unroll: int = 1  # a loop-unrolling knob of the reference's scan; results do not depend on it

    def __post_init__(self) -> None:
        if self.jump_thresh <= 0:
            raise ValueError("jump_thresh must be positive")
        if self.n_points_to_scan is not None:
            if int(self.n_points_to_scan) < 1:
                raise ValueError("n_points_to_scan must be a positive integer or None")
        if self.scan_unroll < 1:
            raise ValueError("scan_unroll must be >= 1")


@dataclasses.dataclass(frozen=True, kw_only=True)
class RFCEnvelope:
    """Rooftop-Cut upper envelope (``dcegm.py:113-126``): a candidate below a
    neighbour's tangent line across a policy jump is deleted."""

    jump_thresh: float = 2.0
    search_radius: int = 10

    def __post_init__(self) -> None:
        if self.jump_thresh <= 0:
            raise ValueError("jump_thresh must be positive")
        if int(self.search_radius) < 1:
            raise ValueError("search_radius must be >= 1")


@dataclasses.dataclass(frozen=True, kw_only=True)
class LTMEnvelope:
    """Local-upper-bound brute-force envelope (``dcegm.py:129-132``)."""


@dataclasses.dataclass(frozen=True, kw_only=True)
class MSSEnvelope:
    """HARK-style left-to-right segment envelope with crossing insertion
    (``dcegm.py:135-138``)."""


@dataclasses.dataclass(frozen=True, kw_only=True)
class DCEGM:
    """Discrete-continuous EGM with an upper envelope (``dcegm.py:151-255``).

    ``FUESEnvelope`` (the default), ``RFCEnvelope``, ``LTMEnvelope`` and
    ``MSSEnvelope`` are implemented by this solver (RFC, LTM and MSS on
    candidate rows of up to 4096 points).
    """

    savings_grid: Any
    envelope: Any = dataclasses.field(default_factory=FUESEnvelope)
    refined_grid_factor: float = 2.0
    n_constrained_points: int = 20
    stochastic_node_batch_size: int = 0

    def __post_init__(self) -> None:
        if not isinstance(self.envelope, (FUESEnvelope, RFCEnvelope, LTMEnvelope, MSSEnvelope)):
            raise NotImplementedError(
                f"{type(self.envelope).__name__} is not implemented on the GPU path "
                "(FUESEnvelope, RFCEnvelope, LTMEnvelope and MSSEnvelope are)")
        if self.refined_grid_factor < 1.0:
            raise ValueError("refined_grid_factor must be >= 1")
        if self.n_constrained_points < 1:
            raise ValueError("n_constrained_points must be >= 1")


@dataclasses.dataclass(frozen=True, kw_only=True)
class EGM:
    """The plain one-asset endogenous grid method (``src/_lcm/solution/egm.py:70-90``).

    Accepted as a configuration so that models naming it load; a regime
    declaring it is refused when the regime is built (the GPU path implements
    ``DCEGM``, which solves the same one-state, no-kink problem: its envelope
    keeps every candidate of a monotone row).
    """

    savings_grid: Any


@dataclasses.dataclass(frozen=True, kw_only=True)
class NEGM:
    """Nested EGM: an outer grid search over a second continuous margin with an
    inner ``DCEGM`` solve (``src/_lcm/solution/negm.py:72-120``).  Accepted as a
    configuration; a regime declaring it is refused when the regime is built."""

    inner: Any
    outer_grid: Any
    outer_batch_size: int = 0

    def __post_init__(self) -> None:
        if int(self.outer_batch_size) < 0:
            raise ValueError("outer_batch_size must be >= 0")
