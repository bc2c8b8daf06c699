"""Solver configuration objects (``src/lcm/solvers.py``, ``src/_lcm/solution/dcegm.py:71-255``)."""

from __future__ import annotations

import dataclasses
from typing import Any


@dataclasses.dataclass(frozen=True, kw_only=True)
class GridSearch:
    """Brute-force grid search over the full state-action product (the default)."""


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
class DCEGM:
    """Discrete-continuous EGM with an upper envelope (``dcegm.py:151-255``).

    Only ``FUESEnvelope`` is implemented by this solver.
    """

    savings_grid: Any
    envelope: Any = dataclasses.field(default_factory=FUESEnvelope)
    refined_grid_factor: float = 2.0
    n_constrained_points: int = 20
    stochastic_node_batch_size: int = 0

    def __post_init__(self) -> None:
        if not isinstance(self.envelope, FUESEnvelope):
            raise NotImplementedError("only FUESEnvelope is implemented on the GPU path")
        if self.refined_grid_factor < 1.0:
            raise ValueError("refined_grid_factor must be >= 1")
        if self.n_constrained_points < 1:
            raise ValueError("n_constrained_points must be >= 1")
