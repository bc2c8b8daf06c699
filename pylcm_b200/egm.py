"""DC-EGM regime description (host side).

Traces what the endogenous-grid step of a ``ConsumptionSavingsRegime`` solved
by ``DCEGM`` needs, restating the pieces the reference assembles in
``src/_lcm/egm/step.py:565-940`` and ``src/_lcm/egm/step_core.py:156-616``:

- utility u(c, discrete) and its derivative u'(c) (the reference uses
  ``jax.grad``; here :func:`pylcm_b200.ir.diff`);
- the regime's ``inverse_marginal_utility``;
- per next-period target: the regime probability, the laws of the target's
  discrete states, and the liquid state's law written in the post-decision
  state A (the savings function is replaced by A), with dR'/dA;
- the exogenous savings grid, the constrained-segment sampling
  (``CONSTRAINED_OFFSET_FRACTION = 1e-4``, ratio (1/1e-4)^(1/(n-1)),
  ``step_core.py:54``, ``step.py:914``) and the refined-row length
  ``ceil(refined_grid_factor * n_candidates)``.

Rows are the combinations of the regime's discrete states (in canonical
order) and discrete actions (discrete actions vary fastest), like the
reference's per-combo vmap.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Any

import numpy as np

from pylcm_b200 import ir
from pylcm_b200.exceptions import ModelInitializationError, TracingError
from pylcm_b200.regime import MarkovTransition
from pylcm_b200.solvers import DCEGM
from pylcm_b200.spec import (
    BETA_ARG,
    BETA_FUNC,
    NextState,
    ParamResolver,
    RegimeSpec,
    _as_bool,
    _Tracer,
    proc_P_name,
    proc_grid_name,
)

CONSTRAINED_OFFSET_FRACTION = 1e-4


def is_egm(spec: RegimeSpec) -> bool:
    return isinstance(spec.solver, DCEGM)


@dataclasses.dataclass
class EgmTarget:
    spec: RegimeSpec
    prob: ir.Expr
    disc_laws: dict  # state name -> NextState (target's discrete states)
    next_R: ir.Expr | None  # law of the liquid state in A (None: stateless target)
    dR_dA: ir.Expr | None
    # no law for one of the target's states: the source cannot reach the
    # target; a non-zero probability toward it poisons the continuation (NaN)
    unreachable: bool = False
    # a target solved without the endogenous grid (terminal or grid search):
    # its carry is its value array on its own state grid with the marginal
    # value of its Euler state (``value_euler``) beside it
    value_euler: str | None = None

    @property
    def is_value(self) -> bool:
        return self.value_euler is not None


def value_child_euler(tg: RegimeSpec) -> str:
    """The Euler state of a target that publishes its value array as a carry
    (``regime_building/processing.py:1270-1386``): the first declared state,
    which must be continuous; further continuous (passive) states are not
    carried here; a terminal target has no actions and no process states
    (its marginal value is the gradient of its utility)."""
    first = tg.state(next(iter(tg.user.states)))
    cont = [a for a in tg.states if a.kind == "continuous"]
    if first.kind != "continuous":
        raise ModelInitializationError(
            f"DCEGM target {tg.name!r}: its first state must be its continuous (Euler) state"
        )
    if len(cont) > 1:
        raise ModelInitializationError(
            f"DCEGM target {tg.name!r}: passive continuous states in a carried value are not supported"
        )
    if tg.terminal and (tg.actions or any(a.kind == "process" for a in tg.states)):
        raise ModelInitializationError(
            f"terminal DCEGM target {tg.name!r} must have no actions and no process states"
        )
    return first.name


@dataclasses.dataclass
class EgmRegime:
    spec: RegimeSpec
    E: str  # liquid (Euler) state
    C: str  # continuous action
    disc_states: list
    disc_actions: list
    U: ir.Expr
    dU: ir.Expr
    invmu: ir.Expr
    beta: ir.Expr
    targets: list
    savings: np.ndarray
    n_constrained: int
    ratio: float
    n_pad: int
    jump_thresh: float
    scan_window: int  # FUES same-segment look-ahead (0: exhaustive)
    taste_scale: float | None
    feasible: ir.Expr
    tracer: Any
    envelope: str = "fues"  # the upper envelope: "fues" | "ltm" | "rfc" | "mss"
    search_radius: int = 10  # RFC: neighbours inspected on each side

    @property
    def n_rows(self) -> int:
        n = 1
        for a in self.disc_states + self.disc_actions:
            n *= a.size
        return n

    @property
    def n_disc_actions(self) -> int:
        n = 1
        for a in self.disc_actions:
            n *= a.size
        return n

    @property
    def n_cand(self) -> int:
        return self.n_constrained + len(self.savings)

    def row_env(self, row: int) -> dict:
        """(kind, name) -> code for the discrete variables of a row."""
        env = {}
        rem = row
        for a in reversed(self.disc_states + self.disc_actions):
            env[("state" if a in self.disc_states else "action", a.name)] = rem % a.size
            rem //= a.size
        return env


MU = ir.var("egm", "mu", "f")
A_VAR = ir.var("egm", "A", "f")


def trace_egm_regime(spec: RegimeSpec, specs: list, resolver: ParamResolver, targets: tuple) -> EgmRegime:
    solver = spec.solver
    liq = spec.user.liquid
    E, C = liq.state, liq.action
    if liq.resources != E:
        raise ModelInitializationError("DCEGM here needs resources equal to the liquid state")
    cont_states = [a for a in spec.states if a.kind == "continuous"]
    cont_actions = [a for a in spec.actions if a.kind == "continuous"]
    if [a.name for a in cont_states] != [E] or [a.name for a in cont_actions] != [C]:
        raise ModelInitializationError("DCEGM needs exactly one continuous state and one continuous action")
    if "inverse_marginal_utility" not in spec.functions:
        raise ModelInitializationError("DCEGM needs an inverse_marginal_utility function")
    t = _Tracer(spec, resolver, overrides={liq.post_decision_state: A_VAR})
    U = ir.const(t.trace("utility"))
    cvar = ir.var("action", C, "f")
    dU = ir.diff(U, cvar)
    # inverse marginal utility: its single argument is the marginal continuation
    imu = spec.functions["inverse_marginal_utility"]
    import inspect

    from pylcm_b200.spec import _rebind_numpy_namespace

    fn = _rebind_numpy_namespace(imu)
    sig = list(inspect.signature(fn).parameters)
    kwargs = {sig[0]: MU}
    for p in sig[1:]:
        kwargs[p] = t.resolve_arg("inverse_marginal_utility", p, inspect.Parameter.empty)
    invmu = ir.const(fn(**kwargs))
    ok, bval = resolver.find(spec.name, BETA_FUNC, BETA_ARG)
    if not ok:
        raise TracingError(f"regime {spec.name!r}: missing discount_factor")
    beta = t.add_param(f"{BETA_FUNC}__{BETA_ARG}", bval, ("arg", BETA_FUNC, BETA_ARG))
    for ax in spec.states:
        if ax.kind == "process":
            pp = resolver.process_params(spec.name, ax.name, ax.grid)
            t.add_param(proc_grid_name(ax.name), ax.grid.compute_gridpoints(**pp), ("proc_nodes", ax.name))
            t.add_param(proc_P_name(ax.name), ax.grid.compute_transition_probs(**pp), ("proc_P", ax.name))
    feasible: ir.Expr = ir.const(True)
    for cn in spec.constraint_names:
        feasible = ir.logical("and", feasible, _as_bool(t.trace(cn)))
    raw = t.trace("next_regime")
    n_reg = len(specs)
    if isinstance(spec.user.transition, MarkovTransition):
        probs = [ir.const(x) for x in raw.items]
    else:
        rid = ir.const(raw)
        probs = [ir.where(ir._cmp("==", rid, k), 1.0, 0.0) for k in range(n_reg)]
    by = {s.name: s for s in specs}
    tgs = []
    for tname in targets:
        tg = by[tname]
        if not tg.states:
            tgs.append(EgmTarget(tg, probs[tg.rid], {}, None, None))
            continue
        euler = tg.user.liquid.state if is_egm(tg) else value_child_euler(tg)
        laws = {}
        nextR = None
        src_states = {a.name for a in spec.states}
        unreachable = False
        for ax in tg.states:
            if ax.kind == "process":
                if ax.name not in src_states:
                    unreachable = True
                    break
                laws[ax.name] = NextState("process", None, ax.name)
                continue
            fname = f"next_{ax.name}"
            if fname not in spec.functions:
                if ax.kind == "continuous" or ax.name not in src_states:
                    unreachable = True
                    break
                laws[ax.name] = NextState("det", ir.var("state", ax.name, "i"))
                continue
            law = spec.functions[fname]
            val = t.trace(fname)
            if ax.name == euler:
                nextR = ir.const(val)
            elif isinstance(law, MarkovTransition):
                laws[ax.name] = NextState("markov", val)
            else:
                laws[ax.name] = NextState("det", ir.const(val))
        if unreachable or nextR is None:
            tgs.append(EgmTarget(tg, probs[tg.rid], {}, None, None, unreachable=True))
            continue
        tgs.append(EgmTarget(tg, probs[tg.rid], laws, nextR, ir.diff(nextR, A_VAR),
                             value_euler=None if is_egm(tg) else euler))
    sav = np.asarray(solver.savings_grid.to_numpy(), dtype=np.float64)
    nc = int(solver.n_constrained_points)
    ratio = (1.0 / CONSTRAINED_OFFSET_FRACTION) ** (1.0 / max(nc - 1, 1))
    n_pad = int(math.ceil(solver.refined_grid_factor * (nc + len(sav))))
    taste = resolver.taste_scale(spec.name) if spec.taste_shocks else None
    return EgmRegime(
        spec=spec,
        E=E,
        C=C,
        disc_states=[a for a in spec.states if a.kind != "continuous"],
        disc_actions=[a for a in spec.actions if a.kind != "continuous"],
        U=U,
        dU=dU,
        invmu=invmu,
        beta=beta,
        targets=tgs,
        savings=sav,
        n_constrained=nc,
        ratio=ratio,
        n_pad=n_pad,
        jump_thresh=float(getattr(solver.envelope, "jump_thresh", 2.0)),
        scan_window=int(getattr(solver.envelope, "n_points_to_scan", None) or 0),
        envelope={"FUESEnvelope": "fues", "LTMEnvelope": "ltm", "RFCEnvelope": "rfc",
                  "MSSEnvelope": "mss"}[type(solver.envelope).__name__],
        search_radius=int(getattr(solver.envelope, "search_radius", 10)),
        taste_scale=taste,
        feasible=feasible,
        tracer=t,
    )


def _as_traced(er: "EgmRegime"):
    """A TracedRegime view of the EGM tracer's parameters (layout / packing)."""
    from pylcm_b200.spec import TracedRegime

    t = er.tracer
    return TracedRegime(
        spec=er.spec, U=er.U, F=ir.const(True), regime_probs=None, regime_id=None, next_states={},
        param_values=t.param_values, param_order=t.param_order, param_sources=t.param_sources,
        beta=er.beta, taste_scale=er.taste_scale, process_tables={},
    )


def _tracer_layout(self):
    return _as_traced(self).param_layout()


def _pack_for(self, resolver):
    tr = _as_traced(self)
    return tr.pack_params(tr.values_for(resolver))


def _pack_many(self, resolvers, memo=None):
    return _as_traced(self).pack_many(resolvers, memo)


EgmRegime.tracer_layout = _tracer_layout
EgmRegime.pack_for = _pack_for
EgmRegime.pack_many = _pack_many
