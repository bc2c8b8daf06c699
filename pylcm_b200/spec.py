"""Model processing: canonical axis order, parameter resolution, tracing.

This is the host-side step between the user's ``Model``/``Regime`` declaration
and the CUDA code generator.  It restates the parts of the reference's model
build that decide *what* is computed:

- canonical state order (discrete states incl. processes, then continuous; each
  group by ``(not distributed, batch_size)``, stable) and action order
  (discrete actions first, then continuous), ``src/_lcm/variables.py:156-198`` and
  ``src/_lcm/engine.py:244-247``;
- resolution of function arguments by name (the ``dags`` rule used at
  ``src/_lcm/regime_building/Q_and_F.py:1321-1351``): an argument is another
  function's output, a state, an action, ``period``/``age``, or a parameter;
- parameter lookup: function level ``params[regime][func][arg]``, then regime
  level ``params[regime][arg]``, then model level ``params[arg]``; the same
  for ``fixed_params`` (``src/lcm/model.py:927-955``);
- the regime transition as a probability vector over regimes (a deterministic
  ``next_regime`` becomes one-hot), ``Q_and_F.py:466-681``.
"""

from __future__ import annotations

import dataclasses
import inspect
import math
from collections.abc import Mapping
from typing import Any, Callable, Sequence

import numpy as np

from pylcm_b200 import ir
from pylcm_b200.exceptions import (
    InvalidParamsError,
    ModelInitializationError,
    TracingError,
)
from pylcm_b200.grids import ContinuousGrid, DiscreteGrid, Grid
from pylcm_b200.processes import _Process
from pylcm_b200.regime import MarkovTransition

SPECIAL_ARGS = ("period", "age")
BETA_FUNC = "koopmans_aggregator"
BETA_ARG = "discount_factor"


@dataclasses.dataclass(frozen=True)
class Axis:
    """One state or action axis in canonical order."""

    name: str
    kind: str  # 'discrete' | 'process' | 'continuous'
    grid: Grid

    @property
    def size(self) -> int:
        return len(self.grid)

    @property
    def is_discrete(self) -> bool:
        return self.kind in ("discrete", "process")


def _axis_kind(grid: Grid) -> str:
    if isinstance(grid, _Process):
        return "process"
    if isinstance(grid, DiscreteGrid):
        return "discrete"
    if isinstance(grid, ContinuousGrid):
        return "continuous"
    raise ModelInitializationError(f"unsupported grid type {type(grid).__name__}")


def _state_sort_key(grid: Grid) -> tuple:
    bs = getattr(grid, "batch_size", 0)
    return (not getattr(grid, "distributed", False), bs if bs != 0 else math.inf)


@dataclasses.dataclass
class RegimeSpec:
    name: str
    rid: int
    user: Any
    states: list[Axis]
    actions: list[Axis]
    functions: dict[str, Callable]
    constraint_names: tuple[str, ...]
    active_periods: tuple[int, ...]

    @property
    def terminal(self) -> bool:
        return self.user.terminal

    @property
    def taste_shocks(self) -> bool:
        return self.user.taste_shocks is not None

    @property
    def state_shape(self) -> tuple[int, ...]:
        return tuple(a.size for a in self.states)

    @property
    def n_states(self) -> int:
        return int(np.prod(self.state_shape)) if self.states else 1

    @property
    def discrete_actions(self) -> list[Axis]:
        return [a for a in self.actions if a.is_discrete]

    @property
    def continuous_actions(self) -> list[Axis]:
        return [a for a in self.actions if not a.is_discrete]

    @property
    def n_actions(self) -> int:
        return int(np.prod([a.size for a in self.actions])) if self.actions else 1

    @property
    def n_discrete_actions(self) -> int:
        return int(np.prod([a.size for a in self.discrete_actions])) if self.discrete_actions else 1

    @property
    def n_continuous_actions(self) -> int:
        return int(np.prod([a.size for a in self.continuous_actions])) if self.continuous_actions else 1

    def state(self, name: str) -> Axis:
        for a in self.states:
            if a.name == name:
                return a
        raise KeyError(name)

    @property
    def solver(self) -> Any:
        return self.user.solver


def build_regime_specs(regimes: Mapping[str, Any], regime_id_class: type, ages) -> list[RegimeSpec]:
    """Canonicalise user regimes into `RegimeSpec`s ordered by regime id."""
    from pylcm_b200.grids import _field_names_and_values

    ids = _field_names_and_values(regime_id_class)
    if set(ids) != set(regimes):
        raise ModelInitializationError(
            f"regime_id_class fields {sorted(ids)} do not match regimes {sorted(regimes)}"
        )
    specs = []
    for name, rid in sorted(ids.items(), key=lambda kv: kv[1]):
        reg = regimes[name]
        sgrids = dict(reg.states)
        disc = [n for n in sgrids if _axis_kind(sgrids[n]) in ("discrete", "process")]
        cont = [n for n in sgrids if _axis_kind(sgrids[n]) == "continuous"]
        disc.sort(key=lambda n: _state_sort_key(sgrids[n]))
        cont.sort(key=lambda n: _state_sort_key(sgrids[n]))
        states = [Axis(n, _axis_kind(sgrids[n]), sgrids[n]) for n in disc + cont]
        agrids = dict(reg.actions)
        for n, g in agrids.items():
            if isinstance(g, _Process):
                raise ModelInitializationError(f"action {n!r} cannot be a stochastic process")
        dacts = [n for n in agrids if _axis_kind(agrids[n]) == "discrete"]
        cacts = [n for n in agrids if _axis_kind(agrids[n]) == "continuous"]
        actions = [Axis(n, _axis_kind(agrids[n]), agrids[n]) for n in dacts + cacts]
        funcs: dict[str, Callable] = dict(reg.functions)
        for cname, c in reg.constraints.items():
            if cname in funcs:
                raise ModelInitializationError(f"constraint {cname!r} clashes with a function name")
            funcs[cname] = c
        for sname, law in reg.state_transitions.items():
            if sname not in sgrids:
                raise ModelInitializationError(
                    f"regime {name!r}: state_transitions has {sname!r}, which is not a state"
                )
            if isinstance(sgrids[sname], _Process):
                raise ModelInitializationError(
                    f"regime {name!r}: process state {sname!r} has an intrinsic transition"
                )
            funcs[f"next_{sname}"] = law
        if reg.transition is not None:
            funcs["next_regime"] = reg.transition
        active = ages.get_periods_where(reg.active)
        specs.append(
            RegimeSpec(
                name=name,
                rid=int(rid),
                user=reg,
                states=states,
                actions=actions,
                functions=funcs,
                constraint_names=tuple(reg.constraints),
                active_periods=active,
            )
        )
    return specs


# --------------------------------------------------------------------------
# parameters
# --------------------------------------------------------------------------
def _is_leaf(v: Any) -> bool:
    return not isinstance(v, Mapping)


class ParamResolver:
    """Looks up a function argument's value in user params / fixed params."""

    def __init__(self, params: Mapping, fixed_params: Mapping, regime_names: tuple[str, ...]) -> None:
        self.sources = (params or {}, fixed_params or {})
        self.regime_names = regime_names

    def find(self, regime: str, func: str, arg: str) -> tuple[bool, Any]:
        for src in self.sources:
            r = src.get(regime)
            if isinstance(r, Mapping):
                f = r.get(func)
                if isinstance(f, Mapping) and arg in f:
                    return True, f[arg]
                if arg in r and _is_leaf(r[arg]):
                    return True, r[arg]
            f = src.get(func)
            if func not in self.regime_names and isinstance(f, Mapping) and arg in f:
                return True, f[arg]
            if arg in src and arg not in self.regime_names and _is_leaf(src[arg]):
                return True, src[arg]
        return False, None

    def process_params(self, regime: str, state: str, proc: _Process) -> dict:
        key = (regime, state, id(proc))
        cache = self.__dict__.setdefault("_proc_params", {})
        hit = cache.get(key)
        if hit is not None:
            return dict(hit[1])
        out = self._process_params(regime, state, proc)
        cache[key] = (proc, out)  # keeps `proc` alive so its id stays unique
        return dict(out)

    def _process_params(self, regime: str, state: str, proc: _Process) -> dict:
        # the process's fixed parameters and runtime parameter names, kept on
        # the (frozen) process object itself
        ent = proc.__dict__.get("_lcm_param_fields")
        if ent is None:
            ent = (dict(proc.fixed_params), tuple(proc.runtime_param_names))
            object.__setattr__(proc, "_lcm_param_fields", ent)
        out = dict(ent[0])
        for name in ent[1]:
            found = False
            for src in self.sources:
                for holder in (src.get(regime), src):
                    if isinstance(holder, Mapping):
                        d = holder.get(state)
                        if isinstance(d, Mapping) and name in d:
                            out[name] = d[name]
                            found = True
                            break
                if found:
                    break
            if not found:
                raise InvalidParamsError(
                    f"missing process parameter {regime}.{state}.{name}"
                )
        return out

    def taste_scale(self, regime: str) -> float:
        for src in self.sources:
            r = src.get(regime)
            if isinstance(r, Mapping):
                t = r.get("taste_shocks")
                if isinstance(t, Mapping) and "scale" in t:
                    s = float(np.asarray(t["scale"]))
                    if not s > 0:
                        raise InvalidParamsError("taste-shock scale must be strictly positive")
                    return s
        raise InvalidParamsError(f"regime {regime!r} declares taste shocks but no taste_shocks.scale")


# --------------------------------------------------------------------------
# tracing
# --------------------------------------------------------------------------
@dataclasses.dataclass
class NextState:
    """How one state of a target regime is reached from the source regime."""

    kind: str  # 'cont' | 'det' | 'markov' | 'process'
    expr: Any  # Expr (cont/det), VecExpr (markov), None (process)
    source_process: str | None = None  # process state name in the source


@dataclasses.dataclass
class TracedRegime:
    spec: RegimeSpec
    U: ir.Expr
    F: ir.Expr
    regime_probs: list | None  # one Expr per regime id (non-terminal only)
    regime_id: ir.Expr | None  # the next regime id, when the transition is deterministic
    next_states: dict[str, dict[str, NextState]]  # target -> state -> law
    param_values: dict[str, np.ndarray]  # flat name -> value (float64)
    param_order: list[str]
    param_sources: dict[str, tuple]  # flat name -> how to look it up
    beta: ir.Expr | None
    taste_scale: float | None
    process_tables: dict[str, tuple[np.ndarray, np.ndarray]]  # state -> (nodes, P)

    def param_layout(self) -> tuple[dict[str, tuple[int, tuple]], int]:
        """flat name -> (offset, shape) in the packed float64 parameter vector."""
        out = {}
        off = 0
        for name in self.param_order:
            v = np.asarray(self.param_values[name], dtype=np.float64)
            out[name] = (off, v.shape)
            off += max(1, v.size)
        return out, off

    def values_for(self, resolver: "ParamResolver") -> dict[str, np.ndarray]:
        """Parameter values of another parameter set, same layout as the trace."""
        out = {}
        # process tables of this parameter set, shared by every trace of the
        # regime (one per target set) that packs it
        proc_cache = resolver.__dict__.setdefault("_proc_tables", {})
        for flat in self.param_order:
            src = self.param_sources[flat]
            if src[0] == "arg":
                ok, val = resolver.find(self.spec.name, src[1], src[2])
                if not ok:
                    raise InvalidParamsError(f"regime {self.spec.name!r}: missing parameter {src[2]!r} of {src[1]!r}")
                v = np.asarray(val, dtype=np.float64)
            elif src[0] == "proc_field":
                ax = self.spec.state(src[1])
                pp = resolver.process_params(self.spec.name, src[1], ax.grid)
                v = np.asarray(float(pp[src[2]]), dtype=np.float64)
            else:
                state = src[1]
                ck = (self.spec.name, state)
                if ck not in proc_cache:
                    ax = self.spec.state(state)
                    pp = resolver.process_params(self.spec.name, state, ax.grid)
                    proc_cache[ck] = (
                        np.asarray(ax.grid.compute_gridpoints(**pp), dtype=np.float64),
                        np.asarray(ax.grid.compute_transition_probs(**pp), dtype=np.float64),
                    )
                v = proc_cache[ck][0 if src[0] == "proc_nodes" else 1]
            if v.shape != self.param_values[flat].shape:
                raise InvalidParamsError(
                    f"parameter {flat} has shape {v.shape}, expected {self.param_values[flat].shape}"
                )
            out[flat] = v
        return out

    def pack_many(self, resolvers: Sequence["ParamResolver"], memo: dict | None = None) -> np.ndarray:
        """Packed vectors of many parameter sets, one row each: the same
        numbers as ``pack_params(values_for(r))`` row by row, gathered one
        parameter (column) at a time.  `memo` shares the gathered columns
        between the traces of one regime (one per target set) packing the same
        resolvers; process tables are computed once per distinct set of
        process parameters."""
        cached = self.__dict__.get("_layout_cache")
        if cached is None:
            cached = self.__dict__["_layout_cache"] = self.param_layout()
        layout, total = cached
        n = len(resolvers)
        out = np.zeros((n, max(total, 1)), dtype=np.float64)
        memo = {} if memo is None else memo
        name = self.spec.name
        for flat in self.param_order:
            off, shape = layout[flat]
            src = self.param_sources[flat]
            key = (name, *src)
            col = memo.get(key)
            if col is None:
                if src[0] == "arg":
                    vals = []
                    for r in resolvers:
                        ok, val = r.find(name, src[1], src[2])
                        if not ok:
                            raise InvalidParamsError(f"regime {name!r}: missing parameter {src[2]!r} of {src[1]!r}")
                        vals.append(val)
                elif src[0] == "proc_field":
                    pps = self._process_params_of(resolvers, src[1], memo)
                    vals = [float(pp[src[2]]) for pp in pps]
                else:
                    # one table per distinct set of process parameters
                    ax = self.spec.state(src[1])
                    tk_key = ("__proc_table_keys__", name, src[1])
                    keys = memo.get(tk_key)
                    tables: dict = memo.setdefault(("__proc_tables__", name, src[1]), {})
                    if keys is None:
                        keys = []
                        for pp in self._process_params_of(resolvers, src[1], memo):
                            tk = tuple((k, np.asarray(v, dtype=np.float64).tobytes()) for k, v in sorted(pp.items()))
                            if tk not in tables:
                                tables[tk] = (
                                    np.asarray(ax.grid.compute_gridpoints(**pp), dtype=np.float64),
                                    np.asarray(ax.grid.compute_transition_probs(**pp), dtype=np.float64),
                                )
                            keys.append(tk)
                        memo[tk_key] = keys
                    vals = [tables[tk][0 if src[0] == "proc_nodes" else 1] for tk in keys]
                try:
                    col = np.asarray(vals, dtype=np.float64)
                except ValueError:
                    col = None
                want = (n, *np.shape(self.param_values[flat]))
                if col is None or col.shape != want:
                    bad = next(
                        (np.shape(v) for v in vals if np.shape(v) != np.shape(self.param_values[flat])), None
                    )
                    raise InvalidParamsError(
                        f"parameter {flat} has shape {bad}, expected {np.shape(self.param_values[flat])}"
                    )
                col = col.reshape(n, -1)
                memo[key] = col
            width = max(1, col.shape[1])
            if col.shape[1]:
                out[:, off : off + width] = col
        return out

    def _process_params_of(self, resolvers, state: str, memo: dict) -> list:
        """Process parameters of `state` for every resolver (memoised)."""
        key = ("__proc_params__", self.spec.name, state)
        pps = memo.get(key)
        if pps is None:
            ax = self.spec.state(state)
            pps = memo[key] = [r.process_params(self.spec.name, state, ax.grid) for r in resolvers]
        return pps

    def pack_params(self, values: dict | None = None) -> np.ndarray:
        values = self.param_values if values is None else values
        cached = self.__dict__.get("_layout_cache")
        if cached is None:
            cached = self.__dict__["_layout_cache"] = self.param_layout()
        layout, total = cached
        vec = np.zeros(max(total, 1), dtype=np.float64)
        for name, (off, shape) in layout.items():
            v = np.asarray(values[name], dtype=np.float64).ravel()
            vec[off : off + max(1, v.size)] = v if v.size else 0.0
        return vec


def proc_grid_name(state: str) -> str:
    return f"__proc__{state}__nodes"


def proc_P_name(state: str) -> str:
    return f"__proc__{state}__P"


def proc_field_name(state: str, field: str) -> str:
    return f"__proc__{state}__{field}"


class _Tracer:
    def __init__(self, spec: RegimeSpec, resolver: ParamResolver, overrides: dict | None = None) -> None:
        self.spec = spec
        self.resolver = resolver
        self.overrides = dict(overrides or {})
        self.cache: dict[str, Any] = {}
        self.active: list[str] = []
        self.param_values: dict[str, np.ndarray] = {}
        self.param_order: list[str] = []
        self.param_sources: dict[str, tuple] = {}
        self.env: dict[str, Any] = {}
        for ax in spec.states:
            if ax.kind == "continuous":
                self.env[ax.name] = ir.var("state", ax.name, "f")
            elif ax.kind == "process":
                self.env[ax.name] = ir.Expr(
                    "pidx", (proc_grid_name(ax.name), ir.var("state", ax.name, "i")), "f"
                )
            else:
                self.env[ax.name] = ir.var("state", ax.name, "i")
        for ax in spec.actions:
            self.env[ax.name] = ir.var("action", ax.name, "f" if ax.kind == "continuous" else "i")
        self.env["period"] = ir.var("period", "period", "i")
        self.env["age"] = ir.var("age", "age", "f")

    def add_param(self, flat: str, value: Any, source: tuple) -> Any:
        arr = np.asarray(value)
        if arr.dtype == object:
            raise InvalidParamsError(f"parameter {flat} is not numeric")
        if flat not in self.param_values:
            self.param_values[flat] = np.asarray(arr, dtype=np.float64)
            self.param_order.append(flat)
            self.param_sources[flat] = source
        if arr.ndim == 0:
            return ir.param(flat)
        return ir.ParamArray(flat, arr.shape)

    def resolve_arg(self, func: str, arg: str, default: Any) -> Any:
        if arg in self.overrides:
            return self.overrides[arg]
        if arg in self.spec.functions:
            return self.trace(arg)
        if arg in self.env:
            return self.env[arg]
        ok, val = self.resolver.find(self.spec.name, func, arg)
        if ok:
            return self.add_param(f"{func}__{arg}", val, ("arg", func, arg))
        if default is not inspect.Parameter.empty:
            return default
        raise InvalidParamsError(
            f"regime {self.spec.name!r}: argument {arg!r} of {func!r} is neither a "
            "function, state, action, period/age, nor a supplied parameter"
        )

    def call(self, name: str, fn: Callable) -> Any:
        target = fn.func if isinstance(fn, MarkovTransition) else fn
        target = _rebind_numpy_namespace(target)
        sig = inspect.signature(target)
        kwargs = {}
        for p in sig.parameters.values():
            if p.kind in (p.VAR_POSITIONAL, p.VAR_KEYWORD):
                raise TracingError(f"{name}: *args/**kwargs are not supported")
            kwargs[p.name] = self.resolve_arg(name, p.name, p.default)
        try:
            return target(**kwargs)
        except TracingError:
            raise
        except Exception as e:  # noqa: BLE001
            raise TracingError(f"tracing {self.spec.name}.{name} failed: {e!r}") from e

    def trace(self, name: str) -> Any:
        if name in self.cache:
            return self.cache[name]
        if name in self.active:
            raise TracingError(f"cyclic function dependency through {name!r}")
        self.active.append(name)
        out = self.call(name, self.spec.functions[name])
        self.active.pop()
        if isinstance(out, (bool, int, float, np.number, np.bool_)):
            out = ir.const(out)
        self.cache[name] = out
        return out


_NUMPY_LIKE = None


def _rebind_numpy_namespace(fn: Callable) -> Callable:
    """Return `fn` with any global bound to NumPy/JAX's numpy swapped for ours.

    Model code written for the reference refers to ``jnp``; here it may be
    bound to real ``numpy``.  The traced call must see this package's
    ``jnp`` so traced values build IR.
    """
    import types

    from pylcm_b200 import jnp as ours

    g = getattr(fn, "__globals__", None)
    if g is None:
        return fn
    swap = {}
    for k, v in g.items():
        if isinstance(v, types.ModuleType) and v.__name__ in ("numpy", "jax.numpy"):
            swap[k] = ours
    if not swap:
        return fn
    new_g = dict(g)
    new_g.update(swap)
    new = types.FunctionType(fn.__code__, new_g, fn.__name__, fn.__defaults__, fn.__closure__)
    new.__kwdefaults__ = fn.__kwdefaults__
    return new


def _as_bool(e: Any) -> ir.Expr:
    e = ir.const(e) if not isinstance(e, ir.Expr) else e
    if e.dtype != "b":
        return ir._cmp("!=", e, 0)
    return e


def _unreachable(spec: RegimeSpec, tgt: RegimeSpec) -> bool:
    """True when `spec` has no law of motion for one of `tgt`'s states."""
    src = {a.name for a in spec.states}
    for ax in tgt.states:
        if ax.name in src:
            continue
        if ax.kind == "process" or f"next_{ax.name}" not in spec.functions:
            return True
    return False


def _intrinsic_budget(spec: RegimeSpec, t: "_Tracer") -> ir.Expr | None:
    """The budget mask an endogenous-grid regime's grid argmax (simulation)
    needs: continuous action <= resources - lowest savings node
    (``src/_lcm/egm/budget.py:36-100``,
    ``src/_lcm/regime_building/processing.py:1517-1545``)."""
    from pylcm_b200.solvers import DCEGM

    if not isinstance(spec.solver, DCEGM) or spec.terminal:
        return None
    liq = spec.user.liquid
    lb = float(np.asarray(spec.solver.savings_grid.to_numpy(), dtype=np.float64)[0])
    res = t.resolve_arg("utility", liq.resources, inspect.Parameter.empty)
    c = ir.var("action", liq.action, "f")
    return ir._cmp("<=", c, ir.const(res) - lb)


def trace_regime(
    spec: RegimeSpec,
    all_specs: list[RegimeSpec],
    resolver: ParamResolver,
    targets: tuple[str, ...],
) -> TracedRegime:
    """Trace utility, feasibility and the transitions toward `targets`."""
    t = _Tracer(spec, resolver)
    U = t.trace("utility")
    if isinstance(U, ir.VecExpr):
        raise TracingError("utility must be a scalar")
    U = ir.const(U)
    F: ir.Expr = ir.const(True)
    for c in spec.constraint_names:
        F = ir.logical("and", F, _as_bool(t.trace(c)))
    budget = _intrinsic_budget(spec, t)
    if budget is not None:
        F = ir.logical("and", F, budget)
    # process tables (node values, transition matrix) enter the parameter vector
    process_tables = {}
    for ax in spec.states:
        if ax.kind == "process":
            pp = resolver.process_params(spec.name, ax.name, ax.grid)
            nodes = np.asarray(ax.grid.compute_gridpoints(**pp), dtype=np.float64)
            P = np.asarray(ax.grid.compute_transition_probs(**pp), dtype=np.float64)
            process_tables[ax.name] = (nodes, P)
            t.add_param(proc_grid_name(ax.name), nodes, ("proc_nodes", ax.name))
            t.add_param(proc_P_name(ax.name), P, ("proc_P", ax.name))
            # the process's own parameters (used by the simulation's draws)
            for field in sorted(pp):
                t.add_param(proc_field_name(ax.name, field), float(pp[field]), ("proc_field", ax.name, field))
    beta = None
    taste_scale = None
    regime_probs = None
    regime_id = None
    next_states: dict[str, dict[str, NextState]] = {}
    if not spec.terminal:
        ok, bval = resolver.find(spec.name, BETA_FUNC, BETA_ARG)
        if not ok:
            raise InvalidParamsError(f"regime {spec.name!r}: missing discount_factor")
        beta = t.add_param(f"{BETA_FUNC}__{BETA_ARG}", bval, ("arg", BETA_FUNC, BETA_ARG))
        raw = t.trace("next_regime")
        n_reg = len(all_specs)
        if isinstance(spec.user.transition, MarkovTransition):
            if not isinstance(raw, ir.VecExpr) or len(raw) != n_reg:
                raise TracingError(
                    f"regime {spec.name!r}: MarkovTransition must return {n_reg} regime probabilities"
                )
            regime_probs = [ir.const(x).astype("f") if ir.const(x).dtype != "f" else x for x in raw.items]
        else:
            if isinstance(raw, ir.VecExpr):
                raise TracingError(
                    f"regime {spec.name!r}: a vector-valued regime transition must be "
                    "wrapped in MarkovTransition"
                )
            rid = ir.const(raw)
            regime_id = rid if rid.dtype == "i" else rid.astype("i")
            regime_probs = [ir.where(ir._cmp("==", rid, k), 1.0, 0.0) for k in range(n_reg)]
        by_name = {s.name: s for s in all_specs}
        for tname in targets:
            tgt = by_name[tname]
            if _unreachable(spec, tgt):
                # the source has no law for one of the target's states: it
                # cannot move there; a non-zero probability toward it poisons
                # the continuation (NaN)
                next_states[tname] = None
                continue
            laws: dict[str, NextState] = {}
            for ax in tgt.states:
                if ax.kind == "process":
                    src_ax = next((a for a in spec.states if a.name == ax.name), None)
                    if src_ax is None or src_ax.kind != "process" or src_ax.size != ax.size:
                        raise ModelInitializationError(
                            f"{spec.name}->{tname}: process state {ax.name!r} must exist with the "
                            "same node count in the source regime"
                        )
                    laws[ax.name] = NextState("process", None, ax.name)
                    continue
                fname = f"next_{ax.name}"
                if fname in spec.functions:
                    law = spec.functions[fname]
                    val = t.trace(fname)
                    if isinstance(law, MarkovTransition):
                        if ax.kind == "continuous":
                            raise TracingError(f"MarkovTransition on continuous state {ax.name!r}")
                        if not isinstance(val, ir.VecExpr) or len(val) != ax.size:
                            raise TracingError(
                                f"{fname} must return {ax.size} probabilities for {ax.name!r}"
                            )
                        laws[ax.name] = NextState("markov", val)
                    elif ax.kind == "continuous":
                        laws[ax.name] = NextState("cont", ir.const(val).astype("f") if ir.const(val).dtype != "f" else val)
                    else:
                        v = ir.const(val)
                        laws[ax.name] = NextState("det", v.astype("i") if v.dtype != "i" else v)
                elif ax.name in t.env and any(a.name == ax.name for a in spec.states):
                    # a state without an explicit law keeps its value (identity law)
                    laws[ax.name] = NextState(
                        "cont" if ax.kind == "continuous" else "det",
                        ir.var("state", ax.name, "f" if ax.kind == "continuous" else "i"),
                    )
                else:
                    raise ModelInitializationError(
                        f"{spec.name}->{tname}: no law of motion for target state {ax.name!r}"
                    )
            next_states[tname] = laws
    if spec.taste_shocks:
        taste_scale = resolver.taste_scale(spec.name)
    return TracedRegime(
        spec=spec,
        U=U,
        F=F,
        regime_probs=regime_probs,
        regime_id=regime_id,
        next_states=next_states,
        param_values=t.param_values,
        param_order=t.param_order,
        param_sources=t.param_sources,
        beta=beta,
        taste_scale=taste_scale,
        process_tables=process_tables,
    )
