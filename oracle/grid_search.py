"""Oracle: brute-force grid-search backward induction in NumPy float64.

Test infrastructure only (see ``oracle/__init__.py``).  Restates, per period
and regime, the reference's Bellman step:

- ``Q_and_F`` (``src/_lcm/regime_building/Q_and_F.py:138-168``): Q = U + beta*CE,
  F = AND of constraints;
- ``compute_CE`` (``Q_and_F.py:466-681``): CE = sum_r p_r * E_r / mass, mass
  check ``_regime_mass_is_a_distribution`` (``Q_and_F.py:1401-1432``);
- ``_expectation_over_stochastic_nodes`` (``Q_and_F.py:1145-1209``):
  E = sum_j w_j v_j / sum_j w_j, zero-weight non-finite values dropped;
- the V interpolator (``V.py:66-183``) with ``map_coordinates``
  (``ndimage.py:29-109``: lower index clipped to [0, n-2], linear
  extrapolation, zero-weight corners ignore +-inf) and the grid coordinate
  functions (``grids/coordinates.py:30-167``);
- ``max_Q_over_a`` (``max_Q_over_a.py:160``) and the first-index argmax
  (``argmax.py:6-69``); with taste shocks the logsum over discrete actions of
  the max over continuous actions (``max_Q_over_a.py:108-138``,
  ``logsum.py:32-64``).

The expectation is taken node by node exactly as the reference does (one
interpolation per stochastic node), not by contracting first.  The package's
model-spec layer (axis order, parameter lookup) is reused so the oracle sees
the same model; the arithmetic here is independent of the CUDA path.
"""

from __future__ import annotations

import inspect
import itertools
from typing import Any

import numpy as np

from pylcm_b200.regime import MarkovTransition
from pylcm_b200.spec import (
    BETA_ARG,
    BETA_FUNC,
    ParamResolver,
    RegimeSpec,
    _rebind_numpy_namespace,
)


# ----------------------------------------------------------------- helpers
def grid_coordinate(grid, values: np.ndarray) -> np.ndarray:
    """Fractional index of `values` on a continuous grid (``coordinates.py``)."""
    kind = grid.kind
    v = np.asarray(values, dtype=np.float64)
    if kind == "lin":
        n = grid.n_points
        step = (float(grid.stop) - float(grid.start)) / (n - 1 if n > 1 else 1)
        return (v - float(grid.start)) / step if n > 1 else np.zeros_like(v)
    if kind == "log":
        a, b = np.log(float(grid.start)), np.log(float(grid.stop))
        n = grid.n_points
        with np.errstate(all="ignore"):
            lv = np.log(v)
            c = (lv - a) / ((b - a) / (n - 1))
            lo = np.floor(c)
            sl = (b - a) / (n - 1)
            lower = np.exp(a + sl * lo)
            upper = np.exp(a + sl * (lo + 1))
            return lo + (v - lower) / (upper - lower)
    if kind == "piece":
        # ``piecewise.py:107-118, 178-188``: the segment by searchsorted(side="right")
        # over the effective starts of segments 1..k-1, plus its offset
        bnds = [seg.effective_bounds() for seg in grid.segments]
        ns = np.array([int(seg.n_points) for seg in grid.segments])
        offs = np.concatenate([[0], np.cumsum(ns[:-1])])
        seg_i = np.searchsorted(np.array([a for a, _ in bnds[1:]]), v, side="right")
        out = np.empty_like(v)
        for k, ((a, b), n) in enumerate(zip(bnds, ns)):
            m = seg_i == k
            if not m.any():
                continue
            if grid.log:
                a_l, b_l = np.log(a), np.log(b)
                sl = (b_l - a_l) / (n - 1)
                with np.errstate(all="ignore"):
                    c = (np.log(v[m]) - a_l) / sl
                    lo = np.floor(c)
                    lower = np.exp(a_l + sl * lo)
                    upper = np.exp(a_l + sl * (lo + 1))
                    out[m] = offs[k] + lo + (v[m] - lower) / (upper - lower)
            else:
                out[m] = offs[k] + (v[m] - a) / ((b - a) / (n - 1))
        return out
    if kind == "irreg":
        pts = grid.to_numpy()
        n = len(pts)
        if n == 1:
            return np.zeros_like(v)
        up = np.clip(np.searchsorted(pts, v, side="right"), 1, n - 1)
        lo = up - 1
        return lo + (v - pts[lo]) / (pts[up] - pts[lo])
    raise ValueError(kind)


def _irreg_coordinate(pts: np.ndarray, v: np.ndarray) -> np.ndarray:
    n = len(pts)
    up = np.clip(np.searchsorted(pts, v, side="right"), 1, n - 1)
    lo = up - 1
    return lo + (v - pts[lo]) / (pts[up] - pts[lo])


def zero_safe(w: np.ndarray, v: np.ndarray) -> np.ndarray:
    """w * v with w == 0 annihilating +-inf/nan (``zero_safe.py:161-251``)."""
    w = np.asarray(w, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    safe_v = np.where((w == 0.0) & ~np.isfinite(v), 0.0, v)
    with np.errstate(all="ignore"):
        return w * safe_v


def interp_rows(rows: np.ndarray, coords: list[np.ndarray]) -> np.ndarray:
    """Multilinear interpolation of `rows[..., c1, c2, ...]` at coords.

    `rows` has shape (*B, n1, ..., nd) where *B broadcasts against the
    coordinate arrays' shape; returns the values at those coordinates.
    """
    d = len(coords)
    shape = rows.shape[-d:]
    data = []
    for c, n in zip(coords, shape):
        lo = np.clip(np.nan_to_num(np.floor(c), nan=0.0), 0, n - 2).astype(np.int64)  # NaN: any index, NaN weight
        wu = c - lo
        wl = 1 - wu
        data.append(((lo, wl), (lo + 1, wu)))
    out = None
    bshape = np.broadcast_shapes(rows.shape[:-d], *(np.shape(c) for c in coords))
    batch_idx = np.indices(bshape, sparse=True) if rows.shape[:-d] else ()
    for corner in itertools.product(*data):
        idxs = tuple(i for i, _ in corner)
        w = corner[0][1]
        for _, ww in corner[1:]:
            w = w * ww
        if rows.ndim > d:
            nb = rows.ndim - d
            bidx = tuple(
                np.broadcast_to(batch_idx[len(bshape) - nb + k], bshape) for k in range(nb)
            )
            vals = rows[bidx + tuple(np.broadcast_to(i, bshape) for i in idxs)]
        else:
            vals = rows[tuple(np.broadcast_to(i, bshape) for i in idxs)]
        term = zero_safe(w, vals)
        out = term if out is None else out + term
    return out


# ------------------------------------------------------- function evaluation
class _Evaluator:
    """Evaluates a regime's functions on broadcast NumPy arrays (dags rule)."""

    def __init__(self, spec: RegimeSpec, resolver: ParamResolver, env: dict, flat: dict) -> None:
        self.spec = spec
        self.resolver = resolver
        self.env = env
        self.flat = flat  # (func, arg) -> value, for recording what was used
        self.cache: dict[str, Any] = {}

    def arg_value(self, func: str, arg: str, default: Any) -> Any:
        if arg in self.spec.functions:
            return self.value(arg)
        if arg in self.env:
            return self.env[arg]
        ok, val = self.resolver.find(self.spec.name, func, arg)
        if ok:
            return np.asarray(val, dtype=np.float64) if np.ndim(val) else float(np.asarray(val))
        if default is not inspect.Parameter.empty:
            return default
        raise KeyError(f"{self.spec.name}: cannot resolve {arg!r} of {func!r}")

    def call(self, name: str) -> Any:
        fn = self.spec.functions[name]
        target = fn.func if isinstance(fn, MarkovTransition) else fn
        target = _rebind_numpy_namespace(target)
        kwargs = {
            p.name: self.arg_value(name, p.name, p.default)
            for p in inspect.signature(target).parameters.values()
        }
        with np.errstate(all="ignore"):
            return target(**kwargs)

    def value(self, name: str) -> Any:
        if name not in self.cache:
            self.cache[name] = self.call(name)
        return self.cache[name]


def _leaf_deps(spec: RegimeSpec, name: str, seen=None) -> set[str]:
    """Names of states/actions/period/age that function `name` depends on."""
    seen = set() if seen is None else seen
    fn = spec.functions[name]
    target = fn.func if isinstance(fn, MarkovTransition) else fn
    out = set()
    leaves = {a.name for a in spec.states} | {a.name for a in spec.actions} | {"period", "age"}
    for p in inspect.signature(target).parameters:
        if p in spec.functions and p not in seen:
            seen.add(p)
            out |= _leaf_deps(spec, p, seen)
        elif p in leaves:
            out.add(p)
    return out


def _vector_function_table(spec, resolver, name, n_out, period, age):
    """Evaluate a vector-valued function (Markov law / regime transition) per
    combination of its leaf inputs, with scalar inputs (the reference vmaps it)."""
    deps = sorted(_leaf_deps(spec, name))
    axes = {a.name: a for a in spec.states + spec.actions}
    dep_axes = [d for d in deps if d in axes]
    values = []
    for d in dep_axes:
        ax = axes[d]
        values.append(range(ax.size))
    table = {}
    for combo in itertools.product(*values):
        env = {"period": period, "age": age}
        for d, i in zip(dep_axes, combo):
            env[d] = _axis_value(spec, resolver, axes[d], i)
        ev = _Evaluator(spec, resolver, env, {})
        out = np.asarray(ev.value(name), dtype=np.float64).reshape(-1)
        if out.size != n_out:
            raise ValueError(f"{name} returned {out.size} values, expected {n_out}")
        table[combo] = out
    return dep_axes, table


def _process_tables(spec, resolver):
    out = {}
    for ax in spec.states:
        if ax.kind == "process":
            pp = resolver.process_params(spec.name, ax.name, ax.grid)
            out[ax.name] = (
                np.asarray(ax.grid.compute_gridpoints(**pp), dtype=np.float64),
                np.asarray(ax.grid.compute_transition_probs(**pp), dtype=np.float64),
            )
    return out


_PROC_CACHE: dict = {}


def _axis_value(spec, resolver, ax, idx):
    if ax.kind == "process":
        nodes, _ = _process_tables(spec, resolver)[ax.name]
        return nodes[idx]
    if ax.kind == "discrete":
        return int(idx)
    return ax.grid.to_numpy()[idx]


# --------------------------------------------------------------- the solve
def bellman_step(
    spec: RegimeSpec,
    specs: list[RegimeSpec],
    resolver: ParamResolver,
    period: int,
    age: float,
    next_V: dict[str, np.ndarray],
    state_rows: np.ndarray | None = None,
    state_values: dict | None = None,
    return_qf: bool = False,
):
    """V and policy (flat action index) of `spec` at `period`.

    `next_V` maps each regime active next period to its value array.
    `state_rows` optionally restricts the computation to a subset of flat
    state indices (used for bounded CPU timing samples).  `state_values`
    (name -> array) evaluates at arbitrary, off-grid states instead (the
    simulation): a process state's transition weights are then the
    transition-matrix rows interpolated at the value's node coordinate
    (``processing.py:2780-2839``).  With `return_qf` the (Q, F) matrices are
    returned instead of (V, policy).
    """
    sshape = spec.state_shape
    n_s = spec.n_states
    if state_values is not None:
        n_rows = len(next(iter(state_values.values()))) if state_values else 1
        rows = np.arange(n_rows)
    else:
        rows = np.arange(n_s) if state_rows is None else np.asarray(state_rows)
    s_idx = np.unravel_index(rows, sshape) if (spec.states and state_values is None) else ()
    ashape = tuple(a.size for a in spec.actions)
    n_a = spec.n_actions
    a_idx = np.unravel_index(np.arange(n_a), ashape) if spec.actions else ()
    procs = _process_tables(spec, resolver)

    env: dict[str, Any] = {"period": period, "age": age}
    sidx_of: dict[str, np.ndarray] = {}
    blend: dict[str, tuple] = {}
    for k, ax in enumerate(spec.states):
        if state_values is not None:
            x = np.asarray(state_values[ax.name], dtype=np.float64)[:, None]
            if ax.kind == "process":
                nodes = procs[ax.name][0]
                c = _irreg_coordinate(nodes, x)
                lo = np.clip(np.floor(c), 0, len(nodes) - 2).astype(np.int64)
                blend[ax.name] = (lo, c - lo)
                sidx_of[ax.name] = lo
                env[ax.name] = x
            elif ax.kind == "discrete":
                sidx_of[ax.name] = x.astype(np.int64)
                env[ax.name] = x.astype(np.int64)
            else:
                env[ax.name] = x
            continue
        i = s_idx[k][:, None]
        sidx_of[ax.name] = i
        if ax.kind == "process":
            env[ax.name] = procs[ax.name][0][i]
        elif ax.kind == "discrete":
            env[ax.name] = i.astype(np.int64)
        else:
            env[ax.name] = ax.grid.to_numpy()[i]
    aidx_of: dict[str, np.ndarray] = {}
    for k, ax in enumerate(spec.actions):
        i = a_idx[k][None, :]
        aidx_of[ax.name] = i
        env[ax.name] = i.astype(np.int64) if ax.kind == "discrete" else ax.grid.to_numpy()[i]
    bshape = (len(rows), n_a)
    ev = _Evaluator(spec, resolver, env, {})

    U = np.broadcast_to(np.asarray(ev.value("utility"), dtype=np.float64), bshape)
    F = np.ones(bshape, dtype=bool)
    for c in spec.constraint_names:
        F = F & np.broadcast_to(np.asarray(ev.value(c), dtype=bool), bshape)
    if _is_egm(spec) and not spec.terminal:
        # intrinsic budget of an endogenous-grid regime's grid argmax
        # (src/_lcm/egm/budget.py:36-100): c <= resources - lowest savings node
        liq = spec.user.liquid
        lb = float(np.asarray(spec.solver.savings_grid.to_numpy(), dtype=np.float64)[0])
        res = ev.value(liq.resources) if liq.resources in spec.functions else ev.env[liq.resources]
        F = F & np.broadcast_to(np.asarray(env[liq.action]) <= np.asarray(res) - lb, bshape)

    if spec.terminal:
        Q = U
    else:
        ok, beta = resolver.find(spec.name, BETA_FUNC, BETA_ARG)
        beta = float(np.asarray(beta))
        n_reg = len(specs)
        # regime transition probabilities, one (N_s, N_a) array per regime
        if isinstance(spec.user.transition, MarkovTransition):
            deps, table = _vector_function_table(spec, resolver, "next_regime", n_reg, period, age)
            probs = _lookup_table(deps, table, sidx_of, aidx_of, bshape, n_reg)
        else:
            rid = np.broadcast_to(np.asarray(ev.value("next_regime")), bshape)
            probs = [(rid == k).astype(np.float64) for k in range(n_reg)]
        by_name = {s.name: s for s in specs}
        targets = [s for s in specs if s.name in next_V]
        scalar_t = [s for s in targets if not s.states]
        state_t = [s for s in targets if s.states]
        CE = np.zeros(bshape)
        mass = np.zeros(bshape)
        neg = np.zeros(bshape, dtype=bool)
        for tgt in scalar_t + state_t:
            p = probs[tgt.rid]
            mass = mass + p
            neg = neg | (p < 0)
            if not tgt.states:
                E = np.broadcast_to(np.asarray(next_V[tgt.name], dtype=np.float64), bshape)
            elif _unreachable(spec, tgt):
                # no law for one of the target's states: NaN where p != 0
                E = np.full(bshape, np.nan)
            else:
                E = _expected_next_value(
                    spec, tgt, resolver, ev, next_V[tgt.name], procs, sidx_of, aidx_of, bshape, period, age, blend
                )
            CE = CE + zero_safe(p, E)
        valid = (np.abs(mass - 1.0) <= 1e-3) & ~neg
        with np.errstate(all="ignore"):
            CE = CE / np.where(valid, mass, np.nan)
        Q = U + beta * CE

    if return_qf:
        return Q, F
    if spec.taste_shocks:
        scale = resolver.taste_scale(spec.name)
        nd = spec.n_discrete_actions
        nc = spec.n_continuous_actions
        Qm = np.where(F, Q, -np.inf).reshape(len(rows), nd, nc)
        Qc = Qm.max(axis=2)
        vmax = Qc.max(axis=1, keepdims=True)
        fin = np.where(np.isneginf(vmax), 0.0, vmax)
        with np.errstate(all="ignore"):
            sh = (Qc - fin) / scale
            m = sh.max(axis=1, keepdims=True)
            m = np.where(np.isfinite(m), m, 0.0)
            lse = np.log(np.exp(sh - m).sum(axis=1)) + m[:, 0]
        V = fin[:, 0] + scale * lse
        # policy: the hard argmax of the choice-specific values (no noise)
        cont_arg = Qm.argmax(axis=2)
        d_arg = Qc.argmax(axis=1)
        pol = (d_arg * nc + cont_arg[np.arange(len(rows)), d_arg]).astype(np.int32)
    else:
        Qm = np.where(F, Q, -np.inf)
        V = np.max(Qm, axis=1, initial=-np.inf)
        has_nan = np.isnan(np.where(F, Q, 0.0)).any(axis=1)
        V = np.where(has_nan, np.nan, V)
        mask = (Q == V[:, None]) & F
        pol = np.argmax(mask, axis=1).astype(np.int32)
    # gap between the best and the second-best feasible action (inf if < 2)
    Qg = np.where(F, np.nan_to_num(Q, nan=-np.inf), -np.inf)
    if Qg.shape[1] >= 2:
        top2 = np.partition(Qg, Qg.shape[1] - 2, axis=1)[:, -2:]
        with np.errstate(invalid="ignore"):
            gap = np.where(np.isfinite(top2[:, 0]), top2[:, 1] - top2[:, 0], np.inf)
    else:
        gap = np.full(Qg.shape[0], np.inf)
    global LAST_GAP
    LAST_GAP = gap
    if state_rows is None:
        return V.reshape(sshape), pol.reshape(sshape)
    return V, pol


LAST_GAP = None


def _is_egm(spec) -> bool:
    from pylcm_b200.solvers import DCEGM

    return isinstance(spec.solver, DCEGM)


def _unreachable(spec, tgt) -> bool:
    """True when `spec` has no law of motion for one of `tgt`'s states."""
    src = {a.name for a in spec.states}
    for ax in tgt.states:
        if ax.name in src:
            continue
        if ax.kind == "process" or f"next_{ax.name}" not in spec.functions:
            return True
    return False


def _lookup_table(deps, table, sidx_of, aidx_of, bshape, n_out):
    """Broadcast a per-combination vector table to (N_s, N_a) arrays."""
    idx = []
    for d in deps:
        i = sidx_of.get(d)
        if i is None:
            i = aidx_of[d]
        idx.append(np.broadcast_to(i, bshape))
    out = []
    if not deps:
        vec = table[()]
        return [np.full(bshape, vec[k]) for k in range(n_out)]
    keys = list(table)
    arr = np.stack([table[k] for k in keys])  # (n_combo, n_out)
    # map combination -> row
    sizes = [max(k[j] for k in keys) + 1 for j in range(len(deps))]
    lin = np.zeros(bshape, dtype=np.int64)
    kl = np.zeros(len(keys), dtype=np.int64)
    for j, n in enumerate(sizes):
        lin = lin * n + idx[j]
        kl = kl * n + np.array([k[j] for k in keys])
    pos = np.empty(int(np.prod(sizes)), dtype=np.int64)
    pos[kl] = np.arange(len(keys))
    rows = pos[lin]
    for k in range(n_out):
        out.append(arr[rows, k])
    return out


def _expected_next_value(spec, tgt, resolver, ev, V_next, procs, sidx_of, aidx_of, bshape, period, age, blend=None):
    """E[V'_tgt] at every (state, action): node-by-node interpolation."""
    laws = {}
    stoch_axes = []  # (axis position in tgt, list of weight arrays per node)
    det_idx = {}
    cont_vals = {}
    blend = blend or {}
    for pos, ax in enumerate(tgt.states):
        if ax.kind == "process":
            P = procs[ax.name][1]
            if ax.name in blend:
                lo, t = blend[ax.name]
                ws = [np.broadcast_to(zero_safe(1 - t, P[lo, j]) + zero_safe(t, P[lo + 1, j]), bshape) for j in range(ax.size)]
            else:
                cur = sidx_of[ax.name]
                ws = [np.broadcast_to(P[cur, j], bshape) for j in range(ax.size)]
            stoch_axes.append((pos, ws))
            continue
        fname = f"next_{ax.name}"
        if fname in spec.functions:
            law = spec.functions[fname]
            if isinstance(law, MarkovTransition):
                deps, table = _vector_function_table(spec, resolver, fname, ax.size, period, age)
                ws = _lookup_table(deps, table, sidx_of, aidx_of, bshape, ax.size)
                stoch_axes.append((pos, ws))
            elif ax.kind == "continuous":
                cont_vals[pos] = np.broadcast_to(np.asarray(ev.value(fname), dtype=np.float64), bshape)
            else:
                det_idx[pos] = np.broadcast_to(np.asarray(ev.value(fname)).astype(np.int64), bshape)
        else:
            # identity law
            if ax.kind == "continuous":
                cont_vals[pos] = np.broadcast_to(ev.env[ax.name], bshape)
            else:
                det_idx[pos] = np.broadcast_to(sidx_of[ax.name], bshape)
        laws[pos] = ax
    cont_pos = [p for p, ax in enumerate(tgt.states) if ax.kind == "continuous"]
    coords = [grid_coordinate(tgt.states[p].grid, cont_vals[p]) for p in cont_pos]
    shape = tgt.state_shape
    strides = [int(np.prod(shape[k + 1 :])) for k in range(len(shape))]
    flatV = np.asarray(V_next, dtype=np.float64).ravel()
    # per continuous axis: (lower index, lower weight), (upper index, upper weight)
    cdata = []
    for p, c in zip(cont_pos, coords):
        n = shape[p]
        lo = np.clip(np.nan_to_num(np.floor(c), nan=0.0), 0, n - 2).astype(np.int64)  # NaN: any index, NaN weight
        wu = c - lo
        cdata.append(((lo, 1 - wu), (lo + 1, wu)))
    node_ranges = [range(len(ws)) for _, ws in stoch_axes]
    num = np.zeros(bshape)
    den = np.zeros(bshape)
    for combo in itertools.product(*node_ranges):
        w = None
        for (pos, ws), j in zip(stoch_axes, combo):
            w = ws[j] if w is None else w * ws[j]
        if w is None:
            w = np.ones(bshape)
        stoch_map = {pos: j for (pos, _), j in zip(stoch_axes, combo)}
        base = np.zeros(bshape, dtype=np.int64)
        for pos, ax in enumerate(tgt.states):
            if ax.kind == "continuous":
                continue
            i = stoch_map[pos] if pos in stoch_map else det_idx[pos]
            base = base + np.asarray(i, dtype=np.int64) * strides[pos]
        if cont_pos:
            vals = None
            for corner in itertools.product(*cdata):
                cw = corner[0][1]
                for _, ww in corner[1:]:
                    cw = cw * ww
                flat = base
                for (ci, _), p in zip(corner, cont_pos):
                    flat = flat + ci * strides[p]
                term = zero_safe(cw, flatV[flat])
                vals = term if vals is None else vals + term
        else:
            vals = flatV[base]
        den = den + w
        safe = np.where((w == 0) & ~np.isfinite(vals), 0.0, vals)
        with np.errstate(all="ignore"):
            num = num + w * safe
    with np.errstate(all="ignore"):
        return num / np.where(den > 0.0, den, 1.0)


def solve(model, params: dict, gaps: dict | None = None) -> tuple[dict, dict]:
    """Backward induction over all periods; returns (V, policy) dicts
    ``{period: {regime: array}}`` like ``Model.solve``.  If `gaps` is a dict
    it receives, per period and regime, the gap between the best and the
    second-best feasible Q at every state (for argmax comparisons)."""
    specs = model.regime_specs
    resolver = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    T = model.n_periods
    V: dict[int, dict[str, np.ndarray]] = {}
    pol: dict[int, dict[str, np.ndarray]] = {}
    for period in range(T - 1, -1, -1):
        age = float(model.ages.values[period])
        V[period] = {}
        pol[period] = {}
        nxt = V.get(period + 1, {})
        for spec in specs:
            if period not in spec.active_periods:
                continue
            if not spec.terminal and period == T - 1:
                raise ValueError(f"non-terminal regime {spec.name} active in the last period")
            v, p = bellman_step(spec, specs, resolver, period, age, nxt)
            V[period][spec.name] = v
            pol[period][spec.name] = p
            if gaps is not None:
                gaps.setdefault(period, {})[spec.name] = LAST_GAP.reshape(spec.state_shape)
    return V, pol
