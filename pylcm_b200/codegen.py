"""Lower a traced regime to CUDA C for sm_100a.

Two kernels are generated per (regime, set of next-period targets):

``lcm_bellman_<tag>`` -- kernel (a), the fused Q_and_F + max/argmax step.
    One CTA owns a tile of ``BLOCK / LANES`` states; ``LANES`` consecutive
    threads share a state and stride over its actions.  Actions are processed
    in chunks whose action-only sub-expressions (typically the utility) are
    evaluated once per chunk into shared memory; state-only sub-expressions are
    evaluated once per thread; only the mixed part runs in the inner loop.
    Infeasible actions are rejected before the continuation is touched.  The
    running (max, first argmax) is combined across lanes with warp shuffles.

``lcm_expect_<tag>_<target>`` -- kernel (b), the shock expectation
    EV[k, col] = sum_j W[k, j] V'[j, col] / sum_j W[k, j]
    where j runs over the target's stochastic node axes (Markov laws and
    processes), k over the discrete inputs the weights depend on, and col over
    the remaining (deterministic discrete x continuous) axes.  The weight
    table is built in shared memory per tile; each thread owns one column and
    keeps all k accumulators in registers, so V' is read once.

Precision modes: ``fp64`` runs both kernels in double precision.  ``fp32``
runs the inner search of (a) in single precision on a float copy of EV and then
re-evaluates Q at the chosen action in double precision from the double EV, so
the published V is a double-precision Bellman value at the single-precision
argmax.

Reference semantics restated here: ``Q_and_F.py:138-168, 466-681, 1145-1209``,
``max_Q_over_a.py:160``, ``argmax.py:6-69``, ``ndimage.py:29-109``,
``coordinates.py:30-167``.
"""

from __future__ import annotations

import dataclasses
import hashlib
import math
from pathlib import Path

import numpy as np

from pylcm_b200 import ir
from pylcm_b200.exceptions import TracingError
from pylcm_b200.spec import RegimeSpec, TracedRegime, proc_P_name

KERNEL_DIR = Path(__file__).resolve().parent / "csrc" / "kernels"


def device_header() -> str:
    return (KERNEL_DIR / "lcm_device.cuh").read_text()


def tc_header() -> str:
    """The tcgen05 expectation (lcm_tc.cuh), for modules with a tensor-core
    form of kernel (b)."""
    return (KERNEL_DIR / "lcm_tc.cuh").read_text()


# ---------------------------------------------------------------------------
# expression emission
# ---------------------------------------------------------------------------
_CMP = {"<": "<", "<=": "<=", ">": ">", ">=": ">=", "==": "==", "!=": "!="}
_UNARY_C = {
    "log": "log",
    "log1p": "log1p",
    "log2": "log2",
    "log10": "log10",
    "exp": "exp",
    "expm1": "expm1",
    "exp2": "exp2",
    "sqrt": "sqrt",
    "cbrt": "cbrt",
    "sin": "sin",
    "cos": "cos",
    "tan": "tan",
    "tanh": "tanh",
    "sinh": "sinh",
    "cosh": "cosh",
    "arctan": "atan",
    "floor": "floor",
    "ceil": "ceil",
    "round": "rint",
    "trunc": "trunc",
    "erf": "erf",
}


def _c_float(v: float, ftype: str) -> str:
    if math.isnan(v):
        return f"lcm_lim<{ftype}>::nan()"
    if math.isinf(v):
        return f"({'-' if v < 0 else ''}lcm_lim<{ftype}>::inf())"
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r:
        r += ".0"
    return f"(({ftype}){r})"


class Emitter:
    """Emits C statements for IR nodes, memoising node -> C expression."""

    def __init__(self, ftype: str, param_off: dict, provided: dict, prefix: str) -> None:
        self.ftype = ftype
        self.param_off = param_off  # flat name -> (offset, shape)
        self.vals: dict[int, str] = dict(provided)  # id(node) -> C expression
        self.lines: list[str] = []
        self.prefix = prefix
        self.n = 0

    def ctype(self, dt: str) -> str:
        return {"f": self.ftype, "i": "int", "b": "bool"}[dt]

    def emit(self, node: ir.Expr) -> str:
        if id(node) in self.vals:
            return self.vals[id(node)]
        # post-order walk that stops at nodes already bound (provided / emitted)
        stack: list[tuple[ir.Expr, bool]] = [(node, False)]
        while stack:
            n, done = stack.pop()
            if id(n) in self.vals:
                continue
            if done:
                self.vals[id(n)] = self._emit_one(n)
                continue
            stack.append((n, True))
            for a in reversed(n.args):
                if isinstance(a, ir.Expr) and id(a) not in self.vals:
                    stack.append((a, False))
        return self.vals[id(node)]

    def _tmp(self, dt: str, expr: str) -> str:
        name = f"{self.prefix}{self.n}"
        self.n += 1
        self.lines.append(f"{self.ctype(dt)} {name} = {expr};")
        return name

    def _arg(self, a: ir.Expr, want: str | None = None) -> str:
        s = self.vals[id(a)]
        if want == "f" and a.dtype != "f":
            return f"(({self.ftype}){s})"
        return s

    def _emit_one(self, n: ir.Expr) -> str:
        op = n.op
        ft = self.ftype
        if op == "const":
            v = n.args[0]
            if n.dtype == "b":
                return "true" if v else "false"
            if n.dtype == "i":
                return f"({int(v)})"
            return _c_float(v, ft)
        if op == "var":
            raise TracingError(f"internal: unbound variable {n.args}")
        if op == "param":
            off, shape = self.param_off[n.args[0]]
            return self._tmp("f", f"(({ft})PV[{off}])")
        if op == "pidx":
            name = n.args[0]
            off, shape = self.param_off[name]
            idx = [self._arg(a) for a in n.args[1:]]
            if len(idx) != len(shape):
                raise TracingError(f"array parameter {name} needs {len(shape)} indices")
            # JAX clamps out-of-range gathers; clamp likewise (and stay in bounds)
            lin = "0"
            for k, (i, s) in enumerate(zip(idx, shape)):
                ci = f"min(max((int)({i}), 0), {s - 1})"
                lin = ci if k == 0 else f"({lin}) * {s} + {ci}"
            return self._tmp("f", f"(({ft})PV[{off} + {lin}])")
        if op == "bin":
            o, a, b = n.args
            if n.dtype == "f":
                xa, xb = self._arg(a, "f"), self._arg(b, "f")
            else:
                xa, xb = self._arg(a), self._arg(b)
            if o in "+-*":
                return self._tmp(n.dtype, f"{xa} {o} {xb}")
            if o == "/":
                return self._tmp("f", f"{xa} / {xb}")
            if o == "//":
                if n.dtype == "f":
                    return self._tmp("f", f"floor({xa} / {xb})")
                return self._tmp("i", f"lcm_floordiv({xa}, {xb})")
            if o == "%":
                if n.dtype == "f":
                    return self._tmp("f", f"({xa} - floor({xa} / {xb}) * {xb})")
                return self._tmp("i", f"lcm_floormod({xa}, {xb})")
            if o == "pow":
                if b.op == "const" and b.dtype in ("i", "f") and float(b.args[0]) == 2.0:
                    return self._tmp(n.dtype, f"{xa} * {xa}")
                if n.dtype == "i":
                    return self._tmp("i", f"(int)rint(pow((double){xa}, (double){xb}))")
                return self._tmp("f", f"pow({xa}, {xb})")
            if o == "min":
                if n.dtype == "f":
                    return self._tmp("f", f"lcm_min({xa}, {xb})")
                return self._tmp(n.dtype, f"min({xa}, {xb})")
            if o == "max":
                if n.dtype == "f":
                    return self._tmp("f", f"lcm_max({xa}, {xb})")
                return self._tmp(n.dtype, f"max({xa}, {xb})")
            raise TracingError(f"unsupported binary op {o}")
        if op == "un":
            f, a = n.args
            x = self._arg(a, "f" if n.dtype == "f" else None)
            if f == "neg":
                return self._tmp(n.dtype, f"-{x}")
            if f == "abs":
                return self._tmp(n.dtype, f"fabs({x})" if n.dtype == "f" else f"abs({x})")
            if f == "isfinite":
                return self._tmp("b", f"lcm_isfinite(({ft}){x})")
            if f == "isnan":
                return self._tmp("b", f"lcm_isnan(({ft}){x})")
            if f == "isinf":
                return self._tmp("b", f"(!lcm_isfinite(({ft}){x}) && !lcm_isnan(({ft}){x}))")
            if f == "signbit":
                return self._tmp("b", f"signbit(({ft}){x})")
            if f in _UNARY_C:
                return self._tmp("f", f"{_UNARY_C[f]}(({ft}){x})")
            raise TracingError(f"unsupported function {f}")
        if op == "cmp":
            o, a, b = n.args
            if "f" in (a.dtype, b.dtype):
                xa, xb = self._arg(a, "f"), self._arg(b, "f")
            else:
                xa, xb = self._arg(a), self._arg(b)
            return self._tmp("b", f"{xa} {_CMP[o]} {xb}")
        if op == "where":
            c, a, b = n.args
            want = "f" if n.dtype == "f" else None
            return self._tmp(n.dtype, f"{self._arg(c)} ? {self._arg(a, want)} : {self._arg(b, want)}")
        if op == "and":
            return self._tmp("b", f"{self._arg(n.args[0])} && {self._arg(n.args[1])}")
        if op == "or":
            return self._tmp("b", f"{self._arg(n.args[0])} || {self._arg(n.args[1])}")
        if op == "not":
            return self._tmp("b", f"!{self._arg(n.args[0])}")
        if op == "cast":
            t, a = n.args
            x = self._arg(a)
            if t == "f":
                return self._tmp("f", f"(({ft}){x})")
            if t == "i":
                if a.dtype == "f":
                    return self._tmp("i", f"(int)trunc({x})")
                return self._tmp("i", f"(int)({x})")
            return self._tmp("b", f"(({x}) != 0)")
        raise TracingError(f"unsupported IR op {op}")


_EXTRA_DEVICE = r"""
__device__ __forceinline__ int lcm_floordiv(int a, int b) { int q = a / b; return (q * b != a && ((a < 0) != (b < 0))) ? q - 1 : q; }
__device__ __forceinline__ int lcm_floormod(int a, int b) { int m = a % b; return (m != 0 && ((m < 0) != (b < 0))) ? m + b : m; }
// NaN-propagating min/max (jnp.minimum / jnp.maximum semantics)
__device__ __forceinline__ double lcm_min(double a, double b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }
__device__ __forceinline__ double lcm_max(double a, double b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
__device__ __forceinline__ float lcm_min(float a, float b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }
__device__ __forceinline__ float lcm_max(float a, float b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
template <typename E> struct lcm_evsel;
template <> struct lcm_evsel<double> { static __device__ __forceinline__ const double* get(const i64* it, int w64, int w32) { return reinterpret_cast<const double*>(it[w64]); } };
template <> struct lcm_evsel<float> { static __device__ __forceinline__ const float* get(const i64* it, int w64, int w32) { return reinterpret_cast<const float*>(it[w32]); } };
"""


def _phase(node: ir.Expr) -> str:
    d = node.deps()
    has_s = any(k == "state" for k, _ in d)
    has_a = any(k == "action" for k, _ in d)
    if has_s and has_a:
        return "SA"
    if has_s:
        return "S"
    if has_a:
        return "A"
    return "P"


def _boundary(roots: list[ir.Expr]) -> list[ir.Expr]:
    """Non-SA nodes whose values the SA phase consumes (roots included)."""
    out: dict[int, ir.Expr] = {}
    seen: set[int] = set()
    stack = [r for r in roots if isinstance(r, ir.Expr)]
    while stack:
        n = stack.pop()
        if id(n) in seen:
            continue
        seen.add(id(n))
        if n.op == "const":
            continue
        if _phase(n) != "SA":
            out[id(n)] = n
            continue
        for a in n.args:
            if isinstance(a, ir.Expr):
                stack.append(a)
    return list(out.values())


def _affine_split(x, cnames: set) -> tuple | None:
    """Split x = x0 + sum_k coef_k * a_k over the continuous actions a_k named
    in `cnames`, with x0 and every coef_k free of those actions, by walking
    the expression: sums, differences, negation, float casts, products with
    an action-free factor and quotients by an action-free divisor keep the
    form; any other node that reads a continuous action (a power, a
    transcendental, a comparison, a select, floor ...) rejects it.  Returns
    (x0, {name: coef}) or None.  The split is exact in real arithmetic."""
    memo: dict[int, tuple | None] = {}
    zero = ir.const(0.0)

    def acts(e) -> bool:
        return isinstance(e, ir.Expr) and any(k == "action" and nm in cnames for k, nm in e.deps())

    def add(p, q, sign: float):
        (a0, A), (b0, Bc) = p, q
        if sign > 0:
            c0 = b0 if ir.is_const(a0) and a0.args[0] == 0.0 else (a0 if ir.is_const(b0) and b0.args[0] == 0.0 else a0 + b0)
        else:
            c0 = -b0 if ir.is_const(a0) and a0.args[0] == 0.0 else (a0 if ir.is_const(b0) and b0.args[0] == 0.0 else a0 - b0)
        C = dict(A)
        for k, v in Bc.items():
            C[k] = (C[k] + v if sign > 0 else C[k] - v) if k in C else (v if sign > 0 else -v)
        return c0, C

    def mul(v, f, div: bool):
        if ir.is_const(v) and v.args[0] in (1.0, -1.0) and not div:
            return f if v.args[0] == 1.0 else -f
        return v / f if div else v * f

    def scale(p, f, div: bool):
        a0, A = p
        s0 = zero if ir.is_const(a0) and a0.args[0] == 0.0 else mul(a0, f, div)
        return s0, {k: mul(v, f, div) for k, v in A.items()}

    def rec(e):
        if not acts(e):
            return (ir.const(e), {})
        if id(e) in memo:
            return memo[id(e)]
        r = None
        if e.dtype != "f":
            r = None
        elif e.op == "var":
            r = (zero, {e.args[1]: ir.const(1.0)})
        elif e.op == "cast":
            r = rec(e.args[1]) if e.args[1].dtype == "f" else None
        elif e.op == "un" and e.args[0] == "neg":
            p = rec(e.args[1])
            r = None if p is None else add((zero, {}), p, -1.0)
        elif e.op == "bin" and e.args[0] in ("+", "-"):
            p, q = rec(e.args[1]), rec(e.args[2])
            r = None if p is None or q is None else add(p, q, 1.0 if e.args[0] == "+" else -1.0)
        elif e.op == "bin" and e.args[0] == "*":
            a, b = e.args[1], e.args[2]
            if acts(a) and not acts(b):
                p = rec(a)
                r = None if p is None else scale(p, b, False)
            elif acts(b) and not acts(a):
                p = rec(b)
                r = None if p is None else scale(p, a, False)
        elif e.op == "bin" and e.args[0] == "/":
            a, b = e.args[1], e.args[2]
            if not acts(b):
                p = rec(a)
                r = None if p is None else scale(p, b, True)
        memo[id(e)] = r
        return r

    return rec(x)


@dataclasses.dataclass
class TargetPlan:
    spec: RegimeSpec
    scalar: bool
    prob: ir.Expr
    stoch_pos: list[int]  # positions (in target state order) of stochastic axes
    det_pos: list[int]
    cont_pos: list[int]
    key_vars: list[tuple[str, str, int]]  # (kind, name, size) in key order
    laws: dict
    w_ev64: int = -1
    w_ev32: int = -1
    w_sizes: int = -1
    w_coord: int = -1
    w_scalar: int = -1
    w_vraw: int = -1
    w_bst: int = -1
    unreachable: bool = False  # no law for one of the target's states

    @property
    def K(self) -> int:
        return int(np.prod([s for _, _, s in self.key_vars])) if self.key_vars else 1

    @property
    def J(self) -> int:
        return int(np.prod([self.spec.states[p].size for p in self.stoch_pos])) if self.stoch_pos else 1

    @property
    def needs_contraction(self) -> bool:
        return bool(self.stoch_pos)


def _target_plan(tr: TracedRegime, tgt: RegimeSpec) -> TargetPlan:
    spec = tr.spec
    prob = tr.regime_probs[tgt.rid]
    if not tgt.states:
        return TargetPlan(tgt, True, prob, [], [], [], [], {})
    laws = tr.next_states[tgt.name]
    if laws is None:
        return TargetPlan(tgt, True, prob, [], [], [], [], {}, unreachable=True)
    stoch, det, cont = [], [], []
    key_deps: set = set()
    for pos, ax in enumerate(tgt.states):
        law = laws[ax.name]
        if law.kind in ("markov", "process"):
            stoch.append(pos)
            if law.kind == "process":
                key_deps.add(("state", law.source_process))
            else:
                for it in law.expr.items:
                    key_deps |= set(it.deps())
        elif law.kind == "det":
            det.append(pos)
        else:
            cont.append(pos)
    key_vars = []
    for ax in spec.states:
        if ("state", ax.name) in key_deps:
            if ax.kind == "continuous":
                raise TracingError(
                    f"{spec.name}->{tgt.name}: transition weights that depend on the continuous "
                    f"state {ax.name!r} are not supported"
                )
            key_vars.append(("state", ax.name, ax.size))
    for ax in spec.actions:
        if ("action", ax.name) in key_deps:
            if ax.kind == "continuous":
                raise TracingError(
                    f"{spec.name}->{tgt.name}: transition weights that depend on the continuous "
                    f"action {ax.name!r} are not supported"
                )
            key_vars.append(("action", ax.name, ax.size))
    return TargetPlan(tgt, False, prob, stoch, det, cont, key_vars, laws)


@dataclasses.dataclass(frozen=True)
class LaunchConfig:
    block: int = 256
    lanes: int = 1  # threads sharing one state (power of two <= 32)
    chunk: int = 512  # actions per shared-memory table chunk
    sb: int = 1  # states per thread (register blocking)
    min_blocks: int = 0  # __launch_bounds__ min CTAs per SM (0 = compiler's choice)
    prune: bool = True  # single-precision search: exact skipping of action groups where eligible
    # ... also in regimes with several continuous actions (measured slower than
    # the full search on the human-capital model: off unless asked for)
    prune_multi: bool = False
    group: int = 16  # actions per skipped group (raised to `lanes` if smaller)
    # single-precision search: read a target with two continuous axes from
    # per-tile collapsed rows where eligible (see RegimeKernels._collapse_info)
    collapse: bool = True

    @property
    def states_per_tile(self) -> int:
        return self.sb * self.block // self.lanes


class RegimeKernels:
    """Generated source + item-record layout for one regime / target set."""

    def __init__(
        self,
        tr: TracedRegime,
        targets: list[RegimeSpec],
        precision: str,
        cfg: LaunchConfig,
    ) -> None:
        if precision not in ("fp64", "fp32"):
            raise ValueError(precision)
        self.tr = tr
        self.spec = tr.spec
        self.precision = precision
        self.cfg = cfg
        self.param_off, self.param_len = tr.param_layout()
        order = sorted(targets, key=lambda s: (bool(s.states), s.rid))
        self.targets = [_target_plan(tr, t) for t in order] if not self.spec.terminal else []
        self._layout()
        self._affine = self._affine_laws()
        self._groups = self._group_plan()
        tag_src = repr(
            (self.spec.name, [t.spec.name for t in self.targets], precision, dataclasses.astuple(cfg))
        )
        self.tag = self.spec.name.replace("-", "_") + "_" + hashlib.sha1(tag_src.encode()).hexdigest()[:8]

    # -------------------------------------------------------------- layout
    def _layout(self) -> None:
        spec = self.spec
        w = 0

        def take(n: int = 1) -> int:
            nonlocal w
            k = w
            w += n
            return k

        self.W_P = take()
        self.W_V = take()
        self.W_POL = take()
        self.W_PERIOD = take()
        self.W_AGE = take()
        self.W_NSTATES = take()
        self.W_NACT = take()
        self.W_SSIZE = take(len(spec.states))
        self.W_SGRID = take(len(spec.states))
        self.W_ASIZE = take(len(spec.actions))
        self.W_AGRID = take(len(spec.actions))
        self.W_TASTE = take()
        self.W_ATAB = take()  # global action table (kernel a0 output) of this item
        for t in self.targets:
            if t.unreachable:
                continue
            if t.scalar:
                t.w_scalar = take()
            else:
                t.w_ev64 = take()
                t.w_ev32 = take()
                t.w_sizes = take(len(t.spec.states))
                t.w_coord = take(3 * len(t.cont_pos))
                # the target's value array itself (node-by-node reads in the
                # simulation, for process values outside the process grid)
                t.w_vraw = take()
                # block statistics of the float table (group skipping; 0: none)
                t.w_bst = take()
        self.n_words = max(w, 1)

    # -------------------------------------------------------------- source
    def source(self) -> str:
        parts = [device_header(), _EXTRA_DEVICE, self._bellman_source()]
        tc = [t for t in self.targets if self.tc_ok(t)]
        if tc:
            parts.insert(1, tc_header())
        for t in self.targets:
            if not t.scalar and (t.needs_contraction or self.precision == "fp32"):
                parts.append(self._expect_source(t))
        for t in tc:
            parts.append(self._expect_tc_source(t))
        if any(self.group_stats(t) == 2 for t in self.targets):
            parts.append(f'extern "C" __global__ void __launch_bounds__(256) {self.stats_name()}('
                         "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, "
                         "int n_tiles) {\n  lcm_tile_stats2(items, tile_prefix, n_items, n_tiles);\n}")
        return "\n".join(parts)

    def e_words_for(self, t: TargetPlan) -> int:
        return 9 + len(t.spec.states)

    def bellman_name(self) -> str:
        return f"lcm_bellman_{self.tag}"

    def atab_name(self) -> str:
        return f"lcm_atab_{self.tag}"

    def expect_name(self, t: TargetPlan) -> str:
        return f"lcm_expect_{self.tag}_{t.spec.name}"

    # ..................................................................
    def _sim_extrapolated_expectation(self, ti, t, T, E, blend, proc_names, dn, mk) -> list[str]:
        """Simulation, process value outside its grid: the transition row is
        the extrapolation of the two bracketing rows (a weight may be
        negative), and blending the two contracted rows is then not the
        reference's expectation wherever a node's value is infinite.  Redo it
        (and, for a target reached with several process laws, always do it)
        node by node as the reference does (``processing.py:2780-2839``,
        ``Q_and_F.py:1145-1209``): per combination of the target's stochastic
        states, the interpolated value times the product of the node weights
        (a zero weight ignoring a non-finite value), over the sum of the
        weights."""
        spec = self.spec
        tg = t.spec
        # blend None: always (targets reached with several process laws)
        L = ["{"] if blend is None else [f"if (!(PT[{blend}] >= 0.0 && PT[{blend}] <= 1.0)) {{"]
        L.append(f"  {T} num = ({T})0, den = ({T})0;")
        cblk = "1"
        for pos in t.cont_pos:
            cblk = f"{cblk} * C.n{ti}_{pos}"
        # nested loops over the stochastic axes
        depth = 0
        for pos in t.stoch_pos:
            ax = tg.states[pos]
            L.append("  " * (depth + 1) + f"for (int j{pos} = 0; j{pos} < {ax.size}; ++j{pos}) {{")
            depth += 1
        ind = "  " * (depth + 1)
        wexpr = f"({T})1"
        for pos in t.stoch_pos:
            ax = tg.states[pos]
            law = t.laws[ax.name]
            if law.kind == "process":
                off, shape = self.param_off[proc_P_name(law.source_process)]
                pi = proc_names.index(law.source_process)
                L.append(ind + f"const {T} w{pos} = lcm_zs(({T})1 - ({T})PT[{pi}], ({T})PV[{off} + PLO[{pi}] * {shape[1]} + j{pos}])"
                         f" + lcm_zs(({T})PT[{pi}], ({T})PV[{off} + (PLO[{pi}] + 1) * {shape[1]} + j{pos}]);")
            else:
                items = mk[(ti, pos)]
                L.append(ind + f"{T} w{pos} = ({T})0;")
                for q, v in enumerate(items):
                    L.append(ind + f"if (j{pos} == {q}) w{pos} = ({T})({v});")
            wexpr = f"{wexpr} * w{pos}" if wexpr != f"({T})1" else f"w{pos}"
        L.append(ind + f"const {T} w = {wexpr};")
        # flat index of the node row (non-continuous axes in declaration order)
        flat = "(i64)0"
        for pos, ax in enumerate(tg.states):
            if ax.kind == "continuous":
                continue
            if pos in t.stoch_pos:
                flat = f"({flat}) * {ax.size} + j{pos}"
            else:
                sz = f"C.n{ti}_{pos}"
                flat = f"({flat}) * {sz} + min(max((int)({dn[(ti, pos)]}), 0), {sz} - 1)"
        L.append(ind + f"const double* vrow = C.vr{ti} + ({flat}) * ({cblk});")
        if len(t.cont_pos) == 0:
            L.append(ind + f"const {T} v = ({T})vrow[0];")
        elif len(t.cont_pos) == 1:
            L.append(ind + f"const {T} v = lcm_interp1<{T}, double>(vrow, C.n{ti}_{t.cont_pos[0]}, c0);")
        else:
            L.append(ind + f"const {T} v = lcm_interp2<{T}, double>(vrow, C.n{ti}_{t.cont_pos[0]}, "
                           f"C.n{ti}_{t.cont_pos[1]}, c0, c1);")
        L.append(ind + "den = den + w;")
        L.append(ind + "num = num + ((w == 0 && !lcm_isfinite(v)) ? w * 0 : w * v);")
        for _ in t.stoch_pos:
            depth -= 1
            L.append("  " * (depth + 1) + "}")
        L.append(f"  ev = num / (den > 0 ? den : ({T})1);")
        L.append("}")
        return L

    def _affine_laws(self) -> dict:
        """Continuous next-state laws that are affine in the one continuous
        action they read: {(target, state position): (law at action 0,
        d law / d action, action var)}.  The single-precision search then
        computes the grid coordinate as K + M * action with K and M fixed per
        (state, discrete action) -- one fused multiply-add per action.  Its
        candidates are re-evaluated in double precision, so the search's
        rounding does not reach the published values beyond that search's
        tolerance; the double-precision form keeps the law as written."""
        out: dict = {}
        if self.precision != "fp32":
            return out
        dnames = {a.name for a in self.spec.actions if a.kind != "continuous"}
        for ti, t in enumerate(self.targets):
            if t.scalar:
                continue
            for pos in t.cont_pos:
                if t.spec.states[pos].grid.kind != "lin":
                    continue  # the coordinate is affine in the law only on a linear grid
                x = ir.const(t.laws[t.spec.states[pos].name].expr)
                if not isinstance(x, ir.Expr):
                    continue
                acts = {nm for k, nm in x.deps() if k == "action" and nm not in dnames}
                if len(acts) != 1:
                    continue
                cv = ir.var("action", next(iter(acts)), "f")
                if _affine_split(x, {cv.args[1]}) is None:
                    continue  # a non-affine piece (floor, select ...) that the derivative would miss
                g = ir.const(ir.diff(x, cv))
                if not isinstance(g, ir.Expr) or any(n is cv for n in ir.topo_order([g])):
                    continue
                x0 = ir.substitute(x, cv, 0.0)
                out[(ti, pos)] = (x0, g, cv)
        return out

    COLLAPSE_MAX_OUTER = 8  # largest action grid read in the collapsed rows

    def _collapse_info(self, ti: int, t) -> dict | None:
        """Collapsed rows for target `t` in the single-precision search.

        Eligible when `t` has two continuous axes and no deterministic
        discrete ones, its expectation row is keyed by discrete states only,
        and one axis (B) has an affine coordinate in one continuous action
        `ob` of at most COLLAPSE_MAX_OUTER points whose state part does not
        read the *line state* -- the current regime's continuous state named
        like the other axis (A).  The kernel then walks the states with the
        line state fastest, so that a tile covers at most two lines (all
        other states fixed); per tile it interpolates axis B once per (line,
        value of `ob`) into rows over axis A in shared memory, and each
        (state, action) pair reads its row with a 1-D interpolation instead
        of the bilinear read.  The candidates are re-evaluated in double
        precision as everywhere in this search."""
        spec = self.spec
        if self.precision != "fp32" or not self.cfg.collapse or self._groups or spec.terminal:
            return None
        if t.scalar or t.unreachable or len(t.cont_pos) != 2 or t.det_pos:
            return None
        if any(kind != "state" for kind, _, _ in t.key_vars):
            return None
        cont_states = [a.name for a in spec.states if a.kind == "continuous"]
        names = [a.name for a in spec.actions]
        for cb, posB in enumerate(t.cont_pos):
            if (ti, posB) not in self._affine:
                continue
            ca, posA = 1 - cb, t.cont_pos[1 - cb]
            line = t.spec.states[posA].name
            if line not in cont_states:
                continue
            x0, g, cv = self._affine[(ti, posB)]
            ob = cv.args[1]
            kob = names.index(ob)
            if spec.actions[kob].size > self.COLLAPSE_MAX_OUTER:
                continue
            if any(a.kind != "continuous" for a in spec.actions[kob:]):
                continue
            deps: set = set()
            for e in (x0, g):
                if isinstance(e, ir.Expr):
                    deps |= set(e.deps())
            if any(k not in ("state", "param", "period", "age") for k, _ in deps) or ("state", line) in deps:
                continue
            namax = (t.spec.states[posA].size + 31) // 32 * 32
            return {"ti": ti, "ca": ca, "cb": cb, "posA": posA, "posB": posB, "line": line,
                    "kline": [a.name for a in spec.states].index(line), "ob": ob, "kob": kob,
                    "nob": spec.actions[kob].size, "x0": x0, "g": g, "namax": namax}
        return None

    def _budget_bound(self):
        """(action position, bound node, strict) of a constraint a <= b (or
        b >= a, or strict) in F, where `a` is the slowest continuous action --
        every action before it discrete, so that its index is the slowest
        part of the continuous-action index and, its grid being ascending, the
        feasible actions of a state form a prefix of the table -- and `b` reads
        no action.  None if F has no such constraint."""
        spec = self.spec
        names = [a.name for a in spec.actions]
        kc = next((k for k, a in enumerate(spec.actions) if a.kind == "continuous"), None)
        if kc is None:
            return None
        cname = names[kc]
        F = ir.const(self.tr.F)
        stack = [F] if isinstance(F, ir.Expr) else []
        while stack:
            n = stack.pop()
            if n.op == "and":
                stack.extend(a for a in n.args if isinstance(a, ir.Expr))
                continue
            if n.op != "cmp" or n.args[0] not in ("<", "<=", ">", ">="):
                continue
            lhs, rhs = n.args[1], n.args[2]
            if n.args[0] in (">", ">="):
                lhs, rhs = rhs, lhs
            if not (isinstance(lhs, ir.Expr) and lhs.op == "var" and tuple(lhs.args[:2]) == ("action", cname)):
                continue
            if isinstance(rhs, ir.Expr) and any(k == "action" for k, _ in rhs.deps()):
                continue
            return kc, rhs
        return None

    # group skipping: tiles of the block statistics of a target with two
    # continuous axes (axis 1 x axis 2); one continuous axis uses 16-column blocks
    GROUP_TILE = (16, 2)
    GROUP_MAX_CHUNK = 2048  # the whole continuous-action table in shared memory

    def _group_plan(self) -> dict | None:
        """Eligibility and the affine pieces of the exact skipping of action
        groups in the single-precision search (kernel (a)).

        A group is a run of consecutive values of one continuous action (the
        scan action, the largest) with the other continuous actions fixed.
        Its Q values are bounded above by its largest utility plus beta times
        the largest expectation-table value among the nodes its next-state
        coordinates can reach.  That needs: the utility and the continuous
        actions in the action table (utility free of the state), a
        state-free non-negative discount factor, and per reached target with
        one or two continuous axes (linear grids, no deterministic discrete
        axis) coordinates x = x0 + sum_k coef_k a_k with x0 and coef_k free of
        the continuous actions, so that interval arithmetic over the group's
        action ranges bounds them.  Constraints of the same affine form
        (lhs - rhs) give a second test: a group all of whose members violate
        one is skipped.  Returns None when nothing qualifies."""
        spec, tr = self.spec, self.tr
        if (self.precision != "fp32" or not self.cfg.prune or spec.terminal or spec.taste_shocks
                or tr.regime_id is None or tr.beta is None):
            return None
        cacts = [a for a in spec.actions if a.kind == "continuous"]
        if not cacts or (len(cacts) > 1 and not self.cfg.prune_multi):
            return None
        cn = {a.name for a in cacts}
        U, beta = ir.const(tr.U), ir.const(tr.beta)
        if not isinstance(U, ir.Expr) or any(k == "state" for k, _ in U.deps()):
            return None
        if not any(k == "action" and nm in cn for k, nm in U.deps()):
            return None
        if isinstance(beta, ir.Expr) and any(k in ("state", "action") for k, _ in beta.deps()):
            return None
        axes: dict[int, list] = {}
        for ti, t in enumerate(self.targets):
            if t.scalar or t.unreachable or t.det_pos or not 1 <= len(t.cont_pos) <= 2:
                continue
            parts = []
            for ci, pos in enumerate(t.cont_pos):
                ax = t.spec.states[pos]
                if ax.grid.kind != "lin":
                    break
                sp = _affine_split(ir.const(t.laws[ax.name].expr), cn)
                if sp is None:
                    break
                parts.append((pos, ci, sp[0], sp[1]))
            else:
                axes[ti] = parts
        if not axes:
            return None
        cons = []
        F = ir.const(tr.F)
        stack = [F] if isinstance(F, ir.Expr) else []
        while stack:
            n = stack.pop()
            if n.op == "and":
                stack.extend(a for a in n.args if isinstance(a, ir.Expr))
                continue
            if n.op != "cmp" or n.args[0] not in ("<", "<=", ">", ">="):
                continue
            lhs, rhs = ir.const(n.args[1]), ir.const(n.args[2])
            if lhs.dtype != "f" and rhs.dtype != "f":
                continue
            sp = _affine_split(lhs - rhs, cn)
            if sp is not None and sp[1]:
                cons.append((n.args[0], sp[0], sp[1]))
        used = set()
        for parts in axes.values():
            for _, _, _, co in parts:
                used |= set(co)
        for _, _, co in cons:
            used |= set(co)
        sizes = [a.size for a in cacts]
        scan = int(np.argmax(sizes))
        return {"axes": axes, "cons": cons, "acts": [a.name for a in cacts if a.name in used],
                "scan": scan, "cacts": [a.name for a in cacts]}

    def _group_roots(self) -> list:
        g = self._groups
        if not g:
            return []
        out = [ir.var("action", nm, "f") for nm in g["acts"]]
        for parts in g["axes"].values():
            for _, _, x0, co in parts:
                out.append(x0)
                out += list(co.values())
        for _, y0, co in g["cons"]:
            out.append(y0)
            out += list(co.values())
        return out

    def group_stats(self, t: TargetPlan) -> int:
        """Block statistics the search's group skipping reads for target `t`:
        0 none, 1 per 16 columns (written by kernel (b)), 2 per GROUP_TILE
        tile of the two continuous axes (written by the statistics kernel)."""
        g = self._groups
        if not g:
            return 0
        ti = next((i for i, x in enumerate(self.targets) if x is t), None)
        if ti is None or ti not in g["axes"]:
            return 0
        return len(g["axes"][ti])

    def stats_name(self) -> str:
        return f"lcm_tile_stats_{self.tag}"

    def inner_flops(self) -> dict:
        """Floating-point operations of one (state, action) evaluation of
        kernel (a)'s inner loop, counted from the traced IR: every
        floating-point node that depends on a continuous action and on the
        state (the part not hoisted to the per-tile, per-state or per-action
        phases) -- arithmetic, comparisons and selects count one, a
        transcendental one (its special-function unit work is not expanded) --
        plus, per target reached with a continuous state, the grid coordinate
        (2 per continuous axis), the multilinear read (2^d - 1 lerps of 2
        flops, 3 for d = 2 with the two interpolation weights), and the Bellman
        combination Q = U + beta CE and the running maximum (3)."""
        spec = self.spec
        dn = {a.name for a in spec.actions if a.kind != "continuous"}
        seen: set[int] = set()
        n_arith = n_trans = 0
        stack = [r for r in self._roots() if isinstance(r, ir.Expr)]
        while stack:
            n = stack.pop()
            if id(n) in seen or n.op in ("const", "var", "param"):
                continue
            seen.add(id(n))
            d = n.deps()
            if not (any(k == "state" for k, _ in d) and any(k == "action" and nm not in dn for k, nm in d)):
                continue
            if n.dtype == "f" or n.op == "cmp":
                if n.op == "un":
                    n_trans += 1
                else:
                    n_arith += 1
            stack.extend(a for a in n.args if isinstance(a, ir.Expr))
        per_target = []
        for t in self.targets:
            if t.scalar or t.unreachable or not t.cont_pos:
                continue
            dim = len(t.cont_pos)
            per_target.append(2 * dim + (2 * (2 ** dim - 1) if dim == 1 else 2 * (2 ** dim - 1) + 2))
        # a deterministic regime transition reads one target per evaluation
        interp = (max(per_target) if self.tr.regime_id is not None else sum(per_target)) if per_target else 0
        total = n_arith + n_trans + interp + 3
        return {"ir_arith": n_arith, "ir_transcendental": n_trans, "interpolation": interp, "total": total}

    def _roots(self):
        """Root IR nodes the per-(state, action) code needs."""
        tr = self.tr
        roots = [tr.F, tr.U]
        for x0, g, cv in getattr(self, "_affine", {}).values():
            roots += [x0, g, cv]
        roots += self._group_roots() if getattr(self, "_groups", None) else []
        if tr.beta is not None:
            roots.append(tr.beta)
        if tr.regime_id is not None and self.targets:
            roots.append(tr.regime_id)
        for t in self.targets:
            if tr.regime_id is None:
                roots.append(t.prob)
            if t.scalar:
                continue
            for pos in t.det_pos:
                roots.append(t.laws[t.spec.states[pos].name].expr)
            for pos in t.cont_pos:
                roots.append(t.laws[t.spec.states[pos].name].expr)
        return [ir.const(r) for r in roots]

    def _bellman_source(self) -> str:
        """Kernel (a0) (action table) and kernel (a) (Bellman step) for this regime.

        Loop structure of kernel (a), per tile of states:

            P  : params / period / age only          -> once per tile
            S  : state only                         -> once per state slot
            for each discrete-action combination d (outer, unrolled):
                D  : discrete actions only           -> once per d
                SD : state x discrete actions        -> once per (slot, d)
                for each chunk of continuous actions (shared-memory table):
                    SA : everything else              -> the inner loop
            A  : continuous-action only              -> precomputed by (a0)

        With a deterministic regime transition whose next regime is known per
        d, the inner loop is specialised to that one target.
        """
        spec = self.spec
        cfg = self.cfg
        fp32 = self.precision == "fp32"
        ST = "float" if fp32 else "double"
        TT = ST
        taste = spec.taste_shocks
        dacts = [a for a in spec.actions if a.kind != "continuous"]
        cacts = [a for a in spec.actions if a.kind == "continuous"]
        dnames = {a.name for a in dacts}
        ND = spec.n_discrete_actions

        def phase(n: ir.Expr) -> str:
            d = n.deps()
            has_s = any(k == "state" for k, _ in d)
            has_ac = any(k == "action" and nm not in dnames for k, nm in d)
            has_ad = any(k == "action" and nm in dnames for k, nm in d)
            if has_ac:
                return "SA" if has_s else "A"
            if has_s:
                return "SD" if has_ad else "S"
            return "D" if has_ad else "P"

        roots = self._roots()
        det = self.tr.regime_id is not None and bool(self.targets)
        rid_phase = phase(self.tr.regime_id) if det else None
        unswitch = det and rid_phase in ("P", "D")
        # boundary nodes the inner loop consumes, by phase
        bnd: dict[str, list] = {k: [] for k in ("P", "D", "S", "SD", "A")}
        seen: set[int] = set()
        stack = [r for r in roots if isinstance(r, ir.Expr)]
        while stack:
            n = stack.pop()
            if id(n) in seen or n.op == "const":
                continue
            seen.add(id(n))
            ph = phase(n)
            if ph != "SA":
                bnd[ph].append(n)
                continue
            stack.extend(a for a in n.args if isinstance(a, ir.Expr))
        bP, bD, bS, bSD, bA = bnd["P"], bnd["D"], bnd["S"], bnd["SD"], bnd["A"]
        if unswitch and id(self.tr.regime_id) not in {id(x) for x in bP + bD}:
            (bP if rid_phase == "P" else bD).append(self.tr.regime_id)
        # action-table columns: float fields / int fields
        slot: list[tuple[str, int]] = []
        nf = ni = 0
        for n in bA:
            if n.dtype == "f":
                slot.append(("F", nf))
                nf += 1
            else:
                slot.append(("I", ni))
                ni += 1
        NF, NI = max(nf, 1), max(ni, 1)
        B, LANES, CH, SB = cfg.block, cfg.lanes, cfg.chunk, cfg.sb
        if self._groups:
            CH = max(CH, self.GROUP_MAX_CHUNK)  # group skipping holds the whole table
        SPT = cfg.states_per_tile
        SPB = B // LANES
        dstates = [a for a in spec.states if a.kind != "continuous"]
        NDS = max(len(dstates), 1)
        nP, nD, nS, nSD = (max(len(x), 1) for x in (bP, bD, bS, bSD))
        pv = lambda: {id(ir.var("period", "period", "i")): "period", id(ir.var("age", "age", "f")): "age"}  # noqa: E731
        # targets the single-precision search reads from collapsed rows (one
        # line state for the whole kernel)
        cinfo: dict = {}
        if unswitch and fp32 and not taste:
            for ti_, t_ in enumerate(self.targets):
                c_ = self._collapse_info(ti_, t_)
                if c_ is not None and (not cinfo or c_["kline"] == next(iter(cinfo.values()))["kline"]):
                    cinfo[ti_] = c_
        rows_off = NF * CH * 4 + NI * CH * 4  # the collapsed rows follow the action table
        rows_bytes = max((2 * c["nob"] * c["namax"] * 4 for c in cinfo.values()), default=0)

        L: list[str] = []
        ap = L.append
        ap(f"// ---- regime {spec.name}: Bellman step (kernel a), precision {self.precision}")

        # ----------------------------------------------------------------
        # per-target loop invariants of the Q evaluation
        ap(f"template <typename T, typename E> struct Ctx_{self.tag} {{")
        loads = []
        for ti, t in enumerate(self.targets):
            if t.unreachable:
                continue
            if t.scalar:
                ap(f"  T sv{ti};")
                loads.append(f"sv{ti} = (T)(*lcm_wp<const double>(it, {t.w_scalar}));")
                continue
            ap(f"  const E* ev{ti};")
            loads.append(f"ev{ti} = lcm_evsel<E>::get(it, {t.w_ev64}, {t.w_ev32});")
            ap(f"  const double* vr{ti};")
            loads.append(f"vr{ti} = lcm_wp<const double>(it, {t.w_vraw});")
            ap(f"  const float2* bst{ti};")
            loads.append(f"bst{ti} = lcm_wp<const float2>(it, {t.w_bst});")
            for pos in t.det_pos + t.cont_pos:
                ap(f"  int n{ti}_{pos};")
                loads.append(f"n{ti}_{pos} = lcm_wi(it, {t.w_sizes + pos});")
            for ci, pos in enumerate(t.cont_pos):
                w0 = t.w_coord + 3 * ci
                if t.spec.states[pos].grid.kind == "irreg":
                    ap(f"  const double* p{ti}_{ci};")
                    loads.append(f"p{ti}_{ci} = lcm_wp<const double>(it, {w0 + 2});")
                elif t.spec.states[pos].grid.kind == "piece":
                    ap(f"  const double* p{ti}_{ci}; int k{ti}_{ci}, g{ti}_{ci};")
                    loads.append(f"p{ti}_{ci} = lcm_wp<const double>(it, {w0 + 2}); "
                                 f"k{ti}_{ci} = lcm_wi(it, {w0 + 1}); g{ti}_{ci} = lcm_wi(it, {w0});")
                else:
                    ap(f"  T a{ti}_{ci}, b{ti}_{ci};")
                    loads.append(f"a{ti}_{ci} = (T)lcm_wd(it, {w0}); b{ti}_{ci} = (T)lcm_wd(it, {w0 + 1});")
        ap("  __device__ __forceinline__ void load(const i64* __restrict__ it) {")
        for l_ in loads:
            ap("    " + l_)
        ap("  }")
        ap("};")

        # ----------------------------------------------------------------
        # accessors of the continuous-action table
        ap(
            f"template <typename T> struct AFTab_{self.tag} {{ const {TT}* tabf; const int* tabi; int j;\n"
            f"  __device__ __forceinline__ T F(int f) const {{ return (T)tabf[f * {CH} + j]; }}\n"
            f"  __device__ __forceinline__ int I(int f) const {{ return tabi[f * {CH} + j]; }} }};"
        )
        if cinfo:
            ap(
                f"template <typename T> struct AFCol_{self.tag} {{ const {TT}* tabf; const int* tabi; int j; "
                f"const float* R;\n"
                f"  __device__ __forceinline__ T F(int f) const {{ return (T)tabf[f * {CH} + j]; }}\n"
                f"  __device__ __forceinline__ int I(int f) const {{ return tabi[f * {CH} + j]; }} }};"
            )
        ap(
            f"struct AFLoc_{self.tag} {{ double v[{NF}]; int vi[{NI}];\n"
            f"  __device__ __forceinline__ double F(int f) const {{ return v[f]; }}\n"
            f"  __device__ __forceinline__ int I(int f) const {{ return vi[f]; }} }};"
        )

        # ----------------------------------------------------------------
        # the inner (state, action) evaluation, templated on precision and on
        # the selected target (TSEL < 0: all targets by probability / id)
        proc_names = [a.name for a in spec.states if a.kind == "process"]

        def sa_body(T: str, E: str, tsel: int, sim: bool = False, coll: dict | None = None) -> list[str]:
            prov = pv()
            for i, n in enumerate(bP):
                prov[id(n)] = _cast(f"PVd[{i}]", n.dtype, T)
            for i, n in enumerate(bD):
                prov[id(n)] = _cast(f"DV[{i}]", n.dtype, T)
            for i, n in enumerate(bS):
                prov[id(n)] = _cast(f"SV[{i}]", n.dtype, T)
            for i, n in enumerate(bSD):
                prov[id(n)] = _cast(f"SDV[{i}]", n.dtype, T)
            for i, n in enumerate(bA):
                col, k = slot[i]
                if col == "F":
                    prov[id(n)] = f"(({T})AF.F({k}))"
                elif n.dtype == "b":
                    prov[id(n)] = f"(AF.I({k}) != 0)"
                else:
                    prov[id(n)] = f"AF.I({k})"
            for i, a in enumerate(dstates):
                prov[id(ir.var("state", a.name, "i"))] = f"SI[{i}]"
            for a in dacts:
                prov[id(ir.var("action", a.name, "i"))] = f"DI_{a.name}"
            e = Emitter(T, self.param_off, prov, "q")
            out: list[str] = []
            fexpr = e.emit(self.tr.F)
            out += e.lines
            e.lines = []
            out.append(f"if (!({fexpr})) return false;")
            uexpr = e.emit(self.tr.U)
            out += e.lines
            e.lines = []
            if spec.terminal:
                out.append(f"Q = ({T})({uexpr});")
                return out
            bexpr = e.emit(self.tr.beta)
            out += e.lines
            e.lines = []
            sel = [(ti, t) for ti, t in enumerate(self.targets) if tsel < 0 or ti == tsel]
            pnames, dn, xn, affine_names = {}, {}, {}, {}
            rid_name = e.emit(self.tr.regime_id) if (det and tsel < 0) else None
            mk = {}
            for ti, t in sel:
                if not det:
                    pnames[ti] = e.emit(t.prob)
                if t.scalar:
                    continue
                for pos in t.det_pos:
                    dn[(ti, pos)] = e.emit(t.laws[t.spec.states[pos].name].expr)
                if sim and any(kind == "state" and name in proc_names for kind, name, _ in t.key_vars):
                    for pos in t.stoch_pos:
                        law = t.laws[t.spec.states[pos].name]
                        if law.kind == "markov":
                            mk[(ti, pos)] = [e.emit(x) for x in law.expr.items]
                for pos in t.cont_pos:
                    if not sim and (ti, pos) in self._affine:
                        x0, g, cv = self._affine[(ti, pos)]
                        affine_names[(ti, pos)] = (e.emit(x0), e.emit(g), e.emit(cv))
                        xn[(ti, pos)] = None
                    else:
                        xn[(ti, pos)] = e.emit(t.laws[t.spec.states[pos].name].expr)
            out += e.lines
            e.lines = []
            if det:
                out.append(f"{T} ce = lcm_lim<{T}>::nan();")
            else:
                out.append(f"{T} ce = ({T})0; {T} mass = ({T})0; bool neg = false;")
            for ti, t in sel:
                if det and tsel >= 0:
                    out.append("{ {")
                elif det:
                    out.append(f"{{ if (({rid_name}) == {t.spec.rid}) {{")
                else:
                    out.append(f"{{ {T} p = ({T})({pnames[ti]}); mass += p; neg = neg || (p < ({T})0);")
                    out.append("  if (p != 0) {")
                if t.unreachable:
                    out.append(f"    {T} ev = lcm_lim<{T}>::nan();")
                elif t.scalar:
                    out.append(f"    {T} ev = C.sv{ti};")
                else:
                    inner: list[str] = []
                    key = "0"
                    key_hi = None
                    # two or more process laws: the simulation takes the
                    # node-by-node expectation (each process row interpolated
                    # at its own value), not a blend of contracted rows
                    multi = sim and sum(1 for kd, nm, _ in t.key_vars if kd == "state" and nm in proc_names) > 1
                    for kind, name, size in t.key_vars:
                        if sim and kind == "state" and name in proc_names:
                            if multi:
                                continue
                            pi = proc_names.index(name)
                            key_hi = f"({key}) * {size} + PLO[{pi}] + 1"
                            key = f"({key}) * {size} + PLO[{pi}]"
                            blend = pi
                            continue
                        iv = f"SI[{[a.name for a in dstates].index(name)}]" if kind == "state" else f"DI_{name}"
                        key = f"({key}) * {size} + {iv}"
                        if key_hi is not None:
                            key_hi = f"({key_hi}) * {size} + {iv}"
                    off = key
                    off_hi = key_hi
                    for pos in t.det_pos:
                        sz = f"C.n{ti}_{pos}"
                        off = f"({off}) * {sz} + min(max((int)({dn[(ti, pos)]}), 0), {sz} - 1)"
                        if off_hi is not None:
                            off_hi = f"({off_hi}) * {sz} + min(max((int)({dn[(ti, pos)]}), 0), {sz} - 1)"
                    cblk = "1"
                    for pos in t.cont_pos:
                        cblk = f"{cblk} * C.n{ti}_{pos}"
                    for ci, pos in enumerate(t.cont_pos):
                        if coll is not None and ti == coll["ti"] and ci == coll["cb"]:
                            continue  # axis B comes interpolated in the collapsed row AF.R
                        ax = t.spec.states[pos]
                        x = xn[(ti, pos)]
                        kind = ax.grid.kind
                        if kind == "lin" and not sim and (ti, pos) in affine_names:
                            # (x0 + g c - a) b as K + M c: K, M are loop-invariant
                            x0n, gn, cvn = affine_names[(ti, pos)]
                            cc = (f"((({T})({x0n}) - C.a{ti}_{ci}) * C.b{ti}_{ci} + "
                                  f"(({T})({gn}) * C.b{ti}_{ci}) * ({T})({cvn}))")
                        elif kind == "lin":
                            cc = f"lcm_coord_lin<{T}>(({T})({x}), C.a{ti}_{ci}, C.b{ti}_{ci})"
                        elif kind == "log":
                            cc = f"lcm_coord_log<{T}>(({T})({x}), C.a{ti}_{ci}, C.b{ti}_{ci})"
                        elif kind == "piece":
                            cc = f"lcm_coord_piece<{T}>(({T})({x}), C.p{ti}_{ci}, C.k{ti}_{ci}, C.g{ti}_{ci})"
                        else:
                            cc = f"lcm_coord_irreg<{T}>(({T})({x}), C.p{ti}_{ci}, C.n{ti}_{pos})"
                        inner.append(f"{T} c{ci} = {cc};")
                    rows = [] if multi else [("row", off)] + ([("rowh", off_hi)] if off_hi is not None else [])
                    if coll is not None and ti == coll["ti"]:
                        rows = []
                        inner.append(f"{T} ev = lcm_interp1s<{T}>(AF.R, C.n{ti}_{coll['posA']}, c{coll['ca']});")
                    if multi:
                        inner.append(f"{T} ev = ({T})0;")
                        inner += self._sim_extrapolated_expectation(ti, t, T, E, None, proc_names, dn, mk)
                    for rname, roff in rows:
                        ev_name = "ev" if rname == "row" else "evh"
                        inner.append(f"const {E}* {rname} = C.ev{ti} + (i64)({roff}) * ({cblk});")
                        if len(t.cont_pos) == 0:
                            inner.append(f"{T} {ev_name} = ({T}){rname}[0];")
                        elif len(t.cont_pos) == 1:
                            inner.append(f"{T} {ev_name} = lcm_interp1<{T}, {E}>({rname}, C.n{ti}_{t.cont_pos[0]}, c0);")
                        elif len(t.cont_pos) == 2:
                            inner.append(
                                f"{T} {ev_name} = lcm_interp2<{T}, {E}>({rname}, C.n{ti}_{t.cont_pos[0]}, C.n{ti}_{t.cont_pos[1]}, c0, c1);"
                            )
                        else:
                            raise TracingError("more than two continuous states per target are not supported")
                    if off_hi is not None:
                        # off-grid process value: blend the two bracketing node rows
                        # (the reference interpolates the transition-matrix rows)
                        inner.append(f"ev = lcm_zs(({T})1 - ({T})PT[{blend}], ev) + lcm_zs(({T})PT[{blend}], evh);")
                        inner += self._sim_extrapolated_expectation(ti, t, T, E, blend, proc_names, dn, mk)
                    out += ["    " + s for s in inner]
                if det:
                    out.append("    ce = ev;")
                else:
                    out.append("    ce = ce + (lcm_isfinite(ev) ? p * ev : lcm_zs(p, ev));")
                out.append("  }")
                out.append("}")
            if not det:
                out.append(f"bool valid = (fabs(mass - ({T})1) <= ({T})1e-3) && !neg;")
                # a negative weight poisons the row even when the weights sum
                # to exactly one (Q_and_F.py:1401-1432, 646-653)
                out.append(f"ce = valid ? ((mass == ({T})1) ? ce : ce / mass) : lcm_lim<{T}>::nan();")
            out.append(f"Q = ({T})({uexpr}) + ({T})({bexpr}) * ce;")
            return out

        di_params = "".join(f"int DI_{a.name}, " for a in dacts)
        tsel_values = [-1] + ([ti for ti in range(len(self.targets))] if unswitch else [])
        for tsel in tsel_values:
            ap(
                f"template <typename T, typename E, typename AFN>\n"
                f"__device__ __forceinline__ bool lcm_sa{tsel + 1}_{self.tag}(const Ctx_{self.tag}<T, E>& C, "
                f"const double* __restrict__ PV, const double* PVd, const double* DV, const double* SV, "
                f"const double* SDV, const AFN& AF, const int* SI, {di_params}int period, double age, T& Q) {{"
            )
            for s_ in sa_body("T", "E", tsel):
                ap("  " + s_)
            ap("  return true;\n}")
        for ti_, c_ in cinfo.items():
            # target ti_ read from the collapsed rows (AFCol's R)
            ap(
                f"template <typename T, typename E, typename AFN>\n"
                f"__device__ __forceinline__ bool lcm_sc{ti_ + 1}_{self.tag}(const Ctx_{self.tag}<T, E>& C, "
                f"const double* __restrict__ PV, const double* PVd, const double* DV, const double* SV, "
                f"const double* SDV, const AFN& AF, const int* SI, {di_params}int period, double age, T& Q) {{"
            )
            for s_ in sa_body("T", "E", ti_, coll=c_):
                ap("  " + s_)
            ap("  return true;\n}")

        ap(
            f"template <typename T, typename E, typename AFN>\n"
            f"__device__ __forceinline__ bool lcm_simsa_{self.tag}(const Ctx_{self.tag}<T, E>& C, "
            f"const double* __restrict__ PV, const double* PVd, const double* DV, const double* SV, "
            f"const double* SDV, const AFN& AF, const int* SI, const int* PLO, const double* PT, "
            f"{di_params}int period, double age, T& Q) {{"
        )
        ap("  (void)PLO; (void)PT;")
        for s_ in sa_body("T", "E", -1, sim=True):
            ap("  " + s_)
        ap("  return true;\n}")

        # ----------------------------------------------------------------
        # emitters for the hoisted phases (double precision)
        eP = Emitter("double", self.param_off, pv(), "p")
        pvals = [eP.emit(n) for n in bP]

        def prov_sd(kind: str) -> dict:
            prov = pv()
            for i, n in enumerate(bP):
                prov[id(n)] = f"PVd[{i}]" if n.dtype == "f" else _cast(f"PVd[{i}]", n.dtype, "double")
            for i, a in enumerate(dstates):
                prov[id(ir.var("state", a.name, "i"))] = f"si_{a.name}"
            for a in spec.states:
                if a.kind == "continuous":
                    prov[id(ir.var("state", a.name, "f"))] = f"sv_{a.name}"
            for a in dacts:
                prov[id(ir.var("action", a.name, "i"))] = f"DI_{a.name}"
            if kind == "SD":
                for i, n in enumerate(bD):
                    prov[id(n)] = f"DV[{i}]" if n.dtype == "f" else _cast(f"DV[{i}]", n.dtype, "double")
                for i, n in enumerate(bS):
                    prov[id(n)] = f"SV[kb][{i}]" if n.dtype == "f" else _cast(f"SV[kb][{i}]", n.dtype, "double")
            return prov

        def emit_phase(nodes, kind, pref):
            e = Emitter("double", self.param_off, prov_sd(kind), pref)
            vals = [e.emit(n) for n in nodes]
            return e.lines, vals

        d_lines, d_vals = emit_phase(bD, "D", "d")
        s_lines, s_vals = emit_phase(bS, "S", "s")
        sd_lines, sd_vals = emit_phase(bSD, "SD", "x")

        def decode_disc(lines: list[str], ad_expr: str) -> None:
            lines.append(f"int drem = {ad_expr};")
            for a in reversed(dacts):
                lines.append(f"const int DI_{a.name} = drem % {a.size}; drem /= {a.size};")

        # ----------------------------------------------------------------
        # kernel (a)
        SA = f"lcm_sa{{}}_{self.tag}"
        ap(
            f'extern "C" __global__ void __launch_bounds__({B}{", " + str(cfg.min_blocks) if cfg.min_blocks else ""}) '
            f"{self.bellman_name()}(const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles) {{"
        )
        ap("  extern __shared__ __align__(16) unsigned char lcm_smem[];")
        gumax_at = len(L)  # a per-group utility maximum is declared here when groups are skipped
        ap(f"  {TT}* tabf = reinterpret_cast<{TT}*>(lcm_smem);")
        ap(f"  int* tabi = reinterpret_cast<int*>(lcm_smem + {NF * CH * (4 if fp32 else 8)});")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.n_words};")
        ap(f"    Ctx_{self.tag}<{ST}, {ST}> C; C.load(it);")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD});")
        ap(f"    const double age = lcm_wd(it, {self.W_AGE});")
        ap(f"    const int n_states = lcm_wi(it, {self.W_NSTATES});")
        ap(f"    const int n_actions = lcm_wi(it, {self.W_NACT});")
        ap(f"    const int n_ac = n_actions / {ND};")
        ap(f"    const double* __restrict__ atf = lcm_wp<const double>(it, {self.W_ATAB});")
        ap(f"    const int* __restrict__ ati = reinterpret_cast<const int*>(atf + (i64){nf} * n_actions);")
        ap(f"    const int sbase = (tile - tile_prefix[item]) * {SPT} + (int)threadIdx.x / {LANES};")
        ap(f"    const int lane = (int)threadIdx.x % {LANES};")
        ap("    (void)period; (void)age; (void)ati; (void)PV;")
        for s_ in eP.lines:
            ap("    " + s_)
        ap(f"    double PVd[{nP}];")
        for i, v in enumerate(pvals):
            ap(f"    PVd[{i}] = (double)({v});")
        if not bP:
            ap("    PVd[0] = 0.0;")
        ap(f"    int SI[{SB}][{NDS}]; double SV[{SB}][{nS}]; bool act[{SB}]; int sidx[{SB}];")
        kline = next(iter(cinfo.values()))["kline"] if cinfo else -1
        if cinfo:
            # states walked with the line state fastest (a tile then covers at
            # most two lines); sidx is the state's index in the declared order
            ap(f"    int lslot[{SB}];")
            ap(f"    const int nLine = lcm_wi(it, {self.W_SSIZE + kline});")
            ap(f"    const int line0 = ((tile - tile_prefix[item]) * {SPT}) / nLine;")
        ap(f"    #pragma unroll\n    for (int kb = 0; kb < {SB}; ++kb) {{")
        ap(f"      const int s = sbase + kb * {SPB};")
        ap("      act[kb] = s < n_states; sidx[kb] = s;")
        ap("      int srem = act[kb] ? s : 0;")
        order = list(range(len(spec.states) - 1, -1, -1))
        if cinfo:
            order = [kline] + [k for k in order if k != kline]
        for k in order:
            ax = spec.states[k]
            ap(f"      const int si_{ax.name} = srem % lcm_wi(it, {self.W_SSIZE + k}); srem /= lcm_wi(it, {self.W_SSIZE + k});")
        if cinfo:
            phys = "0"
            for k, ax in enumerate(spec.states):
                phys = f"({phys}) * lcm_wi(it, {self.W_SSIZE + k}) + si_{ax.name}"
            ap(f"      if (act[kb]) sidx[kb] = {phys};")
            ap("      lslot[kb] = act[kb] ? s / nLine - line0 : 0;")
        for k, ax in enumerate(spec.states):
            if ax.kind == "continuous":
                ap(f"      const double sv_{ax.name} = lcm_wp<const double>(it, {self.W_SGRID + k})[si_{ax.name}];")
        for s_ in s_lines:
            ap("      " + s_)
        for i, v in enumerate(s_vals):
            ap(f"      SV[kb][{i}] = (double)({v});")
        if not bS:
            ap("      SV[kb][0] = 0.0;")
        for i, a in enumerate(dstates):
            ap(f"      SI[kb][{i}] = si_{a.name};")
        if not dstates:
            ap("      SI[kb][0] = 0;")
        ap("    }")
        BEST = "LcmBest2" if (fp32 and not taste) else "LcmBest"
        if taste:
            ap(f"    LcmBest<{ST}> bd[{SB}][{ND}];")
        else:
            ap(f"    {BEST}<{ST}> best[{SB}];")
            ap(f"    #pragma unroll\n    for (int kb = 0; kb < {SB}; ++kb) best[kb].init();")
        # ---- discrete-action loop (unrolled: ND is a compile-time constant)
        ap(f"    #pragma unroll\n    for (int ad = 0; ad < {ND}; ++ad) {{")
        dl: list[str] = []
        decode_disc(dl, "ad")
        for s_ in dl:
            ap("      " + s_)
        for s_ in d_lines:
            ap("      " + s_)
        ap(f"      double DV[{nD}];")
        for i, v in enumerate(d_vals):
            ap(f"      DV[{i}] = (double)({v});")
        if not bD:
            ap("      DV[0] = 0.0;")
        ap(f"      double SDV[{SB}][{nSD}];")
        ap(f"      #pragma unroll\n      for (int kb = 0; kb < {SB}; ++kb) {{")
        if bSD:
            # re-derive the state variables of slot kb for the SD phase
            ap("        int srem = act[kb] ? sidx[kb] : 0;")
            for k in range(len(spec.states) - 1, -1, -1):
                ax = spec.states[k]
                ap(f"        const int si_{ax.name} = srem % lcm_wi(it, {self.W_SSIZE + k}); srem /= lcm_wi(it, {self.W_SSIZE + k});")
            for k, ax in enumerate(spec.states):
                if ax.kind == "continuous":
                    ap(f"        const double sv_{ax.name} = lcm_wp<const double>(it, {self.W_SGRID + k})[si_{ax.name}];")
            for s_ in sd_lines:
                ap("        " + s_)
            for i, v in enumerate(sd_vals):
                ap(f"        SDV[kb][{i}] = (double)({v});")
        else:
            ap("        SDV[kb][0] = 0.0;")
        ap("      }")
        if taste:
            ap(f"      #pragma unroll\n      for (int kb = 0; kb < {SB}; ++kb) bd[kb][ad].init();")

        def inner_loop(sa_fn: str) -> list[str]:
            o = []
            o.append(f"for (int c0 = 0; c0 < n_ac; c0 += {CH}) {{")
            o.append(f"  const int cn = min({CH}, n_ac - c0);")
            o.append("  __syncthreads();")
            o.append(f"  for (int j = threadIdx.x; j < cn; j += {B}) {{")
            o.append("    const i64 a = (i64)ad * n_ac + c0 + j;")
            for k in range(nf):
                o.append(f"    tabf[{k} * {CH} + j] = ({TT})atf[(i64){k} * n_actions + a];")
            for k in range(ni):
                o.append(f"    tabi[{k} * {CH} + j] = ati[(i64){k} * n_actions + a];")
            o.append("  }")
            o.append("  __syncthreads();")
            o.append(f"  for (int j = lane; j < cn; j += {LANES}) {{")
            o.append(f"    AFTab_{self.tag}<{ST}> af{{tabf, tabi, j}};")
            o.append("    const int aidx = ad * n_ac + c0 + j;")
            o.append(f"    #pragma unroll\n    for (int kb = 0; kb < {SB}; ++kb) {{")
            o.append(f"      {ST} q;")
            di_args = "".join(f"DI_{a.name}, " for a in dacts)
            call = f"{sa_fn}<{ST}, {ST}>(C, PV, PVd, DV, SV[kb], SDV[kb], af, SI[kb], {di_args}period, age, q)"
            push = "bd[kb][ad].push(q, aidx);" if taste else "best[kb].push(q, aidx);"
            o.append(f"      if ({call}) {push}")
            o.append("    }")
            o.append("  }")
            o.append("}")
            return o

        # ---- exact skipping of action groups (single-precision search)
        G = max(cfg.group, LANES)
        GP = self._groups
        GMAX = 2 * CH // G  # groups held in shared memory
        MP = 8  # pilot actions per combination of the other continuous actions

        def provider(n, kb: str) -> str | None:
            """Kernel-scope expression of a hoisted boundary node (double)."""
            if isinstance(n, ir.Expr) and n.op == "const":
                return f"((double){_c_float(float(n.args[0]), 'double')})"
            for lst, fmt in ((bP, "PVd[{i}]"), (bD, "DV[{i}]"), (bS, "SV[" + kb + "][{i}]"),
                             (bSD, "SDV[" + kb + "][{i}]")):
                for i, m in enumerate(lst):
                    if m is n:
                        return fmt.format(i=i)
            return None

        def group_info(ti: int) -> dict | None:
            """Kernel-side pieces of the group plan of target ti (None: the
            hoisted values it needs are not all available)."""
            if GP is None or ti not in GP["axes"]:
                return None
            ia = {id(n): i for i, n in enumerate(bA)}

            def fslot(n):
                i = ia.get(id(n))
                return slot[i][1] if i is not None and slot[i][0] == "F" else None

            uf = fslot(ir.const(self.tr.U))
            avf = {nm: fslot(ir.var("action", nm, "f")) for nm in GP["acts"]}
            if uf is None or any(v is None for v in avf.values()):
                return None
            pb = provider(ir.const(self.tr.beta), "kb")
            if pb is None or "[kb]" in pb:
                return None

            def prov_all(x0, co):
                px = provider(ir.const(x0), "kb")
                pc = {nm: provider(ir.const(c), "kb") for nm, c in co.items()}
                if px is None or any(v is None for v in pc.values()):
                    return None
                return px, pc

            axes = []
            for pos, ci, x0, co in GP["axes"][ti]:
                r = prov_all(x0, co)
                if r is None:
                    return None
                axes.append((pos, ci, r[0], r[1]))
            cons = []
            for op, y0, co in GP["cons"]:
                r = prov_all(y0, co)
                if r is not None:
                    cons.append((op, r[0], r[1]))
            t = self.targets[ti]
            key = "0"
            for kind, name, size in t.key_vars:
                iv = f"SI[kb][{[a.name for a in dstates].index(name)}]" if kind == "state" else f"DI_{name}"
                key = f"({key}) * {size} + {iv}"
            return {"uf": uf, "avf": avf, "beta": pb, "axes": axes, "cons": cons, "key": key, "ti": ti,
                    "bst": f"C.bst{ti}"}

        def inner_loop_groups(sa_fn: str, gi: dict) -> list[str]:
            """inner_loop with exact skipping of action groups.

            The whole continuous-action table sits in shared memory.  A group
            is a run of G consecutive values of the scan action with the other
            continuous actions fixed; per group the block records its largest
            utility and each action's range.  Per state and group, interval
            arithmetic over those ranges bounds the next-state coordinates and
            the constraints' left-minus-right sides: a group all of whose
            members violate a constraint is skipped, and so is a group whose
            Q bound -- largest utility + beta x the largest expectation-table
            value (the block statistics) over the nodes its coordinates can
            reach + a rounding margin -- is below the state's running second
            best (or the second best of a pilot pass over a few spread
            actions, never above the final second best).  Such a group cannot
            enter the top two, so the search's two candidates, and V and the
            policy, are exactly those of the full search.  Coordinates are
            widened by 0.02 + 4e-6 x their magnitude (the float rounding of
            the law as the search evaluates it); a group whose widened
            coordinates leave the grid (extrapolation), and NaN bounds, are
            never skipped.  Candidates are added with index-aware ties, as
            the groups visit the flat action indices out of order."""
            o: list[str] = []
            acts = GP["acts"]
            ks = {nm: k for k, nm in enumerate(acts)}
            anames = [a.name for a in spec.actions]
            cnames = GP["cacts"]
            kscan = anames.index(cnames[GP["scan"]])
            later = [anames.index(nm) for nm in cnames[GP["scan"] + 1:]]
            di_args = "".join(f"DI_{a.name}, " for a in dacts)
            call = f"{sa_fn}<float, float>(C, PV, PVd, DV, SV[kb], SDV[kb], af, SI[kb], {di_args}period, age, q)"
            ti = gi["ti"]
            ninf = "-lcm_lim<float>::inf()"
            o.append(f"const float beta_f = (float)({gi['beta']});")
            o.append(f"const int gN = lcm_wi(it, {self.W_ASIZE + kscan});")
            o.append("int gS = 1;")
            for k in later:
                o.append(f"gS *= lcm_wi(it, {self.W_ASIZE + k});")
            o.append(f"const int gpc = (gN + {G - 1}) / {G};")
            o.append("const int ncomb = gN > 0 ? n_ac / gN : 0;")
            o.append("const int NG = ncomb * gpc;")
            o.append(f"const bool grp = {gi['bst']} != nullptr && beta_f >= 0.0f && n_ac <= {CH} && gN >= {G} "
                     f"&& NG <= {GMAX};  // uniform over the CTA (one item per tile)")
            o.append("if (!grp) {")
            o += ["  " + x for x in inner_loop(sa_fn)]
            o.append("} else {")
            b: list[str] = []
            # per-state affine pieces (float), coordinates in grid units
            b.append(f"float gK[{SB}][{len(gi['axes'])}], gE[{SB}][{len(gi['axes'])}]; int keyr[{SB}];")
            nM = sum(len(pc) for _, _, _, pc in gi["axes"])
            nY = len(gi["cons"])
            nH = sum(len(pc) for _, _, pc in gi["cons"])
            b.append(f"float gM[{SB}][{max(nM, 1)}], gY[{SB}][{max(nY, 1)}], gH[{SB}][{max(nH, 1)}];")
            b.append(f"#pragma unroll\nfor (int kb = 0; kb < {SB}; ++kb) {{")
            m_i = 0
            for p, (pos, ci, px, pc) in enumerate(gi["axes"]):
                A, Bs = f"C.a{ti}_{ci}", f"C.b{ti}_{ci}"
                b.append(f"  {{ const float x0 = (float)({px});")
                b.append(f"    gK[kb][{p}] = (x0 - {A}) * {Bs};")
                b.append(f"    gE[kb][{p}] = (fabsf(x0) + fabsf({A})) * fabsf({Bs}); }}")
                for nm, c in pc.items():
                    b.append(f"  gM[kb][{m_i}] = (float)({c}) * {Bs};")
                    m_i += 1
            h_i = 0
            for c_i, (op, py, pc) in enumerate(gi["cons"]):
                b.append(f"  gY[kb][{c_i}] = (float)({py});")
                for nm, c in pc.items():
                    b.append(f"  gH[kb][{h_i}] = (float)({c});")
                    h_i += 1
            b.append(f"  keyr[kb] = {gi['key']};")
            b.append("}")
            # the continuous-action table of this discrete action, whole
            b.append("__syncthreads();")
            b.append(f"for (int j = threadIdx.x; j < n_ac; j += {B}) {{")
            b.append("  const i64 a = (i64)ad * n_ac + j;")
            for k in range(nf):
                b.append(f"  tabf[{k} * {CH} + j] = ({TT})atf[(i64){k} * n_actions + a];")
            for k in range(ni):
                b.append(f"  tabi[{k} * {CH} + j] = ati[(i64){k} * n_actions + a];")
            b.append("}")
            b.append("__syncthreads();")
            # per-group utility maximum and action ranges
            b.append(f"for (int g = threadIdx.x; g < NG; g += {B}) {{")
            b.append("  const int o_ = g / gpc, gi_ = g - o_ * gpc;")
            b.append(f"  const int jb = (o_ / gS) * gN * gS + (o_ % gS) + gi_ * {G} * gS;")
            b.append(f"  const int m = min({G}, gN - gi_ * {G});")
            b.append(f"  float um = {ninf};")
            for k in range(len(acts)):
                b.append(f"  float lo{k} = lcm_lim<float>::inf(), hi{k} = {ninf};")
            b.append("  for (int t = 0; t < m; ++t) {")
            b.append("    const int j = jb + t * gS;")
            b.append(f"    um = lcm_nanmax(um, tabf[{gi['uf']} * {CH} + j]);")
            for nm, k in ks.items():
                b.append(f"    {{ const float v = tabf[{gi['avf'][nm]} * {CH} + j]; lo{k} = fminf(lo{k}, v); "
                         f"hi{k} = fmaxf(hi{k}, v); }}")
            b.append("  }")
            b.append("  gU[g] = um;")
            for k in range(len(acts)):
                b.append(f"  gLo[{k} * {GMAX} + g] = lo{k}; gHi[{k} * {GMAX} + g] = hi{k};")
            b.append("}")
            b.append("__syncthreads();")
            # pilot pass: a few spread actions per combination (every lane of
            # the state one of them) give a first threshold, the state's
            # second best over them (a top-2 reduction over its lanes)
            b.append("const int MPr = max(8, ncomb > 0 ? 32 / ncomb : 8);")
            b.append(f"float thr[{SB}];")
            b.append("{")
            b.append(f"  float p1[{SB}], p2[{SB}];")
            b.append(f"  #pragma unroll\n  for (int kb = 0; kb < {SB}; ++kb) p1[kb] = p2[kb] = {ninf};")
            b.append(f"  for (int p = lane; p < ncomb * MPr; p += {LANES}) {{")
            b.append("    const int o_ = p / MPr, m_ = p - o_ * MPr;")
            b.append("    const int si = ((2 * m_ + 1) * gN) / (2 * MPr);")
            b.append("    const int j = (o_ / gS) * gN * gS + (o_ % gS) + si * gS;")
            b.append(f"    AFTab_{self.tag}<float> af{{tabf, tabi, j}};")
            b.append(f"    #pragma unroll\n    for (int kb = 0; kb < {SB}; ++kb) {{")
            b.append("      float q;")
            b.append(f"      if (act[kb] && {call} && q > p2[kb]) {{")
            b.append("        if (q > p1[kb]) { p2[kb] = p1[kb]; p1[kb] = q; } else { p2[kb] = q; }")
            b.append("      }")
            b.append("    }")
            b.append("  }")
            b.append(f"  #pragma unroll\n  for (int kb = 0; kb < {SB}; ++kb) {{")
            b.append(f"    #pragma unroll\n    for (int o = {LANES} >> 1; o > 0; o >>= 1) {{")
            b.append("      const float b1 = __shfl_xor_sync(0xffffffffu, p1[kb], o), b2 = __shfl_xor_sync(0xffffffffu, p2[kb], o);")
            b.append("      p2[kb] = fmaxf(fminf(p1[kb], b1), fmaxf(p2[kb], b2));")
            b.append("      p1[kb] = fmaxf(p1[kb], b1);")
            b.append("    }")
            b.append("    thr[kb] = p2[kb];")
            b.append("  }")
            b.append("}")

            def skip_lines(ind: str, th_expr: str) -> list[str]:
                """`skip` of group (um, lo_k, hi_k, am_k) for state kb."""
                L2: list[str] = []
                h_i = 0
                for c_i, (op, py, pc) in enumerate(gi["cons"]):
                    L2.append(f"{{ float lo = gY[kb][{c_i}], hi = lo, mag = fabsf(lo);")
                    for nm in pc:
                        k = ks[nm]
                        L2.append(f"  {{ const float h = gH[kb][{h_i}]; lo += h >= 0.0f ? h * lo{k} : h * hi{k}; "
                                  f"hi += h >= 0.0f ? h * hi{k} : h * lo{k}; mag += fabsf(h) * am{k}; }}")
                        h_i += 1
                    if op in ("<", "<="):
                        L2.append("  skip = skip || lo > 4e-6f * mag; }  // every member has lhs > rhs")
                    else:
                        L2.append("  skip = skip || hi < -4e-6f * mag; }  // every member has lhs < rhs")
                L2.append("if (!skip) {")
                L2.append(f"  const float th = {th_expr};")
                L2.append("  bool ok = true;")
                m_i = 0
                lohi = []
                for p, (pos, ci, px, pc) in enumerate(gi["axes"]):
                    L2.append(f"  float lo_{p} = gK[kb][{p}], hi_{p} = lo_{p}, e_{p} = gE[kb][{p}];")
                    for nm in pc:
                        k = ks[nm]
                        L2.append(f"  {{ const float mm = gM[kb][{m_i}]; lo_{p} += mm >= 0.0f ? mm * lo{k} : mm * hi{k}; "
                                  f"hi_{p} += mm >= 0.0f ? mm * hi{k} : mm * lo{k}; e_{p} += fabsf(mm) * am{k}; }}")
                        m_i += 1
                    L2.append(f"  e_{p} = 0.02f + 4e-6f * e_{p};")
                    L2.append(f"  const int n_{p} = C.n{ti}_{pos};")
                    L2.append(f"  ok = ok && lo_{p} - e_{p} >= 0.0f && hi_{p} + e_{p} <= (float)(n_{p} - 1);")
                    lohi.append(p)
                L2.append("  if (ok) {")
                for p in lohi:
                    L2.append(f"    const int L_{p} = (int)(lo_{p} - e_{p}), H_{p} = min((int)(hi_{p} + e_{p}) + 1, n_{p} - 1);")
                L2.append(f"    float mx = {ninf}, ab = 0.0f;")
                if len(lohi) == 1:
                    L2.append(f"    const float2* row = {gi['bst']} + (i64)keyr[kb] * ((n_0 + 15) >> 4);")
                    L2.append("    for (int b1 = L_0 >> 4; b1 <= (H_0 >> 4); ++b1) {")
                    L2.append("      const float2 st = __ldg(row + b1);")
                    L2.append("      mx = lcm_nanmax(mx, st.x); ab = fmaxf(ab, st.y);")
                    L2.append("    }")
                else:
                    T1, T2 = self.GROUP_TILE
                    L2.append(f"    const int nb1 = (n_0 + {T1 - 1}) / {T1}, nb2 = (n_1 + {T2 - 1}) / {T2};")
                    L2.append(f"    const float2* base = {gi['bst']} + (i64)keyr[kb] * nb1 * nb2;")
                    L2.append(f"    for (int b1 = L_0 / {T1}; b1 <= H_0 / {T1}; ++b1) {{")
                    L2.append(f"      for (int b2 = L_1 / {T2}; b2 <= H_1 / {T2}; ++b2) {{")
                    L2.append("        const float2 st = __ldg(base + (i64)b1 * nb2 + b2);")
                    L2.append("        mx = lcm_nanmax(mx, st.x); ab = fmaxf(ab, st.y);")
                    L2.append("      }")
                    L2.append("    }")
                L2.append("    const float ub = um + beta_f * mx;")
                L2.append("    const float marg = 3.8e-6f * (fabsf(um) + beta_f * ab);")
                L2.append("    skip = ub + marg < th;")
                L2.append("  }")
                L2.append("}")
                return [ind + x for x in L2]

            def group_vars(ind: str, g: str) -> list[str]:
                L2 = [f"const float um = gU[{g}];"]
                for k in range(len(acts)):
                    L2.append(f"const float lo{k} = gLo[{k} * {GMAX} + {g}], hi{k} = gHi[{k} * {GMAX} + {g}];")
                    L2.append(f"const float am{k} = fmaxf(fabsf(lo{k}), fabsf(hi{k}));")
                return [ind + x for x in L2]

            def eval_members(ind: str, cond: str) -> list[str]:
                L2 = [f"const int o_ = gg / gpc, gi_ = gg - o_ * gpc;",
                      f"const int jb = (o_ / gS) * gN * gS + (o_ % gS) + gi_ * {G} * gS;",
                      f"const int m = min({G}, gN - gi_ * {G});",
                      f"for (int t = lane; t < m; t += {LANES}) {{",
                      "  const int j = jb + t * gS;",
                      f"  AFTab_{self.tag}<float> af{{tabf, tabi, j}};",
                      "  const int aidx = ad * n_ac + j;",
                      f"  #pragma unroll\n  for (int kb = 0; kb < {SB}; ++kb) {{",
                      "    float q;",
                      f"    if ({cond} && {call}) {{ if (q != q) best[kb].nan = 1; else best[kb].add(q, aidx); }}",
                      "  }",
                      "}"]
                return [ind + x for x in L2]

            if LANES == 32:
                # a warp per state: lane i tests group g0 + i against the
                # pilot threshold; the warp then evaluates the surviving
                # groups, one member per lane -- every decision is uniform
                # over the warp
                b.append("for (int g0 = 0; g0 < NG; g0 += 32) {")
                b.append("  const int gl = min(g0 + lane, NG - 1);")
                b += group_vars("  ", "gl")
                b.append(f"  unsigned need[{SB}]; unsigned anyb = 0u;")
                b.append(f"  #pragma unroll\n  for (int kb = 0; kb < {SB}; ++kb) {{")
                b.append("    bool skip = false;")
                b += skip_lines("    ", f"fmaxf(thr[kb], best[kb].idx2 >= 0 ? best[kb].v2 : {ninf})")
                b.append("    need[kb] = __ballot_sync(0xffffffffu, act[kb] && g0 + lane < NG && !skip);")
                b.append("    anyb |= need[kb];")
                b.append("  }")
                b.append("  while (anyb) {")
                b.append("    const int bit = __ffs(anyb) - 1;")
                b.append("    anyb &= anyb - 1u;")
                b.append("    const int gg = g0 + bit;")
                b += eval_members("    ", "((need[kb] >> bit) & 1u)")
                b.append("  }")
                b.append("}")
            else:
                b.append("for (int gg = 0; gg < NG; ++gg) {")
                b += group_vars("  ", "gg")
                b.append(f"  bool run[{SB}]; bool any = false;")
                b.append(f"  #pragma unroll\n  for (int kb = 0; kb < {SB}; ++kb) {{")
                b.append("    bool skip = false;")
                b.append("    if (act[kb]) {")
                b += skip_lines("      ", f"fmaxf(thr[kb], best[kb].idx2 >= 0 ? best[kb].v2 : {ninf})")
                b.append("    }")
                b.append("    run[kb] = act[kb] && !skip;")
                b.append("    any = any || run[kb];")
                b.append("  }")
                b.append("  if (!any) continue;")
                b += eval_members("  ", "run[kb]")
                b.append("}")
            o += ["  " + x for x in b]
            o.append("}")
            return o

        def inner_loop_collapse(ti: int, c: dict) -> list[str]:
            """The inner loop of target ti read from collapsed rows, built per
            tile in shared memory; the plain loop where an item's sizes do not
            allow them (a line shorter than a tile, rows longer than
            reserved, another size of the outer action grid)."""
            t = self.targets[ti]
            nob, namax, posA, posB, cb = c["nob"], c["namax"], c["posA"], c["posB"], c["cb"]
            o = ["{"]
            o.append(f"  const int nA = C.n{ti}_{posA}, nB = C.n{ti}_{posB};")
            o.append(f"  if (nLine >= {SPT} && nA <= {namax} && lcm_wi(it, {self.W_ASIZE + c['kob']}) == {nob}) {{")
            o.append(f"    float* crow = reinterpret_cast<float*>(lcm_smem + {rows_off});")
            o.append(f"    const double* obg = lcm_wp<const double>(it, {self.W_AGRID + c['kob']});")
            ostr = "1"
            for k in range(c["kob"] + 1, len(spec.actions)):
                ostr = f"{ostr} * lcm_wi(it, {self.W_ASIZE + k})"
            o.append(f"    const int ostr = {ostr};")
            o.append("    const int nLines = n_states / nLine;")
            o.append("    __syncthreads();  // the previous tile's reads of the rows are done")
            o.append(f"    for (int e = threadIdx.x; e < 2 * {nob} * nA; e += {B}) {{")
            o.append(f"      const int w = e % nA, r = e / nA, ob = r % {nob}, line = line0 + r / {nob};")
            o.append("      float val = lcm_lim<float>::nan();")
            o.append("      if (line < nLines) {")
            o.append("        int lrem = line;")
            for k in range(len(spec.states) - 1, -1, -1):
                ax = spec.states[k]
                if k == kline:
                    o.append(f"        const int si_{ax.name} = 0;")
                else:
                    o.append(f"        const int si_{ax.name} = lrem % lcm_wi(it, {self.W_SSIZE + k}); "
                             f"lrem /= lcm_wi(it, {self.W_SSIZE + k});")
            for k, ax in enumerate(spec.states):
                if ax.kind == "continuous":
                    o.append(f"        const double sv_{ax.name} = lcm_wp<const double>(it, {self.W_SGRID + k})[si_{ax.name}];")
            o += ["        " + x for x in s_lines]
            o.append(f"        double SVl[{nS}];")
            for i, v in enumerate(s_vals):
                o.append(f"        SVl[{i}] = (double)({v});")
            if not bS:
                o.append("        SVl[0] = 0.0;")
            prov = pv()
            for i, n in enumerate(bP):
                prov[id(n)] = _cast(f"PVd[{i}]", n.dtype, "float")
            for i, n in enumerate(bS):
                prov[id(n)] = _cast(f"SVl[{i}]", n.dtype, "float")
            for i, a in enumerate(dstates):
                prov[id(ir.var("state", a.name, "i"))] = f"si_{a.name}"
            e = Emitter("float", self.param_off, prov, "w")
            x0s, gs = e.emit(c["x0"]), e.emit(c["g"])
            o += ["        " + x for x in e.lines]
            key = "0"
            for kind, name, size in t.key_vars:
                key = f"({key}) * {size} + si_{name}"
            o.append(f"        const float cB = (((float)({x0s})) - C.a{ti}_{cb}) * C.b{ti}_{cb} + "
                     f"(((float)({gs})) * C.b{ti}_{cb}) * (float)obg[ob];")
            o.append("        float fB; const int lB = lcm_lower(cB, nB, fB); const float uB = cB - fB;")
            o.append(f"        const float* blk = C.ev{ti} + (i64)({key}) * ((i64)nA * nB);")
            if cb == 1:
                o.append("        const float va = blk[(i64)w * nB + lB], vb = blk[(i64)w * nB + lB + 1];")
            else:
                o.append("        const float va = blk[(i64)lB * nA + w], vb = blk[(i64)(lB + 1) * nA + w];")
            o.append("        val = va + uB * (vb - va);")
            o.append("        if (!lcm_isfinite(val)) val = lcm_zs(1.0f - uB, va) + lcm_zs(uB, vb);")
            o.append("      }")
            o.append("      crow[e] = val;")
            o.append("    }")
            # the budget constraint a <= b on the slowest continuous action:
            # a state's feasible actions are a prefix of the table; a warp
            # stops at the longest prefix among its states (two grid points of
            # slack for the single-precision test)
            bb = self._budget_bound()
            bexpr = None
            if bb is not None:
                kc, bnode = bb
                if isinstance(bnode, (int, float)):
                    bexpr = repr(float(bnode))
                elif id(bnode) in {id(x) for x in bS}:
                    bexpr = f"SV[kb][{[id(x) for x in bS].index(id(bnode))}]"
                elif id(bnode) in {id(x) for x in bP}:
                    bexpr = f"PVd[{[id(x) for x in bP].index(id(bnode))}]"
            if bexpr is None:
                o.append("    const int jfe = n_ac;")
            else:
                o.append(f"    const double* cgr = lcm_wp<const double>(it, {self.W_AGRID + kc});")
                o.append(f"    const int ncg = lcm_wi(it, {self.W_ASIZE + kc});")
                o.append("    int jfe = 0;")
                o.append(f"    #pragma unroll\n    for (int kb = 0; kb < {SB}; ++kb) {{")
                o.append("      if (!act[kb]) continue;")
                o.append(f"      const double wv = (double)({bexpr});")
                o.append("      int lo = 0, hi = ncg;  // grid points at or below the bound")
                o.append("      while (lo < hi) { const int mid = (lo + hi) >> 1; if (cgr[mid] <= wv) lo = mid + 1; else hi = mid; }")
                o.append("      jfe = max(jfe, min(lo + 2, ncg) * (n_ac / ncg));")
                o.append("    }")
                o.append("    jfe = __reduce_max_sync(0xffffffffu, jfe);")
            o.append(f"    for (int c0 = 0; c0 < n_ac; c0 += {CH}) {{")
            o.append(f"      const int cn = min({CH}, n_ac - c0);")
            o.append("      __syncthreads();")
            o.append(f"      for (int j = threadIdx.x; j < cn; j += {B}) {{")
            o.append("        const i64 a = (i64)ad * n_ac + c0 + j;")
            for k in range(nf):
                o.append(f"        tabf[{k} * {CH} + j] = ({TT})atf[(i64){k} * n_actions + a];")
            for k in range(ni):
                o.append(f"        tabi[{k} * {CH} + j] = ati[(i64){k} * n_actions + a];")
            o.append("      }")
            o.append("      __syncthreads();")
            o.append("      const int jend = min(cn, jfe - c0);")
            o.append(f"      for (int j = lane; j < jend; j += {LANES}) {{")
            o.append("        const int aidx = ad * n_ac + c0 + j;")
            o.append(f"        const int obi = ((c0 + j) / ostr) % {nob};")
            o.append(f"        #pragma unroll\n        for (int kb = 0; kb < {SB}; ++kb) {{")
            o.append(f"          AFCol_{self.tag}<{ST}> af{{tabf, tabi, j, crow + (lslot[kb] * {nob} + obi) * nA}};")
            o.append(f"          {ST} q;")
            di_args = "".join(f"DI_{a.name}, " for a in dacts)
            o.append(f"          if (lcm_sc{ti + 1}_{self.tag}<{ST}, {ST}>(C, PV, PVd, DV, SV[kb], SDV[kb], af, SI[kb], "
                     f"{di_args}period, age, q)) best[kb].push(q, aidx);")
            o.append("        }")
            o.append("      }")
            o.append("    }")
            o.append("  } else {")
            o += ["    " + x for x in inner_loop(SA.format(ti + 1))]
            o.append("  }")
            o.append("}")
            return o

        any_pruned = False
        n_gacts = 0
        if unswitch:
            rid_expr = f"(int)PVd[{[id(x) for x in bP].index(id(self.tr.regime_id))}]" if rid_phase == "P" else None
            if rid_phase == "D":
                rid_expr = f"(int)DV[{[id(x) for x in bD].index(id(self.tr.regime_id))}]"
            ap(f"      const int rid = {rid_expr};")
            first = True
            for ti, t in enumerate(self.targets):
                ap(f"      {'if' if first else 'else if'} (rid == {t.spec.rid}) {{")
                first = False
                gi = group_info(ti)
                if gi is not None:
                    any_pruned = True
                    n_gacts = max(n_gacts, len(GP["acts"]))
                if ti in cinfo:
                    body = inner_loop_collapse(ti, cinfo[ti])
                else:
                    body = inner_loop(SA.format(ti + 1)) if gi is None else inner_loop_groups(SA.format(ti + 1), gi)
                for s_ in body:
                    ap("        " + s_)
                ap("      }")
            ap("      else {")
            for s_ in inner_loop(SA.format(0)):
                ap("        " + s_)
            ap("      }")
        else:
            for s_ in inner_loop(SA.format(0)):
                ap("      " + s_)
        ap("    }")
        if any_pruned:
            L.insert(gumax_at, f"  __shared__ float gU[{GMAX}], gLo[{max(n_gacts, 1) * GMAX}], gHi[{max(n_gacts, 1) * GMAX}];")
        self.prunes_groups = any_pruned

        # ---- reduction and epilogue
        def final_eval(a_var: str, out_var: str, loc: str) -> list[str]:
            lines = [f"AFLoc_{self.tag} {loc}; Ctx_{self.tag}<double, double> Cd; Cd.load(it);"]
            for k in range(nf):
                lines.append(f"{loc}.v[{k}] = atf[(i64){k} * n_actions + {a_var}];")
            for k in range(ni):
                lines.append(f"{loc}.vi[{k}] = ati[(i64){k} * n_actions + {a_var}];")
            decode_disc(lines, f"{a_var} / n_ac")
            lines += d_lines
            lines.append(f"double DV[{nD}];")
            for i, v in enumerate(d_vals):
                lines.append(f"DV[{i}] = (double)({v});")
            if not bD:
                lines.append("DV[0] = 0.0;")
            lines.append(f"double SDVf[{nSD}];")
            if bSD:
                lines.append("{ int srem = s;")
                for k in range(len(spec.states) - 1, -1, -1):
                    ax = spec.states[k]
                    lines.append(f"const int si_{ax.name} = srem % lcm_wi(it, {self.W_SSIZE + k}); srem /= lcm_wi(it, {self.W_SSIZE + k});")
                for k, ax in enumerate(spec.states):
                    if ax.kind == "continuous":
                        lines.append(f"const double sv_{ax.name} = lcm_wp<const double>(it, {self.W_SGRID + k})[si_{ax.name}];")
                lines += sd_lines
                for i, v in enumerate(sd_vals):
                    lines.append(f"SDVf[{i}] = (double)({v});")
                lines.append("}")
            else:
                lines.append("SDVf[0] = 0.0;")
            di_args = "".join(f"DI_{a.name}, " for a in dacts)
            lines.append(f"double {out_var};")
            lines.append(
                f"if (!{SA.format(0)}<double, double>(Cd, PV, PVd, DV, SV[kb], SDVf, {loc}, SI[kb], {di_args}period, age, {out_var})) {out_var} = -lcm_lim<double>::inf();"
            )
            return lines

        ap(f"    #pragma unroll\n    for (int kb = 0; kb < {SB}; ++kb) {{")
        if taste:
            ap(f"      #pragma unroll\n      for (int d = 0; d < {ND}; ++d) lcm_group_reduce<{LANES}, {ST}>(bd[kb][d]);")
        elif fp32:
            ap(f"      lcm_group_reduce2<{LANES}, {ST}>(best[kb]);")
        else:
            ap(f"      lcm_group_reduce<{LANES}, {ST}>(best[kb]);")
        ap("      if (act[kb] && lane == 0) {")
        ap("        const int s = sidx[kb];")
        ap(f"        double* Vout = lcm_wp<double>(it, {self.W_V});")
        ap(f"        int* Pout = lcm_wp<int>(it, {self.W_POL});")
        if taste:
            ap(f"        double vals[{ND}]; int bdi = -1; double bv = -lcm_lim<double>::inf(); int anynan = 0;")
            ap(f"        for (int d = 0; d < {ND}; ++d) {{")
            ap("          anynan |= bd[kb][d].nan;")
            ap("          if (bd[kb][d].idx < 0) { vals[d] = -lcm_lim<double>::inf(); continue; }")
            if fp32:
                ap("          { const int aa = bd[kb][d].idx;")
                for s_ in final_eval("aa", "qd", "afl"):
                    ap("            " + s_)
                ap("            vals[d] = qd; }")
            else:
                ap("          vals[d] = bd[kb][d].v;")
            ap("          if (bdi < 0 || vals[d] > bv) { bv = vals[d]; bdi = d; }")
            ap("        }")
            ap(f"        const double scale = lcm_wd(it, {self.W_TASTE});")
            ap(f"        double v = lcm_logsum<double, {ND}>(vals, scale);")
            ap("        if (anynan) v = lcm_lim<double>::nan();")
            ap("        int pol = 0;")
            ap(f"        for (int d = 0; d < {ND}; ++d) if (d == bdi) pol = bd[kb][d].idx;")
            ap("        Vout[s] = v; Pout[s] = (bdi < 0 || anynan) ? 0 : pol;")
        else:
            ap("        double v; int pol;")
            ap("        if (best[kb].nan) { v = lcm_lim<double>::nan(); pol = 0; }")
            ap("        else if (best[kb].idx < 0) { v = -lcm_lim<double>::inf(); pol = 0; }")
            if fp32:
                ap("        else { const int aa = best[kb].idx;")
                for s_ in final_eval("aa", "qd", "afl"):
                    ap("          " + s_)
                ap("          v = qd; pol = aa;")
                ap("          if (best[kb].idx2 >= 0) { const int ab = best[kb].idx2;")
                for s_ in final_eval("ab", "qd2", "afl2"):
                    ap("            " + s_)
                ap("            if (qd2 > v || (qd2 == v && ab < pol)) { v = qd2; pol = ab; } }")
                ap("        }")
            else:
                ap("        else { v = (double)best[kb].v; pol = best[kb].idx; }")
            ap("        Vout[s] = v; Pout[s] = pol;")
        ap("      }")
        ap("    }")
        ap("  }")
        ap("}")
        self.smem_bytes = NF * CH * (4 if fp32 else 8) + NI * CH * 4 + rows_bytes
        self.atab_words = nf * 2 + ni

        # ----------------------------------------------------------------
        # kernel (a0): continuous-action-only sub-expressions, one thread per action
        ap(f"// ---- regime {spec.name}: action table (kernel a0)")
        ap(
            f'extern "C" __global__ void __launch_bounds__(256) {self.atab_name()}('
            "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles) {"
        )
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.n_words};")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD});")
        ap(f"    const double age = lcm_wd(it, {self.W_AGE});")
        ap(f"    const int n_actions = lcm_wi(it, {self.W_NACT});")
        ap(f"    double* atf = lcm_wp<double>(it, {self.W_ATAB});")
        ap(f"    int* ati = reinterpret_cast<int*>(atf + (i64){nf} * n_actions);")
        ap("    (void)period; (void)age; (void)ati; (void)PV;")
        ap("    const int a = (tile - tile_prefix[item]) * 256 + (int)threadIdx.x;")
        ap("    if (a < n_actions) {")
        ap("      int arem = a;")
        prov = pv()
        for k in range(len(spec.actions) - 1, -1, -1):
            ax = spec.actions[k]
            ap(f"      const int ai_{ax.name} = arem % lcm_wi(it, {self.W_ASIZE + k}); arem /= lcm_wi(it, {self.W_ASIZE + k});")
        for k, ax in enumerate(spec.actions):
            if ax.kind == "continuous":
                ap(f"      const double av_{ax.name} = lcm_wp<const double>(it, {self.W_AGRID + k})[ai_{ax.name}];")
                prov[id(ir.var("action", ax.name, "f"))] = f"av_{ax.name}"
            else:
                prov[id(ir.var("action", ax.name, "i"))] = f"ai_{ax.name}"
        e = Emitter("double", self.param_off, prov, "t")
        vals = [e.emit(n) for n in bA]
        for s_ in e.lines:
            ap("      " + s_)
        for i, (n, v) in enumerate(zip(bA, vals)):
            col, k = slot[i]
            if col == "F":
                ap(f"      atf[(i64){k} * n_actions + a] = (double)({v});")
            else:
                ap(f"      ati[(i64){k} * n_actions + a] = (int)({v});")
        ap("    }")
        ap("  }")
        ap("}")
        L += self._sim_kernel(locals())
        return "\n".join(L)

    # ------------------------------------------------------------------ (d)
    def _sim_layout(self) -> None:
        spec = self.spec
        w = self.n_words
        self.SW_N, self.SW_RID_IN, self.SW_RID_OUT, self.SW_VAL, self.SW_AIDX = w, w + 1, w + 2, w + 3, w + 4
        self.SW_SEED = w + 5  # XOR-ed into the launch seed: one Philox key per item
        # JAX-stream key table of the item (0: the Philox stream): 2 words per
        # slot -- 0 the regime draw, 1 the taste shocks, then one per state
        # of each target (sim_slot)
        self.SW_JKEYS = w + 6
        w += 7
        self.SW_ACT = w
        w += len(spec.actions)
        self.SW_SIN = w
        w += len(spec.states)
        names: list[str] = []
        if self.targets:
            for t in self.targets:
                for ax in t.spec.states:
                    if ax.name not in names:
                        names.append(ax.name)
        else:
            names = [ax.name for ax in spec.states]
        self.sim_out_names = names
        self.SW_SOUT = w
        w += len(names)
        self.sim_words = w
        self.sim_slot: dict[tuple, int] = {}
        q = 2
        for ti, t in enumerate(self.targets):
            for k, ax in enumerate(t.spec.states):
                self.sim_slot[(t.spec.name, ax.name)] = q
                q += 1
        self.sim_n_slots = q

    def sim_name(self) -> str:
        return f"lcm_sim_{self.tag}"

    def _sim_kernel(self, env: dict) -> list[str]:
        """Kernel (d): one simulated period of this regime for every subject in it.

        One warp per subject: the 32 lanes stride over the actions (double
        precision), the first lane records value and action and draws the next
        regime and next states with the Philox stream of (seed, subject,
        period, stream id).  Stream ids: 0 regime draw, 1 + k the k-th state of
        the drawn target, 64 + d the taste shock of discrete choice d, 128 + k
        the mixture component of the k-th state (normal-mixture processes).
        """
        from pylcm_b200.spec import proc_field_name, proc_grid_name

        self._sim_layout()
        spec = self.spec
        tag = self.tag
        bP, bD, bS, bSD = env["bP"], env["bD"], env["bS"], env["bSD"]
        nf, nP, nD, nS, nSD = env["nf"], env["nP"], env["nD"], env["nS"], env["nSD"]
        dstates, dacts = env["dstates"], env["dacts"]
        ND, taste = env["ND"], env["taste"]
        pv, decode_disc = env["pv"], env["decode_disc"]
        eP, pvals = env["eP"], env["pvals"]
        d_lines, d_vals = env["d_lines"], env["d_vals"]
        proc_names = env["proc_names"]
        NDS = max(len(dstates), 1)
        NPROC = max(len(proc_names), 1)
        L: list[str] = []
        ap = L.append

        def sim_prov(kind: str) -> dict:
            prov = pv()
            for i, n in enumerate(bP):
                prov[id(n)] = f"PVd[{i}]" if n.dtype == "f" else _cast(f"PVd[{i}]", n.dtype, "double")
            for a in spec.states:
                if a.kind == "continuous":
                    prov[id(ir.var("state", a.name, "f"))] = f"sv_{a.name}"
                else:
                    prov[id(ir.var("state", a.name, "i"))] = f"si_{a.name}"
                if a.kind == "process":
                    node = ir.Expr("pidx", (proc_grid_name(a.name), ir.var("state", a.name, "i")), "f")
                    prov[id(node)] = f"pv_{a.name}"
            for a in dacts:
                prov[id(ir.var("action", a.name, "i"))] = f"DI_{a.name}"
            if kind == "SD":
                for i, n in enumerate(bD):
                    prov[id(n)] = f"DV[{i}]" if n.dtype == "f" else _cast(f"DV[{i}]", n.dtype, "double")
                for i, n in enumerate(bS):
                    prov[id(n)] = f"SV[{i}]" if n.dtype == "f" else _cast(f"SV[{i}]", n.dtype, "double")
            return prov

        eS = Emitter("double", self.param_off, sim_prov("S"), "s")
        s_vals = [eS.emit(n) for n in bS]
        eSD = Emitter("double", self.param_off, sim_prov("SD"), "x")
        sdv = [eSD.emit(n) for n in bSD]

        ap(f"struct AFG_{tag} {{ const double* atf; const int* ati; int n; int a;")
        ap("  __device__ __forceinline__ double F(int f) const { return __ldg(atf + (i64)f * n + a); }")
        ap("  __device__ __forceinline__ int I(int f) const { return __ldg(ati + (i64)f * n + a); } };")
        ap(
            f'extern "C" __global__ void __launch_bounds__(256) {self.sim_name()}('
            "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles, u64 seed) {"
        )
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* __restrict__ it = items + (i64)item * {self.sim_words};")
        ap("    const int s = (tile - tile_prefix[item]) * 8 + (int)threadIdx.x / 32;")
        ap("    const int lane = (int)threadIdx.x % 32;")
        ap(f"    if (s >= lcm_wi(it, {self.SW_N})) continue;")
        ap(f"    const int* rid_in = lcm_wp<const int>(it, {self.SW_RID_IN});")
        ap(f"    if (rid_in[s] != {spec.rid}) continue;  // warp-uniform: one subject per warp")
        ap(f"    Ctx_{tag}<double, double> C; C.load(it);")
        ap(f"    const double* __restrict__ PV = lcm_wp<const double>(it, {self.W_P});")
        ap(f"    const int period = lcm_wi(it, {self.W_PERIOD});")
        ap(f"    const double age = lcm_wd(it, {self.W_AGE});")
        ap(f"    const int n_actions = lcm_wi(it, {self.W_NACT});")
        ap(f"    const int n_ac = n_actions / {ND};")
        ap(f"    const double* __restrict__ atf = lcm_wp<const double>(it, {self.W_ATAB});")
        ap(f"    const int* __restrict__ ati = reinterpret_cast<const int*>(atf + (i64){nf} * n_actions);")
        ap("    (void)period; (void)age; (void)ati; (void)PV;")
        ap(f"    const u64 key = seed ^ (u64)it[{self.SW_SEED}];")
        ap("    LcmRng rng; rng.k0 = (u32)key; rng.k1 = (u32)(key >> 32); rng.subject = (u32)s; rng.period = (u32)period;")
        ap(f"    const u32* JK = lcm_wp<const u32>(it, {self.SW_JKEYS});")
        ap("    const LcmJaxRng jr{JK, (u32)s};")
        for s_ in eP.lines:
            ap("    " + s_)
        ap(f"    double PVd[{nP}]; PVd[0] = 0.0;")
        for i, v in enumerate(pvals):
            ap(f"    PVd[{i}] = (double)({v});")
        ap(f"    int SI[{NDS}]; int PLO[{NPROC}]; double PT[{NPROC}]; SI[0] = 0; PLO[0] = 0; PT[0] = 0.0;")
        for k, a in enumerate(spec.states):
            ap(f"    const double x_{a.name} = lcm_wp<const double>(it, {self.SW_SIN + k})[s];")
            if a.kind == "continuous":
                ap(f"    const double sv_{a.name} = x_{a.name};")
            elif a.kind == "discrete":
                ap(f"    const int si_{a.name} = (int)x_{a.name};")
            else:
                off, shape = self.param_off[proc_grid_name(a.name)]
                pi = proc_names.index(a.name)
                ap(f"    const double pv_{a.name} = x_{a.name};")
                ap(f"    const double pc_{a.name} = lcm_coord_irreg<double>(pv_{a.name}, PV + {off}, {shape[0]});")
                ap(f"    double pf_{a.name}; PLO[{pi}] = lcm_lower(pc_{a.name}, {shape[0]}, pf_{a.name}); PT[{pi}] = pc_{a.name} - pf_{a.name};")
                ap(f"    const int si_{a.name} = PLO[{pi}];")
        for i, a in enumerate(dstates):
            ap(f"    SI[{i}] = si_{a.name};")
        for s_ in eS.lines:
            ap("    " + s_)
        ap(f"    double SV[{nS}]; SV[0] = 0.0;")
        for i, v in enumerate(s_vals):
            ap(f"    SV[{i}] = (double)({v});")
        if taste:
            ap(f"    LcmBest<double> bd[{ND}];")
            ap(f"    #pragma unroll\n    for (int d = 0; d < {ND}; ++d) bd[d].init();")
        else:
            ap("    LcmBest<double> best; best.init();")
        ap(f"    #pragma unroll\n    for (int ad = 0; ad < {ND}; ++ad) {{")
        dl: list[str] = []
        decode_disc(dl, "ad")
        for s_ in dl + d_lines:
            ap("      " + s_)
        ap(f"      double DV[{nD}]; DV[0] = 0.0;")
        for i, v in enumerate(d_vals):
            ap(f"      DV[{i}] = (double)({v});")
        for s_ in eSD.lines:
            ap("      " + s_)
        ap(f"      double SDV[{nSD}]; SDV[0] = 0.0;")
        for i, v in enumerate(sdv):
            ap(f"      SDV[{i}] = (double)({v});")
        di_args = "".join(f"DI_{a.name}, " for a in dacts)
        push = "bd[ad].push(q, aidx);" if taste else "best.push(q, aidx);"
        ap("      for (int j = lane; j < n_ac; j += 32) {")
        ap("        const int aidx = ad * n_ac + j;")
        ap(f"        AFG_{tag} af{{atf, ati, n_actions, aidx}};")
        ap("        double q;")
        ap(f"        if (lcm_simsa_{tag}<double, double>(C, PV, PVd, DV, SV, SDV, af, SI, PLO, PT, {di_args}period, age, q)) {push}")
        ap("      }")
        ap("    }")
        if taste:
            ap(f"    #pragma unroll\n    for (int d = 0; d < {ND}; ++d) lcm_group_reduce<32, double>(bd[d]);")
        else:
            ap("    lcm_group_reduce<32, double>(best);")
        ap("    if (lane != 0) continue;")
        if taste:
            ap(f"    const double scale = lcm_wd(it, {self.W_TASTE});")
            # the reference (max_Q_over_a.py:268-297): per discrete cell the
            # first argmax of the masked Q row (a NaN first, an all -inf row
            # its first action), then the first argmax of max + noise over
            # the cells (a NaN cell first)
            ap("    int dstar = -1, dnan = -1; double bn = -lcm_lim<double>::inf(); double vstar = -lcm_lim<double>::inf();")
            ap(f"    for (int d = 0; d < {ND}; ++d) {{")
            ap("      const double qc = bd[d].nan ? lcm_lim<double>::nan() : (bd[d].idx < 0 ? -lcm_lim<double>::inf() : bd[d].v);")
            ap("      const double g = JK ? jr.gumbel(1, d) : rng.gumbel(64u + (u32)d);")
            ap("      const double noisy = qc + scale * (g - 0.5772156649015329);")
            ap("      if (dnan < 0 && noisy != noisy) dnan = d;")
            ap("      if (dstar < 0 || noisy > bn) { bn = noisy; dstar = d; vstar = qc; }")
            ap("    }")
            ap("    if (dnan >= 0) { dstar = dnan; vstar = lcm_lim<double>::nan(); }")
            ap("    int aa = 0;")
            ap(f"    for (int d = 0; d < {ND}; ++d) if (d == dstar) "
               "aa = bd[d].nan ? bd[d].nan - 1 : ((bd[d].idx < 0 || !(bd[d].v > -lcm_lim<double>::inf())) ? d * n_ac : bd[d].idx);")
            ap("    const double value = vstar;")
        else:
            # argmax_and_max (argmax.py:55-69): a NaN maximum matches no
            # entry, so the first action
            ap("    const int aa = (best.nan || best.idx < 0) ? 0 : best.idx;")
            ap("    const double value = best.nan ? lcm_lim<double>::nan() : (best.idx < 0 ? -lcm_lim<double>::inf() : best.v);")
        ap(f"    lcm_wp<double>(it, {self.SW_VAL})[s] = value;")
        ap(f"    lcm_wp<int>(it, {self.SW_AIDX})[s] = aa;")
        ap("    int arem = aa;")
        prov = sim_prov("S")
        for k in range(len(spec.actions) - 1, -1, -1):
            ax = spec.actions[k]
            ap(f"    const int ai_{ax.name} = arem % lcm_wi(it, {self.W_ASIZE + k}); arem /= lcm_wi(it, {self.W_ASIZE + k});")
        for k, ax in enumerate(spec.actions):
            if ax.kind == "continuous":
                ap(f"    const double av_{ax.name} = lcm_wp<const double>(it, {self.W_AGRID + k})[ai_{ax.name}];")
                prov[id(ir.var("action", ax.name, "f"))] = f"av_{ax.name}"
                ap(f"    lcm_wp<double>(it, {self.SW_ACT + k})[s] = av_{ax.name};")
            else:
                prov[id(ir.var("action", ax.name, "i"))] = f"ai_{ax.name}"
                ap(f"    lcm_wp<double>(it, {self.SW_ACT + k})[s] = (double)ai_{ax.name};")
        e = Emitter("double", self.param_off, prov, "n")
        out_idx = {name: self.SW_SOUT + i for i, name in enumerate(self.sim_out_names)}
        rid_out = f"lcm_wp<int>(it, {self.SW_RID_OUT})[s]"
        if spec.terminal:
            ap(f"    {rid_out} = {spec.rid};")
            for a in spec.states:
                ap(f"    lcm_wp<double>(it, {out_idx[a.name]})[s] = x_{a.name};")
        else:
            tr = self.tr
            if tr.regime_id is not None:
                r_expr = e.emit(tr.regime_id)
                for s_ in e.lines:
                    ap("    " + s_)
                e.lines = []
                ap(f"    const int rid = (int)({r_expr});")
            else:
                probs = [e.emit(p) for p in tr.regime_probs]
                for s_ in e.lines:
                    ap("    " + s_)
                e.lines = []
                ap(f"    double rp[{len(probs)}];")
                for i, p_ in enumerate(probs):
                    ap(f"    rp[{i}] = (double)({p_});")
                ap(f"    const int rid = JK ? lcm_jax_choice<{len(probs)}>(rp, jr.uniform(0)) "
                   f": lcm_categorical<{len(probs)}>(rp, rng.uniform(0u));")
            ap(f"    {rid_out} = rid;")
            for t in self.targets:
                if t.unreachable:
                    continue  # the drawn target's states stay NaN
                ap(f"    if (rid == {t.spec.rid}) {{")
                # scoped emitter: expressions bound inside this branch stay in it
                et = Emitter("double", self.param_off, dict(e.vals), f"n{t.spec.rid}_")
                for k, ax in enumerate(t.spec.states):
                    law = t.laws[ax.name]
                    dst = f"lcm_wp<double>(it, {out_idx[ax.name]})[s]"
                    stream = f"{1 + k}u"
                    q = self.sim_slot[(t.spec.name, ax.name)]
                    if law.kind in ("cont", "det"):
                        v = et.emit(law.expr)
                        for s_ in et.lines:
                            ap("      " + s_)
                        et.lines = []
                        ap(f"      {dst} = (double)({v});")
                    elif law.kind == "markov":
                        vs = [et.emit(x) for x in law.expr.items]
                        for s_ in et.lines:
                            ap("      " + s_)
                        et.lines = []
                        ap(f"      {{ double mp[{len(vs)}];")
                        for i, v in enumerate(vs):
                            ap(f"        mp[{i}] = (double)({v});")
                        ap(f"        {dst} = (double)(JK ? lcm_jax_choice<{len(vs)}>(mp, jr.uniform({q})) "
                           f": lcm_categorical<{len(vs)}>(mp, rng.uniform({stream}))); }}")
                    else:  # process: draw from the source process's law
                        src = law.source_process
                        grid = spec.state(src).grid
                        fld = lambda f, src=src: f"PV[{self.param_off[proc_field_name(src, f)][0]}]"  # noqa: E731
                        cls = type(grid).__name__
                        nz = f"(JK ? jr.normal({q}) : rng.normal({stream}))"
                        if cls in ("TauchenAR1Process", "RouwenhorstAR1Process"):
                            ap(f"      {dst} = {fld('mu')} + {fld('rho')} * pv_{src} + {fld('sigma')} * {nz};")
                        elif cls == "NormalIIDProcess":
                            ap(f"      {dst} = {fld('mu')} + {fld('sigma')} * {nz};")
                        elif cls == "LogNormalIIDProcess":
                            ap(f"      {dst} = exp({fld('mu')} + {fld('sigma')} * {nz});")
                        elif cls == "UniformIIDProcess":
                            ap(f"      {dst} = JK ? jr.uniform({q}, {fld('start')}, {fld('stop')}) "
                               f": {fld('start')} + ({fld('stop')} - {fld('start')}) * rng.uniform({stream});")
                        elif cls in ("TauchenNormalMixtureAR1Process", "NormalMixtureIIDProcess"):
                            # component 1 with probability p1 (its own stream), then its normal
                            ar = f"{fld('mu')} + {fld('rho')} * pv_{src} + " if cls.startswith("Tauchen") else ""
                            ap("      { double z; bool c1;")
                            ap(f"        if (JK) {{ c1 = jr.mixture({q}, {fld('p1')}, z); }}")
                            ap(f"        else {{ c1 = rng.uniform({128 + k}u) < {fld('p1')}; z = rng.normal({stream}); }}")
                            ap(f"        {dst} = {ar}(c1 ? {fld('mu1')} + {fld('sigma1')} * z : {fld('mu2')} + {fld('sigma2')} * z); }}")
                        else:
                            raise TracingError(f"no simulation draw for process {cls}")
                ap("    }")
        ap("  }")
        ap("}")
        return L


    # ------------------------------------------------------------------ (b)
    def _weight_fill(self, t: TargetPlan, block: int) -> list[str]:
        """Lines that fill the item's weight table W[k * J + j] (double, in
        shared memory) with a stride of `block` threads; they read the item
        words PV (3), period (4) and age (5) through `PV`, `period`, `age`."""
        tg = t.spec
        K, J = t.K, t.J
        L = [f"for (int e = threadIdx.x; e < {K * J}; e += {block}) {{",
             f"  const int k = e / {J}; const int j = e % {J};",
             "  int kr = k;"]
        for kind, kname, size in reversed(t.key_vars):
            L.append(f"  const int key_{kind}_{kname} = kr % {size}; kr /= {size};")
        L.append("  int jr = j;")
        for pos in reversed(t.stoch_pos):
            ax = tg.states[pos]
            L.append(f"  const int jn_{ax.name} = jr % {ax.size}; jr /= {ax.size};")
        prov = {
            id(ir.var("period", "period", "i")): "period",
            id(ir.var("age", "age", "f")): "age",
        }
        for kind, kname, size in t.key_vars:
            prov[id(ir.var(kind, kname, "i"))] = f"key_{kind}_{kname}"
        e = Emitter("double", self.param_off, prov, "w")
        factors = []
        for pos in t.stoch_pos:
            ax = tg.states[pos]
            law = t.laws[ax.name]
            if law.kind == "process":
                off, shape = self.param_off[proc_P_name(law.source_process)]
                n = shape[0]
                factors.append(f"PV[{off} + key_state_{law.source_process} * {n} + jn_{ax.name}]")
            else:
                # select item j of the Markov vector
                exprs = [e.emit(x) for x in law.expr.items]
                sel = exprs[-1]
                for q in range(len(exprs) - 2, -1, -1):
                    sel = f"(jn_{ax.name} == {q} ? (double)({exprs[q]}) : {sel})"
                factors.append(f"(double)({sel})")
        L += ["  " + s_ for s_ in e.lines]
        prod = factors[0] if factors else "1.0"
        for f_ in factors[1:]:
            prod = f"({prod}) * ({f_})"
        L.append(f"  W[e] = {prod};")
        L.append("}")
        return L

    # ..................................................................
    # tensor-core form of kernel (b) (single-precision search table)
    TC_MAX_J = 64
    TC_MAX_K = 256

    def tc_ok(self, t: TargetPlan) -> bool:
        """The single-precision search table of target `t` comes from the
        tcgen05 kernel: a contraction whose V' rows are the target's
        stochastic node combinations (no deterministic discrete axis), with at
        most 64 nodes and 256 weight rows."""
        return (self.precision == "fp32" and not t.scalar and not t.unreachable and t.needs_contraction
                and not t.det_pos and t.J <= self.TC_MAX_J and t.K <= self.TC_MAX_K)

    def expect_tc_name(self, t: TargetPlan) -> str:
        return f"lcm_expect_tc_{self.tag}_{t.spec.name}"

    @staticmethod
    def tc_shape(K: int, J: int) -> dict:
        """Padded sizes and shared memory of the tensor-core expectation (the
        host-side twin of LcmTcShape in lcm_tc.cuh)."""
        JP = (J + 7) // 8 * 8
        NP = (K + 15) // 16 * 16
        ncol = 32 if NP <= 32 else 64 if NP <= 64 else 128 if NP <= 128 else 256
        dyn = 2 * 128 * JP * 4 + 2 * NP * JP * 4 + 128
        static = K * J * 8 + K * 4 + 8 + 4 + 4 + 64
        # at most 512 / ncol CTAs per SM so that every CTA's tensor-memory
        # allocation succeeds at once: pad the dynamic shared memory so that
        # no more CTAs fit (228 KB per SM, 1 KB reserved per CTA)
        max_ctas = 512 // ncol
        per_sm, reserve = 233472, 1024
        if per_sm // (dyn + static + reserve) > max_ctas:
            dyn = per_sm // (max_ctas + 1) - static - reserve + 1
        return {"JP": JP, "NP": NP, "ncol": ncol, "smem": dyn, "max_ctas": max_ctas}

    def _expect_tc_source(self, t: TargetPlan) -> str:
        """Kernel (b), tensor-core form: EV32 by a 3xTF32 tcgen05 GEMM
        (lcm_tc_expect in lcm_tc.cuh) with this target's weight table."""
        name = self.expect_tc_name(t)
        K, J = t.K, t.J
        L = [f"// ---- expectation {self.spec.name} -> {t.spec.name} on the tensor cores: K={K} J={J}",
             f"struct WFill_{name} {{",
             "  __device__ __forceinline__ void operator()(const i64* __restrict__ it, double* W) const {",
             "    const double* __restrict__ PV = lcm_wp<const double>(it, 3);",
             "    const int period = lcm_wi(it, 4);",
             "    const double age = lcm_wd(it, 5);",
             "    (void)period; (void)age; (void)PV;"]
        L += ["    " + s_ for s_ in self._weight_fill(t, 128)]
        L += ["  }", "};",
              f'extern "C" __global__ void __launch_bounds__(128) {name}('
              "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles) {",
              f"  lcm_tc_expect<{K}, {J}>(items, tile_prefix, n_items, n_tiles, {9 + len(t.spec.states)}, "
              f"{8 + len(t.spec.states)}, WFill_{name}{{}});",
              "}"]
        return "\n".join(L)

    def _expect_source(self, t: TargetPlan) -> str:
        """Kernel (b): contraction of V' over the target's stochastic axes."""
        spec = self.spec
        tg = t.spec
        K, J = t.K, t.J
        stoch = t.stoch_pos
        B = 256
        KC = min(K, 32)
        # weight expressions per stochastic axis
        L: list[str] = []
        ap = L.append
        name = self.expect_name(t)
        # item layout for (b)
        # 0 Vt (double*), 1 EV64 out, 2 EV32 out (0 if none), 3 PV (params of source)
        # 4 period, 5 age, 6 cblk, 7 n_cols, 8.. sizes of target axes
        self.EW = {"V": 0, "EV64": 1, "EV32": 2, "P": 3, "PERIOD": 4, "AGE": 5, "CBLK": 6, "NCOLS": 7, "SIZES": 8,
                   "BSTATS": 8 + len(tg.states)}
        self.e_words = 9 + len(tg.states)
        ap(f"// ---- expectation {spec.name} -> {tg.name}: K={K} J={J}")
        ap(
            f'extern "C" __global__ void __launch_bounds__({B}) {name}('
            "const i64* __restrict__ items, const int* __restrict__ tile_prefix, int n_items, int n_tiles) {"
        )
        ap(f"  __shared__ double W[{K * J}];")
        ap(f"  __shared__ double Winv[{K}];")
        ap("  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {")
        ap("    const int item = lcm_find_item(tile_prefix, n_items, tile);")
        ap(f"    const i64* it = items + (i64)item * {self.e_words};")
        ap("    const double* __restrict__ Vt = lcm_wp<const double>(it, 0);")
        ap("    double* EV64 = lcm_wp<double>(it, 1);")
        ap("    float* EV32 = lcm_wp<float>(it, 2);")
        ap("    const double* __restrict__ PV = lcm_wp<const double>(it, 3);")
        ap("    const int period = lcm_wi(it, 4);")
        ap("    const double age = lcm_wd(it, 5);")
        ap("    const int cblk = lcm_wi(it, 6);")
        ap("    const int n_cols = lcm_wi(it, 7);")
        ap("    (void)period; (void)age;")
        ap("    __syncthreads();")
        for s_ in self._weight_fill(t, B):
            ap("    " + s_)
        ap("    __syncthreads();")
        ap(f"    for (int k = threadIdx.x; k < {K}; k += {B}) {{")
        ap(f"      double sw = 0.0; for (int j = 0; j < {J}; ++j) sw += W[k * {J} + j];")
        ap("      Winv[k] = sw > 0.0 ? sw : 1.0;")
        ap("    }")
        ap("    __syncthreads();")
        # block statistics of the float table (word BSTATS, 0: none): per row k
        # and 16 columns, (max, finite |max|), for the search's group skipping
        ap(f"    float2* BST = EV32 ? lcm_wp<float2>(it, {8 + len(tg.states)}) : nullptr;")
        ap("    const int nb16 = (n_cols + 15) >> 4;")
        ap(f"    const int col_t = (tile - tile_prefix[item]) * {B} + (int)threadIdx.x;")
        ap("    const bool live = col_t < n_cols;")
        ap("    const int col = live ? col_t : 0;")
        ap("    {")
        # decode col -> det indices + cflat ; compute base offset per j
        ap("      const int cflat = col % cblk; int dr = col / cblk;")
        det_names = []
        for pos in reversed(t.det_pos):
            ax = tg.states[pos]
            ap(f"      const int di_{ax.name} = dr % {ax.size}; dr /= {ax.size};")
        # strides over target discrete axes in order
        disc_pos = [p for p, ax in enumerate(tg.states) if ax.kind != "continuous"]
        ap(f"      for (int k0 = 0; k0 < {K}; k0 += {KC}) {{")
        ap(f"        double acc[{KC}];")
        ap(f"        #pragma unroll\n        for (int kk = 0; kk < {KC}; ++kk) acc[kk] = 0.0;")
        ap(f"        for (int j = 0; j < (live ? {J} : 0); ++j) {{")
        ap("          int jr = j;")
        for pos in reversed(stoch):
            ax = tg.states[pos]
            ap(f"          const int jn_{ax.name} = jr % {ax.size}; jr /= {ax.size};")
        off = "0"
        for pos in disc_pos:
            ax = tg.states[pos]
            iv = f"jn_{ax.name}" if pos in stoch else f"di_{ax.name}"
            off = f"({off}) * {ax.size} + {iv}"
        ap(f"          const double v = Vt[(i64)({off}) * cblk + cflat];")
        ap(f"          #pragma unroll\n          for (int kk = 0; kk < {KC}; ++kk) {{")
        ap(f"            const int k = k0 + kk; if (k < {K}) acc[kk] += lcm_zs(W[k * {J} + j], v);")
        ap("          }")
        ap("        }")
        ap(f"        #pragma unroll\n        for (int kk = 0; kk < {KC}; ++kk) {{")
        ap(f"          const int k = k0 + kk; if (k < {K}) {{")
        ap("            const double r = acc[kk] / Winv[k];")
        ap("            if (live) {")
        ap("              EV64[(i64)k * n_cols + col] = r;")
        ap("              if (EV32) EV32[(i64)k * n_cols + col] = (float)r;")
        ap("            }")
        ap("            if (BST) {  // uniform over the CTA (one item per tile)")
        ap("              const float2 st = lcm_block16_stats(live ? (float)r : -lcm_lim<float>::inf());")
        ap("              if (live && (threadIdx.x & 15) == 0) BST[(i64)k * nb16 + (col >> 4)] = st;")
        ap("            }")
        ap("          }")
        ap("        }")
        ap("      }")
        ap("    }")
        ap("  }")
        ap("}")
        return "\n".join(L)


def _ctype(dt: str) -> str:
    return {"f": "double", "i": "int", "b": "bool"}[dt]


def _cast(expr: str, dt: str, T: str) -> str:
    if dt == "f":
        return f"(({T}){expr})"
    if dt == "i":
        return f"((int){expr})"
    return f"(({expr}) != 0)"
