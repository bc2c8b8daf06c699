"""Oracle: forward simulation in NumPy float64 (test infrastructure only).

Restates the reference's per-period simulation step
(``src/_lcm/simulation/simulate.py:465-668``): the first-index argmax of Q at
each subject's state (the taste-shock variant adds centred Gumbel noise to
the per-discrete-choice maxima, ``max_Q_over_a.py:255-297``), then the next
regime and next states (deterministic laws, Markov draws,
``next_state.py:301-341``, and process draws, ``processes/ar1.py:122-132``,
``processes/iid.py``).

Random numbers, two streams:

- ``rng="philox"``: the counter-based Philox-4x32-10 stream of the GPU
  kernel's serving form (counter = (subject, period, stream id, 0), key = the seed),
  restated in NumPy, so GPU and oracle paths can be compared draw for draw;
- ``rng="jax"`` (default): the reference's own stream (``pylcm_b200.jaxrng``, JAX's
  Threefry-2x32 with its key threading): ``key(seed)``; per period, per active
  regime in declaration order, the taste-shock keys (``simulate.py:562-572``)
  and then ``split(key, 3)`` into the next-state key, the regime key and the
  running key (``simulate.py:630``); per subject, one key per stochastic
  next-state function (sorted qualified names, ``transitions.py:111-125``)
  and one for the regime draw (``transitions.py:260-275``); the samplers of
  ``jax.random`` (``choice`` with weights, ``normal``, ``uniform``,
  ``bernoulli``, ``gumbel``).  This stream reproduces the reference's stored
  stochastic simulations.
"""

from __future__ import annotations

import math

import numpy as np

from oracle.grid_search import _process_tables, bellman_step, solve
from pylcm_b200.regime import MarkovTransition
from pylcm_b200.spec import ParamResolver, trace_regime

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
EULER_GAMMA = 0.5772156649015329


def philox4x32(c0, c1, c2, c3, k0, k1):
    """Philox-4x32-10 on uint32 arrays (Salmon et al. 2011)."""
    c = [np.asarray(x, dtype=np.uint32) for x in (c0, c1, c2, c3)]
    k0 = np.uint32(k0)
    k1 = np.uint32(k1)
    with np.errstate(over="ignore"):
        for r in range(10):
            if r > 0:
                k0 = np.uint32((int(k0) + int(_W0)) & 0xFFFFFFFF)
                k1 = np.uint32((int(k1) + int(_W1)) & 0xFFFFFFFF)
            p0 = c[0].astype(np.uint64) * _M0
            p1 = c[2].astype(np.uint64) * _M1
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & np.uint64(0xFFFFFFFF)).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & np.uint64(0xFFFFFFFF)).astype(np.uint32)
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
    return c


def _u53(a, b):
    m = ((a >> np.uint32(5)).astype(np.uint64) << np.uint64(26)) | (b >> np.uint32(6)).astype(np.uint64)
    return (m.astype(np.float64) + 0.5) * 2.0**-53


class Rng:
    def __init__(self, seed: int, period: int, subjects: np.ndarray) -> None:
        self.k0 = seed & 0xFFFFFFFF
        self.k1 = (seed >> 32) & 0xFFFFFFFF
        self.period = period
        self.subjects = np.asarray(subjects, dtype=np.uint32)

    def _raw(self, stream: int):
        n = self.subjects.shape
        return philox4x32(self.subjects, np.full(n, self.period, np.uint32), np.full(n, stream, np.uint32),
                          np.zeros(n, np.uint32), self.k0, self.k1)

    def uniform(self, stream: int):
        r = self._raw(stream)
        return _u53(r[0], r[1])

    def normal(self, stream: int):
        r = self._raw(stream)
        u1, u2 = _u53(r[0], r[1]), _u53(r[2], r[3])
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)

    def gumbel(self, stream: int):
        return -np.log(-np.log(self.uniform(stream)))


def categorical(p: np.ndarray, u: np.ndarray) -> np.ndarray:
    """First index whose cumulative weight exceeds u * total (rows of p)."""
    tot = p.sum(axis=1)
    thr = u * tot
    cum = np.cumsum(p, axis=1)
    idx = (cum > thr[:, None]).argmax(axis=1)
    none = ~(cum > thr[:, None]).any(axis=1)
    return np.where(none, p.shape[1] - 1, idx)


class _JaxStream:
    """The reference's key threading over one simulation (``rng="jax"``)."""

    def __init__(self, seed: int, n: int) -> None:
        from pylcm_b200 import jaxrng

        self.J = jaxrng
        self.key = jaxrng.key(seed)
        self.n = n

    def taste_keys(self):
        self.key, d = self.J.simulation_keys(self.key, ["taste_shock"], self.n)
        return d["taste_shock"]

    def split3(self):
        ks = self.J.split(self.key, 3)
        self.key = ks[2]
        return ks[0], ks[1]


def _reachable_targets(spec, specs, res, model) -> list:
    """Targets the regime's transition reaches with positive probability in
    some period (the reference's simulation reachability)."""
    from pylcm_b200.validation import _regime_probs

    out = set()
    for period in spec.active_periods:
        if period + 1 >= model.n_periods:
            continue
        P, _ = _regime_probs(spec, specs, res, period, float(model.ages.values[period]))
        for s in specs:
            if np.any(np.nan_to_num(P[:, s.rid]) > 0):
                out.add(s.name)
    return [s for s in specs if s.name in out]


def _erfinv(u):
    from scipy.special import erfinv

    return erfinv(u)


def simulate(model, params, initial_conditions, seed: int = 0, V=None, rng: str = "jax") -> dict:
    """Per period: regime_id, value, states, actions (NaN where not defined).
    `rng` selects the random stream (see the module docstring)."""
    specs = model.regime_specs
    res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    if V is None:
        from oracle.grid_search import _is_egm

        if any(_is_egm(s) for s in specs):
            from oracle.dcegm import solve as egm_solve

            V, _ = egm_solve(model, params)
        else:
            V, _ = solve(model, params)
    T = model.n_periods
    ic = dict(initial_conditions)
    rid = np.asarray(ic.pop("regime_id"), dtype=np.int64)
    ic.pop("age", None)
    N = rid.shape[0]
    snames = sorted({a.name for s in specs for a in s.states})
    anames = sorted({a.name for s in specs for a in s.actions})
    S = {n: np.full(N, np.nan) for n in snames}
    for k, v in ic.items():
        S[k] = np.asarray(v, dtype=np.float64).copy()
    out = {}
    by_id = {s.rid: s for s in specs}
    jax_rng = rng == "jax"
    stream = _JaxStream(seed, N) if jax_rng else None
    # the reference walks the active regimes in declaration order
    order = [next(s for s in specs if s.name == nm) for nm in model.user_regimes] if jax_rng else specs
    reach = {s.name: _reachable_targets(s, specs, res, model) for s in specs if not s.terminal} if jax_rng else {}
    for period in range(T):
        age = float(model.ages.values[period])
        val = np.full(N, np.nan)
        A = {n: np.full(N, np.nan) for n in anames}
        newR = np.full(N, -1, dtype=np.int64)
        newS = {n: np.full(N, np.nan) for n in snames}
        nxt = V.get(period + 1, {})
        for spec in order:
            if period not in spec.active_periods:
                continue
            sel = np.nonzero(rid == spec.rid)[0]
            jk = None
            if jax_rng:
                # every active regime advances the running key, members or not
                jk = {"taste": stream.taste_keys() if spec.taste_shocks else None}
                if not spec.terminal:
                    jk["states"], jk["regime"] = stream.split3()
            if sel.size == 0:
                continue
            rng = Rng(seed, period, sel)
            sv = {a.name: S[a.name][sel] for a in spec.states}
            Q, F = bellman_step(spec, specs, res, period, age, nxt, state_values=sv if spec.states else {"_": np.zeros(sel.size)}, return_qf=True)
            Q = np.broadcast_to(Q, F.shape)
            Qm = np.where(F, Q, -np.inf)
            if spec.taste_shocks:
                scale = res.taste_scale(spec.name)
                nd, nc = spec.n_discrete_actions, spec.n_continuous_actions
                Qd = Qm.reshape(len(sel), nd, nc)
                cont_arg = Qd.argmax(axis=2)
                Qc = Qd.max(axis=2)
                if jax_rng:
                    # jax.random.gumbel(key, (nd,)): one uniform per discrete
                    # cell from the counters (0, d) of the subject's key
                    from pylcm_b200 import jaxrng

                    noise = scale * (jaxrng.gumbel_shaped(jk["taste"][sel], nd) - EULER_GAMMA)
                else:
                    noise = np.stack([scale * (rng.gumbel(64 + d) - EULER_GAMMA) for d in range(nd)], axis=1)
                noisy = Qc + noise  # -inf stays -inf, a NaN cell is NaN (argmax: first NaN)
                dstar = noisy.argmax(axis=1)
                aa = dstar * nc + cont_arg[np.arange(len(sel)), dstar]
                v = Qc[np.arange(len(sel)), dstar]
            else:
                # argmax_and_max (argmax.py:55-69): the first feasible action at
                # the max; a NaN max, or no feasible action, matches none: 0
                v = Qm.max(axis=1)
                aa = ((Qm == v[:, None]) & F).argmax(axis=1)
            val[sel] = v
            ashape = tuple(a.size for a in spec.actions)
            aidx = np.unravel_index(aa, ashape) if spec.actions else ()
            chosen = {}
            for k, a in enumerate(spec.actions):
                x = aidx[k].astype(np.int64) if a.kind == "discrete" else a.grid.to_numpy()[aidx[k]]
                A[a.name][sel] = x
                chosen[a.name] = x
            if spec.terminal:
                newR[sel] = spec.rid
                for a in spec.states:
                    newS[a.name][sel] = S[a.name][sel]
                continue
            targets = tuple(s.name for s in specs if (period + 1) in s.active_periods)
            tr = trace_regime(spec, specs, res, targets)
            env = _eval_env(spec, sv, chosen, period, age, res)
            skeys = None
            if jax_rng:
                from pylcm_b200 import jaxrng

                tr_all = trace_regime(spec, specs, res, tuple(t.name for t in reach[spec.name]))
                qnames = sorted(
                    f"{t}__next_{nm}"
                    for t, laws in tr_all.next_states.items() if laws is not None
                    for nm, law in laws.items() if law.kind in ("markov", "process")
                )
                _, skeys = jaxrng.simulation_keys(jk["states"], qnames, N)
                _, rkeys = jaxrng.simulation_keys(jk["regime"], ["regime_transition"], N)
            if tr.regime_id is not None:
                r_new = np.broadcast_to(_ev(tr.regime_id, env, tr), (len(sel),)).astype(np.int64)
            else:
                probs = np.stack([np.broadcast_to(_ev(p, env, tr), (len(sel),)) for p in tr.regime_probs], axis=1)
                if jax_rng:
                    # choice over the regimes active next period, by regime id
                    cand = [s.rid for s in specs if s.name in targets]
                    k = jaxrng.choice_index(rkeys["regime_transition"][sel], probs[:, cand])
                    r_new = np.asarray(cand, dtype=np.int64)[k]
                else:
                    r_new = categorical(probs, rng.uniform(0))
            newR[sel] = r_new
            for tname in targets:
                tgt = next(s for s in specs if s.name == tname)
                m = r_new == tgt.rid
                if not m.any() or tr.next_states.get(tname) is None:
                    continue
                for k, ax in enumerate(tgt.states):
                    law = tr.next_states[tname][ax.name]
                    if law.kind in ("cont", "det"):
                        x = np.broadcast_to(_ev(law.expr, env, tr), (len(sel),)).astype(np.float64)
                    elif law.kind == "markov":
                        p = np.stack([np.broadcast_to(_ev(it, env, tr), (len(sel),)) for it in law.expr.items], axis=1)
                        if jax_rng:
                            x = jaxrng.choice_index(skeys[f"{tname}__next_{ax.name}"][sel], p).astype(np.float64)
                        else:
                            x = categorical(p, rng.uniform(1 + k)).astype(np.float64)
                    elif jax_rng:
                        x = _jax_process_draw(spec, law, res, sv, skeys[f"{tname}__next_{ax.name}"][sel])
                    else:
                        grid = spec.state(law.source_process).grid
                        pp = res.process_params(spec.name, law.source_process, grid)
                        cls = type(grid).__name__
                        y = sv[law.source_process]
                        if cls in ("TauchenAR1Process", "RouwenhorstAR1Process"):
                            x = float(pp["mu"]) + float(pp["rho"]) * y + float(pp["sigma"]) * rng.normal(1 + k)
                        elif cls == "NormalIIDProcess":
                            x = float(pp["mu"]) + float(pp["sigma"]) * rng.normal(1 + k)
                        elif cls == "LogNormalIIDProcess":
                            x = np.exp(float(pp["mu"]) + float(pp["sigma"]) * rng.normal(1 + k))
                        elif cls in ("TauchenNormalMixtureAR1Process", "NormalMixtureIIDProcess"):
                            # mixture innovation (``ar1.py:306-320``, ``iid.py:290-300``):
                            # component 1 with probability p1, then its normal
                            c1 = rng.uniform(128 + k) < float(pp["p1"])
                            z = rng.normal(1 + k)
                            eps = np.where(c1, float(pp["mu1"]) + float(pp["sigma1"]) * z,
                                           float(pp["mu2"]) + float(pp["sigma2"]) * z)
                            x = eps if cls == "NormalMixtureIIDProcess" else float(pp["mu"]) + float(pp["rho"]) * y + eps
                        else:
                            x = float(pp["start"]) + (float(pp["stop"]) - float(pp["start"])) * rng.uniform(1 + k)
                    newS[ax.name][sel[m]] = np.asarray(x)[m]
        out[period] = {"regime_id": rid.copy(), "value": val, "states": {n: S[n].copy() for n in snames}, "actions": A}
        rid = newR
        S = newS
    return out


def _jax_process_draw(spec, law, res, sv, keys):
    """The reference's process draws (``processes/ar1.py:122-132, 191-201,
    305-319``, ``processes/iid.py:58-65, 135-140, 201-206, 286-298``) from
    the subjects' keys."""
    from pylcm_b200 import jaxrng

    grid = spec.state(law.source_process).grid
    pp = {k: float(v) for k, v in res.process_params(spec.name, law.source_process, grid).items()}
    cls = type(grid).__name__
    y = sv[law.source_process]
    if cls in ("TauchenAR1Process", "RouwenhorstAR1Process"):
        return pp["mu"] + pp["rho"] * y + pp["sigma"] * jaxrng.normal(keys, _erfinv)
    if cls == "NormalIIDProcess":
        return pp["mu"] + pp["sigma"] * jaxrng.normal(keys, _erfinv)
    if cls == "LogNormalIIDProcess":
        return np.exp(pp["mu"] + pp["sigma"] * jaxrng.normal(keys, _erfinv))
    if cls == "UniformIIDProcess":
        return jaxrng.uniform(keys, pp["start"], pp["stop"])
    if cls in ("TauchenNormalMixtureAR1Process", "NormalMixtureIIDProcess"):
        k2 = jaxrng.split(keys, 2)
        comp = jaxrng.bernoulli(k2[..., 0, :], pp["p1"])
        z = jaxrng.normal(k2[..., 1, :], _erfinv)
        eps = np.where(comp, pp["mu1"] + pp["sigma1"] * z, pp["mu2"] + pp["sigma2"] * z)
        return eps if cls == "NormalMixtureIIDProcess" else pp["mu"] + pp["rho"] * y + eps
    raise NotImplementedError(cls)


def _eval_env(spec, sv, chosen, period, age, res):
    from oracle.grid_search import _process_tables

    procs = _process_tables(spec, res)
    env = {("period", "period"): period, ("age", "age"): age}
    for a in spec.states:
        if a.kind == "continuous":
            env[("state", a.name)] = sv[a.name]
        elif a.kind == "discrete":
            env[("state", a.name)] = sv[a.name].astype(np.int64)
        else:
            nodes = procs[a.name][0]
            from oracle.grid_search import _irreg_coordinate

            c = _irreg_coordinate(nodes, sv[a.name])
            env[("state", a.name)] = np.clip(np.floor(c), 0, len(nodes) - 2).astype(np.int64)
            env[("procval", a.name)] = sv[a.name]
    for a in spec.actions:
        env[("action", a.name)] = chosen[a.name]
    return env


def _ev(expr, env, tr):
    """Evaluate an IR expression at simulated values (process values directly)."""
    from pylcm_b200 import ir
    from pylcm_b200.spec import proc_grid_name

    # process state values enter user functions as pidx(nodes, index); in the
    # simulation they are the subject's own (off-grid) value
    procvals = {k[1]: v for k, v in env.items() if k[0] == "procval"}
    if procvals:
        expr = _subst_proc(expr, procvals)
    params = {k: v for k, v in tr.param_values.items()}
    return ir.evaluate(expr, env, params)


_SUBST_CACHE: dict = {}


def _subst_proc(expr, procvals):
    from pylcm_b200 import ir
    from pylcm_b200.spec import proc_grid_name

    names = {proc_grid_name(n): n for n in procvals}

    # evaluate with a custom walk: replace pidx(proc nodes) by the value
    cache = {}

    def ev(e):
        if id(e) in cache:
            return cache[id(e)]
        if e.op == "pidx" and e.args[0] in names:
            r = ir.var("procval", names[e.args[0]], "f")
        elif e.op in ("const", "var", "param"):
            r = e
        else:
            args = tuple(ev(a) if isinstance(a, ir.Expr) else a for a in e.args)
            r = ir.Expr(e.op, args, e.dtype)
        cache[id(e)] = r
        return r

    return ev(expr)
