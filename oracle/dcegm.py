"""Oracle: DC-EGM backward induction with the FUES, LTM, RFC or MSS envelope (test
infrastructure only).

Restates the reference's endogenous-grid step
(``src/_lcm/egm/step_core.py:156-616``) in NumPy float64, per (discrete
state x discrete action) row:

1. continuation at every savings node A: for each next-period target (weighted
   by the regime probability) and each combination of the target's discrete
   states (Markov / process / deterministic laws), read the target's carry
   rows at R'(A) and aggregate over the target's discrete choices (hard max,
   or logsum / softmax with taste shocks) -- ``egm/continuation.py:959-1534``;
   E[V'] and E[mu' dR'/dA] are weighted means over the nodes;
2. Euler inversion c = (u')^{-1}(max(beta E[mu'], eps)), R = A + c,
   v = u(c) + beta E[V'] (``egm/euler.py:18-68``);
3. constrained candidates c_k = span 1e-4 ratio^k (``step_core.py:443-514``);
4. the upper envelope: FUES (``oracle/fues.py``), or LTM / RFC / MSS
   (``oracle/envelopes.py``; RFC with the candidates' u'(c) as supgradient,
   0 for dead candidates, ``step_core.py:414-440``);
5. publication on the state grid: the refined value row read with a
   Fritsch-Carlson-limited cubic Hermite interpolant whose node slopes are
   u'(c), floored at (and below the first refined point replaced by) the
   closed-form constrained value (``step_core.py:517-616``); the carry rows
   are the refined grid, value and u'(policy);
6. V over the regime's states: the max over discrete actions (logsum with
   taste shocks).

Reads of refined rows follow the reference's rules (``egm/interp.py:63-131``):
linear extrapolation below the first node, clamp at or above the last, a
duplicated abscissa (kink) read right-continuously.
"""

from __future__ import annotations

import itertools
import math

import numpy as np

from oracle.envelopes import refine_ltm, refine_mss, refine_rfc
from oracle.fues import refine
from oracle.grid_search import _process_tables, bellman_step
from pylcm_b200 import ir
from pylcm_b200.egm import A_VAR, MU, is_egm, trace_egm_regime
from pylcm_b200.spec import ParamResolver, trace_regime

EPS = np.finfo(np.float64).eps


def fc_slopes(f0, f1, d0, d1, h):
    """Fritsch-Carlson (1980) limited node slopes on one bracket."""
    delta = (f1 - f0) / h
    d0 = np.where(delta == 0.0, 0.0, d0)
    d1 = np.where(delta == 0.0, 0.0, d1)
    with np.errstate(all="ignore"):
        a = np.where(delta != 0.0, d0 / delta, 0.0)
        b = np.where(delta != 0.0, d1 / delta, 0.0)
    a = np.maximum(a, 0.0)
    b = np.maximum(b, 0.0)
    r2 = a * a + b * b
    tau = np.where(r2 > 9.0, 3.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 1.0)
    return tau * a * delta, tau * b * delta


def read_row(xq, xp, fp, dp=None):
    """Read a NaN-padded ascending row at queries xq (reference read rules)."""
    xq = np.asarray(xq, dtype=np.float64)
    L = int(np.sum(~np.isnan(xp)))
    if L == 0:
        return np.full(xq.shape, np.nan)
    if L == 1:
        return np.full(xq.shape, fp[0])
    x = xp[:L]
    f = fp[:L]
    idx = np.searchsorted(x, xq, side="right") - 1
    lo = np.clip(idx, 0, L - 2)
    x0, x1 = x[lo], x[lo + 1]
    f0, f1 = f[lo], f[lo + 1]
    h = x1 - x0
    with np.errstate(all="ignore"):
        t = np.where(h > 0, (xq - x0) / np.where(h > 0, h, 1.0), 0.0)
        lin = f0 + t * (f1 - f0)
        lin = np.where(h > 0, lin, f1)
        out = lin
        if dp is not None:
            d = dp[:L]
            d0, d1 = d[lo], d[lo + 1]
            ok = np.isfinite(f0) & np.isfinite(f1) & np.isfinite(d0) & np.isfinite(d1) & (h > 0) & (idx >= 0)
            e0, e1 = fc_slopes(f0, f1, d0, d1, np.where(h > 0, h, 1.0))
            t2, t3 = t * t, t * t * t
            herm = (2 * t3 - 3 * t2 + 1) * f0 + (t3 - 2 * t2 + t) * h * e0 + (-2 * t3 + 3 * t2) * f1 + (t3 - t2) * h * e1
            out = np.where(ok, herm, lin)
        neg = (np.isneginf(f0) | np.isneginf(f1)) & ~((xq == x0) & np.isfinite(f0)) & ~((xq == x1) & np.isfinite(f1))
        out = np.where(neg & (idx >= 0), -np.inf, out)
    out = np.where(idx >= L - 1, f[L - 1], out)
    return out


def _eval(expr, env, tr):
    return ir.evaluate(expr, env, {k: v for k, v in tr.param_values.items()})


def value_carry_marginal(spec, euler, V_arr, specs, res, period, age):
    """Marginal-value rows of a regime whose value array a DC-EGM regime
    reads (``egm/terminal.py:76-330``), in the value array's layout.

    Terminal regime: the derivative of its utility with respect to the Euler
    state at the grid nodes, zero where the value is -inf.  Grid-search
    regime: the value array's slope along the Euler axis -- ``np.gradient``'s
    second-order stencil where both neighbours are feasible (finite), the
    one-sided difference toward the single feasible neighbour, zero without
    one and at infeasible states (``terminal.py:272-314``).
    """
    V_arr = np.asarray(V_arr, dtype=np.float64).reshape(spec.state_shape)
    names = [a.name for a in spec.states]
    ax = names.index(euler)
    grid = spec.state(euler).grid.to_numpy()
    if spec.terminal:
        tr = trace_regime(spec, specs, res, ())
        dU = ir.diff(tr.U, ir.var("state", euler, "f"))
        idx = np.indices(spec.state_shape)
        env = {("period", "period"): period, ("age", "age"): age}
        for k, a in enumerate(spec.states):
            env[("state", a.name)] = grid[idx[k]] if a.name == euler else idx[k]
        with np.errstate(all="ignore"):
            mu = np.broadcast_to(np.asarray(_eval(dU, env, tr), dtype=np.float64), spec.state_shape)
        return np.where(np.isneginf(V_arr), 0.0, mu)
    v = np.moveaxis(V_arr, ax, -1)
    feas = np.isfinite(v)
    safe = np.where(feas, v, 0.0)
    fwd = np.diff(safe, axis=-1) / np.diff(grid)
    pad = np.zeros(v.shape[:-1] + (1,))
    right = np.concatenate([fwd, pad], axis=-1)
    left = np.concatenate([pad, fwd], axis=-1)
    fpad = np.zeros(v.shape[:-1] + (1,), dtype=bool)
    has_r = np.concatenate([feas[..., 1:], fpad], axis=-1)
    has_l = np.concatenate([fpad, feas[..., :-1]], axis=-1)
    interior = np.gradient(safe, grid, axis=-1) if len(grid) > 1 else np.zeros_like(safe)
    m = np.where(has_l & has_r, interior, np.where(has_r, right, np.where(has_l, left, 0.0)))
    m = np.where(feas, m, 0.0)
    return np.moveaxis(m, -1, ax)


def _value_child_read(tg, wlists, Rn, dR, V_arr, M_arr):
    """Continuation read of a carried value array: the expectation over the
    target's discrete states folded into the value and marginal rows (sum of
    w * row over the nodes with a non-zero weight), then one read at R'(A)
    on the target's Euler grid (``egm/continuation.py:551-674, 1460-1520``)."""
    spec = tg.spec
    names = [a.name for a in spec.states]
    ax = names.index(tg.value_euler)
    grid = spec.state(tg.value_euler).grid.to_numpy()
    V = np.moveaxis(np.asarray(V_arr, dtype=np.float64).reshape(spec.state_shape), ax, -1)
    M = np.moveaxis(np.asarray(M_arr, dtype=np.float64).reshape(spec.state_shape), ax, -1)
    fv = np.zeros(len(grid))
    fm = np.zeros(len(grid))
    for combo in itertools.product(*[range(len(w)) for w in wlists]):
        w = 1.0
        for wl, j in zip(wlists, combo):
            w *= wl[j]
        if w == 0.0:
            continue
        with np.errstate(all="ignore"):
            fv = fv + w * V[combo]
            fm = fm + w * M[combo]
    with np.errstate(all="ignore"):
        val = read_row(Rn, grid, fv, fm)
        mar = read_row(Rn, grid, fm)
        mar = np.where(np.isneginf(val), 0.0, mar * dR)
    return val, mar


def _weight_lists(tg, dstates, procs, env, tr):
    """Weights of each discrete state of a target: the process row, the
    Markov row or the one-hot deterministic law."""
    wlists = []
    for ax in dstates:
        law = tg.disc_laws[ax.name]
        if law.kind == "process":
            P = procs[law.source_process][1]
            wlists.append(P[env[("state", law.source_process)], :])
        elif law.kind == "markov":
            wlists.append(np.array([float(_eval(x, env, tr)) for x in law.expr.items]))
        else:
            k = int(_eval(law.expr, env, tr))
            w = np.zeros(ax.size)
            w[min(max(k, 0), ax.size - 1)] = 1.0
            wlists.append(w)
    return wlists


def egm_step(er, specs, res, period, age, carry_next, V_next, grid_R, value_mu=None):
    """Rows of V_d on the state grid and carry rows for one EGM regime.
    `value_mu` holds the marginal-value rows of the targets read as value
    arrays (terminal / grid-search regimes)."""
    tr = er.tracer
    procs = _process_tables(er.spec, res)
    beta = float(_eval(er.beta, {}, tr))
    A = er.savings
    nrow = er.n_rows
    nd = er.n_disc_actions
    n_g = len(grid_R)
    V_rows = np.full((nrow, n_g), np.nan)
    carry = {}
    for row in range(nrow):
        env = {("period", "period"): period, ("age", "age"): age}
        env.update(er.row_env(row))
        for a in er.disc_states:
            if a.kind == "process":
                env[("state", a.name)] = env[("state", a.name)]
        EV = np.zeros_like(A)
        EMU = np.zeros_like(A)
        mass = 0.0
        for tg in er.targets:
            p = float(_eval(tg.prob, env, tr))
            mass += p
            if p == 0.0:
                continue
            if tg.unreachable:
                EV = EV * np.nan
                continue
            if tg.next_R is None:
                EV = EV + p * float(np.asarray(V_next[tg.spec.name]))
                continue
            # joint distribution over the target's discrete states
            dstates = [a for a in tg.spec.states if a.kind != "continuous"]
            wlists = _weight_lists(tg, dstates, procs, env, tr)
            envA = dict(env)
            envA[("egm", "A")] = A
            Rn = np.broadcast_to(np.asarray(_eval(tg.next_R, envA, tr), dtype=np.float64), A.shape)
            dR = np.broadcast_to(np.asarray(_eval(tg.dR_dA, envA, tr), dtype=np.float64), A.shape)
            if tg.is_value:
                val, mar = _value_child_read(tg, wlists, Rn, dR, V_next[tg.spec.name], value_mu[tg.spec.name])
                with np.errstate(all="ignore"):
                    EV = EV + p * val
                    EMU = EMU + p * mar
                continue
            num_v = np.zeros_like(A)
            num_m = np.zeros_like(A)
            den = 0.0
            ct = carry_next[tg.spec.name]
            nd_t = int(np.prod([a.size for a in tg.spec.actions if a.kind != "continuous"])) or 1
            for combo in itertools.product(*[range(len(w)) for w in wlists]):
                w = 1.0
                for wl, j in zip(wlists, combo):
                    w *= wl[j]
                den += w
                if w == 0.0:
                    continue
                base = 0
                for ax, j in zip(dstates, combo):
                    base = base * ax.size + j
                vals, mus = [], []
                for d in range(nd_t):
                    g, v, mu = ct[base * nd_t + d]
                    vals.append(read_row(Rn, g, v, mu))
                    mus.append(read_row(Rn, g, mu))
                vals = np.stack(vals)
                mus = np.stack(mus)
                if tg.spec.taste_shocks:
                    lam = res.taste_scale(tg.spec.name)
                    vmax = vals.max(axis=0)
                    fin = np.where(np.isneginf(vmax), 0.0, vmax)
                    with np.errstate(all="ignore"):
                        ex = np.exp((vals - fin) / lam)
                        s = ex.sum(axis=0)
                        Vs = fin + lam * np.log(s)
                        prob = ex / np.where(s > 0, s, 1.0)
                    MUs = (prob * np.where(prob > 0, mus, 0.0)).sum(axis=0)
                else:
                    arg = vals.argmax(axis=0)
                    Vs = vals.max(axis=0)
                    MUs = mus[arg, np.arange(len(A))]
                with np.errstate(all="ignore"):
                    num_v = num_v + w * np.where((w == 0) & ~np.isfinite(Vs), 0.0, Vs)
                    num_m = num_m + w * MUs * dR
            with np.errstate(all="ignore"):
                EV = EV + p * (num_v / (den if den > 0 else 1.0))
                EMU = EMU + p * (num_m / (den if den > 0 else 1.0))
        if not (abs(mass - 1.0) <= 1e-3):
            EV = EV * np.nan
        elif mass != 1.0:
            EV, EMU = EV / mass, EMU / mass
        disc = beta * EMU
        with np.errstate(all="ignore"):
            tgt = np.where(disc < 0.0, np.nan, np.maximum(disc, EPS))
            envc = dict(env)
            envc[("egm", "mu")] = tgt
            c = np.broadcast_to(np.asarray(_eval(er.invmu, envc, tr), dtype=np.float64), A.shape)
            m = A + c
            envu = dict(env)
            envu[("action", er.C)] = c
            u = np.broadcast_to(np.asarray(_eval(er.U, envu, tr), dtype=np.float64), A.shape)
            v = u + beta * EV
        # constrained candidates
        span = min(m[0], float(np.max(grid_R))) - A[0]
        nc = er.n_constrained
        if span > 0.0 and np.isfinite(span):
            cc = span * 1e-4 * er.ratio ** np.arange(nc, dtype=np.float64)
            envk = dict(env)
            envk[("action", er.C)] = cc
            with np.errstate(all="ignore"):
                vc = np.broadcast_to(np.asarray(_eval(er.U, envk, tr), dtype=np.float64), cc.shape) + beta * EV[0]
        else:
            cc = np.full(nc, np.nan)
            vc = np.full(nc, np.nan)
        cand_g = np.concatenate([A[0] + cc, m])
        cand_c = np.concatenate([cc, c])
        cand_v = np.concatenate([vc, v])
        cand_s = np.concatenate([np.full(nc, A[0]), A])
        dead = np.isneginf(cand_v)
        cand_g = np.where(dead, np.nan, cand_g)
        cand_c = np.where(dead, np.nan, cand_c)
        cand_v = np.where(dead, np.nan, cand_v)
        cand_s = np.where(dead, np.nan, cand_s)
        if er.envelope == "ltm":
            rg, rc, rv, n_kept = refine_ltm(cand_g, cand_c, cand_v, er.n_pad)
        elif er.envelope == "mss":
            rg, rc, rv, n_kept = refine_mss(cand_g, cand_c, cand_v, er.n_pad)
        elif er.envelope == "rfc":
            # candidate supgradient u'(c), 0 for dead candidates (step_core.py:414-440)
            envm = dict(env)
            envm[("action", er.C)] = np.where(dead, 1.0, cand_c)
            with np.errstate(all="ignore"):
                cm = np.broadcast_to(np.asarray(_eval(er.dU, envm, tr), dtype=np.float64), cand_c.shape)
            cm = np.where(dead, 0.0, cm)
            rg, rc, rv, n_kept = refine_rfc(cand_g, cand_c, cand_v, cm, er.n_pad, er.search_radius, er.jump_thresh)
        else:
            rg, rc, rv, n_kept = refine(cand_g, cand_c, cand_v, cand_s, er.n_pad, er.jump_thresh,
                                        er.scan_window or None)
        envr = dict(env)
        envr[("action", er.C)] = np.where(np.isnan(rc), 1.0, rc)
        with np.errstate(all="ignore"):
            mu = np.broadcast_to(np.asarray(_eval(er.dU, envr, tr), dtype=np.float64), rc.shape).copy()
        mu = np.where(np.isnan(rc), np.nan, mu)
        mu = np.where(np.isneginf(rv), 0.0, mu)
        overflow = n_kept > er.n_pad
        val = read_row(grid_R, rg, rv, mu)
        cf = grid_R - A[0]
        envf = dict(env)
        envf[("action", er.C)] = np.maximum(cf, np.finfo(np.float64).tiny)
        with np.errstate(all="ignore"):
            ucf = np.broadcast_to(np.asarray(_eval(er.U, envf, tr), dtype=np.float64), cf.shape)
        vcons = np.where(cf > 0.0, ucf + beta * EV[0], -np.inf)
        Vr = np.where((cf > 0.0) & (grid_R <= rg[0]), vcons, np.maximum(val, vcons))
        if overflow:
            Vr[:] = np.nan
            rv = np.full_like(rv, np.nan)
            mu = np.full_like(mu, np.nan)
        if np.all(dead):
            Vr[:] = -np.inf
            rv = np.full_like(rv, -np.inf)
            mu = np.zeros_like(mu)
        feas = bool(np.all(_eval(er.feasible, env, tr)))
        if not feas:
            Vr[:] = -np.inf
            rv = np.full_like(rv, -np.inf)
            mu = np.zeros_like(mu)
        V_rows[row] = Vr
        carry[row] = (rg, rv, mu)
    # V over the regime's states: aggregate over discrete actions
    ns = nrow // er.n_disc_actions
    Vd = V_rows.reshape(ns, er.n_disc_actions, n_g)
    if er.taste_scale is not None:
        lam = er.taste_scale
        vmax = Vd.max(axis=1, keepdims=True)
        fin = np.where(np.isneginf(vmax), 0.0, vmax)
        with np.errstate(all="ignore"):
            V = fin[:, 0, :] + lam * np.log(np.exp((Vd - fin) / lam).sum(axis=1))
    else:
        V = Vd.max(axis=1)
    shape = tuple(a.size for a in er.disc_states) + (n_g,)
    return V.reshape(shape), carry, V_rows


def solve(model, params):
    """Backward induction where DCEGM regimes take the EGM step and the others
    grid search.  Returns (V, carry) dicts keyed by period then regime."""
    specs = model.regime_specs
    res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    T = model.n_periods
    V, carry = {}, {}
    for period in range(T - 1, -1, -1):
        age = float(model.ages.values[period])
        V[period], carry[period] = {}, {}
        for s in specs:
            if period not in s.active_periods:
                continue
            targets = tuple(x.name for x in specs if (period + 1) in x.active_periods) if not s.terminal else ()
            if is_egm(s) and not s.terminal:
                er = trace_egm_regime(s, specs, res, targets)
                grid_R = s.state(er.E).grid.to_numpy()
                vmu = {
                    t.spec.name: value_carry_marginal(t.spec, t.value_euler, V[period + 1][t.spec.name], specs, res,
                                                      period + 1, float(model.ages.values[period + 1]))
                    for t in er.targets if t.is_value and not t.unreachable
                }
                Vs, cr, _ = egm_step(er, specs, res, period, age, carry.get(period + 1, {}), V.get(period + 1, {}),
                                     grid_R, vmu)
                V[period][s.name] = Vs
                carry[period][s.name] = cr
            else:
                v, _ = bellman_step(s, specs, res, period, age, V.get(period + 1, {}))
                V[period][s.name] = v
    return V, carry
