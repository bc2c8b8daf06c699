"""Full-size parity of the benchmark configurations against the oracle.

Each check takes the GPU's own next-period arrays (value arrays, and for
DC-EGM the refined carry rows that ``return_simulation_policy`` publishes),
runs the oracle's step for one period on them and compares the result with
the GPU's arrays of that period, so the horizon adds no error of its own:

- config 1 (stochastic retirement model: 7-node Tauchen income, wealth and
  consumption 500 / 500, work / retire, T = 40): every state at periods
  T-2, T-3, 20 and 0;
- config 3 (32-state Markov shock x wealth 1000 x human capital 50, 300 x 3
  actions, T = 60): 2000 seeded state rows per checked period;
- config 2 (DC-EGM + FUES retirement model, 2000-point savings and wealth
  grids, 16 Gauss-Hermite income nodes, T = 40, taste scale none / 0.05):
  value arrays and refined rows of both DC-EGM regimes.

Bars, as the reference's ``tests/conftest.py:36`` (12 decimals) for the
double-precision path: V within 1e-12 by |a-b| / max(1, |b|) and by the pure
relative error |a-b| / |b| (both reported); argmax identical wherever the
best-to-second-best gap exceeds 1e-9 relative.  Single-precision search: V
within 1e-6, >= 99.9 % policy agreement, identical argmax where the relative
gap exceeds 1e-5.  DC-EGM: see ``DCEGM_BAR``.
"""

import numpy as np
import pytest

from oracle import dcegm as OD
from oracle import grid_search as OG
from pylcm_b200.egm import is_egm, trace_egm_regime
from pylcm_b200.spec import ParamResolver
from tests import models as M

pytestmark = pytest.mark.gpu

# DC-EGM double precision: the GPU and the oracle insert FUES crossings and
# evaluate the cubic Hermite reads with different roundings (the device
# contracts a*b+c into one fused multiply-add, NumPy rounds the product
# first), so refined rows and values agree to a few ulps of the largest term
# of each expression rather than of the result.
DCEGM_BAR = 1e-10


def _errs(a, b):
    """(max |a-b|/max(1,|b|), max |a-b|/|b|) over entries finite in both;
    the non-finite patterns must be equal."""
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_array_equal(np.isposinf(a), np.isposinf(b))
    np.testing.assert_array_equal(np.isneginf(a), np.isneginf(b))
    fin = np.isfinite(b)
    if not fin.any():
        return 0.0, 0.0
    d = np.abs(a[fin] - b[fin])
    with np.errstate(divide="ignore", invalid="ignore"):
        pure = np.where(b[fin] != 0, d / np.abs(b[fin]), np.where(d == 0, 0.0, np.inf))
    return float((d / np.maximum(1.0, np.abs(b[fin]))).max()), float(pure.max())


def _one_step(model, params, V, periods, n_rows=None, seed=0):
    """Oracle Bellman step of every grid-search regime at each period, fed
    the GPU's value arrays of the next period: yields (regime, period,
    state rows, V, policy, gap)."""
    specs = model.regime_specs
    res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    rng = np.random.default_rng(seed)
    for period in periods:
        age = float(model.ages.values[period])
        nxt = {s.name: np.asarray(V[period + 1][s.name]) for s in specs
               if (period + 1) in s.active_periods} if period + 1 < model.n_periods else {}
        for s in specs:
            if period not in s.active_periods or is_egm(s):
                continue
            rows = None
            if n_rows is not None and s.n_states > n_rows:
                rows = np.sort(rng.choice(s.n_states, n_rows, replace=False))
            Vo, Po = OG.bellman_step(s, specs, res, period, age, nxt, state_rows=rows)
            yield s.name, period, rows, np.asarray(Vo).reshape(-1), np.asarray(Po).reshape(-1), OG.LAST_GAP


def _check_fp64(model, params, periods, n_rows=None):
    V, pol = model.solve(params=params, precision="fp64", return_policy=True, log_level="off")
    worst = [0.0, 0.0]
    n_checked = 0
    for name, period, rows, Vo, Po, gap in _one_step(model, params, V, periods, n_rows):
        g = np.asarray(V[period][name]).reshape(-1)
        p = np.asarray(pol[period][name]).reshape(-1)
        if rows is not None:
            g, p = g[rows], p[rows]
        e_abs, e_rel = _errs(g, Vo)
        worst = [max(worst[0], e_abs), max(worst[1], e_rel)]
        sel = gap / np.maximum(1.0, np.abs(np.nan_to_num(Vo, neginf=0.0))) > 1e-9
        np.testing.assert_array_equal(p[sel], Po[sel], err_msg=f"{name} period {period}")
        n_checked += Vo.size
    assert worst[0] < 1e-12 and worst[1] < 1e-12, (worst, n_checked)
    return worst


def _check_fp32(model, params, periods, n_rows=None):
    V, pol = model.solve(params=params, precision="fp32", return_policy=True, log_level="off")
    worst = [0.0, 0.0]
    n_all = n_agree = 0
    for name, period, rows, Vo, Po, gap in _one_step(model, params, V, periods, n_rows):
        g = np.asarray(V[period][name]).reshape(-1)
        p = np.asarray(pol[period][name]).reshape(-1)
        if rows is not None:
            g, p = g[rows], p[rows]
        e_abs, e_rel = _errs(g, Vo)
        worst = [max(worst[0], e_abs), max(worst[1], e_rel)]
        rel_gap = gap / np.maximum(1.0, np.abs(np.nan_to_num(Vo, neginf=0.0)))
        sel = rel_gap > 1e-5
        np.testing.assert_array_equal(p[sel], Po[sel], err_msg=f"{name} period {period}")
        n_all += p.size
        n_agree += int((p == Po).sum())
    assert worst[0] < 1e-6 and worst[1] < 1e-6, worst
    assert n_agree >= 0.999 * n_all, (n_agree, n_all)
    return worst, n_agree / n_all


# ---------------------------------------------------------------- config 1
def test_config1_fp64_full_size_one_step():
    model = M.stochastic_model(40, 500, 500, 7)
    _check_fp64(model, M.stochastic_params(), periods=(39, 38, 37, 20, 0))


def test_config1_fp32_full_size_one_step():
    model = M.stochastic_model(40, 500, 500, 7)
    _check_fp32(model, M.stochastic_params(beta=0.95, crra=3.0, interest_rate=0.03), periods=(38, 37, 20, 0))


# ---------------------------------------------------------------- config 3
def test_config3_fp64_full_size_sampled_rows():
    model = M.hc_model()
    _check_fp64(model, M.hc_params(1), periods=(59, 58, 57, 30, 0), n_rows=2000)


def test_config3_fp32_full_size_sampled_rows():
    model = M.hc_model()
    _check_fp32(model, M.hc_params(2), periods=(58, 57, 30, 0), n_rows=2000)


# ---------------------------------------------------------------- config 2
@pytest.mark.parametrize("taste", [None, 0.05])
def test_config2_dcegm_full_size_one_step(taste):
    model = M.dcegm_model(40, 2000, 2000, taste=taste is not None)
    params = M.dcegm_params(0, taste_scale=taste)
    V, pub = model.solve(params=params, log_level="off", return_simulation_policy=True)
    specs = model.regime_specs
    res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    worst = {"V": [0.0, 0.0], "rows": [0.0, 0.0]}
    for period in (38, 37, 20, 0):
        age = float(model.ages.values[period])
        nxt_V = {s.name: np.asarray(V[period + 1][s.name]) for s in specs if (period + 1) in s.active_periods}
        carry_next = {}
        for name, sp in pub[period + 1].items():
            g = sp.endog_grid.reshape(-1, sp.endog_grid.shape[-1])
            v = sp.value.reshape(g.shape)
            mu = sp.marginal_utility.reshape(g.shape)
            carry_next[name] = {r: (g[r], v[r], mu[r]) for r in range(g.shape[0])}
        for s in specs:
            if period not in s.active_periods or s.terminal or not is_egm(s):
                continue
            targets = tuple(x.name for x in specs if (period + 1) in x.active_periods)
            er = trace_egm_regime(s, specs, res, targets)
            grid_R = s.state(er.E).grid.to_numpy()
            Vs, rows, _ = OD.egm_step(er, specs, res, period, age, carry_next, nxt_V, grid_R, {})
            e = _errs(V[period][s.name], Vs)
            worst["V"] = [max(x, y) for x, y in zip(worst["V"], e)]
            sp = pub[period][s.name]
            g = sp.endog_grid.reshape(len(rows), -1)
            v = sp.value.reshape(g.shape)
            mu = sp.marginal_utility.reshape(g.shape)
            for r, (rg, rv, rmu) in rows.items():
                for a, b in ((g[r], rg), (v[r], rv), (mu[r], rmu)):
                    e = _errs(a, b)
                    worst["rows"] = [max(x, y) for x, y in zip(worst["rows"], e)]
    assert max(worst["V"]) < DCEGM_BAR and max(worst["rows"]) < DCEGM_BAR, worst
