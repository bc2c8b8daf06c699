"""Normal-mixture processes (``processes/ar1.py:206-320``, ``iid.py:211-300``):
their node and transition tables against a direct restatement of the
mixture-CDF binning, and -- on the GPU -- solve and simulation of a model
holding both, against the oracle."""

import numpy as np
import pytest
from scipy.stats import norm

from pylcm_b200 import NormalMixtureIIDProcess, TauchenNormalMixtureAR1Process
from tests import models as M
from tests.conftest import rel_err

MIX = dict(p1=0.3, mu1=0.2, sigma1=0.1, mu2=-0.1, sigma2=0.4)


def _cdf(x, p1, mu1, sigma1, mu2, sigma2):
    return p1 * norm.cdf(x, mu1, sigma1) + (1 - p1) * norm.cdf(x, mu2, sigma2)


def _moments(p1, mu1, sigma1, mu2, sigma2):
    m = p1 * mu1 + (1 - p1) * mu2
    return m, p1 * (sigma1**2 + mu1**2) + (1 - p1) * (sigma2**2 + mu2**2) - m**2


def test_ar1_mixture_tables():
    proc = TauchenNormalMixtureAR1Process(n_points=7)
    kw = dict(rho=0.9, mu=0.05, n_std=3.0, **MIX)
    nodes = proc.compute_gridpoints(**kw)
    P = proc.compute_transition_probs(**kw)
    m, v = _moments(**MIX)
    lrm, sd = (0.05 + m) / (1 - 0.9), np.sqrt(v / (1 - 0.81))
    np.testing.assert_allclose(nodes, np.linspace(lrm - 3 * sd, lrm + 3 * sd, 7), rtol=1e-14)
    h = nodes[1] - nodes[0]
    for i in range(7):
        z = nodes - 0.05 - 0.9 * nodes[i]
        row = _cdf(z + h / 2, **MIX) - _cdf(z - h / 2, **MIX)
        row[0] = _cdf(z[0] + h / 2, **MIX)
        row[-1] = 1 - _cdf(z[-1] - h / 2, **MIX)
        np.testing.assert_allclose(P[i], row, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(P.sum(axis=1), 1.0, rtol=1e-12)


def test_iid_mixture_tables():
    proc = NormalMixtureIIDProcess(n_points=5)
    kw = dict(n_std=2.0, **MIX)
    nodes = proc.compute_gridpoints(**kw)
    P = proc.compute_transition_probs(**kw)
    m, v = _moments(**MIX)
    np.testing.assert_allclose(nodes, np.linspace(m - 2 * np.sqrt(v), m + 2 * np.sqrt(v), 5), rtol=1e-14)
    h = nodes[1] - nodes[0]
    w = _cdf(nodes + h / 2, **MIX) - _cdf(nodes - h / 2, **MIX)
    w[0], w[-1] = _cdf(nodes[0] + h / 2, **MIX), 1 - _cdf(nodes[-1] - h / 2, **MIX)
    assert (P == P[0]).all()
    np.testing.assert_allclose(P[0], w, rtol=1e-12)


def _ic(n, kind="ar1"):
    rng = np.random.default_rng(2)
    ic = {"wealth": rng.uniform(1, 15, n), "income": rng.normal(0, 0.3, n), "age": np.zeros(n),
          "regime_id": np.zeros(n, dtype=int)}
    if kind == "two":
        ic["shock"] = rng.normal(0, 1.5, n)
    return ic


@pytest.mark.parametrize("kind", ["ar1", "iid", "two"])
def test_oracle_solves_and_simulates_a_mixture_model(kind):
    from oracle.grid_search import solve
    from oracle.simulate import simulate

    model = M.mixture_model(kind)
    V, _ = solve(model, M.mixture_params(kind))
    assert all(np.isfinite(np.asarray(v)).all() for d in V.values() for v in d.values())
    out = simulate(model, M.mixture_params(kind), _ic(40, kind), seed=5)
    inc = np.concatenate([out[p]["states"]["income"] for p in range(1, M.MIX_N_PERIODS - 1)])
    assert np.isfinite(inc).all() and inc.std() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ar1", "iid", "two"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gpu_mixture_model_solve_matches_oracle(precision, kind):
    from oracle.grid_search import solve

    model = M.mixture_model(kind)
    for params in (M.mixture_params(kind), M.mixture_params(kind, p1=0.5)):
        V = model.solve(params=params, precision=precision, log_level="off")
        Vo, _ = solve(model, params)
        for p in Vo:
            for r in Vo[p]:
                assert rel_err(V[p][r], Vo[p][r]) < (1e-12 if precision == "fp64" else 1e-6), (p, r)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ar1", "iid", "two"])
def test_gpu_mixture_model_simulation_matches_oracle(kind):
    """"two": a target reached with two process laws, whose simulated
    expectation is taken node by node."""
    from oracle.simulate import simulate

    model = M.mixture_model(kind)
    params = M.mixture_params(kind)
    ic = _ic(64, kind)
    res = model.simulate(params=params, initial_conditions=ic, seed=5)
    ora = simulate(model, params, ic, seed=5)
    for p in ora:
        np.testing.assert_array_equal(res.periods[p]["regime_id"], ora[p]["regime_id"])
        for name in ("wealth", "income") + (("shock",) if kind == "two" else ()):
            np.testing.assert_allclose(res.periods[p]["states"][name], ora[p]["states"][name], rtol=1e-9, atol=1e-9,
                                       equal_nan=True)
        np.testing.assert_allclose(res.periods[p]["value"], ora[p]["value"], rtol=1e-9, atol=1e-9, equal_nan=True)
