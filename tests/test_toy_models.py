"""Pen-and-paper toy model (discrete actions only): the solved value
functions against the analytic ones, as the reference checks
(`tests/test_solution_on_toy_model_deterministic.py`: interior points of the
first period, all points of the second, decimal 12)."""

import numpy as np
import pytest

from oracle.grid_search import solve as oracle_solve
from tests import models as M

CASES = [(b, n) for b in (0.0, 0.5, 0.9, 1.0) for n in (100, 1000)]


def _check(V, n, beta):
    w = np.linspace(0.0, 2.0, n)
    v0, v1 = M.toy_deterministic_analytic(w, beta)
    np.testing.assert_array_almost_equal(np.asarray(V[0]["alive"])[1:-1], v0[1:-1], decimal=12)
    np.testing.assert_array_almost_equal(np.asarray(V[1]["alive"]), v1, decimal=12)


@pytest.mark.parametrize("beta,n", CASES)
def test_oracle_matches_the_analytic_solution(beta, n):
    V, _ = oracle_solve(M.toy_deterministic_model(n), M.toy_deterministic_params(beta))
    _check(V, n, beta)


@pytest.mark.gpu
@pytest.mark.parametrize("beta,n", CASES)
def test_gpu_matches_the_analytic_solution(beta, n):
    V = M.toy_deterministic_model(n).solve(params=M.toy_deterministic_params(beta))
    _check(V, n, beta)


P_CASES = [[[0.9, 0.1], [0.2, 0.8]], [[0.9, 0.1], [0.0, 1.0]], [[0.5, 0.5], [0.2, 0.8]]]
S_CASES = [(b, n, k) for b in (0.0, 0.5, 0.9, 1.0) for n in (100, 1000) for k in range(3)]


def _check_stochastic(V, n, beta, P):
    w = np.linspace(0.0, 2.0, n)
    V0 = np.asarray(V[0]["alive"])
    V1 = np.asarray(V[1]["alive"])
    health_axis = 0 if V0.shape[0] == 2 else 1
    for h in (0, 1):
        v0, _, _ = M.toy_stochastic_analytic(w, np.full(n, h), beta, P)
        got0 = V0[h] if health_axis == 0 else V0[:, h]
        got1 = V1[h] if health_axis == 0 else V1[:, h]
        np.testing.assert_array_almost_equal(got0[1:-1], v0[1:-1], decimal=12)
        np.testing.assert_array_almost_equal(got1, M.toy_stochastic_v1(w, np.full(n, h)), decimal=12)


@pytest.mark.parametrize("beta,n,k", S_CASES)
def test_stochastic_oracle_matches_the_analytic_solution(beta, n, k):
    P = P_CASES[k]
    V, _ = oracle_solve(M.toy_stochastic_model(n), M.toy_stochastic_params(beta, P))
    _check_stochastic(V, n, beta, P)


@pytest.mark.gpu
@pytest.mark.parametrize("beta,n,k", S_CASES)
def test_stochastic_gpu_matches_the_analytic_solution(beta, n, k):
    P = P_CASES[k]
    V = M.toy_stochastic_model(n).solve(params=M.toy_stochastic_params(beta, P))
    _check_stochastic(V, n, beta, P)


@pytest.mark.gpu
@pytest.mark.parametrize("beta,k", [(0.5, 0), (0.9, 1), (1.0, 2)])
def test_stochastic_simulation_follows_the_analytic_policy(beta, k):
    """Given the simulated period-1 health, the simulated values, wealth and
    choices are the analytic ones (the draws are this package's counter RNG,
    so the health path itself is not compared)."""
    P = P_CASES[k]
    model = M.toy_stochastic_model(100)
    w0 = np.array([0.25, 0.75, 1.25, 1.75, 2.0])
    h0 = np.array([0, 1, 0, 1, 1])
    ic = {"wealth": w0, "health": h0.astype(float), "age": np.zeros(5), "regime_id": np.zeros(5, dtype=int)}
    res = model.simulate(params=M.toy_stochastic_params(beta, P), initial_conditions=ic, seed=3)
    p0, p1 = res.periods[0], res.periods[1]
    v0, c0, l0 = M.toy_stochastic_analytic(w0, h0, beta, P)
    # rows at the wealth boundary (2) are left out, as the reference does: there
    # the grid interpolation of next period's step-shaped value differs from
    # the pen-and-paper value
    k0 = w0 != 2.0
    np.testing.assert_array_almost_equal(p0["value"][k0], v0[k0], decimal=12)
    np.testing.assert_array_equal(p0["actions"]["consumption"][k0], c0[k0])
    np.testing.assert_array_equal(p0["actions"]["labor_supply"][k0], l0[k0])
    w1 = w0 - c0 + l0
    np.testing.assert_array_almost_equal(p1["states"]["wealth"][k0], w1[k0], decimal=12)
    h1 = p1["states"]["health"].astype(int)
    k1 = k0 & (w1 != 2.0)
    np.testing.assert_array_almost_equal(p1["value"][k1], M.toy_stochastic_v1(w1, h1)[k1], decimal=12)
