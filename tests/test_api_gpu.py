"""The reference's solve keywords on the GPU path: the continuation's mass
check (``src/_lcm/regime_building/Q_and_F.py:1401-1432``) against the oracle,
and ``return_simulation_policy`` (``src/lcm/model.py:448, 517-518``) against
the DC-EGM oracle's refined rows."""

import numpy as np
import pytest

from tests import models as M
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize(
    "params",
    [M.mass_params(mass=1.0005), M.mass_params(mass=1.01), M.mass_params(p_survive=-0.1)],
    ids=["mass_within_1e-3", "mass_off_by_1e-2", "negative_weight"],
)
def test_mass_check_matches_the_oracle(params):
    """A continuation mass within 1e-3 of one is divided out; a larger
    deviation or a negative weight gives NaN -- at the same states, with the
    same values elsewhere, on the GPU and in the oracle."""
    from oracle.grid_search import solve as oracle_solve

    model = M.mass_model()
    V = model.solve(params=params, log_level="off")
    Vo, _ = oracle_solve(model, params)
    n_nan = 0
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-12, (p, r)
            n_nan += int(np.isnan(Vo[p][r]).sum())
    assert (n_nan > 0) == (params["mass"] != 1.0005)


def _rows_equal(a, b, tol):
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    fin = np.isfinite(b)
    np.testing.assert_array_equal(np.isfinite(a), fin)
    if fin.any():
        d = np.abs(a[fin] - b[fin]) / np.maximum(1.0, np.abs(b[fin]))
        assert d.max() < tol, d.max()


@pytest.mark.parametrize("taste", [None, 0.05])
def test_return_simulation_policy_publishes_the_dcegm_rows(taste):
    from oracle.dcegm import solve as oracle_solve

    model = M.dcegm_model(n_periods=5, n_savings=200, n_wealth=100, taste=taste is not None)
    params = M.dcegm_params(1, taste_scale=taste)
    V, pol = model.solve(params=params, log_level="off", return_simulation_policy=True)
    V0 = model.solve(params=params, log_level="off")
    for p in V0:
        for r in V0[p]:
            assert np.array_equal(V[p][r], V0[p][r], equal_nan=True)
    Vo, carry = oracle_solve(model, params)
    assert sorted(pol) == list(range(model.n_periods))
    assert dict(pol[model.n_periods - 1]) == {}
    for p in range(model.n_periods - 1):
        assert sorted(pol[p]) == ["retired", "working"]
        for name, sp in pol[p].items():
            rows = carry[p][name]
            n_rows = len(rows)
            g = sp.endog_grid.reshape(n_rows, -1)
            v = sp.value.reshape(n_rows, -1)
            mu = sp.marginal_utility.reshape(n_rows, -1)
            c = sp.policy.reshape(n_rows, -1)
            lead = (16, 2) if name == "working" else ()
            assert sp.endog_grid.shape[:-1] == lead
            for row in range(n_rows):
                rg, rv, rmu = rows[row]
                _rows_equal(g[row], rg, 1e-10)
                _rows_equal(v[row], rv, 1e-10)
                _rows_equal(mu[row], rmu, 1e-10)
                np.testing.assert_array_equal(np.isnan(c[row]), np.isnan(rg))


def test_grid_search_regimes_publish_no_simulation_policy():
    model = M.stochastic_model(4, 30, 40)
    V, pol = model.solve(params=M.stochastic_params(), log_level="off", return_simulation_policy=True)
    assert sorted(pol) == list(range(model.n_periods))
    assert all(len(d) == 0 for d in pol.values())
