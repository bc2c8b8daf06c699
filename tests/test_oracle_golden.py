"""The CPU oracle reproduces the reference's stored float64 solutions.

Golden vectors: the reference's ``tests/data/regression_tests/solution.pkl``
and ``tests/data/processes/solution_*.pkl`` (extracted by
``tests/golden/make_golden.py``).  The reference asserts them at 5 decimals;
the oracle matches them to ~1e-15.
"""

import numpy as np
import pytest

from oracle.grid_search import solve as oracle_solve
from tests import models as M
from tests.conftest import load_golden, rel_err


def test_regression_solution_matches_reference():
    golden = load_golden("regression_solution.npz")
    V, _ = oracle_solve(M.regression_model(4), M.regression_params(4))
    for period, regs in golden.items():
        for regime, ref in regs.items():
            assert rel_err(V[period][regime], ref) < 1e-14, (period, regime)


@pytest.mark.parametrize("kind", ["uniform", "normal", "lognormal", "tauchen", "rouwenhorst"])
def test_processes_solution_matches_reference(kind):
    golden = load_golden(f"processes_solution_{kind}.npz")
    V, _ = oracle_solve(M.processes_model(4, kind), M.processes_params(kind))
    for period, regs in golden.items():
        for regime, ref in regs.items():
            assert rel_err(V[period][regime], ref) < 1e-14, (kind, period, regime)


def test_oracle_planted_mistake_is_detected():
    """A planted error in the oracle's inputs (wrong discount factor) must
    break the golden comparison: the check has teeth."""
    golden = load_golden("regression_solution.npz")
    V, _ = oracle_solve(M.regression_model(4), M.regression_params(4, discount_factor=0.951))
    assert rel_err(V[0]["working_life"], golden[0]["working_life"]) > 1e-6


def test_analytical_retirement_model_is_close():
    """Iskhakov et al. (2017) closed form (loose, like the reference's own
    test: MSE over periods at 1 decimal, first two wealth nodes excluded)."""
    from tests.golden import analytical_models as AM

    for case in ("five_periods", "low_delta"):
        model, params = AM.model_and_params(case)
        V, _ = oracle_solve(model, params)
        periods = sorted(V)
        worker = np.stack([V[p]["working_life"] for p in periods[:-1]])
        retired = np.stack([V[p]["retirement"] for p in periods[:-1]])
        for kind, num in (("worker", worker), ("retired", retired)):
            ana = np.load(f"tests/golden/analytical_{case}__values_{kind}.npy")
            mse = np.mean((ana - num) ** 2, axis=0)
            # numpy's assert_array_almost_equal(mse, 0, decimal=1): |mse| < 1.5e-1
            assert np.all(np.abs(mse[2:]) < 1.5e-1)
