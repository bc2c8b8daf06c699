"""Cross-check against an independent implementation: the IJRS retirement
model with EV1 taste shocks (scale 0.2) solved by the `dcegm` package (the
reference's fixture, extracted to `tests/golden/ijrs_taste_shocks_reference.npz`).
The smoothed value scale * logsumexp([value_work, value_retire] / scale) must
match the brute-force twin's V at the fixture's wealth nodes up to
consumption-grid resolution (rtol = atol = 2e-2, the reference's bar); the
retiree rows at wealth 1 are left out as the reference does (the fixture run's
uniform savings grid under-resolves them)."""

import numpy as np
import pytest

from tests import models as M
from tests.conftest import GOLDEN

SCALE = 0.2
REGIME = {0: "working_life", 1: "retirement"}


def _fixture():
    d = np.load(GOLDEN / "ijrs_taste_shocks_reference.npz")
    vals = np.stack([d["value_work"], d["value_retire"]], axis=1)
    m = np.nanmax(vals, axis=1)
    emax = m + SCALE * np.log(np.nansum(np.exp((vals - m[:, None]) / SCALE), axis=1))
    keep = ~((d["lagged_choice"] == 1) & (d["wealth"] == 1.0))
    return d["period"][keep].astype(int), d["lagged_choice"][keep].astype(int), d["wealth"][keep], emax[keep]


def _check(V):
    grid = np.asarray(M.ijrs_wealth_points())
    period, lag, wealth, emax = _fixture()
    idx = np.searchsorted(grid, wealth - 1e-12)
    np.testing.assert_allclose(grid[idx], wealth, atol=1e-12)
    for p, l, i, e in zip(period, lag, idx, emax):
        got = float(np.asarray(V[p][REGIME[l]])[i])
        np.testing.assert_allclose(got, e, rtol=2e-2, atol=2e-2, err_msg=f"period {p}, regime {REGIME[l]}")


def test_oracle_brute_force_twin_matches_the_independent_solution():
    from oracle.grid_search import solve as oracle_solve

    V, _ = oracle_solve(M.ijrs_brute_model(), M.ijrs_params(SCALE))
    _check(V)


@pytest.mark.gpu
def test_gpu_brute_force_twin_matches_the_independent_solution():
    V = M.ijrs_brute_model().solve(params=M.ijrs_params(SCALE))
    _check(V)
