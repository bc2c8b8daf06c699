"""DC-EGM + FUES oracle against the Iskhakov et al. (2017) closed-form solution.

The reference checks its grid-search solve against these fixtures at a loose
MSE (1 decimal); the endogenous-grid solve is far closer, so the bar here is
1e-3 absolute on every wealth node but the two lowest."""

import numpy as np
import pytest

from oracle.dcegm import read_row, solve
from tests.golden import analytical_models as AM


@pytest.mark.parametrize("case", ["five_periods", "low_delta"])
def test_dcegm_matches_the_closed_form(case):
    model, params = AM.dcegm_model_and_params(case)
    V, _ = solve(model, params)
    periods = sorted(V)
    for kind, reg in (("worker", "working_life"), ("retired", "retirement")):
        num = np.stack([V[p][reg] for p in periods[:-1]])
        ana = np.load(f"tests/golden/analytical_{case}__values_{kind}.npy")
        assert np.abs(num - ana)[:, 2:].max() < 1e-3


def test_row_read_rules():
    xp = np.array([1.0, 2.0, 2.0, 3.0, np.nan])
    fp = np.array([1.0, 2.0, 5.0, 6.0, np.nan])
    # below the first node: linear extrapolation; at/above the last: clamp;
    # at a duplicated abscissa: the right value
    np.testing.assert_allclose(read_row([0.0, 1.5, 2.0, 2.5, 3.0, 9.0], xp, fp), [0.0, 1.5, 5.0, 5.5, 6.0, 6.0])
