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


def test_value_array_carry_marginals():
    """Marginal-value rows of carried value arrays: a terminal regime's
    utility gradient; a grid-search regime's finite-difference slope, one-
    sided next to an infeasible (-inf) neighbour, zero at infeasible states
    (restating ``egm/terminal.py:272-314``)."""
    import numpy as np

    from oracle.dcegm import value_carry_marginal
    from pylcm_b200.spec import ParamResolver
    from tests import models as M

    model = M.value_children_model()
    specs = model.regime_specs
    res = ParamResolver(M.value_children_params(), model.fixed_params, tuple(s.name for s in specs))
    by = {s.name: s for s in specs}
    w = by["done"].state("wealth").grid.to_numpy()
    mu = value_carry_marginal(by["done"], "wealth", np.zeros((2, len(w))), specs, res, 5, 5.0)
    np.testing.assert_allclose(mu[0], 2.0 * (w + 1.0) ** -2.0, rtol=1e-13)
    np.testing.assert_allclose(mu[1], 3.0 * (w + 1.0) ** -2.0, rtol=1e-13)
    # grid search: quadratic rows are differentiated exactly by the interior
    # stencil; the node next to -inf takes the one-sided slope
    V = np.stack([w ** 2, 3.0 * w + 1.0])
    V[:, 0] = -np.inf
    m = value_carry_marginal(by["retired"], "wealth", V, specs, res, 1, 1.0)
    assert (m[:, 0] == 0.0).all()
    np.testing.assert_allclose(m[0, 2:-1], 2.0 * w[2:-1], rtol=1e-12)
    np.testing.assert_allclose(m[0, 1], (w[2] ** 2 - w[1] ** 2) / (w[2] - w[1]), rtol=1e-14)
    np.testing.assert_allclose(m[0, -1], (w[-1] ** 2 - w[-2] ** 2) / (w[-1] - w[-2]), rtol=1e-14)
    np.testing.assert_allclose(m[1, 1:], 3.0, rtol=1e-12)


def test_value_children_model_oracle_is_finite_and_monotone():
    import numpy as np

    from tests import models as M

    V, _ = solve(M.value_children_model(taste=True), M.value_children_params(0.1))
    for p in V:
        for r, v in V[p].items():
            v = np.asarray(v)
            assert not np.isnan(v).any(), (p, r)
            fin = np.where(np.isfinite(v), v, -1e300)
            assert (np.diff(fin, axis=-1) >= -1e-9).all(), (p, r)
