"""The reference's stored float64 simulation of its mortality example (three
regimes, 10-year periods, survival probabilities indexed by period in Markov
regime transitions), as in its ``test_regression_mortality``.

With the reference's own seed and subject count the simulation is reproduced
row for row (``tests/test_jax_stream.py``).  Here a larger population under
another seed: survival is drawn, so a subject is compared over the periods
its regime path matches the stored one (every subject retires at 40; most
survive to 60); there values, states and choices agree at the reference's
atol of 1e-5."""

import numpy as np
import pytest

from tests import models as M
from tests.conftest import GOLDEN

N = 32


def _ic():
    return {"wealth": np.full(N, 100.0), "age": np.full(N, 40.0), "regime_id": np.zeros(N, dtype=int)}


def _check(periods):
    g = np.load(GOLDEN / "mortality_simulation.npz")
    sel = g["subject_id"] == 0
    path = g["regime"][sel]
    names = {s.rid: s.name for s in M.mortality_model().regime_specs}
    full = 0
    for subj in range(N):
        matched = 0
        for p in range(len(path)):
            rid = int(np.asarray(periods[p]["regime_id"])[subj])
            if names.get(rid) != path[p]:
                break
            matched += 1
            if path[p] == "dead":
                continue
            np.testing.assert_allclose(np.asarray(periods[p]["value"])[subj], g["value"][sel][p], atol=1e-5)
            np.testing.assert_allclose(np.asarray(periods[p]["states"]["wealth"])[subj], g["wealth"][sel][p], atol=1e-5)
            np.testing.assert_allclose(np.asarray(periods[p]["actions"]["consumption"])[subj],
                                       g["consumption"][sel][p], atol=1e-5)
            if path[p] == "working_life":
                assert int(np.asarray(periods[p]["actions"]["labor_supply"])[subj]) == M.LaborSupply.retire
        assert matched >= 1  # period 0 (working life, retiring) is every subject's
        full += matched == len(path)
    assert full >= N // 2


def test_oracle_reproduces_the_reference_mortality_simulation():
    from oracle.simulate import simulate

    _check(simulate(M.mortality_model(), M.mortality_params(), _ic(), seed=3))


@pytest.mark.gpu
def test_gpu_reproduces_the_reference_mortality_simulation():
    res = M.mortality_model().simulate(params=M.mortality_params(), initial_conditions=_ic(), seed=3)
    _check(res.periods)
