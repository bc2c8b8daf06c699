"""The reference's solve / simulate keyword contract (``src/lcm/model.py:440-519,
648-848``), checked on the host: unknown keywords raise, the reference's
optional keywords are accepted by name and validated."""

import warnings

import pytest

from pylcm_b200.model import _check_compat_kwargs
from tests import models as M


def test_unknown_solve_keywords_raise():
    model = M.retirement_model()
    with pytest.raises(TypeError):
        model.solve(params=M.retirement_params(), log_level="off", subject_batch_size=4)
    with pytest.raises(TypeError):
        model.solve(params=M.retirement_params(), log_level="off", not_a_keyword=True)


def test_unknown_simulate_keywords_raise():
    model = M.retirement_model()
    with pytest.raises(TypeError):
        model.simulate(params=M.retirement_params(), initial_conditions={}, log_level="off", return_policy=True)


def test_subject_batch_size_is_validated():
    model = M.retirement_model()
    with pytest.raises(ValueError, match="subject_batch_size"):
        model.simulate(params=M.retirement_params(), initial_conditions={}, log_level="off",
                       subject_batch_size=-1)


def test_reference_keywords_are_accepted_and_checked():
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        _check_compat_kwargs(None, None, 3)
        _check_compat_kwargs(4, None, 0)
    with pytest.raises(ValueError):
        _check_compat_kwargs(0, None, 3)
    with pytest.raises(ValueError):
        _check_compat_kwargs(None, None, -1)
    with pytest.warns(UserWarning, match="snapshots"):
        _check_compat_kwargs(None, "/tmp/lcm-logs", 3)
