"""The launch-shape autotuner: candidate set and failure rule on the host;
on the GPU, tuned shapes through BatchSolver keep the double-precision bars
(V within 1e-12 of the oracle, argmax identical where the gap exceeds 1e-9)."""

import numpy as np
import pytest

from pylcm_b200 import autotune
from pylcm_b200.engine import default_config
from pylcm_b200.exceptions import KernelError
from tests import models as M


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_candidates_start_with_the_heuristic_and_are_distinct(precision):
    model = M.stochastic_model(5, 40, 50)
    for spec in model.regime_specs:
        cands = autotune.candidates(spec, precision, 64)
        assert cands[0] == default_config(spec, precision, 64)
        assert len(set(cands)) == len(cands)
        for c in cands:
            assert c.block // c.lanes >= 8 and c.block in (128, 256)
            assert c.sb in ((1, 2, 4) if precision == "fp32" else (1, 2))


def test_only_compile_and_launch_refusals_are_skipped():
    assert autotune._skippable(KernelError(2, "nvrtc"))
    assert autotune._skippable(KernelError(4, "too many resources"))
    assert not autotune._skippable(KernelError(5, "an illegal memory access"))
    assert not autotune._skippable(RuntimeError("CUDA error: unspecified launch failure"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tuned_shapes_keep_the_bars(precision, tmp_path, monkeypatch):
    from oracle.grid_search import solve as oracle_solve
    from pylcm_b200.batch import BatchSolver
    from tests.conftest import rel_err

    monkeypatch.setattr(autotune, "CACHE", tmp_path / "autotune.json")
    model = M.stochastic_model(5, 60, 80)
    ps = [M.stochastic_params(beta=b, crra=c) for b, c in ((0.95, 2.0), (0.9, 3.0))]
    bs = BatchSolver(model, len(ps), precision, template_params=ps[0], autotune=True)
    assert (tmp_path / "autotune.json").exists()
    assert bs.configs, "the tuner picked a shape for the regimes"
    Vs, Ps = bs.solve(ps, return_policy=True)
    for p_, V, P in zip(ps, Vs, Ps):
        gaps: dict = {}
        Vo, Po = oracle_solve(model, p_, gaps=gaps)
        for per in Vo:
            for r in Vo[per]:
                bar = 1e-12 if precision == "fp64" else 1e-6
                assert rel_err(V[per][r], Vo[per][r]) < bar, (per, r)
                g = gaps[per][r] / np.maximum(1.0, np.abs(np.nan_to_num(Vo[per][r], neginf=0.0)))
                sel = g > (1e-9 if precision == "fp64" else 1e-5)
                np.testing.assert_array_equal(np.asarray(P[per][r])[sel], Po[per][r][sel])
    # a second solver reads the cached shapes
    bs2 = BatchSolver(model, len(ps), precision, template_params=ps[0], autotune=True)
    assert bs2.configs == bs.configs
