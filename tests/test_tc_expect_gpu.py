"""The tensor-core (tcgen05, 3xTF32) form of kernel (b) against the FP64
contraction of the same plan.

In the single-precision search form the float expectation table the search
reads comes from ``lcm_expect_tc_*``; the double table (the FP64
re-evaluation, the simulation) still comes from the FP64 kernel.  Bar: the
float table within 2e-6 of the double one, |a-b| <= 2e-6 max(1, |b|) (3xTF32
keeps about FP32 resolution: the split drops only the lo x lo product), with
identical non-finite entries (columns with an infeasible node are
recomputed in FP64 with the zero-safe rule)."""

import numpy as np
import pytest

from tests import models as M

pytestmark = pytest.mark.gpu

CASES = {
    # 32-state Markov shock (K = J = 32), wealth x human capital
    "markov32": (lambda: M.hc_model(3, 40, 5, 32, 30), lambda: [M.hc_params(s) for s in range(3)]),
    # 7-node Tauchen income (K = J = 7: reduction padded to 8, N to 16)
    "tauchen7": (lambda: M.stochastic_model(3, 300, 60), lambda: [M.stochastic_params(beta=b) for b in (0.9, 0.95)]),
    # Markov health x Gauss-Hermite income process (K = J = 10)
    "health_x_process": (lambda: M.processes_model(4, "tauchen"), lambda: [M.processes_params("tauchen")]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_tensor_core_table_matches_the_fp64_contraction(case):
    import torch

    from pylcm_b200.engine import SolveEngine

    model = CASES[case][0]()
    ps = CASES[case][1]()
    plan = SolveEngine(model, "fp32").plan(ps)
    tc = [l for l in plan.launches if l.kind == "expect_tc"]
    assert tc, "the single-precision form should use the tensor-core expectation"
    checked = 0
    for period in sorted({l.period for l in tc}):
        # run the plan up to this period's expectation launches
        plan_prepared = plan._prepare()
        stream = torch.cuda.current_stream().cuda_stream
        for l, launch in zip(plan.launches, plan_prepared):
            if l.period < period:
                break
            launch(stream)
        torch.cuda.synchronize()
        plan.check_status()
        for (src, targets, tname), (e64, e32, ncols, cblk) in plan.ev.items():
            if e32 is None:
                continue
            a = e32.double().cpu().numpy()
            b = e64.cpu().numpy()
            fa, fb = np.isfinite(a), np.isfinite(b)
            np.testing.assert_array_equal(fa, fb)
            np.testing.assert_array_equal(a[~fa], b[~fb])
            d = np.abs(a[fb] - b[fb]) / np.maximum(1.0, np.abs(b[fb]))
            assert d.max() <= 2e-6, (case, period, tname, d.max())
            checked += 1
    assert checked > 0


def test_fp32_solve_with_tensor_core_table_meets_the_bars():
    """Single-precision search on the tensor-core table: V within 1e-6 of the
    FP64 oracle, >= 99.9 % policy agreement, identical argmax where the
    relative gap exceeds 1e-5."""
    from oracle.grid_search import solve as oracle_solve
    from tests.conftest import rel_err

    model = M.hc_model(4, 40, 6, 32, 30)
    params = M.hc_params(3)
    V, pol = model.solve(params=params, precision="fp32", return_policy=True, log_level="off")
    gaps: dict = {}
    Vo, Po = oracle_solve(model, params, gaps=gaps)
    n_all = n_agree = 0
    for p in Vo:
        for r in Vo[p]:
            assert rel_err(V[p][r], Vo[p][r]) < 1e-6, (p, r)
            g = gaps[p][r] / np.maximum(1.0, np.abs(np.nan_to_num(Vo[p][r], neginf=0.0)))
            same = np.asarray(pol[p][r]) == Po[p][r]
            assert same[g > 1e-5].all(), (p, r)
            n_all += same.size
            n_agree += int(same.sum())
    assert n_agree >= 0.999 * n_all, (n_agree, n_all)
