"""GPU solve vs the CPU oracle (parity tests proper; call through the C ABI).

Bars: fp64 -- V within 1e-12 (|a-b| / max(1, |b|)), argmax identical wherever
the oracle's best-to-second-best gap exceeds 1e-9; fp32 search with fp64
re-evaluation -- V within 1e-6 and >= 99.9 % policy agreement.
"""

import numpy as np
import pytest

from oracle.grid_search import solve as oracle_solve
from tests import models as M
from tests.conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu

CASES = {
    "regression": (lambda: M.regression_model(4), lambda: M.regression_params(4)),
    "proc_tauchen": (lambda: M.processes_model(4, "tauchen"), lambda: M.processes_params("tauchen")),
    "proc_rouwenhorst": (lambda: M.processes_model(5, "rouwenhorst"), lambda: M.processes_params("rouwenhorst")),
    "proc_uniform": (lambda: M.processes_model(4, "uniform"), lambda: M.processes_params("uniform")),
    "retirement": (lambda: M.retirement_model(5, 100, 100), M.retirement_params),
    "stochastic": (lambda: M.stochastic_model(6, 60, 80), M.stochastic_params),
    "hc": (lambda: M.hc_model(4, 30, 6, 5, 25), lambda: M.hc_params(1, 5)),
    # a wealth line longer than a tile (512 states): the single-precision
    # search reads this model from collapsed rows
    "hc_rows": (lambda: M.hc_model(4, 600, 8, 4, 60), lambda: M.hc_params(2, 4)),
    **{f"grid_{k}": (lambda k=k: M.grid_kinds_model(k), M.grid_kinds_params)
       for k in ("irreg", "log", "piece_lin", "piece_log")},
}


MISMATCH: list = []  # (period, regime, state, GPU policy, oracle policy, gap, GPU V, oracle V)


def _action_values(spec, flat):
    """Action values of flat action indices (row-major over the declared
    actions): one column per action."""
    flat = np.asarray(flat, dtype=np.int64)
    if not spec.actions:
        return np.zeros(flat.shape + (1,))
    cols = []
    for ax in reversed(spec.actions):
        i = flat % ax.size
        flat = flat // ax.size
        cols.append(ax.grid.to_numpy()[i] if ax.kind == "continuous" else i.astype(np.float64))
    return np.stack(cols[::-1], axis=-1)


def _compare(model, params, precision, gap_tol=1e-9):
    """(worst V error, #states with gap > gap_tol, #agreeing among them,
    #states, #agreeing overall).  Overall, two policies agree when they choose
    the same action values: a piecewise grid whose segments meet at an open
    bound holds two points a rounding apart (x and nextafter(x)), whose Q
    values the search cannot order."""
    specs = {s.name: s for s in model.regime_specs}
    V, pol = model.solve(params=params, precision=precision, return_policy=True, log_level="off")
    gaps: dict = {}
    Vo, Po = oracle_solve(model, params, gaps=gaps)
    worst = 0.0
    n_pol = n_agree = n_all = n_all_agree = 0
    for p in Vo:
        for r in Vo[p]:
            worst = max(worst, rel_err(V[p][r], Vo[p][r]))
            g = gaps[p][r] / np.maximum(1.0, np.abs(np.nan_to_num(Vo[p][r], neginf=0.0)))
            sel = g > gap_tol
            same = np.asarray(pol[p][r]) == Po[p][r]
            n_pol += int(sel.sum())
            n_agree += int(same[sel].sum())
            for i in np.argwhere(sel & ~same)[:5]:
                i = tuple(i)
                MISMATCH.append((p, r, i, int(np.asarray(pol[p][r])[i]), int(Po[p][r][i]), float(g[i]),
                                 float(np.asarray(V[p][r])[i]), float(Vo[p][r][i])))
            n_all += same.size
            pa, po = np.asarray(pol[p][r]).reshape(-1), np.asarray(Po[p][r]).reshape(-1)
            av, ao = _action_values(specs[r], pa), _action_values(specs[r], po)
            same_val = np.all(np.abs(av - ao) <= 1e-12 * np.maximum(1.0, np.abs(ao)), axis=-1)
            n_all_agree += int((same.reshape(-1) | same_val).sum())
    return worst, n_pol, n_agree, n_all, n_all_agree


@pytest.mark.parametrize("case", sorted(CASES))
def test_fp64_matches_oracle(case):
    mk, mp = CASES[case]
    worst, n_pol, n_agree, _, _ = _compare(mk(), mp(), "fp64")
    assert worst < 1e-12, worst
    assert n_agree == n_pol, (n_agree, n_pol)


@pytest.mark.parametrize("case", sorted(CASES))
def test_fp32_search_matches_oracle(case):
    mk, mp = CASES[case]
    MISMATCH.clear()
    # single-precision search: exact agreement wherever the relative Q gap is
    # above float resolution; >= 99.9 % agreement over all states
    worst, n_pol, n_agree, n_all, n_all_agree = _compare(mk(), mp(), "fp32", gap_tol=1e-5)
    assert worst < 1e-6, worst
    assert n_agree == n_pol, (n_agree, n_pol, MISMATCH[:10])
    assert n_all_agree >= 0.999 * n_all, (n_all_agree, n_all)


def test_gpu_matches_reference_golden_regression():
    golden = load_golden("regression_solution.npz")
    V = M.regression_model(4).solve(params=M.regression_params(4), log_level="off")
    for p, regs in golden.items():
        for r, ref in regs.items():
            assert rel_err(V[p][r], ref) < 1e-12


@pytest.mark.parametrize("kind", ["uniform", "normal", "lognormal", "tauchen", "rouwenhorst"])
def test_gpu_matches_reference_golden_processes(kind):
    golden = load_golden(f"processes_solution_{kind}.npz")
    V = M.processes_model(4, kind).solve(params=M.processes_params(kind), log_level="off")
    for p, regs in golden.items():
        for r, ref in regs.items():
            assert rel_err(V[p][r], ref) < 1e-12, (kind, p, r)


def test_batch_equals_single():
    model = M.stochastic_model(5, 40, 50)
    ps = [M.stochastic_params(beta=b, crra=c) for b, c in ((0.95, 2.0), (0.9, 3.0), (0.97, 1.5))]
    eng = model.engine("fp64")
    batch = eng.solve_batch(ps)
    for p, (Vb, _) in zip(ps, batch):
        V1, _ = eng.solve(p)
        for per in V1:
            for r in V1[per]:
                assert np.array_equal(V1[per][r].cpu().numpy(), Vb[per][r].cpu().numpy())


def test_deterministic_replay():
    model = M.stochastic_model(5, 40, 50)
    p = M.stochastic_params()
    a = model.solve(params=p, log_level="off")
    b = model.solve(params=p, log_level="off")
    for per in a:
        for r in a[per]:
            assert np.array_equal(a[per][r], b[per][r])


def test_cuda_graph_replay_matches_eager():
    model = M.stochastic_model(5, 40, 50)
    eng = model.engine("fp64")
    plan = eng.plan([M.stochastic_params()])
    plan.run()
    eager = {r: v.clone() for r, v in plan.V.items()}
    for v in plan.V.values():
        v.zero_()
    plan.run_graph()
    import torch

    torch.cuda.synchronize()
    for r in eager:
        assert torch.equal(eager[r], plan.V[r])


@pytest.mark.parametrize("lanes,sb", [(2, 4), (4, 2), (1, 4)])
@pytest.mark.parametrize("case", ["stochastic", "hc", "proc_tauchen"])
def test_launch_shape_keeps_the_fp64_bars(case, lanes, sb):
    """Kernel (a) with several lanes per state and states per thread meets
    the FP64 bars against the default shape: V within 1e-12, argmax identical
    wherever the oracle's best-to-second-best gap exceeds 1e-9.  (Values may
    differ in the last bit: the compiler fuses multiply-adds per code shape.)"""
    import torch

    from pylcm_b200.codegen import LaunchConfig
    from pylcm_b200.engine import SolveEngine

    model = CASES[case][0]()
    params = CASES[case][1]()
    gaps = {}
    oracle_solve(model, params, gaps=gaps)
    ref = SolveEngine(model, "fp64").plan([params] * 2)
    ref.run()
    cfg = {s.name: LaunchConfig(block=256, lanes=lanes, chunk=256, sb=sb) for s in model.regime_specs}
    got = SolveEngine(model, "fp64", configs=cfg).plan([params] * 2)
    got.run()
    torch.cuda.synchronize()
    for k in range(2):
        V1, P1 = ref.result(k)
        V2, P2 = got.result(k)
        for p in V1:
            for r in V1[p]:
                a, b = V2[p][r].cpu().numpy(), V1[p][r].cpu().numpy()
                assert rel_err(a, b) <= 1e-12
                g = np.asarray(gaps[p][r]).reshape(a.shape)
                sel = g > 1e-9
                np.testing.assert_array_equal(P2[p][r].cpu().numpy()[sel], P1[p][r].cpu().numpy()[sel])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_solver_overlapped_download_equals_the_device_arrays(precision):
    """`BatchSolver.solve` reads each period's value and policy slices on a
    copy stream while later periods compute; the host arrays equal the
    device arrays and the graph-replay + whole-array download path."""
    import torch

    from pylcm_b200.batch import BatchSolver

    model = M.stochastic_model(6, 60, 80)
    ps = [M.stochastic_params(beta=b, crra=c) for b, c in ((0.95, 2.0), (0.9, 3.0), (0.97, 1.5))]
    bs = BatchSolver(model, len(ps), precision, template_params=ps[0])
    Vs, Ps = bs.solve(ps, return_policy=True)
    for r, v in bs.plan.V.items():
        assert torch.equal(torch.nan_to_num(bs._host_V[r], nan=5.0), torch.nan_to_num(v.cpu(), nan=5.0))
        assert torch.equal(bs._host_pol[r], bs.plan.pol[r].cpu())
    keep = [{p: {r: np.array(a) for r, a in d.items()} for p, d in V.items()} for V in Vs]
    for h in bs._host_V.values():
        h.zero_()
    bs.upload(bs.pack(ps))
    bs.run()
    bs.download(policy=True)
    torch.cuda.synchronize()
    for i, V in enumerate(bs.results()):
        for p in V:
            for r in V[p]:
                assert np.array_equal(V[p][r], keep[i][p][r], equal_nan=True)
    if precision == "fp32":
        return  # single solves may take another launch shape (last-ulp differences)
    for i, p_ in enumerate(ps):
        V1, _ = model.engine(precision).solve(p_)
        for per in V1:
            for r in V1[per]:
                assert np.array_equal(V1[per][r].cpu().numpy(), keep[i][per][r], equal_nan=True)


def test_collapsed_rows_agree_with_the_bilinear_search():
    """The single-precision search with and without the collapsed rows: the
    same argmax wherever the double-precision gap exceeds the search's
    resolution, values within 1e-6 (both are re-evaluated in FP64)."""
    import dataclasses

    import numpy as np

    from pylcm_b200.engine import SolveEngine, default_config

    model, params = M.hc_model(4, 600, 8, 4, 60), [M.hc_params(s, 4) for s in range(3)]
    out = {}
    for coll in (True, False):
        cfg = {s.name: dataclasses.replace(default_config(s, "fp32", 3), collapse=coll) for s in model.regime_specs}
        eng = SolveEngine(model, "fp32", configs=cfg)
        plan = eng.plan(params)
        plan.run()
        out[coll] = ({r: v.cpu().numpy() for r, v in plan.V.items()}, {r: v.cpu().numpy() for r, v in plan.pol.items()})
        srcs = [rk.src for rk in eng._kernels.values()]
        assert any("lcm_sc" in x for x in srcs) == coll
    (Va, Pa), (Vb, Pb) = out[True], out[False]
    for r in Va:
        fin = np.isfinite(Vb[r])
        assert np.array_equal(np.isfinite(Va[r]), fin)
        rel = np.abs(Va[r][fin] - Vb[r][fin]) / np.maximum(1.0, np.abs(Vb[r][fin]))
        assert rel.max() <= 1e-6
        assert (Pa[r] == Pb[r]).mean() >= 0.999
