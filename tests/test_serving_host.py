"""Serving bookkeeping on the host: the HBM footprint estimates that drive
admission, and the latency summary of a request stream."""

import numpy as np

from pylcm_b200.engine import SolveEngine
from pylcm_b200.serving import Result, footprint_bytes, latency_summary, sim_bytes, solve_bytes
from tests import models as M


def test_solve_bytes_cover_the_value_arrays_and_grow_with_the_grids():
    small = SolveEngine(M.stochastic_model(5, 40, 30), "fp32")
    big = SolveEngine(M.stochastic_model(5, 80, 30), "fp32")
    longer = SolveEngine(M.stochastic_model(9, 40, 30), "fp32")
    for eng in (small, big, longer):
        floor = sum(max(len(s.active_periods), 1) * s.n_states * 12 for s in eng.specs)
        assert solve_bytes(eng) >= floor
    assert solve_bytes(big) > solve_bytes(small) and solve_bytes(longer) > solve_bytes(small)
    # the single-precision search keeps a float32 twin of the expectation tables
    assert solve_bytes(small) > solve_bytes(SolveEngine(M.stochastic_model(5, 40, 30), "fp64"))


def test_dcegm_footprint_counts_carry_rows_and_value_array_marginals():
    eng = SolveEngine(M.value_children_model(), "fp64")
    by = {s.name: s for s in eng.specs}
    work = by["working"]
    n_cand = 20 + 80
    n_pad = int(np.ceil(2.0 * n_cand))
    rows = 2 * 2  # health x work choice
    carry = 2 * rows * (4 * n_pad * 8 + 4)
    marg = 2 * (by["retired"].n_states + by["done"].n_states) * 8
    values = sum(max(len(s.active_periods), 1) * s.n_states * 12 for s in eng.specs)
    assert solve_bytes(eng) >= values + carry + marg
    assert work.n_states == 2 * 60


def test_footprint_adds_the_simulation_buffers():
    eng = SolveEngine(M.stochastic_model(5, 40, 30), "fp32")
    assert footprint_bytes(eng, 1000) == solve_bytes(eng) + sim_bytes(eng, 1000)
    assert sim_bytes(eng, 2000) == 2 * sim_bytes(eng, 1000)


def test_latency_summary():
    res = [Result(rid=i, family="f", moments={}, V=None, arrival=0.1 * i, admitted=0.1 * i,
                  finished=0.1 * i + 0.05 + 0.01 * (i % 3), batch_size=1 + i % 4) for i in range(100)]
    out = latency_summary(res)
    lat = np.array([r.finished - r.arrival for r in res])
    assert out["requests"] == 100
    assert abs(out["p50_ms"] - np.percentile(lat, 50) * 1e3) < 1e-9
    assert abs(out["p99_ms"] - np.percentile(lat, 99) * 1e3) < 1e-9
    assert abs(out["wall_s"] - (res[-1].finished - 0.0)) < 1e-12
    assert abs(out["solves_per_s"] - 100 / out["wall_s"]) < 1e-9
    assert out["mean_batch"] == np.mean([r.batch_size for r in res])
