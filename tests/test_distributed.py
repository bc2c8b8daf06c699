"""The multi-rank bookkeeping on CPU: two gloo ranks, each taking its share of
units, the slowest rank's time, results gathered on rank 0."""

import os
import socket

import numpy as np
import pytest

from pylcm_b200.distributed import partition


def test_partition_covers_every_unit_once_and_balances_footprints():
    rng = np.random.default_rng(0)
    fp = rng.integers(1, 10_000, size=101).tolist()
    for world in (1, 2, 3, 8):
        parts = partition(fp, world)
        assert sorted(i for p in parts for i in p) == list(range(101))
        loads = [sum(fp[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(fp)  # greedy bound
    assert partition([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        partition([1], 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist

    from pylcm_b200.distributed import gather_to_root, max_over_ranks, partition

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        fp = [5, 1, 4, 2, 3, 9, 7]
        mine = partition(fp, world)[rank]
        results = {i: {"unit": i, "rank": rank, "square": i * i} for i in mine}
        t = max_over_ranks(10.0 + rank)
        merged = gather_to_root(results)
        q.put((rank, mine, t, merged))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_units_and_report_the_slowest_time():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, mine, t, merged = q.get(timeout=120)
        out[rank] = (mine, t, merged)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] == 11.0  # slowest rank
    assert sorted(out[0][0] + out[1][0]) == list(range(7))
    assert out[1][2] is None
    merged = out[0][2]
    assert sorted(merged) == list(range(7))
    for i, r in merged.items():
        assert r["square"] == i * i and i in out[r["rank"]][0]


class _StandInServer:
    """CPU stand-in of serving.Server: a footprint per request and a run that
    returns one result per request, in request order."""

    def footprint(self, req) -> int:
        return req["bytes"]

    def run(self, reqs, realtime=False):
        import os as _os

        return [{"rid": r["rid"], "pid": _os.getpid(), "moment": float(r["rid"]) ** 0.5} for r in reqs]


def _serve_main(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist

    from pylcm_b200.distributed import partition, serve_partitioned

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = [{"rid": i, "bytes": (i * 7919) % 97 + 1} for i in range(23)]
        merged, wall = serve_partitioned(reqs, _StandInServer())
        mine = partition([r["bytes"] for r in reqs], world)[rank]
        q.put((rank, os.getpid(), mine, merged, wall))
    finally:
        dist.destroy_process_group()


def test_partitioned_serving_front_end_on_two_gloo_ranks():
    """Each request is served once, by the rank the footprint partition gives
    it; rank 0 receives every result; both ranks report the same job time."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, pid, mine, merged, wall = q.get(timeout=120)
        out[rank] = (pid, mine, merged, wall)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[1][2] is None
    merged = out[0][2]
    assert sorted(merged) == list(range(23))
    assert sorted(out[0][1] + out[1][1]) == list(range(23))
    for i, res in merged.items():
        owner = 0 if i in out[0][1] else 1
        assert res["rid"] == i and res["pid"] == out[owner][0]
        assert res["moment"] == float(i) ** 0.5
    assert out[0][3] == out[1][3]
