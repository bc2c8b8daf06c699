"""Several GPUs: independent solves, one process per GPU.

The solve path shards as whole units -- parameter vectors of a batch, or
serving requests -- with no exchange on the data path: each rank solves its
own units on its own GPU.  What crosses ranks is bookkeeping only:

- `partition`: which rank takes which units, balanced by HBM footprint
  (largest first onto the least-loaded rank);
- `max_over_ranks`: the job's time is the slowest rank's (one all-reduce of
  a scalar);
- `gather_to_root`: per-unit results (moments, summaries) collected on rank 0;
- `serve_partitioned`: the multi-GPU front end of the serving loop -- every
  rank holds the same request stream, serves the requests the footprint
  partition gives it on its own GPU, and rank 0 receives every result.

The process group is `torch.distributed` with NCCL on GPUs (gloo on CPUs).
"""

from __future__ import annotations

from typing import Any, Sequence


def partition(footprints: Sequence[int], world: int) -> list[list[int]]:
    """Unit indices per rank: largest footprint first onto the rank with the
    smallest total so far (ties: lower rank); each rank's list ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(footprints)), key=lambda k: (-int(footprints[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(footprints[i])
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group
    (the value itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(items: dict[int, Any]) -> dict[int, Any] | None:
    """Merge per-rank {unit index: result} dicts on rank 0 (None elsewhere)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return dict(items)
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(dict(items), out, dst=0)
    if dist.get_rank() != 0:
        return None
    merged: dict[int, Any] = {}
    for part in out:
        overlap = merged.keys() & part.keys()
        if overlap:
            raise ValueError(f"units {sorted(overlap)} reported by two ranks")
        merged.update(part)
    return merged


def serve_partitioned(requests: Sequence, server, realtime: bool = False) -> tuple[dict | None, float]:
    """One rank's part of a serving job spread over the ranks of the default
    process group (one process per GPU).

    Every rank passes the same `requests`; `partition` assigns them by
    `server.footprint(request)` (HBM bytes of a solve + simulate), each rank
    serves its share with `server.run` on its own GPU -- no exchange on the
    data path -- and the results are gathered on rank 0.  Returns
    ({request index: result} on rank 0, None elsewhere; the job's wall time,
    the slowest rank's)."""
    import time

    import torch.distributed as dist

    ready = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if ready else 1
    rank = dist.get_rank() if ready else 0
    fps = [int(server.footprint(r)) for r in requests]
    mine = partition(fps, world)[rank]
    t0 = time.perf_counter()
    results = server.run([requests[i] for i in mine], realtime=realtime) if mine else []
    wall = time.perf_counter() - t0
    device = "cuda" if ready and dist.get_backend() == "nccl" else None
    wall = max_over_ranks(wall, device=device)
    merged = gather_to_root({i: res for i, res in zip(mine, results)})
    return merged, wall
