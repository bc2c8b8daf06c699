"""Serving: continuous batching of solve+simulate requests on one GPU.

The reference has no serving layer; its unit of work is one
``model.solve(params)`` followed by ``model.simulate(...)``
(``src/lcm/model.py:440-519, 648-848``) -- the inner loop of a
simulated-moments estimation.  This module runs a stream of such requests:

- a request names a model, a parameter set, the initial conditions of the
  simulated subjects and a seed; its model family groups the requests whose
  kernels are the same (grid sizes, horizons and parameters are item words
  and may differ within a family);
- requests that arrive while others run wait in per-family queues; when one
  of the server's CUDA streams is free, the family whose oldest request has
  waited longest is batched -- every waiting request of it, up to
  `max_batch` -- into one job: one heterogeneous solve plan over the batch
  (one launch per (step, kernel) covers every instance, whatever its grid
  sizes and horizon) and one simulation plan over it;
- the requests' solve slots come from per-model pools kept on the device
  (their item records are built once); a request is admitted when a slot and
  its simulation buffers fit the HBM budget left by the pools and the jobs
  in flight -- idle pools of other models are evicted, least recently used
  first -- and otherwise waits for memory to free up;
- jobs on different streams overlap on the device; a job's result (per
  period simulated moments, optionally the value functions) is copied to
  pinned host memory on its stream and the request completes when the host
  sees the job's event.

A request's numbers do not depend on the batch it lands in: each instance
has its own item records, the launch shape of a family is pinned, and the
simulation's counter RNG is keyed by the request's seed and indexed by
subject and period.
"""

from __future__ import annotations

import collections
import dataclasses
import time
from typing import Any, Hashable, Mapping, Sequence

import numpy as np

from pylcm_b200.engine import LaunchConfig, SolveEngine
from pylcm_b200.exceptions import AdmissionError


@dataclasses.dataclass
class Request:
    """One solve+simulate request.

    `family` groups requests that may share a job: models whose regimes
    generate the same kernels (same functions and state / action structure;
    grid sizes, horizon and parameters may differ).  `key` names the model
    itself (requests with equal keys share one model object and engine).
    """

    family: Hashable
    key: Hashable
    model: Any
    params: Mapping
    initial_conditions: Mapping
    seed: int = 0
    arrival: float = 0.0  # seconds after the start of the request stream
    rid: int = 0
    return_V: bool = False


@dataclasses.dataclass
class Result:
    rid: int
    family: Hashable
    moments: dict  # name -> (T,) per-period mean over the simulated subjects
    V: dict | None  # {period: {regime: array}} when requested
    arrival: float
    admitted: float
    finished: float
    batch_size: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def solve_bytes(eng: SolveEngine) -> int:
    """HBM bytes one solve instance (a pool slot) of `eng`'s model holds:
    T x states value (float64) and policy (int32) arrays per regime, the
    expectation tables (float64, plus float32 copies and their block
    statistics in the single-precision search), the action tables, the DC-EGM carry rows (two-period ring) and
    candidates, and the marginal-value rows of regimes DC-EGM reads as value
    arrays."""
    from pylcm_b200.egm import is_egm

    specs = eng.specs
    fp32 = eng.precision == "fp32"
    any_egm = any(is_egm(s) and not s.terminal for s in specs)
    b = 0
    for s in specs:
        slots = max(len(s.active_periods), 1)
        b += slots * s.n_states * (8 + 4)
        if any_egm and not is_egm(s) and any(a.kind == "continuous" for a in s.states):
            b += 2 * s.n_states * 8  # marginal-value rows of a carried value array
        if is_egm(s) and not s.terminal:
            n_rows = 1
            for a in s.states + s.actions:
                if a.kind != "continuous":
                    n_rows *= a.size
            solver = s.solver
            n_cand = int(solver.n_constrained_points) + len(solver.savings_grid.to_numpy())
            n_pad = int(np.ceil(solver.refined_grid_factor * n_cand))
            b += 2 * n_rows * (4 * n_pad * 8 + 4)  # refined grid, policy, value, u'(c); counts
            b += n_rows * n_cand * 8 * 4 * 2  # candidates + envelope workspace
        # expectation tables of the targets (at most one per target and target set)
        for t in specs:
            if t.states and not s.terminal:
                # double table, float copy and its block statistics (8 B per
                # 16 columns) in the single-precision search
                b += t.n_states * 8 + (t.n_states * 4 + -(-t.n_states // 16) * 8 if fp32 else 0)
        b += 4 * s.n_actions * 4  # action table
    return int(b)


def sim_bytes(eng: SolveEngine, n_agents: int) -> int:
    """HBM bytes of the simulation of `n_agents` subjects: per period their
    states, regime, value, action index and actions."""
    specs = eng.specs
    T = eng.model.n_periods
    names = {a.name for s in specs for a in s.states}
    anames = {a.name for s in specs for a in s.actions}
    return int(n_agents * (T + 1) * (8 * len(names) + 4) + n_agents * T * (8 + 4 + 8 * len(anames)))


def footprint_bytes(eng: SolveEngine, n_agents: int) -> int:
    """HBM bytes one solve+simulate instance of `eng`'s model holds."""
    return solve_bytes(eng) + sim_bytes(eng, n_agents)


class _Pool:
    """Device-resident solve slots of one model: a solve plan over `n_slots`
    instances with its item records (all periods) built once; a request
    borrows a slot for one job."""

    def __init__(self, eng: SolveEngine, params, n_slots: int, nbytes: int) -> None:
        from pylcm_b200.engine import SolvePlan

        self.plan = SolvePlan(eng, [params] * n_slots, upload=False)
        self.plan.ensure_sim_records(upload=False)
        self.n_slots = n_slots
        self.free = list(range(n_slots))
        self.nbytes = nbytes
        self.last_used = 0.0

    @property
    def idle(self) -> bool:
        return len(self.free) == self.n_slots


class _Job:
    def __init__(self, family, reqs, stream, plan, sim, host, event, admitted, v_host, lengths, slots) -> None:
        self.family, self.reqs, self.stream = family, reqs, stream
        self.plan, self.sim, self.host, self.event = plan, sim, host, event
        self.admitted, self.v_host, self.lengths, self.slots = admitted, v_host, lengths, slots


class Server:
    """Continuous-batching solve+simulate server on one GPU.

    precision -- "fp32" (single-precision search, double-precision values;
                 the fast form) or "fp64" (the plain form);
    max_batch -- most requests of one family per job;
    n_streams -- jobs in flight at once;
    hbm_budget_bytes -- admission budget (default: half the free HBM);
    pool_slots -- solve slots allocated at a time for one model.

    Device state: per model, pools of solve slots (value and policy arrays,
    expectation / action tables, DC-EGM carry rows) whose item records are
    built once; a job borrows one slot per request and writes only the
    request's parameters into it.  Admission: a request needs a free slot of
    its model -- or room in the budget for a new pool, after evicting idle
    pools of other models, least recently used first -- and room for its
    simulation buffers.  The budget counts every pool and the simulation
    buffers of the jobs in flight.
    """

    def __init__(self, device: int = 0, precision: str = "fp32", max_batch: int = 32, n_streams: int = 4,
                 hbm_budget_bytes: int | None = None, configs: Mapping | None = None, pool_slots: int = 4,
                 autotune: bool = False) -> None:
        """`autotune=True`: the launch shape of each family's regimes is tuned
        once, on the family's first model at the job size `max_batch`
        (``pylcm_b200.autotune``, cached on disk); it then stays pinned for
        the family, so results still do not depend on the batch."""
        import torch

        self.torch = torch
        self.device = device
        self.precision = precision
        self.max_batch = int(max_batch)
        self.pool_slots = int(pool_slots)
        self.dev = torch.device("cuda", device)
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(int(n_streams))]
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget_bytes = free // 2
        self.budget = int(hbm_budget_bytes)
        self.configs = dict(configs or {})
        self.autotune = bool(autotune)
        self._engines: dict[Hashable, SolveEngine] = {}
        self._family_cfg: dict[Hashable, dict] = {}
        self._pools: dict[Hashable, list[_Pool]] = {}
        self.in_use = 0
        self.peak_in_use = 0
        self.jobs_run = 0
        self.pools_built = 0
        self.pools_evicted = 0
        self.batch_sizes: list[int] = []
        self.job_gpu_ms: list[float] = []  # device time of each job (its first kernel to its result copy)
        self.host_launch_s = 0.0  # host time building and issuing jobs
        self.host_finish_s = 0.0  # host time unpacking results
        self.host_phase_s: dict[str, float] = {}  # host time of the phases of building and issuing jobs

    # ---------------------------------------------------------------- engines
    def engine(self, req: Request) -> SolveEngine:
        """The solve engine of a request's model, with one launch shape per
        regime and family (independent of the batch and of the grid sizes,
        so a family's models share kernels and results do not depend on the
        batch)."""
        eng = self._engines.get(req.key)
        if eng is None:
            cfgs = self._family_cfg.get(req.family)
            if cfgs is None:
                cfgs = {}
                if self.autotune:
                    from pylcm_b200 import autotune as _at

                    cfgs.update(_at.tune(req.model, self.precision, [req.params] * self.max_batch))
                cfgs.update(self.configs.get(req.family, {}))
                for s in req.model.regime_specs:
                    if s.name not in cfgs:
                        # jobs of tens of requests: 2 lanes x 2 states per thread
                        cfgs[s.name] = LaunchConfig(block=256, lanes=2, chunk=512, sb=2)
                self._family_cfg[req.family] = cfgs
            eng = SolveEngine(req.model, self.precision, configs=cfgs, device=self.device)
            self._engines[req.key] = eng
        return eng

    @staticmethod
    def _n_agents(req: Request) -> int:
        return int(np.asarray(req.initial_conditions["regime_id"]).shape[0])

    def footprint(self, req: Request) -> int:
        """HBM bytes of one request alone: a one-slot pool and its simulation."""
        eng = self.engine(req)
        return solve_bytes(eng) + sim_bytes(eng, self._n_agents(req))

    def _evict(self, need: int, keep_key) -> None:
        """Free idle pools of other models (least recently used first) until
        `need` more bytes fit the budget."""
        idle = [(pool.last_used, key, pool) for key, pools in self._pools.items() if key != keep_key
                for pool in pools if pool.idle]
        for _, key, pool in sorted(idle, key=lambda x: x[0]):
            if self.in_use + need <= self.budget:
                return
            self._pools[key].remove(pool)
            self.in_use -= pool.nbytes
            self.pools_evicted += 1

    def _acquire(self, req: Request, now: float):
        """A free slot for `req` (building a pool if the budget allows) and
        the admission of its simulation buffers; None when it must wait."""
        eng = self.engine(req)
        sb = sim_bytes(eng, self._n_agents(req))
        pools = self._pools.setdefault(req.key, [])
        pool = next((p for p in pools if p.free), None)
        n_slots = self.pool_slots
        if pool is None:
            # a smaller pool when a full one does not fit
            self._evict(sb + n_slots * solve_bytes(eng), req.key)
            while n_slots > 1 and self.in_use + sb + n_slots * solve_bytes(eng) > self.budget:
                n_slots //= 2
        need = sb + (0 if pool is not None else n_slots * solve_bytes(eng))
        if self.in_use + need > self.budget:
            return None
        if pool is None:
            pool = _Pool(eng, req.params, n_slots, n_slots * solve_bytes(eng))
            pools.append(pool)
            self.pools_built += 1
            self.in_use += pool.nbytes
        pool.last_used = now
        self.in_use += sb
        self.peak_in_use = max(self.peak_in_use, self.in_use)
        return pool, pool.free.pop(0), sb

    # ------------------------------------------------------------------ jobs
    def _launch(self, family, reqs: list, slots: list, stream, now: float) -> _Job:
        from pylcm_b200.engine import BatchPlan
        from pylcm_b200.simulate import SimPlan

        torch = self.torch
        with torch.cuda.stream(stream):
            t_start = torch.cuda.Event(enable_timing=True)
            # every host->device copy happens here, before the job's first kernel:
            # a pageable copy waits for the work queued before it on the stream
            h = [time.perf_counter()]
            for (pool, slot, _), r in zip(slots, reqs):
                pool.plan.load_params(slot, r.params)
            h.append(time.perf_counter())
            plan = BatchPlan(slots=[(pool.plan, slot) for pool, slot, _ in slots])
            h.append(time.perf_counter())
            sim = SimPlan(plan, instances=[(k, r.initial_conditions, r.seed) for k, r in enumerate(reqs)])
            h.append(time.perf_counter())
            t_start.record(stream)
            plan.run(stream.cuda_stream)
            h.append(time.perf_counter())
            sim.run(stream.cuda_stream)
            h.append(time.perf_counter())
            # per-period moments of every instance: a few ops per group of
            # instances with the same horizon and subject count
            rows, layout = [], []
            off = 0
            specs = sim.inst[0]["eng"].specs
            for g in sim.groups:
                T = g["T"]
                cols = [g["val"]] + [g["S"][n][:, :T] for n in sorted(g["S"])] + [g["A"][n] for n in sorted(g["A"])]
                m = [torch.nanmean(c, dim=-1) for c in cols]
                m += [(g["R"][:, :T] == s.rid).to(torch.float64).mean(dim=-1) for s in specs]
                block = torch.stack(m, dim=1)  # (group members, columns, T)
                names = ["value"] + sorted(g["S"]) + sorted(g["A"]) + [f"share_{s.name}" for s in specs]
                rows.append(block.reshape(-1))
                layout.append((g["members"], names, T, off))
                off += block.numel()
            dev_out = torch.cat(rows)
            host = torch.empty(tuple(dev_out.shape), dtype=torch.float64, pin_memory=True)
            host.copy_(dev_out, non_blocking=True)
            v_host = {}
            for k, r in enumerate(reqs):
                if r.return_V:
                    pl, slot = plan.slots[k]
                    vh = {}
                    for name, v in pl.V.items():
                        t = torch.empty(tuple(v[slot].shape), dtype=torch.float64, pin_memory=True)
                        t.copy_(v[slot], non_blocking=True)
                        vh[name] = t
                    v_host[k] = vh
            event = torch.cuda.Event(enable_timing=True)
            event.record(stream)
            h.append(time.perf_counter())
        for k, name in enumerate(("params", "batch_plan", "sim_plan", "issue_solve", "issue_sim", "results")):
            self.host_phase_s[name] = self.host_phase_s.get(name, 0.0) + h[k + 1] - h[k]
        self.jobs_run += 1
        self.batch_sizes.append(len(reqs))
        job = _Job(family, reqs, stream, plan, sim, host, event, now, v_host, layout, slots)
        job.t_start = t_start
        return job

    def _finish(self, job: _Job, now: float) -> list[Result]:
        arr = job.host.numpy()
        moments: dict[int, dict] = {}
        for members, names, T, off in job.lengths:
            block = arr[off: off + len(members) * len(names) * T].reshape(len(members), len(names), T)
            for k, i in enumerate(members):
                moments[i] = {n: block[k, c].copy() for c, n in enumerate(names)}
        out = []
        for k, r in enumerate(job.reqs):
            eng = job.sim.inst[k]["eng"]
            V = None
            if k in job.v_host:
                V = {}
                pl, slot = job.plan.slots[k]
                for name, t in job.v_host[k].items():
                    spec = next(s for s in eng.specs if s.name == name)
                    for p, sl in pl.slot[name].items():
                        V.setdefault(p, {})[name] = t[sl].numpy().reshape(spec.state_shape).copy()
            out.append(Result(r.rid, job.family, moments[k], V, r.arrival, job.admitted, now, len(job.reqs)))
        for pool, slot, sb in job.slots:
            pool.free.append(slot)
            self.in_use -= sb
        self.job_gpu_ms.append(job.t_start.elapsed_time(job.event))
        return out

    # ------------------------------------------------------------------- run
    def run(self, requests: Sequence[Request], realtime: bool = True) -> list[Result]:
        """Serve `requests`, released at their arrival times (seconds after
        the start) when `realtime`, all at once otherwise.  Returns the
        results in request order; `Result.latency` is end-to-end (arrival to
        the host seeing the result)."""
        torch = self.torch
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            fp = self.footprint(r)
            if fp > self.budget:
                raise AdmissionError(f"request {r.rid}: footprint {fp} B exceeds the HBM budget {self.budget} B")
        waiting: dict[Hashable, collections.deque] = collections.OrderedDict()
        free = list(self.streams)
        inflight: list[_Job] = []
        results: dict[int, Result] = {}
        i = 0
        t0 = time.perf_counter()
        n = len(reqs)
        while len(results) < n:
            now = time.perf_counter() - t0
            while i < n and (not realtime or reqs[i].arrival <= now):
                r = reqs[i]
                if not realtime:
                    r.arrival = 0.0
                waiting.setdefault(r.family, collections.deque()).append(r)
                i += 1
            progressed = False
            for job in list(inflight):
                if job.event.query():
                    h0 = time.perf_counter()
                    for res in self._finish(job, h0 - t0):
                        results[res.rid] = res
                    self.host_finish_s += time.perf_counter() - h0
                    inflight.remove(job)
                    free.append(job.stream)
                    progressed = True
            while free and any(waiting.values()):
                fam = min((k for k, q in waiting.items() if q), key=lambda k: waiting[k][0].arrival)
                q = waiting[fam]
                h0 = time.perf_counter()
                batch, slots = [], []
                while q and len(batch) < self.max_batch:
                    got = self._acquire(q[0], h0 - t0)
                    if got is None:
                        break  # admission: wait for memory to free up
                    slots.append(got)
                    batch.append(q.popleft())
                if not batch:
                    break
                inflight.append(self._launch(fam, batch, slots, free.pop(0), h0 - t0))
                self.host_launch_s += time.perf_counter() - h0
                progressed = True
            if not progressed:
                if inflight:
                    time.sleep(5e-5)
                elif i < n:
                    time.sleep(max(0.0, min(reqs[i].arrival - (time.perf_counter() - t0), 1e-3)))
                elif any(waiting.values()):
                    raise AdmissionError("a waiting request cannot be admitted with no job in flight")
        torch.cuda.synchronize(self.dev)
        return [results[r.rid] for r in sorted(requests, key=lambda r: r.rid)]


def latency_summary(results: Sequence[Result], wall_s: float | None = None) -> dict:
    lat = np.array([r.latency for r in results])
    out = {
        "requests": len(results),
        "p50_ms": float(np.percentile(lat, 50) * 1e3),
        "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "mean_ms": float(lat.mean() * 1e3),
        "mean_batch": float(np.mean([r.batch_size for r in results])),
    }
    if wall_s is None:
        wall_s = max(r.finished for r in results) - min(r.arrival for r in results)
    out["wall_s"] = float(wall_s)
    out["solves_per_s"] = len(results) / wall_s
    return out
