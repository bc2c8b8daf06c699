"""Batched solves: many parameter vectors of one model in one launch per step.

``BatchSolver(model, batch_size, precision)`` allocates every device buffer
once (V, policy, EV, parameter vectors, item records) and captures the whole
backward induction -- all periods, all regimes, all instances -- as one CUDA
graph.  ``solve(params_list)`` then only copies the packed parameter vectors
host->device, replays the graph, and copies V (and optionally the policy)
device->host.

This is the "batching" pattern: one launch per (period, regime) covers every
instance, so small models stop being launch-bound, and the graph removes the
host from the per-period loop entirely.
"""

from __future__ import annotations

from typing import Sequence


from pylcm_b200.engine import SolveEngine, SolvePlan


class BatchSolver:
    def __init__(self, model, batch_size: int, precision: str = "fp32", template_params=None,
                 use_graph: bool = True, configs: dict | None = None, device: int = 0,
                 autotune: bool = False) -> None:
        """`autotune=True` times candidate launch shapes of kernel (a) for
        this model and batch size once (cached on disk per GPU, generated
        code and batch bucket, see ``pylcm_b200.autotune``) and uses the
        fastest; explicit `configs` win over tuned ones."""
        import torch

        self.torch = torch
        self.model = model
        self.n = int(batch_size)
        self.precision = precision
        if template_params is None:
            raise ValueError("template_params (one valid params dict) is required to trace the model")
        cfgs = {}
        if autotune:
            from pylcm_b200 import autotune as _at

            cfgs.update(_at.tune(model, precision, [template_params] * self.n))
        cfgs.update(configs or {})
        self.configs = cfgs
        self.engine = SolveEngine(model, precision, configs=cfgs, device=device)
        self.plan: SolvePlan = self.engine.plan([template_params] * self.n)
        self.use_graph = use_graph
        # pinned host staging for parameters and results
        self._pkeys = list(self.plan.params)
        self._host_params = {
            k: torch.empty(tuple(v.shape), dtype=torch.float64, pin_memory=True) for k, v in self.plan.params.items()
        }
        self._host_V = {
            r: torch.empty(tuple(v.shape), dtype=torch.float64, pin_memory=True) for r, v in self.plan.V.items()
        }
        self._host_pol = {
            r: torch.empty(tuple(v.shape), dtype=torch.int32, pin_memory=True) for r, v in self.plan.pol.items()
        }
        if use_graph:
            self.plan.capture()

    # -------------------------------------------------------------- params
    def pack(self, params_list: Sequence) -> dict:
        """Host-side packing of parameter vectors (float64, plan layout)."""
        if len(params_list) != self.n:
            raise ValueError(f"expected {self.n} parameter sets, got {len(params_list)}")
        resolvers = [self.engine.resolver(p) for p in params_list]
        memo: dict = {}
        return {key: self.plan._pack_many[key](resolvers, memo) for key in self._pkeys}

    def upload(self, packed: dict, non_blocking: bool = True) -> int:
        """Copy packed parameters host->device; returns bytes copied."""
        nbytes = 0
        for key, arr in packed.items():
            h = self._host_params[key]
            h.numpy()[...] = arr
            self.plan.params[key].copy_(h, non_blocking=non_blocking)
            nbytes += arr.nbytes
        return nbytes

    def run(self) -> None:
        if self.use_graph:
            self.plan.run_graph()
        else:
            self.plan.run()

    def download(self, policy: bool = False) -> int:
        nbytes = 0
        for r, v in self.plan.V.items():
            self._host_V[r].copy_(v, non_blocking=True)
            nbytes += v.numel() * 8
        if policy:
            for r, v in self.plan.pol.items():
                self._host_pol[r].copy_(v, non_blocking=True)
                nbytes += v.numel() * 4
        return nbytes

    def run_download(self, policy: bool = False) -> int:
        """Run the backward induction and copy its results to the pinned host
        arrays, each period's slice of every value (and policy) array read on
        a copy stream as soon as that period's launches are done -- the copies
        of late periods overlap the computation of the early ones.  Launches
        are issued eagerly, period by period, on the current stream, which
        waits for the copies at the end.  Returns the bytes copied."""
        from pylcm_b200.runtime import get_context

        torch = self.torch
        plan = self.plan
        ctx = get_context(self.engine.device)
        if plan._prepared is None:
            plan._prepared = plan._prepare()
        comp = torch.cuda.current_stream(plan.dev)
        copy = self.__dict__.get("_copy_stream")
        if copy is None:
            copy = self._copy_stream = torch.cuda.Stream(plan.dev)
        by_period: dict[int, list] = {}
        for s in self.engine.specs:
            for period, k in plan.slot[s.name].items():
                by_period.setdefault(period, []).append((s, k))
        nbytes = 0
        launches = plan.launches
        i = 0
        while i < len(launches):
            period = launches[i].period
            while i < len(launches) and launches[i].period == period:
                plan._prepared[i](comp.cuda_stream)
                i += 1
            ev = torch.cuda.Event()
            ev.record(comp)
            copy.wait_event(ev)
            for s, k in by_period.pop(period, []):
                nbytes += self._copy_slot(ctx, s, k, policy, copy.cuda_stream)
        # periods without launches of their own (none in a solve plan)
        for period, items in by_period.items():
            ev = torch.cuda.Event()
            ev.record(comp)
            copy.wait_event(ev)
            for s, k in items:
                nbytes += self._copy_slot(ctx, s, k, policy, copy.cuda_stream)
        comp.wait_stream(copy)
        return nbytes

    def _copy_slot(self, ctx, s, k: int, policy: bool, stream: int) -> int:
        """Copy slot k (one period) of every instance's value (and policy)
        array of regime `s`: n rows of n_states entries, strided by the slots."""
        nbytes = 0
        arrays = [(self.plan.V[s.name], self._host_V[s.name])]
        if policy:
            arrays.append((self.plan.pol[s.name], self._host_pol[s.name]))
        for dev_t, host_t in arrays:
            es = dev_t.element_size()
            row = dev_t.shape[2] * es
            pitch = dev_t.stride(0) * es
            off = k * dev_t.stride(1) * es
            ctx.copy_rows_d2h(host_t.data_ptr() + off, pitch, dev_t.data_ptr() + off, pitch, row, dev_t.shape[0], stream)
            nbytes += row * dev_t.shape[0]
        return nbytes

    def solve(self, params_list: Sequence, return_policy: bool = False):
        """Solve `params_list` (len == batch_size); returns per-instance
        ``{period: {regime: V}}`` host arrays (and policies)."""
        packed = self.pack(params_list)
        self.upload(packed)
        self.run_download(policy=return_policy)
        self.torch.cuda.current_stream().synchronize()
        return self.results(return_policy)

    def results(self, return_policy: bool = False):
        outV, outP = [], []
        for i in range(self.n):
            V: dict = {}
            P: dict = {}
            for s in self.engine.specs:
                for period, k in self.plan.slot[s.name].items():
                    V.setdefault(period, {})[s.name] = self._host_V[s.name][i, k].numpy().reshape(s.state_shape)
                    if return_policy:
                        P.setdefault(period, {})[s.name] = self._host_pol[s.name][i, k].numpy().reshape(s.state_shape)
            outV.append(dict(sorted(V.items())))
            outP.append(dict(sorted(P.items())))
        return (outV, outP) if return_policy else outV

    @property
    def gpu_launches(self) -> int:
        return self.plan.gpu_launches
