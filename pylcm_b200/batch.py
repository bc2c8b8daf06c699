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
                 use_graph: bool = True, configs: dict | None = None, device: int = 0) -> None:
        import torch

        self.torch = torch
        self.model = model
        self.n = int(batch_size)
        self.precision = precision
        self.engine = SolveEngine(model, precision, configs=configs, device=device)
        if template_params is None:
            raise ValueError("template_params (one valid params dict) is required to trace the model")
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

    def solve(self, params_list: Sequence, return_policy: bool = False):
        """Solve `params_list` (len == batch_size); returns per-instance
        ``{period: {regime: V}}`` host arrays (and policies)."""
        packed = self.pack(params_list)
        self.upload(packed)
        self.run()
        self.download(policy=return_policy)
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
