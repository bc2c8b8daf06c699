"""Backward induction on the GPU.

Restates the reference's solve loop (``src/_lcm/solution/backward_induction.py:44-302``)
B200-first: for a batch of solve *instances* (parameter vectors of one model
structure) every buffer is allocated once, the 64-bit item records of every
launch of every period are packed on the host and uploaded in one copy, and
the per-period work is a fixed list of kernel launches:

    for period = T-1 .. 0:
        kernel (b) for every (source regime, target regime) with stochastic
                   target axes  -> EV buffers
        kernel (a) for every regime active in the period -> V, policy

Each launch covers all instances.  The launch list has no host
synchronisation, so it can be replayed inside a CUDA graph
(``SolvePlan.run_graph``).  V arrays stay on the device between periods.
"""

from __future__ import annotations

import dataclasses
import hashlib
import math
import struct
from typing import Any, Sequence

import numpy as np

from pylcm_b200.codegen import LaunchConfig, RegimeKernels
from pylcm_b200.exceptions import ModelInitializationError
from pylcm_b200.runtime import bundle
from pylcm_b200.egm import is_egm
from pylcm_b200.spec import ParamResolver, RegimeSpec, TracedRegime, trace_regime


def _f2w(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", float(x)))[0]


@dataclasses.dataclass
class Launch:
    kind: str  # 'bellman' | 'expect'
    module: Any
    kernel: str
    item_off: int  # word offset into the item buffer
    prefix_off: int  # int offset into the prefix buffer
    n_items: int
    n_tiles: int
    block: int
    smem: int
    period: int
    grid: int = 0  # CTAs of the launch (0: SM count x resident CTAs per SM)


class _Records:
    """Item records and the launch list of a plan.

    Launches are collected with their host records (a 2-D int64 array, one
    row per item) and tiles per item; `tensors()` lays the records out in one
    int64 item buffer and the tile prefixes in one int32 buffer (each prefix
    16-byte aligned) and fills in the launches' offsets.
    """

    def __init__(self) -> None:
        self.launches: list[Launch] = []
        # per launch: (records, tiles per item), None for a launch without records
        self.host: list[tuple | None] = []
        self.shared: list[int] = []  # launch whose records this one reuses (-1: own)

    def add(self, kind, rk, kernel, recs, tiles_per_item, block, smem, period) -> None:
        arr = recs if isinstance(recs, np.ndarray) and recs.ndim == 2 else np.stack(recs)
        if arr.dtype != np.int64:
            arr = arr.astype(np.int64)
        tiles = np.asarray(tiles_per_item, dtype=np.int64)
        self.launches.append(Launch(kind, rk, kernel, 0, 0, arr.shape[0], int(tiles.sum()), block, smem, period))
        self.host.append((arr, tiles))
        self.shared.append(-1)

    def add_same_records(self, kind, rk, kernel, tiles_per_item, block, smem, period) -> None:
        """A launch over the previous launch's item records, own tiling."""
        src = len(self.launches) - 1
        tiles = np.asarray(tiles_per_item, dtype=np.int64)
        last = self.launches[src]
        self.launches.append(Launch(kind, rk, kernel, 0, 0, last.n_items, int(tiles.sum()), block, smem, period))
        self.host.append((self.host[src][0], tiles))
        self.shared.append(src)

    def append(self, launch: Launch) -> None:
        self.launches.append(launch)
        self.host.append(None)
        self.shared.append(-1)

    def keep(self, pred) -> None:
        """Drop the launches `pred` rejects.  A kept launch that reused the
        records of a dropped one takes them over as its own."""
        idx = [k for k, l in enumerate(self.launches) if pred(l)]
        new_of = {k: j for j, k in enumerate(idx)}
        self.launches = [self.launches[k] for k in idx]
        self.host = [self.host[k] for k in idx]
        self.shared = [new_of.get(self.shared[k], -1) if self.shared[k] >= 0 else -1 for k in idx]

    def tensors(self, torch, dev):
        words: list[np.ndarray] = []
        prefs: list[np.ndarray] = []
        w_off = p_off = 0
        for l, h, src in zip(self.launches, self.host, self.shared):
            if h is None:
                continue
            arr, tiles = h
            if src >= 0:
                l.item_off = self.launches[src].item_off
            else:
                l.item_off = w_off
                words.append(arr.reshape(-1))
                w_off += arr.size
            npre = len(tiles) + 1
            pre = np.zeros(npre + (-npre) % 4, dtype=np.int32)
            np.cumsum(tiles, out=pre[1:npre])
            l.prefix_off = p_off
            prefs.append(pre)
            p_off += pre.size
        words_a = np.concatenate(words) if words else np.zeros(1, dtype=np.int64)
        pre_a = np.concatenate(prefs) if prefs else np.zeros(4, dtype=np.int32)
        return (
            torch.as_tensor(words_a, dtype=torch.int64, device=dev),
            torch.as_tensor(pre_a, dtype=torch.int32, device=dev),
        )


SM_COUNT = 148
RESIDENT_THREADS_PER_SM = 1024
FUES_SMEM_MAX_N = 4096  # longest candidate row of the item-form FUES launch
ENVELOPE_MAX_N = 4096  # longest candidate row of the LTM / RFC / MSS envelope kernels


def default_config(spec: RegimeSpec, precision: str, n_items: int = 1) -> LaunchConfig:
    """Launch shape of kernel (a).  Preferred: 2 lanes per state and, in the
    single-precision search, 4 states per thread (each thread's states share
    the shared-memory action loads and give the scheduler independent work --
    the fastest shapes measured on the B200; in double precision more states
    per thread cost more registers than they save); fewer states per thread,
    then more lanes per state, only while the batch's states would not fill
    the GPU (SM count x resident threads)."""
    n_a = spec.n_actions
    total = max(1, spec.n_states * n_items)
    want = SM_COUNT * RESIDENT_THREADS_PER_SM
    lanes = 2 if n_a >= 64 else 1
    sb = 4 if precision == "fp32" else 1
    while sb > 1 and total * lanes < want * sb:
        sb //= 2
    while lanes < 32 and total * lanes < want * sb and n_a >= 8 * lanes * 2:
        lanes *= 2
    chunk = 512 if precision == "fp32" else 256
    return LaunchConfig(block=256, lanes=lanes, chunk=chunk, sb=sb)


class SolveEngine:
    """Compiles and runs the per-period kernels of one model structure."""

    def __init__(self, model, precision: str = "fp64", configs: dict | None = None, device: int = 0) -> None:
        self.model = model
        self.precision = precision
        self.configs = dict(configs or {})
        self.device = device
        self.specs = model.regime_specs
        self._kernels: dict[tuple, RegimeKernels] = {}
        self._traces: dict[tuple, TracedRegime] = {}
        self._targets: dict[tuple, tuple] = {}

    # ------------------------------------------------------------ helpers
    def targets_at(self, spec: RegimeSpec, period: int) -> tuple[str, ...]:
        key = (spec.name, period)
        t = self._targets.get(key)
        if t is None:
            t = () if spec.terminal else tuple(s.name for s in self.specs if (period + 1) in s.active_periods)
            self._targets[key] = t
        return t

    def resolver(self, params) -> ParamResolver:
        return ParamResolver(params, self.model.fixed_params, tuple(s.name for s in self.specs))

    def config_for(self, spec: RegimeSpec, n_items: int = 1) -> LaunchConfig:
        return self.configs.get(spec.name) or default_config(spec, self.precision, n_items)

    def kernels(self, spec: RegimeSpec, targets: tuple[str, ...], params, n_items: int = 1) -> RegimeKernels:
        cfg = self.config_for(spec, n_items)
        key = (spec.name, targets, cfg)
        rk = self._kernels.get(key)
        if rk is None:
            tr = trace_regime(spec, self.specs, self.resolver(params), targets)
            by = {s.name: s for s in self.specs}
            rk = RegimeKernels(tr, [by[t] for t in targets], self.precision, cfg)
            src = rk.source()
            rk.src = src
            rk.key = "lcm_" + hashlib.sha1(src.encode()).hexdigest()[:24]
            self._kernels[key] = rk
        return rk

    def egm_kernels(self, spec: RegimeSpec, targets: tuple[str, ...], params):
        """Generated DC-EGM kernels of a regime for one next-period target set."""
        from pylcm_b200.egm import trace_egm_regime
        from pylcm_b200.egm_codegen import EgmKernels

        key = ("egm", spec.name, targets)
        ek = self._kernels.get(key)
        if ek is None:
            er = trace_egm_regime(spec, self.specs, self.resolver(params), targets)
            ek = EgmKernels(er)
            self._kernels[key] = ek
        return ek

    def value_carry_kernel(self, spec: RegimeSpec, euler: str, params):
        """The marginal-value kernel of a terminal or grid-search regime that
        a DC-EGM regime reads as a carried value array."""
        from pylcm_b200.egm_codegen import ValueCarryKernel

        key = ("vmu", spec.name)
        vk = self._kernels.get(key)
        if vk is None:
            if spec.terminal:
                rk = self.kernels(spec, (), params)
                vk = ValueCarryKernel(spec, euler, rk.tr.U, rk.param_off)
            else:
                vk = ValueCarryKernel(spec, euler)
            self._kernels[key] = vk
        return vk

    def module(self, rk: RegimeKernels):
        from pylcm_b200.runtime import get_context

        mod = getattr(rk, "module", None)
        if mod is None:
            ctx = get_context(self.device)
            mod = ctx.compile(rk.src, rk.key)
            rk.module = mod
        return mod

    # --------------------------------------------------------------- plan
    def plan(self, params_list: Sequence) -> "SolvePlan":
        return SolvePlan(self, list(params_list))

    def solve(self, params, collect_carries: bool = False):
        """(V, policy) of one parameter set; with ``collect_carries`` also
        each period's DC-EGM carry rows (see
        ``SolvePlan.run_collecting_carries``) as a third element."""
        plan = self.plan([params])
        if not collect_carries:
            plan.run()
            plan.check_status()
            return plan.result(0)
        carries = plan.run_collecting_carries()
        plan.check_status()
        return (*plan.result(0), carries)

    def solve_batch(self, params_list: Sequence) -> list[tuple[dict, dict]]:
        plan = self.plan(params_list)
        plan.run()
        return [plan.result(i) for i in range(len(params_list))]


class SolvePlan:
    """Buffers, item records and the launch list for a batch of instances."""

    def __init__(self, eng: SolveEngine, params_list: list, upload: bool = True) -> None:
        import torch

        self.eng = eng
        self.torch = torch
        model = eng.model
        specs = eng.specs
        T = model.n_periods
        n = len(params_list)
        if n == 0:
            raise ValueError("empty batch")
        self.n = n
        dev = torch.device("cuda", eng.device)
        self.dev = dev
        fp32 = eng.precision == "fp32"
        resolvers = [eng.resolver(p) for p in params_list]
        self.params_list = params_list

        # ---- per regime: slots (active periods), V / policy buffers, grids
        self.slot: dict[str, dict[int, int]] = {}
        self.V: dict[str, Any] = {}
        self.pol: dict[str, Any] = {}
        self.sgrid: dict[str, list] = {}
        self.agrid: dict[str, list] = {}
        for s in specs:
            per = list(s.active_periods)
            self.slot[s.name] = {p: k for k, p in enumerate(per)}
            ns = s.n_states
            self.V[s.name] = torch.empty((n, max(len(per), 1), ns), dtype=torch.float64, device=dev)
            self.pol[s.name] = torch.empty((n, max(len(per), 1), ns), dtype=torch.int32, device=dev)
            self.sgrid[s.name] = [
                torch.as_tensor(ax.grid.to_numpy(), dtype=torch.float64, device=dev) if ax.kind == "continuous" else None
                for ax in s.states
            ]
            self.agrid[s.name] = [
                torch.as_tensor(ax.grid.to_numpy(), dtype=torch.float64, device=dev) if ax.kind == "continuous" else None
                for ax in s.actions
            ]

        # ---- kernels per (regime, target set); params per (regime, target set)
        by = {s.name: s for s in specs}
        self.params: dict[tuple, Any] = {}
        self._packers: dict[tuple, Any] = {}  # params key -> packer(resolver) -> float64 vector
        self._pack_many: dict[tuple, Any] = {}  # params key -> packer(resolvers, memo) -> rows
        self.ev: dict[tuple, tuple] = {}
        step_list: list[tuple[int, RegimeSpec, tuple, Any]] = []
        egm_steps: list = []
        pack_memo: dict = {}  # parameter columns shared by a regime's target sets
        for period in range(T - 1, -1, -1):
            for s in specs:
                if period not in s.active_periods:
                    continue
                if not s.terminal and period == T - 1:
                    raise ModelInitializationError(f"non-terminal regime {s.name} active in the last period")
                targets = eng.targets_at(s, period)
                key = (s.name, targets)
                if is_egm(s) and not s.terminal:
                    ek = eng.egm_kernels(s, targets, params_list[0])
                    if key not in self.params:
                        vecs = ek.er.pack_many(resolvers, pack_memo)
                        self.params[key] = torch.as_tensor(vecs, dtype=torch.float64, device=dev)
                        self._packers[key] = ek.er.pack_for
                        self._pack_many[key] = ek.er.pack_many
                    egm_steps.append((period, s, targets, ek))
                    step_list.append((period, s, targets, ek))
                    continue
                rk = eng.kernels(s, targets, params_list[0], n)
                if key not in self.params:
                    vecs = rk.tr.pack_many(resolvers, pack_memo)
                    self.params[key] = torch.as_tensor(vecs, dtype=torch.float64, device=dev)
                    self._packers[key] = lambda r, tr=rk.tr: tr.pack_params(tr.values_for(r))
                    self._pack_many[key] = rk.tr.pack_many
                step_list.append((period, s, targets, rk))
        # DC-EGM buffers: carry rows per active period, scratch per regime
        self.egm: dict[str, dict] = {}
        for period, s, targets, ek in egm_steps:
            if s.name in self.egm:
                continue
            er = ek.er
            # carry rows are read only by the step of the period before: a
            # two-slot ring indexed by period parity
            nslot = 2
            npad, nrow, ncand = er.n_pad, er.n_rows, er.n_cand
            f64 = dict(dtype=torch.float64, device=dev)
            self.egm[s.name] = {
                "rg": torch.full((nslot, n, nrow, npad), float("nan"), **f64),
                "rc": torch.full((nslot, n, nrow, npad), float("nan"), **f64),
                "rv": torch.full((nslot, n, nrow, npad), float("nan"), **f64),
                "mu": torch.full((nslot, n, nrow, npad), float("nan"), **f64),
                "nk": torch.zeros((nslot, n, nrow), dtype=torch.int32, device=dev),
                "cand": [torch.empty((n, nrow, ncand), **f64) for _ in range(4)],
                # candidate marginal utilities (the RFC envelope's tangent slopes)
                "cm": torch.empty((n, nrow, ncand), **f64) if er.envelope == "rfc" else None,
                "ev0": torch.empty((n, nrow), **f64),
                "npad": npad,
                "nrow": nrow,
                "ncand": ncand,
                "sav": torch.as_tensor(er.savings, **f64),
            }
            from pylcm_b200.runtime import get_context

            wb = get_context(eng.device).fues_workspace_bytes(n * nrow, ncand)
            self.egm[s.name]["ws"] = torch.empty(max(wb, 8), dtype=torch.uint8, device=dev)
            self.egm[s.name]["wb"] = wb

        # marginal-value rows of the terminal / grid-search regimes DC-EGM
        # regimes read as carried value arrays (two-slot ring by period parity)
        self.vmu: dict[str, Any] = {}
        self._vck: dict[str, Any] = {}
        self._vmu_need: set = set()
        for period, s, targets, ek in egm_steps:
            for t in ek.er.targets:
                if not t.is_value or t.unreachable:
                    continue
                self._vmu_need.add((t.spec.name, period + 1))
                if t.spec.name not in self.vmu:
                    self.vmu[t.spec.name] = torch.zeros((2, n, t.spec.n_states), dtype=torch.float64, device=dev)
                    self._vck[t.spec.name] = eng.value_carry_kernel(t.spec, t.value_euler, params_list[0])

        # EV buffers per (source, target set, target)
        self.bst: dict[tuple, Any] = {}
        for period, s, targets, rk in step_list:
            if not isinstance(rk, RegimeKernels):
                continue
            for t in rk.targets:
                if t.scalar:
                    continue
                if not (t.needs_contraction or fp32):
                    continue
                k = (s.name, targets, t.spec.name)
                if k in self.ev:
                    continue
                cblk = int(np.prod([t.spec.states[p].size for p in t.cont_pos])) if t.cont_pos else 1
                ncols = int(np.prod([t.spec.states[p].size for p in t.det_pos])) * cblk if t.det_pos else cblk
                e64 = torch.empty((n, t.K, ncols), dtype=torch.float64, device=dev)
                e32 = torch.empty((n, t.K, ncols), dtype=torch.float32, device=dev) if fp32 else None
                self.ev[k] = (e64, e32, ncols, cblk)
                # block statistics of the float table rows (max, finite |max|)
                # for the search's exact group skipping: per 16 columns of a
                # one-axis table (kernel b), per 16 x 2 tile of a two-axis one
                # (the statistics kernel)
                gs = rk.group_stats(t)
                if gs == 1:
                    self.bst[k] = torch.empty((n, t.K, (ncols + 15) // 16, 2), dtype=torch.float32, device=dev)
                elif gs == 2:
                    n1, n2 = (t.spec.states[p].size for p in t.cont_pos)
                    T1, T2 = rk.GROUP_TILE
                    nt = ((n1 + T1 - 1) // T1) * ((n2 + T2 - 1) // T2)
                    self.bst[k] = torch.empty((n, t.K, nt, 2), dtype=torch.float32, device=dev)

        # action tables (kernel a0 output) per (regime, target set), reused across periods
        self.atab: dict[tuple, Any] = {}
        for period, s, targets, rk in step_list:
            if not isinstance(rk, RegimeKernels):
                continue
            k = (s.name, targets)
            if k not in self.atab:
                words = max(1, rk.atab_words) * s.n_actions
                words += words % 2  # keep each instance's table 8-byte aligned
                self.atab[k] = torch.empty((n, words), dtype=torch.int32, device=dev)

        # ---- item records
        # host copies of the Bellman item records per (period, regime), reused
        # by the simulation (same layout, extended with simulation words)
        self.records: dict[tuple, tuple] = {}
        self.resolvers = resolvers
        self._grp: dict[tuple, dict] = {}  # per (regime, target set) group: records of all periods
        self._geo: dict[tuple, tuple] = {}
        self._ar = np.arange(n, dtype=np.int64)
        b = _Records()
        ages = model.ages.values
        for period, s, targets, rk in step_list:
            if not isinstance(rk, RegimeKernels):
                self._egm_launches(rk, period, s, targets, float(ages[period]), resolvers, b)
                continue
            self._gs_launches(b, rk, period, s, targets, (s.name, targets))
            if (s.name, period) in self._vmu_need:
                self._vmu_launch(b, s, targets, period)
        self.launches = b.launches
        self._rec = b
        for rk in {id(l.module): l.module for l in self.launches if l.kind not in ("fues", "env")}.values():
            eng.module(rk)
        if upload:
            self.items, self.prefix = b.tensors(torch, dev)
        self.graph = None
        self._prepared = None
        self._bundled = None
        # grid-search records of endogenous-grid regimes (simulation only)
        self.sim_launches: list[Launch] = []
        self._sim_prepared = None
        self._egm_steps = [(p_, s_, t_) for p_, s_, t_, _ in egm_steps]

    def _gs_template(self, rk: RegimeKernels, period: int, s: RegimeSpec, targets, pkey) -> dict:
        """Records of one grid-search step at `period` (every instance); the
        other periods of the same regime and target set differ only in the
        period, the age and the slot addresses."""
        n = self.n
        fp32 = self.eng.precision == "fp32"
        resolvers = self.resolvers
        age = float(self.eng.model.ages.values[period])
        pbuf = self.params[pkey]
        out = {"expect": [], "tv": [], "stats": []}
        # kernel (b) records
        for t in rk.targets:
            if t.scalar:
                continue
            if not (t.needs_contraction or fp32):
                continue
            e64, e32, ncols, cblk = self.ev[(s.name, targets, t.spec.name)]
            bst = self.bst.get((s.name, targets, t.spec.name))
            Vt = self.V[t.spec.name]
            tslot = self.slot[t.spec.name][period + 1]
            gs = rk.group_stats(t) if bst is not None else 0
            if gs == 2:
                # the statistics kernel's records (the same every period)
                n1, n2 = (t.spec.states[p].size for p in t.cont_pos)
                srec = np.zeros((n, 5), dtype=np.int64)
                srec[:, 0] = [e32[i].data_ptr() for i in range(n)]
                srec[:, 1] = [bst[i].data_ptr() for i in range(n)]
                srec[:, 2], srec[:, 3], srec[:, 4] = t.K, n1, n2
                out["stats"].append((t, srec, [t.K * ((n1 + rk.GROUP_TILE[0] - 1) // rk.GROUP_TILE[0])] * n))
            recs = []
            for i in range(n):
                r = np.zeros(rk.e_words_for(t), dtype=np.int64)
                r[8 + len(t.spec.states)] = bst[i].data_ptr() if gs == 1 else 0
                r[0] = Vt[i, tslot].data_ptr()
                r[1] = e64[i].data_ptr()
                r[2] = e32[i].data_ptr() if e32 is not None else 0
                r[3] = pbuf[i].data_ptr()
                r[4] = period
                r[5] = _f2w(age)
                r[6] = cblk
                r[7] = ncols
                for k, ax in enumerate(t.spec.states):
                    r[8 + k] = ax.size
                recs.append(r)
            out["expect"].append((t, np.stack(recs).astype(np.int64), [math.ceil(ncols / 256)] * n))
        # kernel (a)
        slot = self.slot[s.name][period]
        recs = []
        for i in range(n):
            r = np.zeros(rk.n_words, dtype=np.int64)
            r[rk.W_P] = pbuf[i].data_ptr()
            r[rk.W_V] = self.V[s.name][i, slot].data_ptr()
            r[rk.W_POL] = self.pol[s.name][i, slot].data_ptr()
            r[rk.W_PERIOD] = period
            r[rk.W_AGE] = _f2w(age)
            r[rk.W_NSTATES] = s.n_states
            r[rk.W_NACT] = s.n_actions
            for k, ax in enumerate(s.states):
                r[rk.W_SSIZE + k] = ax.size
                g = self.sgrid[s.name][k]
                r[rk.W_SGRID + k] = g.data_ptr() if g is not None else 0
            for k, ax in enumerate(s.actions):
                r[rk.W_ASIZE + k] = ax.size
                g = self.agrid[s.name][k]
                r[rk.W_AGRID + k] = g.data_ptr() if g is not None else 0
            r[rk.W_TASTE] = _f2w(rk.tr.taste_scale if rk.tr.taste_scale else 0.0)
            r[rk.W_ATAB] = self.atab[(s.name, targets)][i].data_ptr()
            if s.taste_shocks:
                r[rk.W_TASTE] = _f2w(resolvers[i].taste_scale(s.name))
            for t in rk.targets:
                if t.unreachable:
                    continue
                tV = self.V[t.spec.name]
                tslot = self.slot[t.spec.name][period + 1]
                if t.scalar:
                    r[t.w_scalar] = tV[i, tslot].data_ptr()
                    if i == 0:
                        out["tv"].append((t.w_scalar, t.spec.name))
                    continue
                if t.needs_contraction or fp32:
                    e64, e32, ncols, cblk = self.ev[(s.name, targets, t.spec.name)]
                    r[t.w_ev64] = e64[i].data_ptr()
                    r[t.w_ev32] = e32[i].data_ptr() if e32 is not None else 0
                    bst = self.bst.get((s.name, targets, t.spec.name))
                    r[t.w_bst] = bst[i].data_ptr() if bst is not None else 0
                else:
                    r[t.w_ev64] = tV[i, tslot].data_ptr()
                    r[t.w_ev32] = 0
                    if i == 0:
                        out["tv"].append((t.w_ev64, t.spec.name))
                r[t.w_vraw] = tV[i, tslot].data_ptr()
                if i == 0:
                    out["tv"].append((t.w_vraw, t.spec.name))
                for k, ax in enumerate(t.spec.states):
                    r[t.w_sizes + k] = ax.size
                for ci, pos in enumerate(t.cont_pos):
                    ax = t.spec.states[pos]
                    kind, a, bb, npts = ax.grid.coordinate_spec()
                    base = t.w_coord + 3 * ci
                    if kind == "lin":
                        r[base] = _f2w(a)
                        r[base + 1] = _f2w(1.0 / bb if npts > 1 else 0.0)
                    elif kind == "log":
                        r[base] = _f2w(a)
                        r[base + 1] = _f2w(bb)
                    elif kind == "piece":
                        r[base] = int(a)  # 1: log-spaced segments
                        r[base + 1] = int(bb)  # segments
                        r[base + 2] = self._coord_table(t.spec, pos).data_ptr()
                    else:
                        r[base + 2] = self.sgrid[t.spec.name][pos].data_ptr()
            recs.append(r)
        spt = rk.cfg.states_per_tile
        out["bell"] = np.stack(recs).astype(np.int64)
        out["tiles"] = [math.ceil(s.n_states / spt)] * n
        out["atab_tiles"] = [math.ceil(s.n_actions / 256)] * n
        return out

    def _coord_table(self, spec: RegimeSpec, pos: int):
        """Device copy of a piecewise grid's coordinate table (one per plan)."""
        tabs = self.__dict__.setdefault("_ctabs", {})
        key = (spec.name, pos)
        if key not in tabs:
            tab = spec.states[pos].grid.coordinate_table()
            tabs[key] = self.torch.as_tensor(tab, dtype=self.torch.float64, device=self.dev)
        return tabs[key]

    # ---- device addresses of slot-indexed buffers, per instance
    def _geom(self, key, t, slot_axis: int):
        """(base address, per-instance offsets, per-slot step) of a buffer."""
        g = self._geo.get(key)
        if g is None:
            st = [x * t.element_size() for x in t.stride()]
            g = self._geo[key] = (t.data_ptr(), self._ar * st[1 - slot_axis], st[slot_axis])
        return g

    def _vptrs_many(self, name: str, periods: np.ndarray, pol: bool = False) -> np.ndarray:
        """(periods, instances) device addresses of V[name] (or the policy)."""
        base, inst, step = self._geom(("pol" if pol else "V", name), (self.pol if pol else self.V)[name], 1)
        slots = np.array([self.slot[name][int(p)] for p in periods], dtype=np.int64)
        return base + inst[None, :] + slots[:, None] * step

    def _mptrs_many(self, name: str, periods: np.ndarray) -> np.ndarray:
        """(periods, instances) device addresses of a carried value array's
        marginal-value rows (a two-slot ring indexed by period parity)."""
        base, inst, step = self._geom(("vmu", name), self.vmu[name], 0)
        return base + inst[None, :] + (np.asarray(periods, dtype=np.int64)[:, None] % 2) * step

    def _vmu_launch(self, b: "_Records", s: RegimeSpec, targets, period: int) -> None:
        """Marginal-value rows of regime `s` at `period`, from its value array."""
        vk = self._vck[s.name]
        n = self.n
        pa = np.array([period], dtype=np.int64)
        pbuf = self.params[(s.name, targets)]
        grid = self.sgrid[s.name][[a.name for a in s.states].index(vk.euler)]
        rows = np.zeros((n, vk.n_words), dtype=np.int64)
        rows[:, vk.W_P] = pbuf.data_ptr() + self._ar * pbuf.stride(0) * pbuf.element_size()
        rows[:, vk.W_PERIOD] = period
        rows[:, vk.W_AGE] = self._age_words(pa)[0]
        rows[:, vk.W_V] = self._vptrs_many(s.name, pa)[0]
        rows[:, vk.W_M] = self._mptrs_many(s.name, pa)[0]
        rows[:, vk.W_G] = grid.data_ptr()
        rows[:, vk.W_NG] = grid.numel()
        b.add("egm", vk, vk.name(), rows, [math.ceil(s.n_states / 256)] * n, 256, 0, period)

    def _cptrs_many(self, name: str, field: str, periods: np.ndarray) -> np.ndarray:
        """(periods, instances) device addresses of a DC-EGM carry field
        (a two-slot ring indexed by period parity)."""
        base, inst, step = self._geom(("egm", name, field), self.egm[name][field], 0)
        return base + inst[None, :] + (np.asarray(periods, dtype=np.int64)[:, None] % 2) * step

    def _group_periods(self, s: RegimeSpec, targets) -> np.ndarray:
        return np.array([p for p in s.active_periods if self.eng.targets_at(s, p) == targets], dtype=np.int64)

    def _age_words(self, periods: np.ndarray) -> np.ndarray:
        ages = self.eng.model.ages.values
        return np.array([_f2w(float(ages[int(p)])) for p in periods], dtype=np.int64)

    def _gs_group(self, rk: RegimeKernels, s: RegimeSpec, targets, pkey) -> dict:
        """Records of every period of one grid-search (regime, target set)
        group: (periods, instances, words) arrays built from one template and
        the words that vary with the period (period, age, slot addresses)."""
        pa = self._group_periods(s, targets)
        tm = self._gs_template(rk, int(pa[0]), s, targets, pkey)
        P = len(pa)
        agew = self._age_words(pa)
        g = {"index": {int(p): k for k, p in enumerate(pa)}, "tiles": tm["tiles"], "atab_tiles": tm["atab_tiles"],
             "taste_words": [(rk.W_TASTE, s)] if s.taste_shocks else [], "rk": rk, "spec": s, "periods": pa}
        G = np.repeat(tm["bell"][None], P, axis=0)
        G[:, :, rk.W_V] = self._vptrs_many(s.name, pa)
        G[:, :, rk.W_POL] = self._vptrs_many(s.name, pa, pol=True)
        G[:, :, rk.W_PERIOD] = pa[:, None]
        G[:, :, rk.W_AGE] = agew[:, None]
        for w, tname in tm["tv"]:
            G[:, :, w] = self._vptrs_many(tname, pa + 1)
        g["rows"] = G
        g["expect"] = []
        for t, erows, tiles in tm["expect"]:
            X = np.repeat(erows[None], P, axis=0)
            X[:, :, 0] = self._vptrs_many(t.spec.name, pa + 1)
            X[:, :, 4] = pa[:, None]
            X[:, :, 5] = agew[:, None]
            g["expect"].append((t, X, tiles))
        g["stats"] = {id(t): (srec, tiles) for t, srec, tiles in tm["stats"]}
        return g

    def _gs_launches(self, b: "_Records", rk: RegimeKernels, period: int, s: RegimeSpec, targets, pkey) -> None:
        """Kernel (b) and (a0, a) launches of one grid-search step."""
        key = ("gs", s.name, targets, pkey)
        g = self._grp.get(key)
        if g is None:
            g = self._grp[key] = self._gs_group(rk, s, targets, pkey)
        k = g["index"][period]
        for t, X, tiles in g["expect"]:
            if rk.tc_ok(t):
                # single-precision search: the float table comes from the
                # tensor-core kernel, the double table (the FP64 re-evaluation
                # and the simulation) from kernel (b) with its float output off
                X64 = g.setdefault("x64", {}).get(id(t))
                if X64 is None:
                    X64 = g["x64"][id(t)] = X.copy()
                    X64[:, :, 2] = 0
                b.add("expect", rk, rk.expect_name(t), X64[k], tiles, 256, 0, period)
                sh = rk.tc_shape(t.K, t.J)
                ncols = int(X[k][0, 7])
                b.add("expect_tc", rk, rk.expect_tc_name(t), X[k], [math.ceil(ncols / 128)] * len(tiles), 128,
                      sh["smem"], period)
                # the driver's occupancy query answers one CTA per SM for this
                # kernel; registers and shared memory allow three, and the
                # padded shared memory keeps every CTA's tensor-memory
                # allocation within the SM's 512 columns
                b.launches[-1].grid = SM_COUNT * min(3, sh["max_ctas"])
            else:
                b.add("expect", rk, rk.expect_name(t), X[k], tiles, 256, 0, period)
            st = g["stats"].get(id(t))
            if st is not None:
                b.add("stats", rk, rk.stats_name(), st[0], st[1], 256, 0, period)
        rows = g["rows"][k]
        self.records[(period, s.name)] = (rk, rows)
        b.add("atab", rk, rk.atab_name(), rows, g["atab_tiles"], 256, 0, period)
        # kernel (a) reads the same records
        b.add_same_records("bellman", rk, rk.bellman_name(), g["tiles"], rk.cfg.block, rk.smem_bytes, period)


    def ensure_sim_records(self, upload: bool = True) -> None:
        """Grid-search records of the endogenous-grid regimes.

        The simulate phase decides a DC-EGM regime's actions by the grid
        argmax of Q over its action grid (with the intrinsic budget mask)
        against the solved value functions, like a brute-force regime
        (``src/_lcm/simulation/simulate.py:671-770``: the off-grid policy
        read is disabled for every shipped envelope,
        ``src/_lcm/regime_building/processing.py:1662-1699, 1765-1800``).
        Their expectation / action-table launches run only before a
        simulated period, never in the solve.
        """
        if self.sim_launches or not self._egm_steps:
            return
        self._sim_upload = upload
        torch = self.torch
        eng = self.eng
        n = self.n
        dev = self.dev
        fp32 = eng.precision == "fp32"
        b = _Records()
        for period, s, targets in self._egm_steps:
            rk = eng.kernels(s, targets, self.params_list[0], n)
            pkey = (s.name, targets, "gs")
            if pkey not in self.params:
                self.params[pkey] = torch.as_tensor(rk.tr.pack_many(self.resolvers), dtype=torch.float64, device=dev)
                self._packers[pkey] = lambda r, tr=rk.tr: tr.pack_params(tr.values_for(r))
                self._pack_many[pkey] = rk.tr.pack_many
            for t in rk.targets:
                if t.scalar or not (t.needs_contraction or fp32):
                    continue
                k = (s.name, targets, t.spec.name)
                if k not in self.ev:
                    cblk = int(np.prod([t.spec.states[p].size for p in t.cont_pos])) if t.cont_pos else 1
                    ncols = int(np.prod([t.spec.states[p].size for p in t.det_pos])) * cblk if t.det_pos else cblk
                    e64 = torch.empty((n, t.K, ncols), dtype=torch.float64, device=dev)
                    e32 = torch.empty((n, t.K, ncols), dtype=torch.float32, device=dev) if fp32 else None
                    self.ev[k] = (e64, e32, ncols, cblk)
            k = (s.name, targets)
            if k not in self.atab:
                words = max(1, rk.atab_words) * s.n_actions
                words += words % 2
                self.atab[k] = torch.empty((n, words), dtype=torch.int32, device=dev)
            self._gs_launches(b, rk, period, s, targets, pkey)
        # only the inputs of the simulation: drop the Bellman launches
        b.keep(lambda l: l.kind != "bellman")
        self.sim_launches = b.launches
        self._sim_rec = b
        if upload:
            self.sim_items, self.sim_prefix = b.tensors(torch, dev)
        for rk in {id(l.module): l.module for l in self.sim_launches}.values():
            eng.module(rk)

    def instance(self, idx: int):
        """(engine, Bellman records per (period, regime), row) of instance `idx`."""
        return self.eng, self.records, idx

    def instance_plan(self, idx: int):
        return self, idx

    def sim_groups(self) -> dict:
        """Per regime: (kernels, (periods, instances, words) Bellman records,
        periods) of its grid-search groups -- the records the simulation
        extends (built for every period the regime is active in)."""
        out: dict[str, list] = {}
        for key, g in self._grp.items():
            if key[0] == "gs":
                out.setdefault(g["spec"].name, []).append((g["rk"], g["rows"], g["periods"]))
        return out

    def load_params(self, slot: int, params) -> None:
        """Make instance `slot` solve `params`: its parameter vectors (device,
        copied on the current stream) and its taste-shock words (host
        records: build the launches after this)."""
        torch = self.torch
        res = self.eng.resolver(params)
        self.resolvers[slot] = res
        for key, pack in self._packers.items():
            self.params[key][slot].copy_(torch.from_numpy(np.asarray(pack(res), dtype=np.float64)))
        for g in self._grp.values():
            for w, spec in g["taste_words"]:
                g["rows"][:, slot, w] = _f2w(res.taste_scale(spec.name) if spec.taste_shocks else 0.0)

    # ------------------------------------------------------------- DC-EGM
    def _egm_template(self, ek, period, s, targets, age, resolvers) -> dict:
        """Records of one DC-EGM period (every instance); other periods of the
        same regime and target set differ only in the period, the age and the
        slot addresses."""
        out = {"carry": []}
        n = self.n
        er = ek.er
        b = self.egm[s.name]
        slot = self.slot[s.name][period]
        pbuf = self.params[(s.name, targets)]
        grid = self.sgrid[s.name][[a.name for a in s.states].index(er.E)]
        recs = []
        for i in range(n):
            r = np.zeros(ek.n_words, dtype=np.int64)
            r[ek.W_P] = pbuf[i].data_ptr()
            r[ek.W_PERIOD] = period
            r[ek.W_AGE] = _f2w(age)
            r[ek.W_NSAV] = len(er.savings)
            r[ek.W_SAV] = b["sav"].data_ptr()
            r[ek.W_NGRID] = grid.numel()
            r[ek.W_GRID] = grid.data_ptr()
            for wname, arr in zip(("W_CG", "W_CC", "W_CV", "W_CS"), b["cand"]):
                r[getattr(ek, wname)] = arr[i].data_ptr()
            if b["cm"] is not None:
                r[ek.W_CM] = b["cm"][i].data_ptr()
            r[ek.W_EV0] = b["ev0"][i].data_ptr()
            cslot = period % 2
            r[ek.W_RG] = b["rg"][cslot, i].data_ptr()
            r[ek.W_RC] = b["rc"][cslot, i].data_ptr()
            r[ek.W_RV] = b["rv"][cslot, i].data_ptr()
            r[ek.W_MU] = b["mu"][cslot, i].data_ptr()
            r[ek.W_NK] = b["nk"][cslot, i].data_ptr()
            r[ek.W_V] = self.V[s.name][i, slot].data_ptr()
            r[ek.W_POL] = self.pol[s.name][i, slot].data_ptr()
            r[ek.W_NPAD] = b["npad"]
            r[ek.W_TASTE] = _f2w(resolvers[i].taste_scale(s.name) if s.taste_shocks else 0.0)
            for t, w in zip(er.targets, ek.W_T):
                tslot = self.slot[t.spec.name][period + 1]
                if t.unreachable:
                    continue
                if t.next_R is None:
                    r[w["scalar"]] = self.V[t.spec.name][i, tslot].data_ptr()
                    if i == 0:
                        out["carry"].append((w["scalar"], t.spec.name, None))
                    continue
                if t.is_value:
                    tgrid = self.sgrid[t.spec.name][[a.name for a in t.spec.states].index(t.value_euler)]
                    r[w["tv"]] = self.V[t.spec.name][i, tslot].data_ptr()
                    r[w["tm"]] = self.vmu[t.spec.name][(period + 1) % 2, i].data_ptr()
                    r[w["tg"]] = tgrid.data_ptr()
                    r[w["tn"]] = tgrid.numel()
                    if i == 0:
                        out["carry"].append((w["tv"], t.spec.name, None))
                        out["carry"].append((w["tm"], t.spec.name, "vmu"))
                    continue
                if i == 0:
                    for f in ("rg", "rv", "mu", "nk"):
                        out["carry"].append((w[f], t.spec.name, f))
                cb = self.egm[t.spec.name]
                r[w["rg"]] = cb["rg"][(period + 1) % 2, i].data_ptr()
                r[w["rv"]] = cb["rv"][(period + 1) % 2, i].data_ptr()
                r[w["mu"]] = cb["mu"][(period + 1) % 2, i].data_ptr()
                r[w["nk"]] = cb["nk"][(period + 1) % 2, i].data_ptr()
                r[w["npad"]] = cb["npad"]
                r[w["taste"]] = _f2w(resolvers[i].taste_scale(t.spec.name) if t.spec.taste_shocks else 0.0)
            recs.append(r)
        nrow, npad, ncand = b["nrow"], b["npad"], b["ncand"]
        ns = nrow // er.n_disc_actions
        cg, cc, cv, cs = b["cand"]
        frecs = []
        for i in range(n):
            fr = np.zeros(13, dtype=np.int64)
            fr[0], fr[1], fr[2] = cg[i].data_ptr(), cc[i].data_ptr(), cv[i].data_ptr()
            fr[8], fr[9], fr[10] = nrow, ncand, npad
            fr[11] = _f2w(er.jump_thresh)
            if er.envelope == "fues":
                fr[3] = cs[i].data_ptr()  # exogenous savings sources
                fr[12] = er.scan_window
            else:
                # LTM / RFC item words: 3 the candidates' marginal utility
                # (RFC), 12 the search radius
                fr[3] = b["cm"][i].data_ptr() if er.envelope == "rfc" else 0
                fr[12] = er.search_radius
            frecs.append(fr)
        out["recs"] = np.stack(recs).astype(np.int64)
        out["fues"] = np.stack(frecs).astype(np.int64)
        out["tiles_c"] = [math.ceil(nrow * len(er.savings) / 256)] * n
        out["tiles_f"] = [nrow] * n
        out["tiles_u"] = [math.ceil(nrow * npad / 256)] * n
        out["tiles_p"] = [math.ceil(ns * grid.numel() / 256)] * n
        return out

    def _egm_group(self, ek, s: RegimeSpec, targets, resolvers) -> dict:
        """Records of every period of one DC-EGM (regime, target set) group."""
        pa = self._group_periods(s, targets)
        age0 = float(self.eng.model.ages.values[int(pa[0])])
        tm = self._egm_template(ek, int(pa[0]), s, targets, age0, resolvers)
        P = len(pa)
        name = s.name
        G = np.repeat(tm["recs"][None], P, axis=0)
        G[:, :, ek.W_PERIOD] = pa[:, None]
        G[:, :, ek.W_AGE] = self._age_words(pa)[:, None]
        for w, f in ((ek.W_RG, "rg"), (ek.W_RC, "rc"), (ek.W_RV, "rv"), (ek.W_MU, "mu"), (ek.W_NK, "nk")):
            G[:, :, w] = self._cptrs_many(name, f, pa)
        G[:, :, ek.W_V] = self._vptrs_many(name, pa)
        G[:, :, ek.W_POL] = self._vptrs_many(name, pa, pol=True)
        for w, tname, f in tm["carry"]:
            if f is None:
                G[:, :, w] = self._vptrs_many(tname, pa + 1)
            elif f == "vmu":
                G[:, :, w] = self._mptrs_many(tname, pa + 1)
            else:
                G[:, :, w] = self._cptrs_many(tname, f, pa + 1)
        F = np.repeat(tm["fues"][None], P, axis=0)
        for w, f in ((4, "rg"), (5, "rc"), (6, "rv"), (7, "nk")):
            F[:, :, w] = self._cptrs_many(name, f, pa)
        g = {k: tm[k] for k in ("tiles_c", "tiles_f", "tiles_u", "tiles_p")}
        g.update({"index": {int(p): k for k, p in enumerate(pa)}, "rows": G, "fues": F})
        tw = [(ek.W_TASTE, s)]
        for t, w in zip(ek.er.targets, ek.W_T):
            if not t.unreachable and t.next_R is not None and not t.is_value:
                tw.append((w["taste"], t.spec))
        g["taste_words"] = tw
        return g

    def _egm_launches(self, ek, period, s, targets, age, resolvers, rec: "_Records") -> None:
        """Launches of one DC-EGM period: candidates (c1), FUES, carry
        marginal utilities, publication on the state grid."""
        key = ("egm", s.name, targets)
        g = self._grp.get(key)
        if g is None:
            g = self._grp[key] = self._egm_group(ek, s, targets, resolvers)
        k = g["index"][period]
        er = ek.er
        name = s.name
        rows = g["rows"][k]
        cname, uname, pname = ek.names()
        rec.add("egm", ek, cname, rows, g["tiles_c"], 256, 0, period)
        # FUES over every instance's candidate rows (one tile per row)
        b = self.egm[name]
        ncand = b["ncand"]
        if er.envelope != "fues":
            if ncand > ENVELOPE_MAX_N:
                raise NotImplementedError(
                    f"{name}: the {er.envelope.upper()} envelope handles candidate rows of up to "
                    f"{ENVELOPE_MAX_N} points ({ncand} here)")
            rec.add("env", None, f"lcmx_envelope_step:{ {'ltm': 1, 'rfc': 2, 'mss': 3}[er.envelope]}", g["fues"][k],
                    g["tiles_f"], 0, ncand, period)
        elif ncand <= FUES_SMEM_MAX_N:
            rec.add("fues", None, "lcmx_fues_step", g["fues"][k], g["tiles_f"], 0, ncand, period)
        else:
            rec.append(
                Launch("fues", ("fues", name, period % 2, er.jump_thresh, er.scan_window), "lcmx_fues_scan", 0, 0,
                       self.n * b["nrow"], 0, 0, 0, period)
            )
        rec.add("egm", ek, uname, rows, g["tiles_u"], 256, 0, period)
        rec.add("egm", ek, pname, rows, g["tiles_p"], 256, 0, period)

    def _fues_item_launch(self, l: Launch, ib: int, pb: int):
        from pylcm_b200.runtime import get_context

        ctx = get_context(self.eng.device if hasattr(self, "eng") else self.plans[0].eng.device)
        args = (ib + 8 * l.item_off, pb + 4 * l.prefix_off, l.n_items, l.n_tiles, l.smem)

        def launch(stream):
            ctx.fues_step(*args, stream)

        return launch

    def _env_item_launch(self, l: Launch, ib: int, pb: int):
        """The LTM / RFC envelope over item records (kind in the kernel name)."""
        from pylcm_b200.runtime import get_context

        ctx = get_context(self.eng.device if hasattr(self, "eng") else self.plans[0].eng.device)
        kind = int(l.kernel.rsplit(":", 1)[1])
        args = (ib + 8 * l.item_off, pb + 4 * l.prefix_off, l.n_items, l.n_tiles, l.smem)

        def launch(stream):
            ctx.envelope_step(kind, *args, stream)

        return launch

    def _fues_launch(self, spec_name, slot, thr, window=0, instances=None):
        from pylcm_b200.runtime import get_context

        ctx = get_context(self.eng.device)
        b = self.egm[spec_name]
        cg, cc, cv, cs = b["cand"]
        nrow, ncand, npad = b["nrow"], b["ncand"], b["npad"]
        if instances is None:
            instances = list(range(self.n))
        calls = []
        # one call per instance: a call touches only its instance's rows and
        # its own part of the workspace
        for i in instances:
            ptrs = (cg[i].data_ptr(), cc[i].data_ptr(), cv[i].data_ptr(), cs[i].data_ptr())
            outs = (b["rg"][slot, i].data_ptr(), b["rc"][slot, i].data_ptr(), b["rv"][slot, i].data_ptr())
            nk = b["nk"][slot, i].data_ptr()
            wb = ctx.fues_workspace_bytes(nrow, ncand)
            ws = b["ws"].data_ptr() + i * wb
            calls.append((ptrs, outs, nk, ws, wb))

        def launch(stream):
            for ptrs, outs, nk, ws, wb in calls:
                ctx.fues_scan(*ptrs, nrow, ncand, thr, *outs, npad, nk, ws, wb, stream, n_points_to_scan=window)

        return launch

    # ---------------------------------------------------------------- run
    def _prepare(self, launches=None, items=None, prefix=None) -> list:
        if launches is None:
            launches, items, prefix = self.launches, self.items, self.prefix
        ib = items.data_ptr()
        pb = prefix.data_ptr()
        out = []
        for l in launches:
            if l.kind == "fues":
                out.append(self._fues_item_launch(l, ib, pb) if l.module is None else self._fues_launch(*l.module[1:5]))
                continue
            if l.kind == "env":
                out.append(self._env_item_launch(l, ib, pb))
                continue
            out.append(
                l.module.module.prepared(
                    l.kind, l.kernel, ib + 8 * l.item_off, pb + 4 * l.prefix_off, l.n_items, l.n_tiles, l.block, l.smem,
                    grid=l.grid,
                )
            )
        return out

    def run(self, stream: int | None = None) -> None:
        """Issue every launch of the plan (all periods) on `stream`."""
        if stream is None:
            stream = self.torch.cuda.current_stream(self.dev).cuda_stream
        if self._prepared is None:
            self._prepared = self._prepare()
        if self._bundled is None:
            self._bundled = bundle(self._prepared)
        for launch in self._bundled:
            launch(stream)

    def run_collecting_carries(self) -> dict:
        """Issue every launch on the current stream and keep a copy of each
        period's DC-EGM carry rows before the two-slot ring overwrites them.

        Returns ``{period: {regime: {"rg", "rc", "rv", "mu", "nk"}}}`` with
        device tensors of shape (instances, rows, n_pad) (``nk``: (instances,
        rows)): the refined endogenous grid, policy, value and marginal utility
        of every discrete-state x discrete-action row and its kept count, the
        arrays the reference publishes as ``EGMSimPolicy``
        (``src/_lcm/egm/published_policy.py:76-120``)."""
        stream = self.torch.cuda.current_stream(self.dev).cuda_stream
        if self._prepared is None:
            self._prepared = self._prepare()
        egm_at: dict[int, list] = {}
        for p_, s_, _ in self._egm_steps:
            egm_at.setdefault(p_, []).append(s_.name)
        out: dict[int, dict] = {}

        def snap(period):
            for name in egm_at.get(period, ()):
                b = self.egm[name]
                slot = period % 2
                out.setdefault(period, {})[name] = {f: b[f][slot].clone() for f in ("rg", "rc", "rv", "mu", "nk")}

        cur = None
        for l, launch in zip(self.launches, self._prepared):
            if cur is not None and l.period != cur:
                snap(cur)
            cur = l.period
            launch(stream)
        if cur is not None:
            snap(cur)
        return dict(sorted(out.items()))

    def period_input_ops(self, period: int) -> list:
        """The expectation and action-table launches of one period (the
        simulation reads EV and the action table of that period), then the
        simulation-only launches of that period, as per-launch callables."""
        self.ensure_sim_records()
        by_period = self.__dict__.get("_inputs_by_period")
        if by_period is None:
            if self._prepared is None:
                self._prepared = self._prepare()
            by_period = {}
            for l, launch in zip(self.launches, self._prepared):
                if l.kind in ("expect", "atab"):
                    by_period.setdefault(l.period, []).append(launch)
            if self.sim_launches:
                if self._sim_prepared is None:
                    self._sim_prepared = self._prepare(self.sim_launches, self.sim_items, self.sim_prefix)
                for l, launch in zip(self.sim_launches, self._sim_prepared):
                    by_period.setdefault(l.period, []).append(launch)
            self._inputs_by_period = by_period
        return list(by_period.get(period, []))

    def run_period_inputs(self, period: int, stream: int) -> None:
        """Re-issue the expectation and action-table launches of one period
        (the simulation reads EV and the action table of that period)."""
        if self._prepared is None:
            self._prepared = self._prepare()
        for l, launch in zip(self.launches, self._prepared):
            if l.period == period and l.kind in ("expect", "atab"):
                launch(stream)
        if self.sim_launches:
            if self._sim_prepared is None:
                self._sim_prepared = self._prepare(self.sim_launches, self.sim_items, self.sim_prefix)
            for l, launch in zip(self.sim_launches, self._sim_prepared):
                if l.period == period:
                    launch(stream)

    def capture(self) -> None:
        """Capture the launch list in a CUDA graph (replayed by run_graph)."""
        torch = self.torch
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.run(s.cuda_stream)  # warm-up (module attributes, caches)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        with torch.cuda.graph(g):
            self.run(torch.cuda.current_stream(self.dev).cuda_stream)
        self.graph = g

    def run_graph(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    @property
    def gpu_launches(self) -> int:
        return len(self.launches)

    def check_status(self) -> None:
        """Raise if a bounded device-side wait of this plan's kernels gave up
        (the tensor-core expectation's mbarrier wait).  Synchronous."""
        from pylcm_b200.exceptions import KernelError

        for rk in {id(l.module): l.module for l in self.launches if l.kind == "expect_tc"}.values():
            if rk.module.status(reset=True):
                raise KernelError(7, f"{rk.key}: a tensor-core wait gave up; its float expectation table is incomplete")

    def result(self, i: int) -> tuple[dict, dict]:
        V: dict[int, dict[str, Any]] = {}
        P: dict[int, dict[str, Any]] = {}
        for s in self.eng.specs:
            for period, k in self.slot[s.name].items():
                shape = s.state_shape
                V.setdefault(period, {})[s.name] = self.V[s.name][i, k].reshape(shape)
                P.setdefault(period, {})[s.name] = self.pol[s.name][i, k].reshape(shape)
        return dict(sorted(V.items())), dict(sorted(P.items()))


class BatchPlan:
    """Instances of different models of one family in one launch per kernel.

    A family is a set of models whose regimes generate the same kernels:
    the same functions and state / action structure, with grid sizes,
    horizons (T) and parameters free per instance -- they are item words.
    The instances are slots of solve plans (`slots`: (plan, slot) pairs,
    e.g. a server's pooled plans) or, from `members` ((engine, params)
    pairs), one-slot plans built here.  Their launches are merged:

    - the solve aligns instances by steps from the end (step k is period
      T_i - 1 - k of instance i) and, within a step, merges the i-th launch
      of every instance by kernel: one launch per (step, position, kernel)
      covers every instance with its own tiles;
    - the simulation inputs (expectation and action tables of a period) are
      merged by (period, position, kernel) the same way.
    """

    def __init__(self, members: Sequence = (), slots: Sequence | None = None) -> None:
        import torch

        self.torch = torch
        if slots is None:
            slots = [(SolvePlan(eng, [p], upload=False), 0) for eng, p in members]
        if not slots:
            raise ValueError("empty batch")
        self.slots = list(slots)
        self.n = len(self.slots)
        by_plan: dict[int, tuple] = {}
        for pl, k in self.slots:
            by_plan.setdefault(id(pl), (pl, []))[1].append(k)
        self._by_plan = list(by_plan.values())
        self.plans = [pl for pl, _ in self._by_plan]
        self.dev = self.slots[0][0].dev
        self.launches, self.items, self.prefix = self._merge(
            [(pl, pl._rec, pl.launches, lambda l, pl=pl: pl.eng.model.n_periods - 1 - l.period, sl, "solve")
             for pl, sl in self._by_plan]
        )
        self._prepared = None
        self._bundled = None
        self._inputs = None

    def _merge(self, sources):
        """Merge launch lists (restricted to the given slots of each plan) by
        (key, position within key, kernel)."""
        by_key: dict[int, list] = {}
        for pl, rec, launches, key_of, sl, tag in sources:
            # a plan's launches grouped by key never change: cached on the plan
            cache = pl.__dict__.setdefault("_seq_cache", {})
            seq = cache.get(tag)
            if seq is None:
                seq = {}
                for l, h in zip(launches, rec.host):
                    legacy = l.kind == "fues" and l.module is not None
                    gk = None if legacy else (l.kind, l.kernel, l.module.key if hasattr(l.module, "key") else id(l.module))
                    seq.setdefault(key_of(l), []).append((pl, l, h, gk))
                cache[tag] = seq
            n_pl = pl.n
            sub = None if list(sl) == list(range(n_pl)) else np.asarray(sl, dtype=np.int64)
            for k, lst in seq.items():
                by_key.setdefault(k, []).append((lst, sl, sub))
        b = _Records()
        for k in sorted(by_key):
            lists = by_key[k]
            depth = max(len(x) for x, _, _ in lists)
            for j in range(depth):
                groups: dict[tuple, list] = {}
                for lst, sl, sub in lists:
                    if j >= len(lst):
                        continue
                    pl, l, h, gk = lst[j]
                    if gk is None:
                        b.append(Launch("fues", (pl,) + tuple(l.module[1:5]) + (tuple(sl),), l.kernel, 0, 0,
                                        l.n_items, 0, 0, 0, k))
                        continue
                    arr, tiles = h
                    if sub is not None:
                        arr = arr[sub]
                        tiles = tiles[sub]
                    g = groups.get(gk)
                    if g is None:
                        groups[gk] = [(l, arr, tiles)]
                    else:
                        g.append((l, arr, tiles))
                for gk, members in groups.items():
                    l0 = members[0][0]
                    if len(members) == 1:
                        recs, tiles, smem = members[0][1], members[0][2], l0.smem
                    else:
                        recs = np.concatenate([a for _, a, _ in members])
                        tiles = np.concatenate([ts for _, _, ts in members])
                        smem = max(l.smem for l, _, _ in members)  # FUES: the longest candidate row
                    b.add(l0.kind, l0.module, l0.kernel, recs, tiles, l0.block, smem, k)
                    b.launches[-1].grid = l0.grid
        items, prefix = b.tensors(self.torch, self.dev)
        return b.launches, items, prefix

    def _prepare(self, launches, items, prefix) -> list:
        ib = items.data_ptr()
        pb = prefix.data_ptr()
        out = []
        for l in launches:
            if l.kind == "fues":
                if l.module is None:
                    out.append(SolvePlan._fues_item_launch(self, l, ib, pb))
                else:
                    pl, name, slot, thr, window, sl = l.module
                    out.append(pl._fues_launch(name, slot, thr, window, sl))
                continue
            if l.kind == "env":
                out.append(SolvePlan._env_item_launch(self, l, ib, pb))
                continue
            out.append(
                l.module.module.prepared(
                    l.kind, l.kernel, ib + 8 * l.item_off, pb + 4 * l.prefix_off, l.n_items, l.n_tiles, l.block, l.smem,
                    grid=l.grid,
                )
            )
        return out

    def run(self, stream: int | None = None) -> None:
        if stream is None:
            stream = self.torch.cuda.current_stream(self.dev).cuda_stream
        if self._prepared is None:
            self._prepared = self._prepare(self.launches, self.items, self.prefix)
        if self._bundled is None:
            self._bundled = bundle(self._prepared)
        for launch in self._bundled:
            launch(stream)

    @property
    def gpu_launches(self) -> int:
        return len(self.launches)

    # -------------------------------------------------------- simulation
    def ensure_sim_records(self) -> None:
        if self._inputs is not None:
            return
        sources = []
        for pl, sl in self._by_plan:
            pl.ensure_sim_records(upload=False)
            rec = pl.__dict__.get("_sim_input_rec")
            if rec is None:
                rec = _Records()
                rec.launches, rec.host, rec.shared = list(pl._rec.launches), list(pl._rec.host), list(pl._rec.shared)
                rec.keep(lambda l: l.kind in ("expect", "atab"))
                pl._sim_input_rec = rec
            sources.append((pl, rec, rec.launches, lambda l: l.period, sl, "sim_inputs"))
            if pl.sim_launches:
                sources.append((pl, pl._sim_rec, pl.sim_launches, lambda l: l.period, sl, "sim_only"))
        launches, items, prefix = self._merge(sources)
        self._inputs = (launches, items, prefix, self._prepare(launches, items, prefix))

    def period_input_ops(self, period: int) -> list:
        self.ensure_sim_records()
        by_period = self.__dict__.get("_inputs_by_period")
        if by_period is None:
            launches, _, _, prepared = self._inputs
            by_period = {}
            for l, launch in zip(launches, prepared):
                by_period.setdefault(l.period, []).append(launch)
            self._inputs_by_period = by_period
        return by_period.get(period, [])

    def run_period_inputs(self, period: int, stream: int) -> None:
        for launch in bundle(self.period_input_ops(period)):
            launch(stream)

    def instance(self, idx: int):
        pl, slot = self.slots[idx]
        return pl.eng, pl.records, slot

    def instance_plan(self, idx: int):
        return self.slots[idx]

    def result(self, i: int) -> tuple[dict, dict]:
        pl, slot = self.slots[i]
        return pl.result(slot)
