"""Forward simulation on the GPU (kernel (d)).

Restates the reference's simulation loop (``src/_lcm/simulation/simulate.py:74-668``):
for each period, for each regime active in it, every subject currently in
that regime takes the argmax of Q at its own (off-grid) state -- the same
Q evaluation as the solve, reading next period's value function -- and then
draws its next regime and next states.

Two random streams, both independent of the batch a subject is simulated
in:

- ``rng="jax"`` (``Model.simulate``'s default): the reference's own stream,
  JAX's Threefry-2x32 with the reference's key threading
  (``pylcm_b200.jaxrng``): the host walks the key chain of each simulation
  (a handful of hashes per period and regime) and hands every (period,
  regime) item the keys the reference splits per subject; the kernel derives
  each subject's key and draw on the device.  Simulations reproduce the
  reference's stored ones;
- ``rng="philox"`` (the serving loop): a counter-based Philox-4x32-10 stream
  keyed by the seed and indexed by (subject, period, stream id), with no
  host-side key chain.
"""

from __future__ import annotations

import math
from typing import Mapping

import numpy as np

from pylcm_b200.exceptions import InvalidInitialConditionsError, InvalidParamsError
from pylcm_b200.grids import DiscreteGrid
from pylcm_b200.runtime import bundle


class SimulationResult:
    """Raw simulated arrays plus ``to_dataframe()`` (``src/lcm/result.py``)."""

    def __init__(self, model, periods: dict) -> None:
        self.model = model
        self.periods = periods  # period -> dict of arrays

    @property
    def n_subjects(self) -> int:
        return len(next(iter(self.periods.values()))["regime_id"])

    def to_dataframe(self, terminal_rows: str = "all"):
        import pandas as pd

        specs = self.model.regime_specs
        by_id = {s.rid: s for s in specs}
        state_names = sorted({a.name for s in specs for a in s.states})
        action_names = sorted({a.name for s in specs for a in s.actions})
        grids = {}
        for s in specs:
            for a in s.states + s.actions:
                grids.setdefault(a.name, a.grid)
        cols: dict[str, list] = {k: [] for k in ["subject_id", "period", "regime_name", "value", *state_names, *action_names, "age"]}
        ages = self.model.ages.values
        for p in sorted(self.periods):
            d = self.periods[p]
            rid = d["regime_id"]
            for i in range(len(rid)):
                r = int(rid[i])
                if r < 0:
                    continue
                spec = by_id[r]
                if spec.terminal and terminal_rows == "none":
                    continue
                cols["subject_id"].append(i)
                cols["period"].append(p)
                cols["regime_name"].append(spec.name)
                cols["value"].append(float(d["value"][i]))
                own_s = {a.name for a in spec.states}
                own_a = {a.name for a in spec.actions}
                for n in state_names:
                    cols[n].append(float(d["states"][n][i]) if n in own_s else np.nan)
                for n in action_names:
                    cols[n].append(float(d["actions"][n][i]) if n in own_a else np.nan)
                cols["age"].append(float(ages[p]))
        df = pd.DataFrame(cols)
        df["regime_name"] = pd.Categorical(df["regime_name"], categories=[s.name for s in specs])
        for n in state_names + action_names:
            g = grids[n]
            if isinstance(g, DiscreteGrid):
                codes = df[n].to_numpy()
                labels = np.array([g.categories[int(c)] if np.isfinite(c) else None for c in codes], dtype=object)
                df[n] = pd.Categorical(labels, categories=list(g.categories))
        return df


def _initial_arrays(model, initial_conditions: Mapping) -> tuple[np.ndarray, dict]:
    ic = dict(initial_conditions)
    rid = ic.pop("regime_id", ic.pop("regime", None))
    if rid is None:
        raise InvalidInitialConditionsError("initial_conditions needs 'regime_id'")
    rid = np.asarray(rid).astype(np.int64)
    n = rid.shape[0]
    if "age" in ic:
        ages = np.asarray(ic.pop("age"), dtype=np.float64)
        if not np.all(ages == model.ages.values[0]):
            raise InvalidInitialConditionsError("all subjects must start at the first age of the age grid")
    states = {}
    for k, v in ic.items():
        a = np.asarray(v, dtype=np.float64)
        if a.shape != (n,):
            raise InvalidInitialConditionsError(f"initial condition {k!r} must have shape ({n},)")
        states[k] = a
    return rid, states


def _stochastic_names(spec, specs, model, resolver) -> list[tuple[str, str, str]]:
    """(qualified name, target, state) of the stochastic next-state functions
    whose per-subject keys the reference splits for regime `spec`, sorted by
    name (``transitions.py:111-125``): the Markov and process laws toward
    every target the regime's transition reaches with positive probability in
    some period and that it has a law for every state of."""
    from pylcm_b200.regime import MarkovTransition
    from pylcm_b200.spec import _unreachable
    from pylcm_b200.validation import _regime_probs

    reach = set()
    for period in spec.active_periods:
        if period + 1 >= model.n_periods:
            continue
        P, _ = _regime_probs(spec, specs, resolver, period, float(model.ages.values[period]))
        for t in specs:
            if np.any(np.nan_to_num(P[:, t.rid]) > 0):
                reach.add(t.name)
    out = []
    for t in specs:
        if t.name not in reach or not t.states or _unreachable(spec, t):
            continue
        for ax in t.states:
            law = spec.functions.get(f"next_{ax.name}")
            if ax.kind == "process" or isinstance(law, MarkovTransition):
                out.append((f"{t.name}__next_{ax.name}", t.name, ax.name))
    return sorted(out)


def jax_key_chain(model, params, seed: int) -> dict:
    """The reference's key threading over one simulation
    (``simulate.py:275, 562-572, 630``, ``transitions.py:119, 260``):
    {(period, regime): {"regime": key, "taste": key, (target, state): key}},
    each the key the reference splits into one key per subject."""
    from pylcm_b200 import jaxrng
    from pylcm_b200.spec import ParamResolver

    specs = model.regime_specs
    res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    # the names depend on the params (reachability): cached for the last
    # params object (kept alive with its entry, so its id is not reused)
    cache = model.__dict__.setdefault("_jax_names", {})
    hit = cache.get(id(params))
    if hit is not None and hit[0] is params:
        names = hit[1]
    else:
        names = {s.name: _stochastic_names(s, specs, model, res) for s in specs if not s.terminal}
        cache.clear()
        cache[id(params)] = (params, names)
    by_name = {s.name: s for s in specs}
    order = [by_name[n] for n in model.user_regimes]
    key = jaxrng.key(seed)
    chain = {}
    for period in range(model.n_periods):
        for s in order:
            if period not in s.active_periods:
                continue
            d = {}
            if s.taste_shocks:
                d["taste"] = key
                key = jaxrng.split(key, 1)[0]  # the running key: counters (0, 0)
            if not s.terminal:
                ks = jaxrng.split(key, 3)
                run, d["regime"], key = ks[0], ks[1], ks[2]
                for _, tname, state in names[s.name]:
                    d[(tname, state)] = run
                    run = jaxrng.split(run, 1)[0]
            chain[(period, s.name)] = d
    return chain


class SimPlan:
    """Device buffers and launches of the simulations of solve instances.

    `instances` lists (solve-plan instance, initial conditions, seed).  Per
    period, one kernel (d) launch per kernel covers every listed instance
    whose regime uses it, each instance with its own subjects, buffers,
    horizon and seed (the Philox key of an item is the launch seed XOR the
    item's seed word; the launch seed is 0 here).  `solve_plan` is a
    `SolvePlan` (one model) or a `BatchPlan` (a model family).
    """

    def __init__(self, solve_plan, initial_conditions: Mapping | None = None, seed: int = 0,
                 instances: list | None = None, rng: str = "philox", params: Mapping | None = None) -> None:
        """`rng="jax"` draws from the reference's stream and needs the
        instances' `params` (one mapping, or one per instance) for its key
        chain; "philox" draws from the counter stream."""
        import torch

        self.torch = torch
        self._bundled = None
        self.plan = solve_plan
        dev = solve_plan.dev
        if rng not in ("philox", "jax"):
            raise ValueError("rng must be 'philox' or 'jax'")
        if instances is None:
            instances = [(0, initial_conditions, seed)]
        solve_plan.ensure_sim_records()
        nan = float("nan")
        self.inst = []
        for ii, (idx, ic, sd) in enumerate(instances):
            if not 0 <= idx < solve_plan.n:
                raise InvalidParamsError(f"instance {idx} outside the solve plan's batch of {solve_plan.n}")
            eng, records, row = solve_plan.instance(idx)
            model = eng.model
            specs = eng.specs
            rid0, states0 = _initial_arrays(model, ic)
            for s in specs:
                for a in s.states:
                    if a.name not in states0 and (rid0 == s.rid).any():
                        raise InvalidInitialConditionsError(f"initial_conditions lacks state {a.name!r} of regime {s.name!r}")
            self.inst.append({
                "idx": idx,
                "eng": eng,
                "records": records,
                "row": row,
                "T": model.n_periods,
                "N": rid0.shape[0],
                "seed": int(sd) & 0xFFFFFFFFFFFFFFFF,
                "names": sorted({a.name for s in specs for a in s.states}),
                "anames": sorted({a.name for s in specs for a in s.actions}),
                "rid0": rid0,
                "states0": states0,
                "chain": (jax_key_chain(model, params if isinstance(params, Mapping) or params is None else params[ii],
                                        int(sd)) if rng == "jax" else None),
            })
            if rng == "jax" and params is None:
                raise InvalidParamsError("rng='jax' needs the instances' params for the key chain")
        # one (instances, periods, subjects) buffer per array for each group of
        # instances with the same horizon and subject count; each instance
        # works on its own slice (contiguous rows of N subjects)
        by_shape: dict[tuple, list] = {}
        for i, b in enumerate(self.inst):
            by_shape.setdefault((b["T"], b["N"]), []).append(i)
        self.groups = []
        for (T, N), members in by_shape.items():
            n_g = len(members)
            names = sorted({n for i in members for n in self.inst[i]["names"]})
            anames = sorted({n for i in members for n in self.inst[i]["anames"]})
            g = {
                "T": T,
                "N": N,
                "members": members,
                "S": {n: torch.full((n_g, T + 1, N), nan, dtype=torch.float64, device=dev) for n in names},
                "A": {n: torch.full((n_g, T, N), nan, dtype=torch.float64, device=dev) for n in anames},
                "R": torch.full((n_g, T + 1, N), -1, dtype=torch.int32, device=dev),
                "val": torch.full((n_g, T, N), nan, dtype=torch.float64, device=dev),
                "aidx": torch.zeros((n_g, T, N), dtype=torch.int32, device=dev),
            }
            # initial states and regimes: one host array and one copy per array
            for n in names:
                h = np.full((n_g, N), np.nan)
                for k, i in enumerate(members):
                    if n in self.inst[i]["states0"]:
                        h[k] = self.inst[i]["states0"][n]
                g["S"][n][:, 0, :].copy_(torch.from_numpy(h))
            g["R"][:, 0, :].copy_(torch.from_numpy(np.stack([self.inst[i]["rid0"] for i in members]).astype(np.int32)))
            for k, i in enumerate(members):
                b = self.inst[i]
                b["S"] = {n: g["S"][n][k] for n in b["names"]}
                b["A"] = {n: g["A"][n][k] for n in b["anames"]}
                b["R"] = g["R"][k]
                b["val"] = g["val"][k]
                b["aidx"] = g["aidx"][k]
                del b["rid0"], b["states0"]
            self.groups.append(g)
        self.T = max(b["T"] for b in self.inst)
        # item records: the Bellman record of (period, regime, instance) +
        # simulation words, built per (instance, regime, kernel) for all its
        # periods at once, then grouped per (period, kernel) with one sort
        by_kernel: dict[tuple, list] = {}
        jtabs: list[np.ndarray] = []  # JAX-stream key tables, laid out in one device buffer
        jrefs: list[tuple] = []  # (rows array, row indices, table offsets in words)
        jwords = 0
        for b in self.inst:
            N, T = b["N"], b["T"]
            sbytes = N * 8  # one period of a subject array (float64)
            ibytes = N * 4  # one period of an int32 subject array
            S0 = {n: t.data_ptr() for n, t in b["S"].items()}
            A0 = {n: t.data_ptr() for n, t in b["A"].items()}
            R0, V0, X0 = b["R"].data_ptr(), b["val"].data_ptr(), b["aidx"].data_ptr()
            seed_w = np.uint64(b["seed"]).astype(np.int64)
            tiles = math.ceil(N / 8)
            pl, row = self.plan.instance_plan(b["idx"])
            for s in b["eng"].specs:
                for rk, G, gp in pl.sim_groups().get(s.name, []):
                    keep = gp < T
                    if not keep.any():
                        continue
                    b["eng"].module(rk)
                    pa = gp[keep]
                    rows = np.zeros((len(pa), rk.sim_words), dtype=np.int64)
                    rows[:, : rk.n_words] = G[keep, row, :]
                    rows[:, rk.SW_N] = N
                    rows[:, rk.SW_RID_IN] = R0 + pa * ibytes
                    rows[:, rk.SW_RID_OUT] = R0 + (pa + 1) * ibytes
                    rows[:, rk.SW_VAL] = V0 + pa * sbytes
                    rows[:, rk.SW_AIDX] = X0 + pa * ibytes
                    rows[:, rk.SW_SEED] = seed_w
                    for k, a in enumerate(s.actions):
                        rows[:, rk.SW_ACT + k] = A0[a.name] + pa * sbytes
                    for k, a in enumerate(s.states):
                        rows[:, rk.SW_SIN + k] = S0[a.name] + pa * sbytes
                    for k, name in enumerate(rk.sim_out_names):
                        rows[:, rk.SW_SOUT + k] = S0[name] + (pa + 1) * sbytes
                    if b["chain"] is not None:
                        offs = []
                        for p_ in pa:
                            tab = np.zeros((rk.sim_n_slots, 2), dtype=np.uint32)
                            d = b["chain"].get((int(p_), s.name), {})
                            if "regime" in d:
                                tab[0] = d["regime"]
                            if "taste" in d:
                                tab[1] = d["taste"]
                            for (tname, state), q in rk.sim_slot.items():
                                if (tname, state) in d:
                                    tab[q] = d[(tname, state)]
                            # 16-byte aligned tables (uint32 words)
                            jtabs.append(np.concatenate([tab.reshape(-1), np.zeros((-tab.size) % 4, np.uint32)]))
                            offs.append(jwords)
                            jwords += jtabs[-1].size
                        jrefs.append((rows, rk.SW_JKEYS, np.asarray(offs, dtype=np.int64)))
                    g = by_kernel.setdefault((rk.sim_name(), rk.key), [rk, [], [], []])
                    g[1].append(rows)
                    g[2].append(pa)
                    g[3].append(np.full(len(pa), tiles, dtype=np.int64))
        # the key tables' device buffer; the item words point into it
        # uint32 words, moved bit for bit through an int32 view
        self.jkeys = torch.from_numpy(np.concatenate(jtabs).view(np.int32)).to(dev) if jtabs else None
        if jtabs:
            base = self.jkeys.data_ptr()
            for rows, w, offs in jrefs:
                rows[:, w] = base + 4 * offs
        pieces = []  # (period, kernel order, rk, rows, tiles)
        for order, (rk, rows_l, per_l, til_l) in enumerate(by_kernel.values()):
            rows = np.concatenate(rows_l)
            per = np.concatenate(per_l)
            til = np.concatenate(til_l)
            o = np.argsort(per, kind="stable")
            rows, per, til = rows[o], per[o], til[o]
            cuts = np.flatnonzero(np.diff(per)) + 1
            for r_, p_, t_ in zip(np.split(rows, cuts), np.split(per, cuts), np.split(til, cuts)):
                pieces.append((int(p_[0]), order, rk, r_, t_))
        pieces.sort(key=lambda x: (x[0], x[1]))
        recs = []
        prefs = []
        self.launches = []
        off = 0
        poff = 0
        for period, _, rk, rows, tiles in pieces:
            npre = len(tiles) + 1
            pre = np.zeros(npre + (-npre) % 4, dtype=np.int32)
            np.cumsum(tiles, out=pre[1:npre])
            prefs.append(pre)
            recs.append(rows.reshape(-1))
            self.launches.append((period, rk, off, poff, len(rows), int(pre[npre - 1])))
            off += rows.size
            poff += pre.size
        self.items = torch.as_tensor(np.concatenate(recs), dtype=torch.int64, device=dev)
        self.prefix = torch.as_tensor(np.concatenate(prefs), dtype=torch.int32, device=dev)

    def run(self, stream: int | None = None) -> None:
        torch = self.torch
        if stream is None:
            stream = torch.cuda.current_stream(self.plan.dev).cuda_stream
        if self._bundled is None:
            # each period's inputs (expectation and action tables), then its
            # simulation launches: one launch list per run of item launches
            ib, pb = self.items.data_ptr(), self.prefix.data_ptr()
            ops: list = []
            done_inputs = set()
            for period, rk, off, poff, n_items, tiles in self.launches:
                if period not in done_inputs:
                    ops += self.plan.period_input_ops(period)
                    done_inputs.add(period)
                ops.append(rk.module.prepared("sim", rk.sim_name(), ib + 8 * off, pb + 4 * poff, n_items, tiles, 256, 0,
                                              seed=0))
            self._bundled = bundle(ops)
        for launch in self._bundled:
            launch(stream)

    @property
    def gpu_launches(self) -> int:
        return len(self.launches)

    def result(self, model=None, k: int = 0) -> SimulationResult:
        torch = self.torch
        torch.cuda.current_stream(self.plan.dev).synchronize()
        b = self.inst[k]
        model = b["eng"].model if model is None else model
        periods = {}
        R = b["R"].cpu().numpy()
        V = b["val"].cpu().numpy()
        S = {n: v.cpu().numpy() for n, v in b["S"].items()}
        A = {n: v.cpu().numpy() for n, v in b["A"].items()}
        for p in range(b["T"]):
            periods[p] = {
                "regime_id": R[p],
                "value": V[p],
                "states": {n: S[n][p] for n in S},
                "actions": {n: A[n][p] for n in A},
            }
        return SimulationResult(model, periods)


def simulate(model, *, params, initial_conditions, V_arr=None, seed: int = 0, precision: str = "fp64",
             log_level: str = "progress", rng: str = "jax") -> SimulationResult:
    """Solve (unless `V_arr` is given) and simulate `initial_conditions`
    (random stream `rng`: "jax", the reference's, or "philox")."""
    import torch

    eng = model.engine(precision)
    plan = eng.plan([params])
    if V_arr is None:
        plan.run()
    else:
        for p, regs in V_arr.items():
            for r, v in regs.items():
                k = plan.slot[r].get(int(p))
                if k is not None:
                    plan.V[r][0, k].copy_(torch.as_tensor(np.asarray(v, dtype=np.float64).reshape(-1)))
    sim = SimPlan(plan, initial_conditions, seed, rng=rng, params=params)
    sim.run()
    return sim.result(model)
