"""Forward simulation on the GPU (kernel (d)).

Restates the reference's simulation loop (``src/_lcm/simulation/simulate.py:74-668``):
for each period, for each regime active in it, every subject currently in
that regime takes the argmax of Q at its own (off-grid) state -- the same
Q evaluation as the solve, reading next period's value function -- and then
draws its next regime and next states.

Draws use a counter-based Philox-4x32-10 stream keyed by the seed and
indexed by (subject, period, stream id), so a subject's path does not depend
on the batch it is simulated in.  The reference draws with JAX's threefry
keys, so paths with stochastic draws agree with it in distribution, not
bitwise; paths without draws agree exactly.
"""

from __future__ import annotations

import math
from typing import Any, Mapping

import numpy as np

from pylcm_b200.exceptions import InvalidInitialConditionsError, InvalidParamsError
from pylcm_b200.grids import DiscreteGrid


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
                 instances: list | None = None) -> None:
        import torch

        self.torch = torch
        self.plan = solve_plan
        dev = solve_plan.dev
        if instances is None:
            instances = [(0, initial_conditions, seed)]
        solve_plan.ensure_sim_records()
        nan = float("nan")
        self.inst = []
        for idx, ic, sd in instances:
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
            })
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
                    g = by_kernel.setdefault((rk.sim_name(), rk.key), [rk, [], [], []])
                    g[1].append(rows)
                    g[2].append(pa)
                    g[3].append(np.full(len(pa), tiles, dtype=np.int64))
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
        ib, pb = self.items.data_ptr(), self.prefix.data_ptr()
        done_inputs = set()
        for period, rk, off, poff, n_items, tiles in self.launches:
            if period not in done_inputs:
                self.plan.run_period_inputs(period, stream)
                done_inputs.add(period)
            rk.module.simulate(rk.sim_name(), ib + 8 * off, pb + 4 * poff, n_items, tiles, 256, 0, 0, stream)

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
             log_level: str = "progress") -> SimulationResult:
    """Solve (unless `V_arr` is given) and simulate `initial_conditions`."""
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
    sim = SimPlan(plan, initial_conditions, seed)
    sim.run()
    return sim.result(model)
