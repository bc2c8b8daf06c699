"""Benchmark: model solves/sec of the stochastic retirement model.

Workload (one "step" = one batched backward-induction solve):
    stochastic consumption-savings model with a work/retire choice -- 7-node
    Tauchen AR(1) log income (rho=0.9, sigma=0.1, +-3 sd) multiplying the wage,
    wealth and consumption on linspace(1, 400, 500), labour {work, retire},
    CRRA utility, T=40: 40 x 7 x 500 states x 500 x 2 actions per solve.
    A step solves B seeded parameter draws (beta ~ U[0.94, 0.97],
    crra ~ U[1.5, 2.5], r ~ U[0.03, 0.05]) at once.

Forms measured on the GPU:
    fast  -- batched, single-precision search with double-precision
             re-evaluation, one CUDA graph per step (`value`);
    plain -- one solve at a time, FP64, eager launches, per-solve NaN check.
Accuracy of fast vs plain (max relative V error, policy agreement) is
measured on every run.

``--impl reference`` times the CPU oracle (a NumPy float64 restatement of the
reference's solve; the reference itself is JAX, which cannot run here).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "model solves/sec (stochastic retirement model, T=40, 7x500 states, 1000 actions)"
UNIT = "solves/s"


def make_workload(n_periods: int, n_wealth: int, n_cons: int, batch: int, seed: int = 0):
    from tests import models as M

    model = M.stochastic_model(n_periods, n_wealth, n_cons)
    rng = np.random.default_rng(seed)
    params = [
        M.stochastic_params(
            beta=float(rng.uniform(0.94, 0.97)),
            crra=float(rng.uniform(1.5, 2.5)),
            interest_rate=float(rng.uniform(0.03, 0.05)),
        )
        for _ in range(batch)
    ]
    return model, params


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = (
        "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device: int = 0) -> None:
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL,
                text=True,
            )
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        self.out = out

    def summary(self) -> dict:
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": sorted(reasons)}
        loaded = [x for x in sm if x > 0.5 * (smax or max(sm))] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(torch, buf) -> None:
    buf.add_(1.0)  # writes 256 MiB > 126 MB L2


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# --------------------------------------------------------------------------
def run_ours(args) -> dict:
    import torch
    import torch.distributed as dist

    from pylcm_b200.batch import BatchSolver

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://")
    model, params = make_workload(args.periods, args.wealth, args.cons, args.batch, seed=1000 * rank)
    fast = BatchSolver(model, args.batch, "fp32", template_params=params[0], device=local)
    packed = fast.pack(params)
    fast.upload(packed)
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        fast.run()
    torch.cuda.synchronize()

    # ---- device-timed fast form (inputs resident, L2 flushed between steps)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush_l2(torch, flush)
            ev[k][0].record(stream)
            fast.run()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([t_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    value = world * args.batch * args.steps / (t_ms / 1e3)

    # ---- end to end through the public batch API (host params -> host V)
    torch.cuda.synchronize()
    e2e_ms = []
    h2d = d2h = 0
    for k in range(max(1, min(args.steps, 3))):
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        s0.record(stream)
        pk = fast.pack(params)
        h2d = fast.upload(pk)
        fast.run()
        d2h = fast.download(policy=False)
        s1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_value = args.batch / (statistics.median(e2e_ms) / 1e3) * world

    # ---- kernel-level timing of the dominant kernel (kernel a), eager, events
    plan = fast.plan
    prepared = plan._prepare()
    k_times, k_bytes, k_evals = [], [], []
    e_times = []
    flush_l2(torch, flush)
    torch.cuda.synchronize()
    for l, launch in zip(plan.launches, prepared):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        launch(stream.cuda_stream)
        b.record(stream)
        if l.kind == "bellman":
            spec = l.module.spec
            ns, na = spec.n_states, spec.n_actions
            # algorithmic bytes: read EV (float copy) rows of every target + write V, policy
            rd = sum(
                (t.K * (np.prod([t.spec.states[p].size for p in t.det_pos + t.cont_pos]) if not t.scalar else 1)) * 4
                for t in l.module.targets
            )
            k_bytes.append(l.n_items * (rd + ns * (8 + 4)))
            k_evals.append(l.n_items * ns * na)
            k_times.append((a, b))
        else:
            e_times.append((a, b))
    torch.cuda.synchronize()
    kt = [a.elapsed_time(b) for a, b in k_times]
    et = [a.elapsed_time(b) for a, b in e_times]
    avg_k_ms = float(np.mean(kt))
    bytes_per_launch = float(np.mean(k_bytes))
    evals_per_launch = float(np.mean(k_evals))
    pk_ = peaks()
    achieved_gbs = bytes_per_launch / (avg_k_ms / 1e3) / 1e9

    # ---- plain form: FP64, one solve at a time, eager launches
    from pylcm_b200.engine import SolveEngine

    n_plain = min(args.plain_samples, args.batch)
    plain_eng = SolveEngine(model, "fp64", device=local)
    plain_plan = plain_eng.plan([params[0]])
    plain_plan.run(stream.cuda_stream)  # warm-up: first launches load the kernels
    torch.cuda.synchronize()
    pl_ms = []
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    from pylcm_b200.runtime import get_context

    ctx = get_context(local)
    Vplain = []
    for i in range(n_plain):
        rk_pk = {}
        for key in plain_plan.params:
            name, targets = key
            spec = next(s for s in plain_eng.specs if s.name == name)
            rk = plain_eng.kernels(spec, targets, params[0], 1)
            rk_pk[key] = rk.tr.pack_params(rk.tr.values_for(plain_eng.resolver(params[i])))
        for key, arr in rk_pk.items():
            plain_plan.params[key].copy_(torch.as_tensor(arr[None], device="cuda"))
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plain_plan.run(stream.cuda_stream)
        counts.zero_()
        for r, v in plain_plan.V.items():
            ctx.count_nonfinite(v.data_ptr(), v.numel(), counts.data_ptr(), stream.cuda_stream)
        _ = counts.cpu()
        b.record(stream)
        torch.cuda.synchronize()
        pl_ms.append(a.elapsed_time(b))
        Vplain.append({r: v.clone() for r, v in plain_plan.V.items()})
    plain_value = 1e3 / float(np.mean(pl_ms))

    # ---- accuracy of the fast form against FP64 (first n_plain instances)
    torch.cuda.synchronize()
    fast.run()
    torch.cuda.synchronize()
    max_rel = 0.0
    agree = tot = 0
    for i in range(n_plain):
        for r, v in Vplain[i].items():
            vf = fast.plan.V[r][i]
            vp = v[0]
            fin = torch.isfinite(vp)
            if fin.any():
                d = ((vf - vp).abs() / vp.abs().clamp_min(1.0))[fin].max().item()
                max_rel = max(max_rel, d)
    # policy agreement on instance 0 (re-solve it with the plain form)
    for key in plain_plan.params:
        name, targets = key
        spec = next(s for s in plain_eng.specs if s.name == name)
        rk = plain_eng.kernels(spec, targets, params[0], 1)
        plain_plan.params[key].copy_(
            torch.as_tensor(rk.tr.pack_params(rk.tr.values_for(plain_eng.resolver(params[0])))[None], device="cuda")
        )
    plain_plan.run(stream.cuda_stream)
    torch.cuda.synchronize()
    for r in plain_plan.pol:
        a_ = plain_plan.pol[r][0]
        b_ = fast.plan.pol[r][0]
        vp = plain_plan.V[r][0]
        m = torch.isfinite(vp)
        agree += int((a_ == b_)[m].sum().item())
        tot += int(m.sum().item())

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return {}
    spec0 = model.regime_specs
    evals_per_solve = sum(s.n_states * s.n_actions * len(s.active_periods) for s in spec0)
    fl_per_eval = 20  # ~20 flops per (state, action) evaluation of the mixed part
    clocks = clk.summary()
    return {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 search + f64 re-evaluation (fast); f64 (plain)",
        "data": "synthetic (seeded parameter draws)",
        "config": {
            "workload": "stochastic retirement model (Tauchen 7-node income), T=40, wealth/consumption 500/500, 2 labour choices",
            "batch_per_gpu": args.batch,
            "periods": args.periods,
            "wealth_points": args.wealth,
            "consumption_points": args.cons,
            "precision": "fp32 search, fp64 value",
            "parallelism": f"replicas x{world} (independent solves per GPU)",
            "l2": "flushed between timed steps (256 MiB write)",
        },
        "plain": {
            "value": plain_value,
            "unit": UNIT,
            "ms_per_solve": float(np.mean(pl_ms)),
            "form": "fp64, one solve at a time, eager launches + per-solve NaN/Inf count",
            "samples": n_plain,
        },
        "fast_vs_plain": value / world / plain_value,
        "accuracy": {
            "max_rel_V_err_vs_fp64": max_rel,
            "policy_agreement_vs_fp64": agree / max(tot, 1),
            "instances_checked": n_plain,
        },
        "e2e": {
            "value": e2e_value,
            "unit": UNIT,
            "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h),
            "api": "pylcm_b200.batch.BatchSolver pack+upload+run+download (host params -> host V)",
        },
        "gpu_launches": fast.gpu_launches * args.steps,
        "roofline": {
            "kernel": "lcm_bellman (kernel a: fused Q_and_F + max/argmax)",
            "bound": "hbm",
            "achieved": achieved_gbs,
            "peak": pk_["hbm_gbs"],
            "unit": "GB/s",
            "frac": achieved_gbs / pk_["hbm_gbs"],
            "traffic": None,
            "peak_source": pk_["source"],
            "avg_launch_ms": avg_k_ms,
            "algorithmic_bytes_per_launch": bytes_per_launch,
            "note": "kernel (a) is SIMT-compute-bound (~1e3 evaluations per byte); see compute",
            "compute": {
                "q_evals_per_launch": evals_per_launch,
                "q_evals_per_s": evals_per_launch / (avg_k_ms / 1e3),
                "approx_tflops": evals_per_launch * fl_per_eval / (avg_k_ms / 1e3) / 1e12,
                "nominal_fp32_simt_tflops": 74.4,
                "frac_of_nominal_fp32": evals_per_launch * fl_per_eval / (avg_k_ms / 1e3) / 1e12 / 74.4,
            },
            "expectation_kernel_avg_ms": float(np.mean(et)) if et else None,
        },
        "evals_per_solve": evals_per_solve,
        "clocks": clocks,
        "cpu_baseline": cpu_baseline(args) if (rank == 0 and world == 1 and not args.no_cpu) else None,
    }


def cpu_baseline(args) -> dict:
    """The oracle (NumPy FP64 restatement) on a bounded sample: the terminal
    period plus `cpu_periods` decision periods of one solve, extrapolated to
    a full T-period solve."""
    from oracle.grid_search import bellman_step
    from pylcm_b200.spec import ParamResolver

    model, params = make_workload(args.periods, args.wealth, args.cons, 1)
    specs = model.regime_specs
    res = ParamResolver(params[0], model.fixed_params, tuple(s.name for s in specs))
    T = model.n_periods
    V = {}
    t0 = time.perf_counter()
    per_period = []
    for period in range(T - 1, T - 2 - args.cpu_periods, -1):
        ts = time.perf_counter()
        V[period] = {}
        for s in specs:
            if period in s.active_periods:
                V[period][s.name], _ = bellman_step(
                    s, specs, res, period, float(model.ages.values[period]), V.get(period + 1, {})
                )
        per_period.append(time.perf_counter() - ts)
    terminal = per_period[0]
    decision = float(np.mean(per_period[1:]))
    est = terminal + (T - 1) * decision
    return {
        "value": 1.0 / est,
        "unit": UNIT,
        "cores": 1,
        "kind": "port",
        "sample": f"terminal period + {args.cpu_periods} decision periods of one solve timed "
        f"({time.perf_counter() - t0:.1f} s), extrapolated to T={T}",
        "seconds_per_solve_est": est,
    }


def run_reference(args) -> dict:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return {}
    vals = []
    for _ in range(args.warmup):
        pass  # the CPU port has no warm-up state beyond imports
    for _ in range(max(1, min(args.steps, 2))):
        vals.append(cpu_baseline(args)["value"])
    v = float(np.mean(vals))
    cb = cpu_baseline.__doc__
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "stochastic retirement model (Tauchen 7-node income), T=40, wealth/consumption 500/500"},
        "cpu_baseline": {
            "value": v,
            "unit": UNIT,
            "cores": 1,
            "kind": "port",
            "sample": f"terminal + {args.cpu_periods} decision periods per step, extrapolated to a full solve",
        },
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference solve is JAX (not installable here); this is the oracle's NumPy FP64 restatement",
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--periods", type=int, default=40)
    ap.add_argument("--wealth", type=int, default=500)
    ap.add_argument("--cons", type=int, default=500)
    ap.add_argument("--plain-samples", type=int, default=8)
    ap.add_argument("--cpu-periods", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
