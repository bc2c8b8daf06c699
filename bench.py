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
    from pylcm_b200.distributed import max_over_ranks

    t_ms = max_over_ranks(t_ms, device="cuda")  # the slowest rank's time
    value = world * args.batch * args.steps / (t_ms / 1e3)

    # ---- end to end through the public batch API (host params -> host V)
    torch.cuda.synchronize()
    e2e_ms = []
    phases = []
    h2d = d2h = 0
    for k in range(max(1, min(args.steps, 3))):
        flush_l2(torch, flush)
        torch.cuda.synchronize()
        ev4 = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        t0 = time.perf_counter()
        pk = fast.pack(params)
        t1 = time.perf_counter()
        ev4[0].record(stream)
        h2d = fast.upload(pk)
        ev4[1].record(stream)
        ev4[2].record(stream)
        d2h = fast.run_download(policy=False)  # per-period copies overlap the compute
        ev4[3].record(stream)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        phases.append(((t1 - t0) * 1e3, ev4[0].elapsed_time(ev4[1]), ev4[1].elapsed_time(ev4[2]),
                       ev4[2].elapsed_time(ev4[3])))
    # the job's end-to-end time is the slowest rank's (every rank runs this)
    e2e_value = args.batch * world / (max_over_ranks(statistics.median(e2e_ms), device="cuda") / 1e3)
    ph = np.median(np.asarray(phases), axis=0)

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
    extra = {}
    if world == 1 and not args.no_extra:
        extra["serving"] = run_serving(args, local)
        extra["dcegm"] = run_dcegm(args, local)
        extra["hc"] = run_hc(args, local)
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
            "api": "pylcm_b200.batch.BatchSolver pack+upload+run_download (host params -> host V)",
            "phases_ms": {"pack_host": float(ph[0]), "h2d": float(ph[1]), "run_and_overlapped_d2h": float(ph[3])},
        },
        "gpu_launches": fast.gpu_launches * args.steps,
        "roofline": {
            "kernel": "lcm_bellman (kernel a: fused Q_and_F + max/argmax)",
            "bound": "hbm",
            "achieved": achieved_gbs,
            "peak": pk_["hbm_gbs"],
            "unit": "GB/s",
            "frac": achieved_gbs / pk_["hbm_gbs"],
            # DRAM bytes of one kernel (a) launch from the ncu capture of the
            # same launch at batch 256 (17.90336 MB read, 256 B written), scaled
            # by the instances per launch for other batch sizes
            "traffic": (17.90336e6 + 256.0) * args.batch / 256,
            "traffic_source": "ncu dram__bytes_read+write of lcm_bellman_working at batch 256 (x batch/256)",
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
        **extra,
        "cpu_baseline": cpu_baseline(args) if (rank == 0 and world == 1 and not args.no_cpu) else None,
    }


def _rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    fin = np.isfinite(b)
    if not fin.any():
        return 0.0
    return float((np.abs(a[fin] - b[fin]) / np.maximum(1.0, np.abs(b[fin]))).max())


def run_serving(args, local: int) -> dict:
    """Serving workload (solve + simulate requests of the stochastic
    retirement and DC-EGM retirement models, grid sizes 100..2000, T in
    {10, 40, 60}, 10,000 simulated subjects each): capacity with every
    request released at once, then Poisson arrivals at 0.75 x capacity for
    end-to-end latency; the plain form is the FP64 server one request at a
    time."""
    import dataclasses

    import torch

    from pylcm_b200 import examples as E
    from pylcm_b200.serving import Server, latency_summary

    n = args.serve_requests
    n_v = min(16, args.plain_requests, n)
    reqs = E.serving_requests(n, seed=7, n_agents=args.agents)
    for r in reqs[:n_v]:
        r.return_V = True
    srv = Server(device=local, precision="fp32", max_batch=args.serve_batch, n_streams=args.serve_streams)
    srv.run([dataclasses.replace(r) for r in reqs], realtime=False)  # kernels compiled, pools built
    srv.job_gpu_ms, srv.batch_sizes = [], []
    t = time.perf_counter()
    srv.run([dataclasses.replace(r) for r in reqs], realtime=False)
    cap_wall = time.perf_counter() - t
    capacity = n / cap_wall
    cap_gpu = sum(srv.job_gpu_ms)
    rate = 0.75 * capacity  # offered load within 70-90 % of the measured capacity
    arr = np.cumsum(np.random.default_rng(8).exponential(1.0 / rate, size=n))
    reqs_p = [dataclasses.replace(r, arrival=float(a)) for r, a in zip(reqs, arr)]
    srv.job_gpu_ms, srv.batch_sizes, srv.host_launch_s = [], [], 0.0
    with ClockSampler(local) as clk:
        t = time.perf_counter()
        res = srv.run(reqs_p, realtime=True)
        wall = time.perf_counter() - t
    summ = latency_summary(res, wall)
    # plain: FP64, one request at a time (compile pass first)
    sample = reqs[: args.plain_requests]
    pl = Server(device=local, precision="fp64", max_batch=1, n_streams=1)
    pl.run([dataclasses.replace(r) for r in sample], realtime=False)
    t = time.perf_counter()
    pres = pl.run([dataclasses.replace(r) for r in sample], realtime=False)
    pwall = time.perf_counter() - t
    plain_rate = len(sample) / pwall
    plain_lat = np.array([r.finished - r.admitted for r in pres]) * 1e3
    err = 0.0
    for a, b in zip(res[:n_v], pres[:n_v]):
        for per in b.V:
            for name in b.V[per]:
                err = max(err, _rel_err(a.V[per][name], b.V[per][name]))
    torch.cuda.synchronize()
    return {
        "workload": "4096-request serving stream of config 4 restated: each request the stochastic retirement "
        "model (grid search) or the DC-EGM retirement model (taste scale none / 0.05) with prob. 1/2, wealth grid "
        "n in {100,250,500,1000,2000}, T in {10,40,60}, beta~U[.90,.99], crra~U[1,5], r~U[.01,.06]; solve + "
        "simulate 10,000 subjects (w0~U[1,50], income state from its stationary distribution)",
        "requests": n,
        "agents_per_request": args.agents,
        "capacity_solves_per_s": capacity,
        "arrival_rate_per_s": rate,
        "solves_per_s": summ["solves_per_s"],
        "p50_ms": summ["p50_ms"],
        "p99_ms": summ["p99_ms"],
        "mean_batch": summ["mean_batch"],
        "gpu_busy_frac_at_capacity": cap_gpu / 1e3 / cap_wall,
        "host_launch_s": srv.host_launch_s,
        "plain": {
            "solves_per_s": plain_rate,
            "p50_service_ms": float(np.percentile(plain_lat, 50)),
            "p99_service_ms": float(np.percentile(plain_lat, 99)),
            "form": "fp64, max_batch 1, one stream: one request at a time",
            "requests": len(sample),
        },
        "fast_vs_plain": summ["solves_per_s"] / plain_rate,
        "capacity_vs_plain": capacity / plain_rate,
        "max_rel_V_err_vs_fp64": err,
        "V_checked_requests": n_v,
        "pools_built": srv.pools_built,
        "clocks": clk.summary(),
    }


def run_dcegm(args, local: int) -> dict:
    """DC-EGM + FUES (config 2): T=40, 2000-point cubic savings grid on
    [0, 500], wealth grid 2000 points, 16-node Gauss-Hermite income weights,
    CRRA 2, beta 0.97, r 0.04; taste scale none / 0.05.  One solve at a time
    (FP64, eager) and batches of `dcegm_batch` parameter draws."""
    import torch

    from pylcm_b200 import examples as E
    from pylcm_b200.engine import SolveEngine
    from pylcm_b200.runtime import get_context

    out = {}
    stream = torch.cuda.current_stream()
    ctx = get_context(local)
    for taste in (None, 0.05):
        model = E.dcegm_model(n_periods=40, n_savings=2000, n_wealth=2000, taste=taste is not None)
        rng = np.random.default_rng(11)
        plist = [E.dcegm_params(seed=int(rng.integers(1 << 30)), taste_scale=taste) for _ in range(args.dcegm_batch)]
        eng = SolveEngine(model, "fp64", device=local)
        one = eng.plan([plist[0]])
        one.run(stream.cuda_stream)
        torch.cuda.synchronize()
        counts = torch.zeros(2, dtype=torch.int64, device="cuda")
        ms = []
        for _ in range(3):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one.run(stream.cuda_stream)
            counts.zero_()
            for v in one.V.values():
                ctx.count_nonfinite(v.data_ptr(), v.numel(), counts.data_ptr(), stream.cuda_stream)
            _ = counts.cpu()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        batch = eng.plan(plist)
        batch.run(stream.cuda_stream)
        torch.cuda.synchronize()
        bms = []
        for _ in range(2):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            batch.run(stream.cuda_stream)
            b.record(stream)
            torch.cuda.synchronize()
            bms.append(a.elapsed_time(b))
        err = max(_rel_err(batch.V[r][0].cpu().numpy(), one.V[r][0].cpu().numpy()) for r in one.V)
        out["taste_none" if taste is None else "taste_0.05"] = {
            "plain_ms_per_solve": float(np.median(ms)),
            "plain_solves_per_s": 1e3 / float(np.median(ms)),
            "batch": args.dcegm_batch,
            "batched_solves_per_s": args.dcegm_batch / (float(np.median(bms)) / 1e3),
            "batched_vs_plain": (args.dcegm_batch / float(np.median(bms))) / (1.0 / float(np.median(ms))),
            "max_rel_V_err_batch_vs_single": err,
        }
    return out


def run_hc(args, local: int) -> dict:
    """Two continuous states (config 3): wealth 1000 x human capital 50 x a
    32-state Markov shock (Dirichlet(1) rows), 300 consumption x 3 hours
    actions, T=60; a batch of `hc_batch` parameter draws (beta~U[.90,.99],
    crra~U[1,5], r~U[.01,.06]) in the fast form against one FP64 solve."""
    import torch

    from pylcm_b200 import examples as E
    from pylcm_b200.engine import SolveEngine

    stream = torch.cuda.current_stream()
    model = E.hc_model(60, 1000, 50, 32, 300)
    plist = [E.hc_params(seed=k) for k in range(args.hc_batch)]
    fast = SolveEngine(model, "fp32", device=local).plan(plist)
    plain = SolveEngine(model, "fp64", device=local).plan(plist[:1])
    fast.run(stream.cuda_stream)
    plain.run(stream.cuda_stream)
    torch.cuda.synchronize()
    res = {}
    for name, plan, n in (("fast", fast, args.hc_batch), ("plain", plain, 1)):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.run(stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        res[name] = n / (a.elapsed_time(b) / 1e3)
    err = max(_rel_err(fast.V[r][0].cpu().numpy(), plain.V[r][0].cpu().numpy()) for r in plain.V)
    agree = tot = 0
    for r in plain.pol:
        m = torch.isfinite(plain.V[r][0])
        agree += int((fast.pol[r][0] == plain.pol[r][0])[m].sum().item())
        tot += int(m.sum().item())
    evals = sum(s.n_states * s.n_actions * len(s.active_periods) for s in model.regime_specs)
    return {
        "batch": args.hc_batch,
        "fast_solves_per_s": res["fast"],
        "plain_solves_per_s": res["plain"],
        "fast_vs_plain": res["fast"] / res["plain"],
        "q_evals_per_solve": evals,
        "fast_q_evals_per_s": evals * res["fast"],
        "max_rel_V_err_vs_fp64": err,
        "policy_agreement_vs_fp64": agree / max(tot, 1),
    }


_W = {}


def _cpu_init(periods, wealth, cons):
    from pylcm_b200.spec import ParamResolver

    model, params = make_workload(periods, wealth, cons, 1)
    _W["model"] = model
    _W["res"] = ParamResolver(params[0], model.fixed_params, tuple(s.name for s in model.regime_specs))


def _cpu_rows(job):
    from oracle.grid_search import bellman_step

    name, period, rows, nxt = job
    model = _W["model"]
    specs = model.regime_specs
    spec = next(s for s in specs if s.name == name)
    V, _ = bellman_step(spec, specs, _W["res"], period, float(model.ages.values[period]), nxt, state_rows=rows)
    return name, rows, V


def cpu_baseline(args) -> dict:
    """The oracle (NumPy FP64 restatement of the reference's solve) on a
    bounded sample: the terminal period plus `cpu_periods` decision periods of
    one solve, each period's state rows split over a pool of host processes,
    extrapolated to a full T-period solve."""
    import concurrent.futures as cf
    import multiprocessing as mp

    model, _ = make_workload(args.periods, args.wealth, args.cons, 1)
    specs = model.regime_specs
    T = model.n_periods
    cores = max(1, min(args.cpu_cores or (os.cpu_count() or 1), 64))
    V = {}
    per_period = []
    with cf.ProcessPoolExecutor(cores, mp_context=mp.get_context("spawn"), initializer=_cpu_init,
                                initargs=(args.periods, args.wealth, args.cons)) as ex:
        list(ex.map(_cpu_rows, [(specs[-1].name, T - 1, np.arange(1), {})] * cores))  # start the workers
        t0 = time.perf_counter()
        for period in range(T - 1, T - 2 - args.cpu_periods, -1):
            ts = time.perf_counter()
            nxt = V.get(period + 1, {})
            jobs = []
            for s in specs:
                if period in s.active_periods:
                    for rows in np.array_split(np.arange(s.n_states), cores):
                        if rows.size:
                            jobs.append((s.name, period, rows, nxt))
            out = {}
            for name, rows, v in ex.map(_cpu_rows, jobs):
                out.setdefault(name, np.empty(next(x for x in specs if x.name == name).n_states))[rows] = v
            V[period] = {n: v.reshape(next(x for x in specs if x.name == n).state_shape) for n, v in out.items()}
            per_period.append(time.perf_counter() - ts)
    terminal = per_period[0]
    decision = float(np.mean(per_period[1:]))
    est = terminal + (T - 1) * decision
    return {
        "value": 1.0 / est,
        "unit": UNIT,
        "cores": cores,
        "kind": "port",
        "sample": f"terminal period + {args.cpu_periods} decision periods of one solve timed "
        f"({time.perf_counter() - t0:.1f} s, state rows split over {cores} processes), extrapolated to T={T}",
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
    cores = max(1, min(args.cpu_cores or (os.cpu_count() or 1), 64))
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
            "cores": cores,
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
    ap.add_argument("--cpu-cores", type=int, default=0, help="host processes of the CPU baseline (0: all)")
    ap.add_argument("--serve-requests", type=int, default=512)
    ap.add_argument("--agents", type=int, default=10_000)
    ap.add_argument("--serve-batch", type=int, default=32)
    ap.add_argument("--serve-streams", type=int, default=2)
    ap.add_argument("--plain-requests", type=int, default=32)
    ap.add_argument("--no-extra", action="store_true", help="skip the serving / DC-EGM / two-state sections")
    ap.add_argument("--dcegm-batch", type=int, default=32)
    ap.add_argument("--hc-batch", type=int, default=8)
    ap.add_argument("--only", choices=["serving", "dcegm", "hc"], default=None,
                    help="run one extra section alone on GPU 0 and print its JSON (for profiling)")
    args = ap.parse_args()
    if args.only:
        import torch

        torch.cuda.set_device(0)
        fn = {"serving": run_serving, "dcegm": run_dcegm, "hc": run_hc}[args.only]
        print(json.dumps({args.only: fn(args, 0)}))
        return
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
