"""Benchmark: model solves/sec of the stochastic retirement model.

Workload (one "step" = one batched backward-induction solve):
    stochastic consumption-savings model with a work/retire choice -- 7-node
    Tauchen AR(1) log income (rho=0.9, sigma=0.1, +-3 sd) multiplying the wage,
    wealth and consumption on linspace(1, 400, 500), labour {work, retire},
    CRRA utility, T=40: 40 x 7 x 500 states x 500 x 2 actions per solve.
    A step solves B seeded parameter draws (beta ~ U[0.94, 0.97],
    crra ~ U[1.5, 2.5], r ~ U[0.03, 0.05]) at once.

Forms measured on the GPU:
    fast  -- batched, single-precision search (expectation table from the
             tensor-core kernel) with double-precision re-evaluation, one
             CUDA graph per step (`value`);
    plain -- one solve at a time, FP64, eager launches, per-solve NaN check.
Extra sections: the two-continuous-state model at batch 256 (config 3), DC-EGM
(config 2), the 4096-request serving stream (config 4); per-kernel rooflines.

The CPU leg (``cpu_baseline``) times the oracle -- a NumPy float64
restatement of the reference's solve, test infrastructure -- on one full
T=40 solve over the host cores, and uses the same oracle as the checker of
the GPU results (``accuracy_vs_oracle``, configs 1-3).  ``--impl reference``
times that oracle alone (the reference itself is JAX, which cannot be
installed here).
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


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def time_launches(plan, torch, stream) -> list:
    """Run a plan's launch list once, eagerly, with CUDA events around every
    launch on `stream`: [(Launch, ms)]."""
    prepared = plan._prepare()
    ev = []
    for l, launch in zip(plan.launches, prepared):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        launch(stream.cuda_stream)
        b.record(stream)
        ev.append((l, a, b))
    torch.cuda.synchronize()
    return [(l, a.elapsed_time(b)) for l, a, b in ev]


def _expect_target(l):
    rk = l.module
    for t in rk.targets:
        if t.scalar or t.unreachable:
            continue
        if l.kernel in (rk.expect_name(t), getattr(rk, "expect_tc_name", lambda _: None)(t)):
            return rk, t
    return rk, None


def kernel_bytes(l) -> float | None:
    """Algorithmic bytes of one launch (every instance of it):
    (a)  EV rows read once (float table in the single-precision search,
         double otherwise) + V (8 B) and policy (4 B) written per state;
    (b)  V' read once (8 B per node x column) + the table(s) written per
         weight row x column (double 8 B, float 4 B);
    None for the other kernels (tiny, or counted per section)."""
    if l.kind == "bellman":
        rk = l.module
        spec = rk.spec
        e = 4 if rk.precision == "fp32" else 8
        rd = 0
        for t in rk.targets:
            if t.scalar or t.unreachable:
                continue
            cols = int(np.prod([t.spec.states[p].size for p in t.det_pos + t.cont_pos]))
            rd += t.K * cols * e
        return float(l.n_items * (rd + spec.n_states * 12))
    if l.kind in ("expect", "expect_tc"):
        rk, t = _expect_target(l)
        if t is None:
            return None
        cols = int(np.prod([t.spec.states[p].size for p in t.det_pos + t.cont_pos]))
        if l.kind == "expect_tc":
            w = 4
        else:
            w = 8 + (4 if (rk.precision == "fp32" and not rk.tc_ok(t)) else 0)
        return float(l.n_items * cols * (t.J * 8 + t.K * w))
    return None


def roofline_of(timed, kinds, pk) -> dict | None:
    """Achieved GB/s of the launches of `kinds` (algorithmic bytes / average
    launch time) against the measured HBM peak."""
    sel = [(l, ms) for l, ms in timed if l.kind in kinds]
    if not sel:
        return None
    by = [(kernel_bytes(l), ms) for l, ms in sel]
    by = [(b, ms) for b, ms in by if b is not None]
    if not by:
        return None
    avg_ms = float(np.mean([ms for _, ms in by]))
    avg_b = float(np.mean([b for b, _ in by]))
    gbs = avg_b / (avg_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": gbs, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": gbs / pk["hbm_gbs"],
            "peak_source": pk["source"], "launches": len(by), "avg_launch_ms": avg_ms,
            "algorithmic_bytes_per_launch": avg_b, "share_of_plan_time": float(
                sum(ms for _, ms in sel) / max(sum(ms for _, ms in timed), 1e-9))}


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
    from pylcm_b200.distributed import max_over_ranks, partition

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://")
    # the job: world x batch independent parameter vectors, partitioned over
    # the ranks by HBM footprint (equal here: round robin), no collective on
    # the data path
    model, job = make_workload(args.periods, args.wealth, args.cons, world * args.batch, seed=0)
    mine = partition([1] * len(job), world)[rank]
    params = [job[i] for i in mine]
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
    t_ms = max_over_ranks(t_ms, device="cuda")  # the slowest rank's time
    value = world * args.batch * args.steps / (t_ms / 1e3)
    fast.plan.check_status()

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

    # ---- per-launch device times of one fast step (eager, events)
    flush_l2(torch, flush)
    torch.cuda.synchronize()
    timed = time_launches(fast.plan, torch, stream)
    pk_ = peaks()
    rf_a = roofline_of(timed, ("bellman",), pk_)
    bell = [(l, ms) for l, ms in timed if l.kind == "bellman"]
    flops = [l.module.inner_flops()["total"] * l.n_items * l.module.spec.n_states * l.module.spec.n_actions
             for l, _ in bell]
    evals = [l.n_items * l.module.spec.n_states * l.module.spec.n_actions for l, _ in bell]
    bell_ms = sum(ms for _, ms in bell)
    rf_kernels = {
        "a_bellman": rf_a,
        "b_expectation_fp64": roofline_of(timed, ("expect",), pk_),
        "b_expectation_tcgen05": roofline_of(timed, ("expect_tc",), pk_),
        "a0_action_table": {"share_of_plan_time": float(
            sum(ms for l, ms in timed if l.kind == "atab") / max(sum(ms for _, ms in timed), 1e-9))},
    }

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

    def load_plain(i):
        for key in plain_plan.params:
            name, targets = key
            spec = next(s for s in plain_eng.specs if s.name == name)
            rk = plain_eng.kernels(spec, targets, params[0], 1)
            plain_plan.params[key].copy_(
                torch.as_tensor(rk.tr.pack_params(rk.tr.values_for(plain_eng.resolver(params[i])))[None],
                                device="cuda"))

    for i in range(n_plain):
        load_plain(i)
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
    load_plain(0)
    plain_plan.run(stream.cuda_stream)
    torch.cuda.synchronize()
    for r in plain_plan.pol:
        a_ = plain_plan.pol[r][0]
        b_ = fast.plan.pol[r][0]
        vp = plain_plan.V[r][0]
        m = torch.isfinite(vp)
        agree += int((a_ == b_)[m].sum().item())
        tot += int(m.sum().item())
    # host copies of instance 0 for the oracle check (plain FP64 and fast)
    check1 = {
        "model": model, "params": params[0],
        "plain": {r: (plain_plan.V[r][0].cpu().numpy(), plain_plan.pol[r][0].cpu().numpy()) for r in plain_plan.V},
        "fast": {r: (fast.plan.V[r][0].cpu().numpy(), fast.plan.pol[r][0].cpu().numpy()) for r in fast.plan.V},
        "slots": {s.name: dict(plain_plan.slot[s.name]) for s in model.regime_specs},
    }

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return {}
    extra = {}
    checks = {"config1": check1}
    if world == 1 and not args.no_extra:
        extra["serving"] = run_serving(args, local)
        extra["dcegm"], checks["config2"] = run_dcegm(args, local)
        extra["hc"], checks["config3"] = run_hc(args, local)
    spec0 = model.regime_specs
    evals_per_solve = sum(s.n_states * s.n_actions * len(s.active_periods) for s in spec0)
    clocks = clk.summary()
    cpu = cpu_baseline(args, checks) if (rank == 0 and world == 1 and not args.no_cpu) else None
    accuracy_vs_oracle = cpu.pop("accuracy_vs_oracle", None) if cpu else None
    roofline = dict(rf_a)
    roofline.update({
        "kernel": "lcm_bellman (kernel a: fused Q_and_F + max/argmax)",
        # DRAM bytes of one kernel (a) launch from the ncu capture of the
        # same launch at batch 256 (17.90336 MB read, 256 B written), scaled
        # by the instances per launch for other batch sizes
        "traffic": (17.90336e6 + 256.0) * args.batch / 256,
        "traffic_source": "ncu dram__bytes_read+write of lcm_bellman_working at batch 256 (x batch/256)",
        "note": "kernel (a) is SIMT-compute-bound (~1e3 evaluations per byte); its HBM fraction is small by "
        "construction -- see compute",
        "compute": {
            "q_evals_per_s": float(sum(evals) / (bell_ms / 1e3)),
            "flops_per_eval_from_ir": [l.module.inner_flops() for l, _ in bell[:len(spec0)]],
            "tflops": float(sum(flops) / (bell_ms / 1e3) / 1e12),
            "nominal_fp32_simt_tflops": 74.4,
            "frac_of_nominal_fp32_simt": float(sum(flops) / (bell_ms / 1e3) / 1e12 / 74.4),
            "nominal_source": "148 SMs x 128 FP32 lanes x 2 flops x 1.965 GHz",
        },
    })
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
        "dtype": "f32 search on a 3xTF32 tensor-core expectation table + f64 re-evaluation (fast); f64 (plain)",
        "data": "synthetic (seeded parameter draws)",
        "config": {
            "workload": "stochastic retirement model (Tauchen 7-node income), T=40, wealth/consumption 500/500, 2 labour choices",
            "batch_per_gpu": args.batch,
            "periods": args.periods,
            "wealth_points": args.wealth,
            "consumption_points": args.cons,
            "precision": "fp32 search, fp64 value",
            "parallelism": f"replicas x{world} (parameter vectors partitioned over GPUs, no data-path collective)",
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
        "accuracy_vs_oracle": accuracy_vs_oracle,
        "e2e": {
            "value": e2e_value,
            "unit": UNIT,
            "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h),
            "api": "pylcm_b200.batch.BatchSolver pack+upload+run_download (host params -> host V)",
            "phases_ms": {"pack_host": float(ph[0]), "h2d": float(ph[1]), "run_and_overlapped_d2h": float(ph[3])},
        },
        "gpu_launches": fast.gpu_launches * args.steps,
        "roofline": roofline,
        "roofline_kernels": rf_kernels,
        "evals_per_solve": evals_per_solve,
        "clocks": clocks,
        **extra,
        "cpu_baseline": cpu,
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
    srv.host_phase_s, srv.host_launch_s, srv.host_finish_s, srv.jobs_run = {}, 0.0, 0.0, 0
    t = time.perf_counter()
    srv.run([dataclasses.replace(r) for r in reqs], realtime=False)
    cap_wall = time.perf_counter() - t
    capacity = n / cap_wall
    cap_gpu = sum(srv.job_gpu_ms)
    cap_host = {"launch_s": srv.host_launch_s, "finish_s": srv.host_finish_s, "jobs": srv.jobs_run,
                "phases_s": dict(srv.host_phase_s)}
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
        "host_at_capacity": cap_host,
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


def _egm_bytes(l, plan) -> float | None:
    """Algorithmic bytes of a DC-EGM launch over all its instances:
    (c1) candidates: the target carry rows read once (grid, value, marginal,
         8 B each per refined point) + 4 candidate arrays written (8 B per
         candidate);
    FUES: 4 candidate arrays read + 3 refined arrays written per row."""
    eg = plan.egm
    if l.kind == "fues":
        b = next(iter(eg.values()))
        per = b["nrow"] * (4 * b["ncand"] + 3 * b["npad"]) * 8
        return float(plan.n * per)
    if l.kind == "egm" and l.kernel.startswith("lcm_egmc_"):
        ek = l.module
        er = ek.er
        b = eg[er.spec.name]
        rd = 0
        for t in er.targets:
            if t.spec.name in eg:
                tb = eg[t.spec.name]
                rd += tb["nrow"] * tb["npad"] * 3 * 8
        return float(plan.n * (rd + b["nrow"] * b["ncand"] * 4 * 8))
    return None


def run_dcegm(args, local: int):
    """DC-EGM + FUES (config 2): T=40, 2000-point cubic savings grid on
    [0, 500], wealth grid 2000 points, 16-node Gauss-Hermite income weights,
    CRRA 2, beta 0.97, r 0.04; taste scale none / 0.05.  One solve at a time
    (FP64, eager) and batches of `dcegm_batch` parameter draws; per-launch
    device times of one batched solve (kernel c1 and FUES rooflines).
    Returns (section, host copies for the oracle check)."""
    import torch

    from pylcm_b200 import examples as E
    from pylcm_b200.engine import SolveEngine
    from pylcm_b200.runtime import get_context

    out = {}
    check = {}
    stream = torch.cuda.current_stream()
    ctx = get_context(local)
    pk = peaks()
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
        timed = time_launches(batch, torch, stream)
        tot = sum(ms_ for _, ms_ in timed)
        kern = {}
        for label, pred in (("c1_candidates", lambda l: l.kind == "egm" and l.kernel.startswith("lcm_egmc_")),
                            ("fues", lambda l: l.kind == "fues")):
            sel = [(l, ms_) for l, ms_ in timed if pred(l)]
            if not sel:
                continue
            by = [(_egm_bytes(l, batch), ms_) for l, ms_ in sel]
            avg_ms = float(np.mean([m for _, m in by]))
            avg_b = float(np.mean([x for x, _ in by]))
            gbs = avg_b / (avg_ms / 1e3) / 1e9
            kern[label] = {"bound": "hbm", "achieved": gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
                           "frac": gbs / pk["hbm_gbs"], "avg_launch_ms": avg_ms, "launches": len(sel),
                           "algorithmic_bytes_per_launch": avg_b,
                           "share_of_plan_time": float(sum(m for _, m in sel) / max(tot, 1e-9))}
        key = "taste_none" if taste is None else "taste_0.05"
        out[key] = {
            "plain_ms_per_solve": float(np.median(ms)),
            "plain_solves_per_s": 1e3 / float(np.median(ms)),
            "batch": args.dcegm_batch,
            "batched_solves_per_s": args.dcegm_batch / (float(np.median(bms)) / 1e3),
            "batched_vs_plain": (args.dcegm_batch / float(np.median(bms))) / (1.0 / float(np.median(ms))),
            "max_rel_V_err_batch_vs_single": err,
            "kernels": kern,
        }
        # FP64 solve of draw 0 with its published rows, for the oracle check
        V, pub = model.solve(params=plist[0], log_level="off", return_simulation_policy=True)
        keep = (38, 20, 0)
        check[key] = {
            "model": model, "params": plist[0],
            "V": {p: dict(V[p]) for p in set(keep) | {p + 1 for p in keep}},
            "pub": {p: {n: (sp.endog_grid, sp.value, sp.marginal_utility) for n, sp in pub[p].items()}
                    for p in set(keep) | {p + 1 for p in keep}},
            "periods": keep,
        }
    return out, check


def run_hc(args, local: int):
    """Two continuous states (config 3): wealth 1000 x human capital 50 x a
    32-state Markov shock (Dirichlet(1) rows), 300 consumption x 3 hours
    actions, T=60; `hc_batch` parameter draws (beta~U[.90,.99], crra~U[1,5],
    r~U[.01,.06]) in the fast form, in chunks of `hc_chunk` instances (the
    value arrays of 256 instances, 193 GB in FP64, do not fit one GPU), timed
    chunk by chunk end to end on the device; the plain form solves one draw at
    a time in FP64.  Returns (section, host copies for the oracle check)."""
    import torch

    from pylcm_b200 import examples as E
    from pylcm_b200.engine import SolveEngine

    stream = torch.cuda.current_stream()
    model = E.hc_model(args.hc_periods, 1000, 50, 32, 300)
    plist = [E.hc_params(seed=k) for k in range(args.hc_batch)]
    chunk = min(args.hc_chunk, args.hc_batch)
    fast_eng = SolveEngine(model, "fp32", device=local)
    fast = fast_eng.plan(plist[:chunk])
    # parameter vectors of every chunk, packed once on the host
    chunks = [plist[i:i + chunk] for i in range(0, len(plist), chunk)]
    packed = []
    for c in chunks:
        resolvers = [fast_eng.resolver(p) for p in c]
        memo: dict = {}
        packed.append({k: torch.as_tensor(fast._pack_many[k](resolvers, memo), dtype=torch.float64, device="cuda")
                       for k in fast.params})
    fast.run(stream.cuda_stream)  # warm-up (module load)
    torch.cuda.synchronize()
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")
    with ClockSampler(local) as clk:
        evs = []
        for c, pv in zip(chunks, packed):
            for k, v in pv.items():
                fast.params[k][: len(c)].copy_(v)
            flush_l2(torch, flush)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fast.run(stream.cuda_stream)
            b.record(stream)
            evs.append((a, b, len(c)))
        torch.cuda.synchronize()
    fast.check_status()
    fast_ms = sum(a.elapsed_time(b) for a, b, _ in evs)
    fast_rate = args.hc_batch / (fast_ms / 1e3)
    # per-launch times of the last chunk: kernel (a) vs the expectation
    timed = time_launches(fast, torch, stream)
    pk = peaks()
    tot = sum(ms for _, ms in timed)
    kern = {"a_bellman": roofline_of(timed, ("bellman",), pk),
            "b_expectation_tcgen05": roofline_of(timed, ("expect_tc",), pk),
            "b_expectation_fp64": roofline_of(timed, ("expect",), pk)}
    bell = [(l, ms) for l, ms in timed if l.kind == "bellman"]
    ev_s = sum(l.n_items * l.module.spec.n_states * l.module.spec.n_actions for l, _ in bell) / (
        sum(ms for _, ms in bell) / 1e3)
    # fast instance 0 of the first chunk, for the accuracy check
    for k, v in packed[0].items():
        fast.params[k][: len(chunks[0])].copy_(v)
    fast.run(stream.cuda_stream)
    plain = SolveEngine(model, "fp64", device=local).plan(plist[:1])
    plain.run(stream.cuda_stream)
    torch.cuda.synchronize()
    pms = []
    for _ in range(2):
        flush_l2(torch, flush)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plain.run(stream.cuda_stream)
        b.record(stream)
        torch.cuda.synchronize()
        pms.append(a.elapsed_time(b))
    plain_rate = 1e3 / float(np.median(pms))
    err = max(_rel_err(fast.V[r][0].cpu().numpy(), plain.V[r][0].cpu().numpy()) for r in plain.V)
    agree = tot_s = 0
    for r in plain.pol:
        m = torch.isfinite(plain.V[r][0])
        agree += int((fast.pol[r][0] == plain.pol[r][0])[m].sum().item())
        tot_s += int(m.sum().item())
    keep = (58, 30, 0)
    slots = {s.name: dict(plain.slot[s.name]) for s in model.regime_specs}

    def host(plan, i):
        out = {}
        for s in model.regime_specs:
            for p in set(keep) | {p + 1 for p in keep}:
                k = slots[s.name].get(p)
                if k is not None:
                    out.setdefault(p, {})[s.name] = (plan.V[s.name][i, k].cpu().numpy(),
                                                     plan.pol[s.name][i, k].cpu().numpy())
        return out

    check = {"model": model, "params": plist[0], "plain": host(plain, 0), "fast": host(fast, 0), "periods": keep}
    evals = sum(s.n_states * s.n_actions * len(s.active_periods) for s in model.regime_specs)
    return {
        "batch": args.hc_batch,
        "chunk": chunk,
        "fast_solves_per_s": fast_rate,
        "fast_ms_total": fast_ms,
        "plain_solves_per_s": plain_rate,
        "fast_vs_plain": fast_rate / plain_rate,
        "q_evals_per_solve": evals,
        "fast_q_evals_per_s": evals * fast_rate,
        "kernel_a_q_evals_per_s": ev_s,
        "max_rel_V_err_vs_fp64": err,
        "policy_agreement_vs_fp64": agree / max(tot_s, 1),
        "kernels": kern,
        "l2": "flushed before each chunk (256 MiB write); each chunk's arrays exceed L2",
        "clocks": clk.summary(),
    }, check


# --------------------------------------------------------------------------
# CPU leg: the oracle, timed as the baseline and used as the checker
_W = {}


def _cpu_init(periods, wealth, cons, seed_draw):
    from pylcm_b200.spec import ParamResolver

    model, params = make_workload(periods, wealth, cons, seed_draw + 1)
    _W["model"] = model
    _W["res"] = ParamResolver(params[seed_draw], model.fixed_params, tuple(s.name for s in model.regime_specs))


def _cpu_rows(job):
    import oracle.grid_search as OG

    name, period, rows, nxt = job
    model = _W["model"]
    specs = model.regime_specs
    spec = next(s for s in specs if s.name == name)
    V, P = OG.bellman_step(spec, specs, _W["res"], period, float(model.ages.values[period]), nxt, state_rows=rows)
    return name, rows, V, P, OG.LAST_GAP


def _errs(a, b) -> tuple[float, float]:
    """(max |a-b|/max(1,|b|), max |a-b|/|b|) over entries finite in b; inf
    when the non-finite patterns differ."""
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    if not (np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(np.isinf(a), np.isinf(b))):
        return float("inf"), float("inf")
    fin = np.isfinite(b)
    if not fin.any():
        return 0.0, 0.0
    d = np.abs(a[fin] - b[fin])
    with np.errstate(divide="ignore", invalid="ignore"):
        pure = np.where(b[fin] != 0, d / np.abs(b[fin]), np.where(d == 0, 0.0, np.inf))
    return float((d / np.maximum(1.0, np.abs(b[fin]))).max()), float(pure.max())


def _oracle_solve_parallel(ex, specs, T, cores):
    """A full backward induction by the oracle with every period's state rows
    split over the pool: {period: {regime: (V, policy, gap)}}."""
    V = {}
    out_all = {}
    for period in range(T - 1, -1, -1):
        nxt = V.get(period + 1, {})
        jobs = []
        for s in specs:
            if period in s.active_periods:
                for rows in np.array_split(np.arange(s.n_states), cores):
                    if rows.size:
                        jobs.append((s.name, period, rows, nxt))
        out = {}
        for name, rows, v, pol, gap in ex.map(_cpu_rows, jobs):
            n_s = next(x for x in specs if x.name == name).n_states
            o = out.setdefault(name, [np.empty(n_s), np.empty(n_s, dtype=np.int32), np.empty(n_s)])
            o[0][rows], o[1][rows], o[2][rows] = v, pol, gap
        V[period] = {n: o[0].reshape(next(x for x in specs if x.name == n).state_shape) for n, o in out.items()}
        out_all[period] = out
    return out_all


def _check_config1(check, oracle_out) -> dict:
    res = {}
    for form in ("plain", "fast"):
        worst = [0.0, 0.0]
        n_gap = n_gap_same = n_all = n_same = 0
        for period, regs in oracle_out.items():
            for name, (Vo, Po, gap) in regs.items():
                k = check["slots"][name].get(period)
                Vg, Pg = check[form][name]
                Vg, Pg = Vg[k], Pg[k]
                e = _errs(Vg, Vo)
                worst = [max(worst[0], e[0]), max(worst[1], e[1])]
                rel_gap = gap / np.maximum(1.0, np.abs(np.nan_to_num(Vo, neginf=0.0)))
                sel = rel_gap > (1e-9 if form == "plain" else 1e-5)
                n_gap += int(sel.sum())
                n_gap_same += int((Pg[sel] == Po[sel]).sum())
                n_all += Po.size
                n_same += int((Pg == Po).sum())
        res[form] = {"max_abs_rel_V_err": worst[0], "max_pure_rel_V_err": worst[1],
                     "policy_agreement": n_same / max(n_all, 1),
                     "policy_identical_where_gap_above": n_gap_same / max(n_gap, 1),
                     "gap_bar": 1e-9 if form == "plain" else 1e-5}
    res["states_checked"] = "every state of every period of one full T=40 solve (parameter draw 0)"
    return res


def _check_config3(check, n_rows=2000) -> dict:
    import oracle.grid_search as OG
    from pylcm_b200.spec import ParamResolver

    model, params = check["model"], check["params"]
    specs = model.regime_specs
    res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
    rng = np.random.default_rng(0)
    out = {}
    for form in ("plain", "fast"):
        worst = [0.0, 0.0]
        n_all = n_same = n_gap = n_gap_same = 0
        for period in check["periods"]:
            by_name = {x.name: x for x in specs}
            nxt = {n: v.reshape(by_name[n].state_shape) for n, (v, _) in check[form].get(period + 1, {}).items()}
            for s in specs:
                if period not in s.active_periods:
                    continue
                rows = np.sort(rng.choice(s.n_states, min(n_rows, s.n_states), replace=False))
                Vo, Po = OG.bellman_step(s, specs, res, period, float(model.ages.values[period]), nxt, state_rows=rows)
                gap = OG.LAST_GAP
                Vg, Pg = check[form][period][s.name]
                Vg, Pg = Vg.reshape(-1)[rows], Pg.reshape(-1)[rows]
                e = _errs(Vg, Vo)
                worst = [max(worst[0], e[0]), max(worst[1], e[1])]
                rel_gap = gap / np.maximum(1.0, np.abs(np.nan_to_num(Vo, neginf=0.0)))
                sel = rel_gap > (1e-9 if form == "plain" else 1e-5)
                n_gap += int(sel.sum())
                n_gap_same += int((Pg[sel] == Po[sel]).sum())
                n_all += Po.size
                n_same += int((Pg == Po).sum())
        out[form] = {"max_abs_rel_V_err": worst[0], "max_pure_rel_V_err": worst[1],
                     "policy_agreement": n_same / max(n_all, 1),
                     "policy_identical_where_gap_above": n_gap_same / max(n_gap, 1)}
    out["states_checked"] = f"{n_rows} seeded state rows per regime at periods {list(check['periods'])}, one step " \
                            "from the GPU's own next-period arrays"
    return out


def _check_config2(checks) -> dict:
    import oracle.dcegm as OD
    from pylcm_b200.egm import is_egm, trace_egm_regime
    from pylcm_b200.spec import ParamResolver

    out = {}
    for key, check in checks.items():
        model, params = check["model"], check["params"]
        specs = model.regime_specs
        res = ParamResolver(params, model.fixed_params, tuple(s.name for s in specs))
        wV, wR = [0.0, 0.0], [0.0, 0.0]
        for period in check["periods"]:
            age = float(model.ages.values[period])
            nxt_V = {n: np.asarray(v) for n, v in check["V"][period + 1].items()}
            carry_next = {}
            for n, (g, v, mu) in check["pub"][period + 1].items():
                g2 = g.reshape(-1, g.shape[-1])
                carry_next[n] = {r: (g2[r], v.reshape(g2.shape)[r], mu.reshape(g2.shape)[r]) for r in range(g2.shape[0])}
            for s in specs:
                if period not in s.active_periods or s.terminal or not is_egm(s):
                    continue
                targets = tuple(x.name for x in specs if (period + 1) in x.active_periods)
                er = trace_egm_regime(s, specs, res, targets)
                Vs, rows, _ = OD.egm_step(er, specs, res, period, age, carry_next, nxt_V,
                                          s.state(er.E).grid.to_numpy(), {})
                e = _errs(check["V"][period][s.name], Vs)
                wV = [max(x, y) for x, y in zip(wV, e)]
                g, v, mu = check["pub"][period][s.name]
                g2 = g.reshape(len(rows), -1)
                for r, (rg, rv, rmu) in rows.items():
                    for a_, b_ in ((g2[r], rg), (v.reshape(g2.shape)[r], rv), (mu.reshape(g2.shape)[r], rmu)):
                        e = _errs(a_, b_)
                        wR = [max(x, y) for x, y in zip(wR, e)]
        out[key] = {"max_abs_rel_V_err": wV[0], "max_pure_rel_V_err": wV[1],
                    "max_abs_rel_refined_row_err": wR[0], "max_pure_rel_refined_row_err": wR[1],
                    "periods": list(check["periods"]), "form": "fp64 (DC-EGM runs in double precision)"}
    return out


def cpu_baseline(args, checks=None) -> dict:
    """The oracle (NumPy FP64 restatement of the reference's solve) timed on
    one full T=40 solve of the workload (parameter draw 0), every period's
    state rows split over a pool of spawned single-threaded host processes;
    with `checks`, the same oracle output checks the GPU's results (config 1:
    every state of that solve; configs 2 and 3: one step from the GPU's own
    next-period arrays at a few periods)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    model, _ = make_workload(args.periods, args.wealth, args.cons, 1)
    specs = model.regime_specs
    T = model.n_periods
    cores = max(1, min(args.cpu_cores or (os.cpu_count() or 1), 64))
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"  # one BLAS thread per worker process (inherited by the spawned pool)
    with cf.ProcessPoolExecutor(cores, mp_context=mp.get_context("spawn"), initializer=_cpu_init,
                                initargs=(args.periods, args.wealth, args.cons, 0)) as ex:
        list(ex.map(_cpu_rows, [(specs[-1].name, T - 1, np.arange(1), {})] * cores))  # start the workers
        t0 = time.perf_counter()
        oracle_out = _oracle_solve_parallel(ex, specs, T, cores)
        dt = time.perf_counter() - t0
    out = {
        "value": 1.0 / dt,
        "unit": UNIT,
        "cores": cores,
        "kind": "port",
        "sample": f"one full T={T} solve of the workload (parameter draw 0): every period's state rows split over "
        f"{cores} spawned single-threaded processes ({dt:.1f} s)",
        "seconds_per_solve": dt,
        "cpu_model": cpu_model(),
        "blas_threads_per_process": 1,
    }
    if checks:
        acc = {}
        if "config1" in checks:
            acc["config1"] = _check_config1(checks["config1"], oracle_out)
        if "config3" in checks:
            acc["config3"] = _check_config3(checks["config3"])
        if "config2" in checks:
            acc["config2"] = _check_config2(checks["config2"])
        out["accuracy_vs_oracle"] = acc
    return out


def run_reference(args) -> dict:
    """The reference arm: the oracle's full T=40 solve of the workload on the
    host cores, `warmup` untimed solves then `steps` timed ones (each step one
    full solve)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return {}
    model, _ = make_workload(args.periods, args.wealth, args.cons, 1)
    specs = model.regime_specs
    T = model.n_periods
    cores = max(1, min(args.cpu_cores or (os.cpu_count() or 1), 64))
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    times = []
    with cf.ProcessPoolExecutor(cores, mp_context=mp.get_context("spawn"), initializer=_cpu_init,
                                initargs=(args.periods, args.wealth, args.cons, 0)) as ex:
        list(ex.map(_cpu_rows, [(specs[-1].name, T - 1, np.arange(1), {})] * cores))
        for k in range(min(args.warmup, 1) + args.steps):
            t0 = time.perf_counter()
            _oracle_solve_parallel(ex, specs, T, cores)
            if k >= min(args.warmup, 1):
                times.append(time.perf_counter() - t0)
    v = len(times) / float(sum(times))
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / v,
        "higher_is_better": True,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "stochastic retirement model (Tauchen 7-node income), T=40, wealth/consumption 500/500"},
        "cpu_baseline": {
            "value": v,
            "unit": UNIT,
            "cores": cores,
            "kind": "port",
            "sample": f"each step one full T={T} solve (parameter draw 0), state rows split over {cores} processes; "
            f"{min(args.warmup, 1)} untimed warm-up solve",
            "cpu_model": cpu_model(),
            "blas_threads_per_process": 1,
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
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-cores", type=int, default=0, help="host processes of the CPU baseline (0: all)")
    ap.add_argument("--serve-requests", type=int, default=4096)
    ap.add_argument("--agents", type=int, default=10_000)
    ap.add_argument("--serve-batch", type=int, default=64)
    ap.add_argument("--serve-streams", type=int, default=4)
    ap.add_argument("--plain-requests", type=int, default=32)
    ap.add_argument("--no-extra", action="store_true", help="skip the serving / DC-EGM / two-state sections")
    ap.add_argument("--dcegm-batch", type=int, default=32)
    ap.add_argument("--hc-batch", type=int, default=256)
    ap.add_argument("--hc-chunk", type=int, default=32)
    ap.add_argument("--hc-periods", type=int, default=60, help="periods of the two-state model (60: the config)")
    ap.add_argument("--only", choices=["serving", "dcegm", "hc"], default=None,
                    help="run one extra section alone on GPU 0 and print its JSON (for profiling)")
    args = ap.parse_args()
    if args.only:
        import torch

        torch.cuda.set_device(0)
        fn = {"serving": run_serving, "dcegm": run_dcegm, "hc": run_hc}[args.only]
        res = fn(args, 0)
        print(json.dumps({args.only: res[0] if isinstance(res, tuple) else res}))
        return
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
