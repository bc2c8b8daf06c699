"""Autotuner for the launch shape of kernel (a).

For each regime of a model and a batch size, candidate ``LaunchConfig``s
(lanes per state, states per thread, block size, action chunk) are compiled
and timed on the device with CUDA events on the regime's most expensive
Bellman launch; the fastest is kept.  Results are cached in a JSON file keyed
by the GPU name, the structure hash of the regime's generated code and the
batch-size bucket, so tuning runs once per (model structure, batch bucket).

The candidate set is built around the occupancy heuristic of
``engine.default_config``: lanes in {L/2, L, 2L} (L the heuristic), states per
thread in {1, 2} (and 4 in the single-precision search), block in {128, 256},
action chunk in {256, 512}.

A candidate that NVRTC cannot compile, or whose launch the driver refuses
(resources), is skipped.  Any other failure -- in particular an error left
on the context by a launch that ran -- is raised: the context would be
unusable for the remaining candidates and for the caller.

Used by ``BatchSolver(..., autotune=True)`` and ``Server(..., autotune=True)``.
"""

from __future__ import annotations

import hashlib
import itertools
import json
import os
from pathlib import Path

from pylcm_b200.codegen import LaunchConfig
from pylcm_b200.engine import SolveEngine, default_config

CACHE = Path(os.environ.get("LCMX_CACHE_DIR", Path.home() / ".cache" / "pylcm_b200")) / "autotune.json"


def _bucket(n: int) -> int:
    b = 1
    while b < n:
        b *= 2
    return b


def _structure_key(eng: SolveEngine, spec, params) -> str:
    tg = eng.targets_at(spec, min(spec.active_periods))
    rk = eng.kernels(spec, tg, params, 1)
    src = rk.src.split("// ---- regime", 1)[-1]
    # drop the config-dependent tag so all variants share a key
    return hashlib.sha1((src.replace(rk.tag, "TAG") + eng.precision).encode()).hexdigest()[:20]


def candidates(spec, precision: str, n_items: int) -> list[LaunchConfig]:
    """Launch shapes around the heuristic's; the heuristic's own shape first."""
    base = default_config(spec, precision, n_items)
    lanes_set = sorted({max(1, base.lanes // 2), base.lanes, min(32, base.lanes * 2)})
    sbs = (1, 2, 4) if precision == "fp32" else (1, 2)
    out = [base]
    for lanes, sb, block, chunk in itertools.product(lanes_set, sbs, (128, 256), (256, 512)):
        if lanes * 8 > max(8, spec.n_actions) or block // lanes < 8:
            continue
        cfg = LaunchConfig(block=block, lanes=lanes, chunk=chunk, sb=sb)
        if cfg not in out:
            out.append(cfg)
    return out


def _skippable(e: Exception) -> bool:
    """A candidate failure that leaves the context usable: NVRTC rejected
    the source (LCMX_ERR_COMPILE) or the driver refused the launch
    configuration (LCMX_ERR_LAUNCH before anything ran)."""
    from pylcm_b200.exceptions import KernelError

    return isinstance(e, KernelError) and e.status in (2, 4)


def _time_regime(model, precision: str, params_list, spec, cfg: LaunchConfig, reps: int = 2) -> float:
    import torch

    eng = SolveEngine(model, precision, configs={spec.name: cfg})
    plan = eng.plan(params_list)
    plan.run()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    ib, pb = plan.items.data_ptr(), plan.prefix.data_ptr()
    launches = [l for l in plan.launches if l.kind == "bellman" and l.module.spec.name == spec.name]
    # the heaviest launch: most targets, earliest period
    launches.sort(key=lambda l: (-len(l.module.targets), l.period))
    l = launches[0]
    best = float("inf")
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(s)
        l.module.module.bellman_step(
            l.kernel, ib + 8 * l.item_off, pb + 4 * l.prefix_off, l.n_items, l.n_tiles, l.block, l.smem, s.cuda_stream
        )
        b.record(s)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def tune(model, precision: str, params_list, regimes: list[str] | None = None, verbose: bool = False) -> dict:
    """Return {regime: LaunchConfig} for this batch (tuning uncached regimes)."""
    import torch

    n = len(params_list)
    eng = SolveEngine(model, precision)
    cache = json.loads(CACHE.read_text()) if CACHE.exists() else {}
    gpu = torch.cuda.get_device_name(0)
    out = {}
    # a small horizon is enough to time one Bellman launch
    for spec in model.regime_specs:
        if regimes is not None and spec.name not in regimes:
            continue
        if spec.n_states * spec.n_actions < 4096:
            continue
        key = f"{gpu}|{_structure_key(eng, spec, params_list[0])}|{_bucket(n)}"
        hit = cache.get(key)
        if hit is not None:
            out[spec.name] = LaunchConfig(**hit)
            continue
        results = []
        for cfg in candidates(spec, precision, n):
            try:
                t = _time_regime(model, precision, params_list, spec, cfg)
            except Exception as e:
                if not _skippable(e):
                    raise
                # the refused candidate must not have left an error behind
                torch.cuda.synchronize()
                if verbose:
                    print("autotune: skip", cfg, repr(e)[:120])
                continue
            results.append((t, cfg))
            if verbose:
                print(f"autotune {spec.name} {cfg}: {t:.3f} ms")
        if not results:
            continue
        results.sort(key=lambda r: r[0])
        best = results[0][1]
        out[spec.name] = best
        cache[key] = {"block": best.block, "lanes": best.lanes, "chunk": best.chunk, "sb": best.sb, "min_blocks": best.min_blocks}
        CACHE.parent.mkdir(parents=True, exist_ok=True)
        tmp = CACHE.with_suffix(".tmp")
        tmp.write_text(json.dumps(cache, indent=1))
        tmp.replace(CACHE)
    return out
