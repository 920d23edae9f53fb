"""Project autotuner for the launch parameters of a context.

The tunable choices (``cfem_ctx_set_param``) are the number of Tet10
elements (one warp each) per block of the batched element kernel, the
threads per block of the P1 element kernels, and the iterations per body of
the graph scheduler's device-side solve loop. For a workload the tuner times
every candidate on the device (CUDA events on the current stream, median of
a few runs after one warm-up run), keeps the fastest, and records it in a
JSON cache keyed by the GPU and the workload's shape, so later runs of the
same shape start from the tuned values without timing.

Cache file: ``$CLOUDFEM_B200_TUNE_CACHE`` or
``~/.cache/cloudfem_b200/autotune.json``.
"""

import itertools
import json
import math
import os
import tempfile

from . import _native as N

T10_WARPS = (2, 4, 8)
P1_THREADS = (32, 64, 128)
GRAPH_ITERS = (1, 2, 4, 8)


def cache_path():
    return os.environ.get("CLOUDFEM_B200_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "cloudfem_b200", "autotune.json")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(entries):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path), suffix=".tmp")
        with os.fdopen(fd, "w") as f:
            json.dump(entries, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass                       # a read-only home only loses the cache


def device_key(rt):
    import torch
    p = torch.cuda.get_device_properties(rt.device)
    return f"{p.name}|sm{p.major}{p.minor}|{p.multi_processor_count}sm"


def time_ms(fn, repeat=3):
    """Median device time of fn() (CUDA events on the current stream)."""
    import torch
    fn()                                        # warm-up
    ts = []
    for _ in range(repeat):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ts.sort()
    return ts[len(ts) // 2]


def tune(rt, key, space, run, repeat=3, use_cache=True):
    """Grid search over space {param: candidates}; returns (best, timings).

    run() is one execution of the workload with the context's current
    parameters. The best setting is applied to rt and cached under key."""
    full_key = f"{device_key(rt)}|{key}"
    entries = _load() if use_cache else {}
    if use_cache and full_key in entries:
        best = {int(k): v for k, v in entries[full_key]["best"].items()}
        for p, v in best.items():
            rt.set_param(p, v)
        return best, entries[full_key].get("timings_ms", {})
    params = sorted(space)
    timings = {}
    best, best_t = None, math.inf
    for combo in itertools.product(*(space[p] for p in params)):
        for p, v in zip(params, combo):
            rt.set_param(p, v)
        t = time_ms(run, repeat)
        timings[",".join(f"{p}={v}" for p, v in zip(params, combo))] = t
        if t < best_t:
            best, best_t = dict(zip(params, combo)), t
    for p, v in best.items():
        rt.set_param(p, v)
    if use_cache:
        entries = _load()
        entries[full_key] = {"best": {str(p): v for p, v in best.items()},
                             "timings_ms": timings}
        _store(entries)
    return best, timings


def _shape_key(kind, batch):
    dofs = sum(it["dm"].n_nodes for it in batch.items)
    return f"{kind}|n{len(batch.items)}|dofs2^{int(math.log2(max(dofs, 1)))}"


def tune_batch(batch, precision="mixed", rtol=1e-10, solve=True, repeat=3,
               use_cache=True):
    """Tune a prepared cloudfem_b200.batch.Batch: element-kernel block
    shape on its assembly, then the solve-loop body length on its solve.
    Returns {"assembly": {...}, "solve": {...}} with names and values."""
    rt = batch.rt
    npes = {it["dm"].npe for it in batch.items}
    space = {}
    if 10 in npes:
        space[N.PARAM_T10_WARPS] = T10_WARPS
    if 4 in npes:
        space[N.PARAM_P1_THREADS] = P1_THREADS
    out = {}
    if space:
        best, t = tune(rt, _shape_key("assemble", batch), space, batch.assemble,
                       repeat, use_cache)
        out["assembly"] = {"best": _names(best), "timings_ms": t}
    batch.assemble()
    if solve:
        def run():
            batch.solve(precision, rtol=rtol)
        best, t = tune(rt, _shape_key(f"solve-{precision}", batch),
                       {N.PARAM_GRAPH_ITERS: GRAPH_ITERS}, run, max(1, repeat - 2),
                       use_cache)
        out["solve"] = {"best": _names(best), "timings_ms": t}
    return out


def _names(best):
    names = {N.PARAM_T10_WARPS: "t10_elements_per_block",
             N.PARAM_P1_THREADS: "p1_threads_per_block",
             N.PARAM_GRAPH_ITERS: "iterations_per_loop_body"}
    return {names[p]: v for p, v in best.items()}
