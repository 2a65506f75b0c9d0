"""Launch-shape autotuner for the FP32 derivative pass.

The derivative kernel is compiled in several shapes (points per tile =
threads per block, resident blocks per SM; see ndt.kernel_variants()).  The
best shape depends on the workload (scan sizes, neighbour counts, map
density), so tune() runs the caller's step once per shape, times it with CUDA
events on the context's stream and selects the fastest on the context.  The
step may be anything enqueued on the context's stream (the benchmark's step
builds the grid and aligns a batch).  C and C++ callers tune an alignment
batch with the library's own ndt_autotune_batch / ndt_autotune_batch_device
(Context.autotune_device here), which the DAPHNE harness front end calls on
its first batch.
"""
from __future__ import annotations

import json
import pathlib


def tune(ctx, step, repeats: int = 2, torch_mod=None):
    """Time `step()` (work enqueued on ctx.stream) for every kernel variant.

    Returns (best_variant, {variant: ms}) and leaves the best one selected.
    """
    import torch

    torch = torch_mod or torch
    st = torch.cuda.ExternalStream(ctx.stream)
    shapes = ctx.L.ndt_kernel_variants()
    times = {}
    for v in range(shapes):
        ctx.set_kernel_variant(v)
        step()  # warm (allocations, caches)
        ctx.synchronize()
        best = None
        for _ in range(repeats):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            step()
            e1.record(st)
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        times[v] = best
    winner = min(times, key=times.get)
    ctx.set_kernel_variant(winner)
    return winner, times


def save(path, workload: str, winner: int, times: dict, shapes):
    p = pathlib.Path(path)
    table = json.loads(p.read_text()) if p.exists() else {}
    table[workload] = {"variant": winner, "shape": list(shapes[winner]),
                       "ms": {str(k): v for k, v in times.items()}}
    p.write_text(json.dumps(table, indent=1))
