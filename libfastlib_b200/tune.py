"""Autotuner for the launch shapes of libwahgpu (results never depend on
them): times each candidate on the caller's own workload with CUDA events
and leaves the fastest set on the context.

    best, table = tune_batch(ctx, batch)                  # range batches
    best, table = tune_dense(ctx, [(a, b, op, out), ...])  # dense-path operators
"""
from __future__ import annotations

import itertools

from . import TUNE_DENSE_ENGINE, TUNE_DENSE_TILE, TUNE_RANGE_CTAS, TUNE_RANGE_ORDER


def _time(fn, reps: int) -> float:
    import torch
    fn()  # warm-up (first-launch attribute setting, allocation)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_batch(ctx, batch, count_only: bool = True, ctas=(0, 1, 2, 4), reps: int = 2):
    """Work order x resident CTAs per SM for the persistent range launch,
    timed on `batch`.  Count-only batches try query by query (0) and tile by
    tile (1); batches with row ids try query by query with the look-back (0)
    and two tile-by-tile passes around a scan (2)."""
    orders = (0, 1) if count_only else (0, 2)
    table = {}
    for order, c in itertools.product(orders, ctas):
        ctx.set_tuning(TUNE_RANGE_ORDER, order)
        ctx.set_tuning(TUNE_RANGE_CTAS, c)
        table[(order, c)] = _time(batch.run, reps)
    best = min(table, key=table.get)
    ctx.set_tuning(TUNE_RANGE_ORDER, best[0])
    ctx.set_tuning(TUNE_RANGE_CTAS, best[1])
    return best, table


def tune_dense_tile(ctx, a, b, op: int, out, tiles=(1024, 2048, 4096), reps: int = 5):
    """Groups per tile of the dense-path kernel, timed on a OP b into out."""
    table = {}
    for t in tiles:
        ctx.set_tuning(TUNE_DENSE_TILE, t)
        table[t] = _time(lambda: a.binop_into(op, b, out), reps)
    best = min(table, key=table.get)
    ctx.set_tuning(TUNE_DENSE_TILE, best)
    return best, table


def tune_dense(ctx, calls, engines=((5, 2048), (4, 1024), (4, 2048), (4, 4096), (3, 2048)), reps: int = 5):
    """Engine x tile size for the canonical-result (dense-path) operators,
    timed on the caller's calls [(a, b, op, out), ...] together: the
    single-pass kernel over warp tiles (5), the single-pass kernel over CTA
    tiles of 1024 / 2048 / 4096 groups (4: its look-back chain shortens as
    tiles grow, its occupancy falls) and the two-pass kernels (3).  Leaves
    the fastest set on the context."""
    table = {}
    for eng, tile in engines:
        ctx.set_tuning(TUNE_DENSE_ENGINE, eng)
        ctx.set_tuning(TUNE_DENSE_TILE, tile)
        table[(eng, tile)] = _time(lambda: [a.binop_into(op, b, out) for a, b, op, out in calls], reps)
    best = min(table, key=table.get)
    ctx.set_tuning(TUNE_DENSE_ENGINE, best[0])
    ctx.set_tuning(TUNE_DENSE_TILE, best[1])
    return best, table
