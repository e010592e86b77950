"""Autotuner for the launch shape of the pair kernel.

The pair kernel's work per particle is set by the neighbour count, which
varies with density and cutoff, so its launch shape is measured rather than
assumed: the number of in-range pairs a thread keeps per pass, the block size,
and whether each block stages its neighbourhood in shared memory or reads it
through the caches.  Each candidate runs a few hundred real time steps of the
system (the state advances; tuning doubles as equilibration) and the fastest
shape is kept.  Results do not depend on the shape.
"""
from __future__ import annotations

import time

CANDIDATES = ((4, 128, True), (8, 128, True), (4, 64, True),
              (2, 128, False), (4, 128, False), (4, 256, False), (8, 256, False))


def tune_pair_shape(system, steps: int = 300, candidates=CANDIDATES, repeats: int = 2) -> dict:
    """Time `steps` fused time steps per candidate (best of `repeats`), set the
    fastest shape on `system` and return {shape: seconds}."""
    timings = {}
    for k, block, tiled in candidates:
        system.set_pair_shape(k, block, tiled)
        system.step(10)          # capture the graphs outside the timed window
        system.sync()
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            system.step(steps)
            system.sync()
            best = min(best, time.perf_counter() - t0)
        timings[(k, block, tiled)] = best
    k, block, tiled = min(timings, key=timings.get)
    system.set_pair_shape(k, block, tiled)
    return timings
