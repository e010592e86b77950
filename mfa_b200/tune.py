"""Autotuner for the launch shape of the pair kernel.

The pair kernel's work per particle is set by the neighbour count, which
varies with density and cutoff, so the best number of threads sharing one
particle's list and the best block size are measured rather than assumed:
each candidate runs a few hundred real time steps of the system (the state
advances; tuning doubles as equilibration) and the fastest shape is kept.
"""
from __future__ import annotations

import time

CANDIDATES = ((1, 128), (1, 256), (2, 128), (2, 256), (4, 128), (4, 256))


def tune_pair_shape(system, steps: int = 300, candidates=CANDIDATES, repeats: int = 2) -> dict:
    """Time `steps` fused time steps per candidate (best of `repeats`), set the
    fastest shape on `system` and return {shape: seconds}."""
    timings = {}
    for tpp, block in candidates:
        system.set_pair_shape(tpp, block)
        system.step(10)          # capture the graphs outside the timed window
        system.sync()
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            system.step(steps)
            system.sync()
            best = min(best, time.perf_counter() - t0)
        timings[(tpp, block)] = best
    tpp, block = min(timings, key=timings.get)
    system.set_pair_shape(tpp, block)
    return timings
