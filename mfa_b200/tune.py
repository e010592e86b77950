"""Autotuner: cell size, Verlet skin and the pair kernel's launch shape.

A larger skin lists more pairs per particle but rebuilds the lists less often;
the pair kernel's best shape (list entries a thread tests per round, block
size, shared-memory tiling or not, a work queue of a fixed number of CTAs per
multiprocessor or not, the pieces each chunk's list is cut into) depends on
the neighbour count and the system size.  None of them changes the forces, so
all are measured rather than assumed: each candidate runs a few hundred real
time steps of the system (the state advances; tuning doubles as
equilibration) and the fastest is kept.
"""
from __future__ import annotations

import time

import math

# (entries per lane and round, threads per block, tiled, work-queue CTAs per SM)
CANDIDATES = ((2, 128, True, 0), (4, 64, True, 0),
              (2, 128, False, 0), (4, 128, False, 0), (2, 256, False, 0), (4, 256, False, 0),
              (2, 128, False, 6), (2, 128, False, 8), (2, 256, False, 3), (2, 256, False, 4))
SKINS = (0.2, 0.3, 0.4, 0.5, 0.6)
# pieces per chunk tried for the best untiled shape
SPLITS = (1, 2, 4, 8, 16, 32)


def list_radius(params, skin: float) -> float:
    """Verlet-list radius for a skin: max LJ range + skin (or the Ewald
    real-space cutoff + skin when that is decoupled from the LJ range)."""
    rcm = math.sqrt(max(params.range_2[k] for k in range(64)))
    r = rcm + skin
    if params.charged and not (params.quirks & 1):
        r = max(r, math.sqrt(params.ewald_rc_2) + skin)
    return r


def cells_for(params, skin: float):
    """Finest grid whose cells still hold the list radius (at least 1 cell)."""
    r = list_radius(params, skin)
    return [max(1, int(params.boundary[d] / r)) for d in range(3)]


def _time(system, steps, repeats):
    system.step(10)              # rebuild / capture outside the timed window
    system.sync()
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        system.step(steps)
        system.sync()
        best = min(best, time.perf_counter() - t0)
    return best


def tune_cells(system, steps: int = 300, skins=SKINS, repeats: int = 2) -> dict:
    """Try each skin with the finest valid cell grid, keep the fastest.
    Returns {skin: seconds}."""
    timings = {}
    for skin in skins:
        nb = cells_for(system.params, skin)
        system.set_cells(nb, skin)
        timings[skin] = _time(system, steps, repeats)
    best = min(timings, key=timings.get)
    system.set_cells(cells_for(system.params, best), best)
    return timings


def autotune(system, steps: int = 300) -> dict:
    """Cell size and skin, then the pair kernel's launch shape, then the skin
    again for that shape (a cheaper pair kernel moves the skin's optimum)."""
    cells = tune_cells(system, steps)
    shape = tune_pair_shape(system, steps)
    cells2 = tune_cells(system, steps)
    return {"skin": cells, "pair_shape": shape, "skin_for_shape": cells2}


def set_shape(system, k, block, tiled, queue, split):
    """The pair kernel's launch shape on `system`: list entries per lane and
    round, threads per block, tiled or not, work-queue CTAs per SM (untiled;
    0: static) and pieces per chunk (untiled)."""
    system.set_pair_shape(k, block, tiled)
    system.set_pair_queue(0 if tiled else queue)
    system.set_pair_split(1 if tiled else split)


def tune_pair_shape(system, steps: int = 300, candidates=CANDIDATES, splits=SPLITS, repeats: int = 2) -> dict:
    """Time `steps` fused time steps per candidate (best of `repeats`), set the
    fastest shape on `system` and return {shape: seconds}.  The candidates run
    with the context's default pieces per chunk; the best untiled one is then
    timed with each count in `splits`."""
    split0 = system.pair_split()
    timings = {}
    for k, block, tiled, queue in candidates:
        set_shape(system, k, block, tiled, queue, split0)
        timings[(k, block, tiled, queue, 1 if tiled else split0)] = _time(system, steps, repeats)
    untiled = [c for c in timings if not c[2]]
    if untiled:
        k, block, _, queue, _ = min(untiled, key=timings.get)
        for split in splits:
            if (k, block, False, queue, split) not in timings:
                set_shape(system, k, block, False, queue, split)
                timings[(k, block, False, queue, split)] = _time(system, steps, repeats)
    set_shape(system, *min(timings, key=timings.get))
    return timings
