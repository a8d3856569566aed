"""Many independent designs over the ranks of a job.

The reference places one design per process (main/ePlace_main.cpp); a batch
of designs is independent units of work.  Each rank places its share on its
own GPU (on one GPU the engines' loops interleave through ep_run_batch), with
no collective during placement; at the end one object gather brings every
design's result to rank 0.  Designs are dealt to ranks by estimated cost,
pins + B log2 B for B bins (the per-net passes scale with pins, the Poisson
solve with the bin grid), longest first onto the least-loaded rank, so the
ranks finish close together.
"""
import math

import numpy as np


def reference_bins(nl, target_density=None):
    """Bins per side that the engine picks when none are given: the
    reference's rule (EPlace/eplace.cpp:230-261; csrc/engine.cu
    bin_dimension) in float: the largest 2^k, k in 2..10, whose square does
    not exceed core area / (average node area / target density)."""
    if getattr(nl, "bins", 0):
        return int(nl.bins)
    td = np.float32(nl.target_density if target_density is None else target_density)
    f32 = np.float32
    left, right = f32(np.min(nl.row_llx)), f32(np.max(nl.row_urx))
    bottom = f32(nl.row_lly[0])
    top = f32(np.float64(nl.row_lly[-1]) + np.float64(nl.row_h[-1]))
    area = np.asarray(nl.node_w, np.float32) * np.asarray(nl.node_h, np.float32)
    node_area = f32(np.sum(area, dtype=np.float32))
    avg = f32(node_area / f32(len(area)))
    ideal = f32(avg / td)
    core_area = f32((right - left) * (top - bottom))
    count = int(np.float64(core_area / ideal) + 0.5)
    for i in range(1, 10):
        a, b = (2 << i) ** 2, (2 << (i + 1)) ** 2
        if a <= count < b:
            return 2 << i
    return 1024


def design_cost(nl, target_density=None):
    """Estimated work of placing a design: pins + B log2 B, B = bins^2."""
    b = reference_bins(nl, target_density) ** 2
    return float(nl.num_pins) + b * math.log2(b)


def partition(costs, world):
    """Design indices per rank: longest first, each onto the rank with the
    least load so far (ties: the lower rank); within a rank in ascending
    index order.  Deterministic, and the busiest rank carries at most the
    mean load plus one design."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    share = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in share]


def place_designs(netlists, place_batch, rank=0, world=1, dist=None, costs=None):
    """Place `netlists` over `world` ranks; this rank places its share with
    place_batch(list of netlists) -> list of per-design results.  With
    `dist` (torch.distributed, initialised) the results are gathered to rank
    0, which returns all of them in design order; other ranks return None.
    Without it, returns this rank's results as {design index: result}."""
    costs = [design_cost(nl) for nl in netlists] if costs is None else costs
    mine = partition(costs, world)[rank]
    results = place_batch([netlists[i] for i in mine]) if mine else []
    if len(results) != len(mine):
        raise RuntimeError("place_batch returned a result count that differs from its designs")
    local = dict(zip(mine, results))
    if dist is None:
        return local
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(local, gathered, dst=0)
    if rank != 0:
        return None
    merged = {}
    for part in gathered:
        merged.update(part)
    return [merged[i] for i in range(len(netlists))]


def engine_batch(netlists, device=0, max_steps=0, **params):
    """place_batch for the GPU: one engine per design on `device`, each
    initialised, all loops run together (ep_run_batch); returns per design
    its run statistics and final movable-node centres."""
    from . import placer
    engines = []
    try:
        engines = placer.create_engines(
            netlists, [placer.default_params(target_density=float(nl.target_density), device=device, **params)
                       for nl in netlists])
        for e in engines:
            e.initialize()
        stats = placer.run_batch(engines, max_steps=max_steps)
        out = []
        for nl, e, st in zip(netlists, engines, stats):
            out.append(dict(st, positions=e.get_positions()[: nl.num_nodes]))
        return out
    finally:
        for e in engines:
            e.close()
