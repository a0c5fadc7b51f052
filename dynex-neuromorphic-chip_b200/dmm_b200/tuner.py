"""Launch-shape autotuner.

Results never depend on the launch shape (canonical per-variable sums, instance-aligned
tiles), so the tuner only measures device time and keeps the fastest shape.  It sweeps
lanes per variable in the dV reduction (var_group, the "threads per clause-occurrence
group"), clause tile, variable tile, persistent blocks per SM and steps per CUDA graph.
"""
from __future__ import annotations

import itertools

from .instance import Instance

VAR_GROUPS = (1, 2, 4, 8, 16, 32)
CLAUSE_TILES = (1024, 2048, 4096)
VAR_TILES = (256, 512, 1024)
STEPS_PER_GRAPH = (16, 64, 256)


def autotune(inst: Instance, x0, steps: int = 6, flush_bytes: int = 0, var_groups=None,
             clause_tiles=CLAUSE_TILES, var_tiles=VAR_TILES, blocks_per_sm=(0,),
             steps_per_graph=STEPS_PER_GRAPH, verbose: bool = False) -> dict:
    """Measures every shape on `inst` from state x0 and applies the fastest.  Returns
    {"best": shape, "table": [(shape, ms_per_step), ...]}.  Leaves the instance at x0."""
    if var_groups is None:
        var_groups = (32,) if inst.precision == "fp64" else VAR_GROUPS
    table = []
    for g, ct, vt, bps in itertools.product(var_groups, clause_tiles, var_tiles, blocks_per_sm):
        shape = dict(var_group=g, clause_tile=ct, var_tile=vt, blocks_per_sm=bps)
        inst.set_tuning(**shape)
        inst.set_state(x0)
        inst.profile(2, flush_bytes)
        a, b = inst.profile(steps, flush_bytes)
        table.append((shape, (a + b) / steps))
        if verbose:
            print(shape, (a + b) / steps)
    best = min(table, key=lambda r: r[1])[0]
    inst.set_tuning(**best)
    # steps per graph: the solver's own launch path
    gtable = []
    for s in steps_per_graph:
        inst.set_tuning(steps_per_graph=s)
        inst.set_state(x0)
        inst.time_steps(s)
        ms = inst.time_steps(2 * s)
        gtable.append((s, ms / (2 * s)))
        if verbose:
            print("steps_per_graph", s, ms / (2 * s))
    best["steps_per_graph"] = min(gtable, key=lambda r: r[1])[0]
    inst.set_tuning(**best)
    inst.set_state(x0)
    return {"best": best, "table": table, "graph_table": gtable}


BATCH_VAR_GROUPS = (1, 4, 8, 32)
BATCH_STEPS_PER_GRAPH = (16, 64, 256)


def autotune_batch(items, max_steps: int, var_groups=BATCH_VAR_GROUPS,
                   steps_per_graph=BATCH_STEPS_PER_GRAPH, sample: int = 512,
                   device: int = 0) -> dict:
    """Batched configuration: integrates the same sample of formulas (the first `sample`
    items, each from its own initial state, to the step cap or its solution) under every
    (lanes per variable, steps per CUDA graph) shape and keeps the shape with the lowest
    device time.  Results are identical for every shape, so only time decides.  Returns
    {"best": {"var_group": g, "steps_per_graph": s}, "table": [((g, s), device_ms), ...]}."""
    from .workloads import run_batched

    part = items[:sample]
    table = []
    for g, s in itertools.product(var_groups, steps_per_graph):
        r = run_batched(part, max_steps, tuning=dict(var_group=g, steps_per_graph=s),
                        device=device)
        table.append(((g, s), r["device_ms"]))
    (g, s), _ = min(table, key=lambda r: r[1])
    return {"best": {"var_group": g, "steps_per_graph": s}, "table": table}
