"""Synthetic workloads of the batched and served configurations, and their drivers.

The reference's benchmark instances (planted 3-SAT, n = 100,000) are not available; these
generators produce seeded planted 3-SAT formulas with the stated parameters instead:

* batched: `count` formulas, n log-uniform in [n_lo, n_hi], m = round(r n), p0 = 0.08, p1 = 0.46,
  integrated together in one pack (`run_batched`), compared with the plain path that solves the
  same formulas one at a time on the same GPU (`run_plain`);
* served: Poisson arrivals at `rate` requests/s, n log-uniform, r drawn from `ratios`, admitted
  by device-memory footprint into a continuous-batching server (`run_served`) and compared with
  the same arrival stream served one request at a time (`run_served_plain`).

Instances use the FP32 production path and initial state V ~ U[-1,1], Xs ~ U[0,1], Xl = 1.
Per-instance results are identical in every mode (the integrator's arithmetic does not depend on
what else is resident), so solve rates are equal by construction for a common step cap.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np

from .batch import Batch
from .cnf import Formula, generate_planted, initial_state_uniform
from .instance import Instance
from .server import Server


@dataclass
class Item:
    formula: Formula
    x0: np.ndarray
    seed: int
    ratio: float


def make_items(count: int, n_lo: int, n_hi: int, ratios=(8.0,), seed: int = 0,
               p0: float = 0.08, p1: float = 0.46) -> list[Item]:
    rng = np.random.default_rng(seed)
    items = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        r = float(rng.choice(ratios))
        m = int(round(r * n))
        s = seed * 1_000_003 + k
        f, _ = generate_planted(n, m, p0, p1, seed=s)
        items.append(Item(f, initial_state_uniform(f, s + 7), s, r))
    return items


def run_batched(items: list[Item], max_steps: int, tuning: dict | None = None,
                device: int = 0) -> dict:
    """All items in one pack; returns throughput, solve counts and per-item results."""
    t0 = time.perf_counter()
    b = Batch.for_formulas([it.formula for it in items], precision="fp32", device=device)
    if tuning:
        b.set_tuning(**tuning)
    for it in items:
        b.add(it.formula, it.x0, max_steps=max_steps)
    t1 = time.perf_counter()
    stats = b.run()
    t2 = time.perf_counter()
    results = [b.result(k)[0] for k in range(len(items))]
    b.close()
    solved = sum(r.solved for r in results)
    return {
        "instances": len(items), "solved": solved, "setup_s": t1 - t0, "run_s": t2 - t1,
        "device_ms": stats["device_ms"], "clause_updates": stats["clause_updates"],
        "clause_updates_per_s": stats["clause_updates"] / (stats["device_ms"] / 1000.0),
        "solves_per_s": solved / (t2 - t0), "solves_per_s_run": solved / (t2 - t1),
        "steps": [r.steps for r in results], "solved_flags": [r.solved for r in results],
    }


def run_plain(items: list[Item], max_steps: int, device: int = 0) -> dict:
    """The same items one at a time through the single-instance path (create + solve)."""
    t0 = time.perf_counter()
    solved = 0
    updates = 0
    steps = []
    flags = []
    for it in items:
        with Instance(it.formula, precision="fp32", device=device) as inst:
            inst.set_state(it.x0)
            r = inst.solve(max_steps=max_steps)
        solved += r.solved
        updates += it.formula.m * r.steps
        steps.append(r.steps)
        flags.append(r.solved)
    dt = time.perf_counter() - t0
    return {"instances": len(items), "solved": solved, "wall_s": dt, "solves_per_s": solved / dt,
            "clause_updates_per_s": updates / dt, "steps": steps, "solved_flags": flags}


def precision_study(n: int = 1_000_000, r: float = 8.0, seeds=range(8),
                    checkpoints=(10, 100, 1000), max_steps: int = 5000, instance_seed: int = 7,
                    device: int = 0) -> dict:
    """FP32 production path against the FP64 path (the reference's arithmetic) on one planted
    formula from several initial states: max |dV| and |dXl| at each checkpoint step (while
    both runs are still integrating), then solve rate and steps-to-solution of each.  A run
    in which either precision stopped (solved) before a checkpoint is counted under that
    checkpoint's "stopped_before" instead."""
    f, _ = generate_planted(n, int(round(r * n)), 0.08, 0.46, seed=instance_seed)
    errs = {c: {"dv": [], "dxl": []} for c in checkpoints}
    stopped = {c: 0 for c in checkpoints}
    res = {"fp32": [], "fp64": []}
    i32 = Instance(f, precision="fp32", device=device)
    i64 = Instance(f, precision="fp64", device=device)
    try:
        for s in seeds:
            x0 = initial_state_uniform(f, 10_000 + s)
            i32.set_state(x0)
            i64.set_state(x0)
            done = 0
            for k, c in enumerate(checkpoints):
                a = i32.step(c - done)
                b = i64.step(c - done)
                done = c
                if a.status != 0 or b.status != 0:
                    for later in checkpoints[k:]:
                        stopped[later] += 1
                    break
                xa, _ = i32.get_state()
                xb, _ = i64.get_state()
                errs[c]["dv"].append(float(np.max(np.abs(xa[:n] - xb[:n]))))
                errs[c]["dxl"].append(float(np.max(np.abs(xa[n + f.m:] - xb[n + f.m:]))))
            for name, inst in (("fp32", i32), ("fp64", i64)):
                rr = inst.solve(max_steps=max_steps)
                res[name].append((rr.solved, rr.solved_step if rr.solved else rr.steps))
    finally:
        i32.close()
        i64.close()
    out = {"n": n, "m": f.m, "r": r, "seeds": len(list(seeds)), "max_steps": max_steps,
           "checkpoints": {}}
    for c in checkpoints:
        row = {"runs": len(errs[c]["dv"]), "stopped_before": stopped[c]}
        if errs[c]["dv"]:
            row.update(max_abs_dv=max(errs[c]["dv"]), max_abs_dxl=max(errs[c]["dxl"]),
                       median_max_abs_dv=float(np.median(errs[c]["dv"])))
        out["checkpoints"][str(c)] = row
    for name in ("fp32", "fp64"):
        solved = [st for ok, st in res[name] if ok]
        out[name] = {"solve_rate": len(solved) / max(1, len(res[name])),
                     "steps_p50": float(np.median(solved)) if solved else None,
                     "steps_p90": float(np.percentile(solved, 90)) if solved else None,
                     "steps": [st for _, st in res[name]]}
    return out


def poisson_times(count: int, rate: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed + 99)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def run_served(items: list[Item], arrivals: np.ndarray, budget_bytes: int, max_steps: int,
               max_slots: int = 4096, steps_per_launch: int = 16, device: int = 0) -> dict:
    """Continuous batching: requests are submitted at their arrival times while earlier ones
    integrate on the device; time-to-solution = finish - arrival."""
    srv = Server(budget_bytes, max_slots=max_slots, steps_per_launch=steps_per_launch,
                 precision="fp32", device=device)
    t0 = time.perf_counter()
    nxt = 0
    done = {}
    ticket_of = {}
    while len(done) < len(items):
        now = time.perf_counter() - t0
        while nxt < len(items) and arrivals[nxt] <= now:
            it = items[nxt]
            t = srv.submit(it.formula, x0=it.x0, max_steps=max_steps)
            ticket_of[t] = (nxt, now)
            nxt += 1
        resident, queued = srv.pump()
        for res in srv.take():
            k, sub = ticket_of[res["ticket"]]
            done[k] = (res, time.perf_counter() - t0 - arrivals[k])
        if resident == 0 and queued == 0 and nxt < len(items):
            time.sleep(max(0.0, min(0.002, arrivals[nxt] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    srv.close()
    tts = np.array([done[k][1] for k in range(len(items))])
    solved = sum(done[k][0]["result"].solved for k in range(len(items)))
    return {"requests": len(items), "solved": solved, "wall_s": wall,
            "solves_per_s": solved / wall, "p50_tts_s": float(np.percentile(tts, 50)),
            "p99_tts_s": float(np.percentile(tts, 99)),
            "steps": [done[k][0]["result"].steps for k in range(len(items))]}


def run_served_plain(items: list[Item], arrivals: np.ndarray, max_steps: int,
                     device: int = 0) -> dict:
    """The same arrival stream served one request at a time (FIFO, single instance path)."""
    t0 = time.perf_counter()
    tts = []
    solved = 0
    for k, it in enumerate(items):
        now = time.perf_counter() - t0
        if arrivals[k] > now:
            time.sleep(arrivals[k] - now)
        with Instance(it.formula, precision="fp32", device=device) as inst:
            inst.set_state(it.x0)
            r = inst.solve(max_steps=max_steps)
        solved += r.solved
        tts.append(time.perf_counter() - t0 - arrivals[k])
    wall = time.perf_counter() - t0
    tts = np.array(tts)
    return {"requests": len(items), "solved": solved, "wall_s": wall,
            "solves_per_s": solved / wall, "p50_tts_s": float(np.percentile(tts, 50)),
            "p99_tts_s": float(np.percentile(tts, 99))}
