"""Regenerates the golden fixtures from the reference (run in a container that has the
reference sources; the committed outputs travel with the repository).

    python tests/golden/make_golden.py [--ref-dir /root/reference]

Outputs, next to this script:
  fixtures.npz        the reference's CNF fixtures n = 100 .. 1000 (cnf/*.cnf) as arrays,
                      with the planted assignment of their first comment line when present
  known_answers.json  the UNMODIFIED reference CLI (oracle/_ref/dynex_ref) on each fixture
                      and seed 0, 1, 2 (plus n = 10000, seed 0): printed step count, T,
                      and the reported `v` assignment; and the reference's per-step harness
                      (oracle/_ref/libdynex_ref.so) from a seeded uniform initial state:
                      SHA-256 of the FP64 state at selected steps, solve step and T;
                      and the reference CLI with its alpha heuristic (-p 1) on a seeded
                      planted formula (n = 2000, m = 8520, no clause agreeing with the
                      planted assignment in all three literals) that needs more than 10^4
                      steps: step count, T, the heuristic's printed counts and median, and
                      the SHA-256 of the `v` assignment.

    python tests/golden/make_golden.py --only heuristics   # adds/refreshes that entry only
    python tests/golden/make_golden.py --only large        # adds/refreshes the entries below
    python tests/golden/make_golden.py --only replicas     # adds/refreshes cli_replicas
    python tests/golden/make_golden.py --only tuner        # adds/refreshes cli_tuner

cli_tuner: the reference CLI's parameter tuner (-t 1) on fixtures n = 1000 (seed 1, three
replicas) and n = 500 (seed 2, two replicas): the initial objective of every replica, the
`c [TUNE] E:` line (dynex.cc:1711-1722), which the reference computes with one Euler step
through odeint's integrate_n_steps (implemented by oracle/boost_stub from Boost.Odeint's
documented behaviour).  The tuner's later iterations run until a wall-clock limit
(dynex.cc's default integrator ignores maxsteps), so only this first objective is
deterministic.

cli_replicas: the reference CLI with three replicas (-w 3, one thread each, dynex.cc:2643-2700:
replica i > 0 runs alpha / i; with seed 0 replicas 0, 1, 2 start at all 1, 0, -1, otherwise
from one shared mt19937) on fixtures n = 200 and 500, seeds 0 and 1: for every replica that
printed its solving right-hand side before the first solution stopped the others, its step
count and T (which replicas get to print depends on thread timing; each printed pair does
not).

The "large" entries pin the benchmarked sizes (formulas and initial states from the
library's seeded generator, restated in oracle/instance_gen.h and built here by the
reference harness library):
  fixture_n10000.npz  the reference's n = 10000 fixture as arrays (its CLI known answer,
                      156 steps and T = 13.62 for seed 0, is in known_answers.json)
  large.c2_bench_fp64     n = 100000, m = 800000, p1 = 0.46 (the bench formula, seed 1,
                          initial state seed 1001): the reference harness until it solves
                          (at most 1000 steps), SHA-256 of the FP64 state every 25 steps
  large.c2_balanced_fp64  n = 100000, m = 800000 with the fixtures' literal split p1 = 0.58
                          (seed 2, initial state seed 1002), which does not solve within
                          1000 steps: the reference harness for 1000 steps, hashes every 50
  large.c2_balanced_fp32  the same formula and state through the oracle's FP32 restatement
                          (the reference has no FP32 mode), hashes every 50 steps
  large.c4_fp64 / c4_fp32 n = 1000000, m = 8000000 (seed 3, initial state seed 1003): the
                          reference harness (FP64) and the oracle (FP32) for 8 steps, a hash
                          after every step
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import REF_CLI, Oracle, Reference, build, planted_instance, read_cnf  # noqa: E402

HASH_STEPS = [0, 1, 2, 3, 5, 10, 20, 50, 100, 150, 200]


def uniform_init(n, m, seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.uniform(-1, 1, n), rng.uniform(0, 1, m), np.ones(m)])


def state_hash(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<f8").tobytes()).hexdigest()


def run_cli(path: str, seed: int, timeout: float = 600.0, extra=()) -> dict:
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, os.path.basename(path))
        shutil.copy(path, p)
        out = subprocess.run([REF_CLI, "-i", p, "-l", str(seed), *extra], capture_output=True,
                             text=True, timeout=timeout, cwd=d).stdout
    text = re.sub(r"\x1b\[[0-9;]*m", "", out.replace("\r", "\n"))
    # The progress line of the solving right-hand side carries T and the step counter
    # (dynex.cc:609-636); it is printed before the reference's display thread starts
    # writing, so it is never interleaved.
    m = None
    steps = None
    for line in text.splitlines():
        mm = re.search(r"T=([0-9.]+) GLOBAL=.*\(LOC=0\) \((\d+)\)", line)
        if mm:
            m, steps = mm, int(mm.group(2))
            break
    v = []
    for line in text.splitlines():
        if line.startswith("v "):
            v += [int(t) for t in line[2:].split()]
    if v and v[-1] == 0:
        v = v[:-1]
    heur = [list(h.groups()) for h in re.finditer(
        r"alpha heuristic changed (\d+) up, (\d+) down, (\d+) max reached \(median = ([0-9.]+)\)",
        text)]
    return {"solved": m is not None, "T": float(m.group(1)) if m else None, "steps": steps,
            "v": v, "heuristics": [[int(a), int(b), int(c), d] for a, b, c, d in heur]}


HEURISTIC_FORMULA = {"n": 2000, "m": 8520, "p0": 0.0, "p1": 0.5, "seed": 16}


def heuristics_case() -> dict:
    """The reference CLI with -p 1 on HEURISTIC_FORMULA (made by this library's generator)."""
    sys.path.insert(0, os.path.join(ROOT, "dynex-neuromorphic-chip_b200"))
    import dmm_b200 as dmm
    from dmm_b200.cnf import write_cnf
    f = HEURISTIC_FORMULA
    form, _ = dmm.generate_planted(f["n"], f["m"], f["p0"], f["p1"], seed=f["seed"])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "heuristics.cnf")
        write_cnf(form, path)
        r = run_cli(path, 0, extra=("-p", "1"))
    out = {"formula": f, "solved": r["solved"], "T": r["T"], "steps": r["steps"],
           "heuristics": r["heuristics"],
           "v_sha256": hashlib.sha256(np.array(r["v"], dtype="<i4").tobytes()).hexdigest()}
    print("heuristics", out["steps"], out["T"], out["heuristics"], file=sys.stderr)
    return out


LARGE_CASES = {
    # name: (n, m, p0, p1, formula seed, initial-state seed, steps, hash every, engine)
    "c2_bench_fp64": (100_000, 800_000, 0.08, 0.46, 1, 1001, 1000, 25, "reference"),
    "c2_balanced_fp64": (100_000, 800_000, 0.08, 0.58, 2, 1002, 1000, 50, "reference"),
    "c2_balanced_fp32": (100_000, 800_000, 0.08, 0.58, 2, 1002, 1000, 50, "oracle_fp32"),
    "c4_fp64": (1_000_000, 8_000_000, 0.08, 0.46, 3, 1003, 8, 1, "reference"),
    "c4_fp32": (1_000_000, 8_000_000, 0.08, 0.46, 3, 1003, 8, 1, "oracle_fp32"),
}


def replicas_case(path: str, seed: int) -> dict:
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, os.path.basename(path))
        shutil.copy(path, p)
        out = subprocess.run([REF_CLI, "-i", p, "-l", str(seed), "-w", "3"], capture_output=True,
                             text=True, timeout=600, cwd=d).stdout
    text = re.sub(r"\x1b\[[0-9;]*m", "", out.replace("\r", "\n"))
    got = {}
    for line in text.splitlines():
        mm = re.search(r"c \[(\d+)\] [0-9.]+s T=([0-9.]+) GLOBAL=.*\(LOC=0\) \((\d+)\)", line)
        if mm:
            got.setdefault(mm.group(1), {"steps": int(mm.group(3)), "T": float(mm.group(2))})
    return got


def replicas_entries(ref_dir: str, answers: dict) -> None:
    answers["cli_replicas"] = {}
    for n in (200, 500):
        path = os.path.join(ref_dir, "cnf",
                            f"transformed_barthel_n_{n}_r_8.000_p0_0.080_instance_001.cnf")
        for seed in (0, 1):
            r = replicas_case(path, seed)
            answers["cli_replicas"][f"n{n}_seed{seed}"] = r
            print("replicas", n, seed, r, file=sys.stderr)


def tuner_case(path: str, seed: int, replicas: int) -> list:
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, os.path.basename(path))
        shutil.copy(path, p)
        out = subprocess.run([REF_CLI, "-i", p, "-l", str(seed), "-w", str(replicas), "-t", "1",
                              "-s", "1", "-u", "1"], capture_output=True, text=True, timeout=600,
                             cwd=d).stdout
    text = re.sub(r"\x1b\[[0-9;]*m", "", out.replace("\r", "\n"))
    mm = re.search(r"c \[TUNE\] E: ((?:\[[0-9.]+\])+)", text)
    return [float(v) for v in re.findall(r"\[([0-9.]+)\]", mm.group(1))]


def tuner_entries(ref_dir: str, answers: dict) -> None:
    answers["cli_tuner"] = {}
    for n, seed, reps in ((1000, 1, 3), (500, 2, 2)):
        path = os.path.join(ref_dir, "cnf",
                            f"transformed_barthel_n_{n}_r_8.000_p0_0.080_instance_001.cnf")
        e = tuner_case(path, seed, reps)
        answers["cli_tuner"][f"n{n}_seed{seed}_w{reps}"] = {"initial_objective": e}
        print("tuner", n, seed, reps, e, file=sys.stderr)


def large_case(name: str) -> dict:
    n, m, p0, p1, seed, init_seed, steps, every, engine = LARGE_CASES[name]
    lits, off, _, x0 = planted_instance(n, m, p0, p1, seed, init_seed)
    if engine == "reference":
        eng = Reference(n, m, lits, off)
    else:
        eng = Oracle(n, m, lits, off, precision="fp32")
    r = eng.run(x0, steps, dump_every=every)
    hashes = {str(k * every): state_hash(r["dump"][k]) for k in range(len(r["dump"]))
              if k * every <= r["steps"]}
    out = {"n": n, "m": m, "p0": p0, "p1": p1, "seed": seed, "init_seed": init_seed,
           "max_steps": steps, "engine": engine, "steps": r["steps"], "solved": r["solved"],
           "solve_step": r["solve_step"], "solve_t": r["solve_t"], "t": r["t"],
           "hashes": hashes,
           "pre_sha256": hashlib.sha256(r["pre"].astype("<i1").tobytes()).hexdigest()
           if r["solved"] else None,
           "post_sha256": hashlib.sha256(r["post"].astype("<i1").tobytes()).hexdigest()
           if r["solved"] else None,
           "loc": r["loc"][: min(len(r["loc"]), 64)].tolist()}
    print(name, out["steps"], out["solved"], out["solve_step"], file=sys.stderr)
    return out


def large_entries(ref_dir: str, answers: dict) -> None:
    path = os.path.join(ref_dir, "cnf",
                        "transformed_barthel_n_10000_r_8.000_p0_0.080_instance_001.cnf")
    n, m, lits, coff = read_cnf(path)
    np.savez_compressed(os.path.join(HERE, "fixture_n10000.npz"), lits=lits.astype(np.int16),
                        off=coff.astype(np.int32), planted=planted_of(path))
    answers.setdefault("large", {})
    import multiprocessing as mp

    # one process per case: the reference keeps its formula in process globals
    with mp.get_context("spawn").Pool(len(LARGE_CASES)) as pool:
        for name, out in zip(LARGE_CASES, pool.map(large_case, list(LARGE_CASES))):
            answers["large"][name] = out


def planted_of(path: str):
    with open(path) as f:
        first = f.readline()
    if first.startswith("c ["):
        return np.array([1 if int(t) > 0 else -1 for t in first[3:].split("]")[0].split()],
                        dtype=np.int8)
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-dir", default="/root/reference")
    ap.add_argument("--only", choices=["heuristics", "large", "replicas", "tuner"], default=None)
    a = ap.parse_args()
    build()
    if a.only is not None:
        path = os.path.join(HERE, "known_answers.json")
        with open(path) as f:
            answers = json.load(f)
        if a.only == "heuristics":
            answers["cli_heuristics"] = heuristics_case()
        elif a.only == "replicas":
            replicas_entries(a.ref_dir, answers)
        elif a.only == "tuner":
            tuner_entries(a.ref_dir, answers)
        else:
            large_entries(a.ref_dir, answers)
        with open(path, "w") as f:
            json.dump(answers, f, indent=1)
        return
    paths = sorted(glob.glob(os.path.join(a.ref_dir, "cnf", "*.cnf")),
                   key=lambda p: int(re.search(r"_n_(\d+)_", p).group(1)))
    arrays = {}
    answers = {"cli": {}, "harness": {}}
    for path in paths:
        n, m, lits, coff = read_cnf(path)
        name = f"n{n}"
        if n <= 1000:
            arrays[f"{name}_lits"] = lits.astype(np.int16)
            arrays[f"{name}_off"] = coff.astype(np.int32)
            pl = planted_of(path)
            if pl is not None:
                arrays[f"{name}_planted"] = pl
            for seed in (0, 1, 2):
                r = run_cli(path, seed)
                answers["cli"][f"{name}_seed{seed}"] = r
                print(name, seed, r["steps"], r["T"], file=sys.stderr)
            ref = Reference(n, m, lits, coff)
            x0 = uniform_init(n, m, 1234 + n)
            res = ref.run(x0, 200, dump_every=1)
            hashes = {str(s): state_hash(res["dump"][s]) for s in HASH_STEPS
                      if s < len(res["dump"]) and s <= res["steps"]}
            answers["harness"][f"{name}_uniform"] = {
                "init_seed": 1234 + n, "max_steps": 200, "steps": res["steps"],
                "solved": res["solved"], "solve_step": res["solve_step"],
                "solve_t": res["solve_t"], "hashes": hashes,
                "loc": res["loc"][: min(len(res["loc"]), 50)].tolist()}
        elif n == 10000:
            r = run_cli(path, 0)
            answers["cli"][f"{name}_seed0"] = {k: r[k] for k in ("solved", "T", "steps")}
            answers["cli"][f"{name}_seed0"]["v_sha256"] = hashlib.sha256(
                np.array(r["v"], dtype="<i4").tobytes()).hexdigest()
            print(name, 0, r["steps"], r["T"], file=sys.stderr)
    answers["cli_heuristics"] = heuristics_case()
    replicas_entries(a.ref_dir, answers)
    tuner_entries(a.ref_dir, answers)
    large_entries(a.ref_dir, answers)
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **arrays)
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(answers, f, indent=1)


if __name__ == "__main__":
    main()
