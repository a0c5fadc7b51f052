"""The drop-in command line: `dynex -i file.cnf` on the GPU reproduces the reference CLI's
known answers (step count, T, reported assignment) and its report and solution file."""
import os
import re
import subprocess

import numpy as np
import pytest

import dmm_b200 as dmm
from dmm_b200 import _lib

pytestmark = pytest.mark.gpu


def run_cli(args, timeout=300):
    r = subprocess.run([_lib.CLI_PATH] + args, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr
    return r.stdout


def formula_of(f):
    return dmm.from_arrays(f["lits"], f["off"], f["n"])


def parse(out):
    m = re.search(r"c \[(\d+)\] T=([0-9.]+) SOLUTION FOUND", out)
    steps = int(re.search(r"STEPS = (\d+)", out).group(1))
    v = []
    for line in out.splitlines():
        if line.startswith("v "):
            v += [int(t) for t in line[2:].split()]
    assert v and v[-1] == 0
    return {"T": float(m.group(2)) if m else None, "steps": steps, "v": v[:-1],
            "verified": "SAT (VERIFIED)" in out, "sat": "SATISFIABLE" in out}


@pytest.mark.parametrize("name,seed", [("n100", 0), ("n200", 1), ("n500", 2), ("n1000", 0)])
def test_cli_matches_reference_known_answers(tmp_path, fixtures, known_answers, name, seed):
    f = fixtures[name]
    path = str(tmp_path / f"{name}.cnf")
    dmm.write_cnf(dmm.from_arrays(f["lits"], f["off"], f["n"]), path)
    out = parse(run_cli(["-i", path, "-l", str(seed)]))
    ka = known_answers["cli"][f"{name}_seed{seed}"]
    assert out["sat"] and out["verified"]
    assert out["steps"] == ka["steps"]
    assert out["T"] == pytest.approx(ka["T"], abs=1e-9)
    assert out["v"] == ka["v"]
    # the solution file in the reference's format (dynex.cc:693-699)
    sol = open(path + ".solution.txt").read().split(",")
    lits = [int(t) for t in sol if t.strip()]
    assert len(lits) == f["n"]
    assign = np.array([1 if l > 0 else -1 for l in lits], np.int8)
    assert dmm.check_assignment(dmm.from_arrays(f["lits"], f["off"], f["n"]), assign) == 0


def test_cli_replicas_and_fp32(tmp_path, fixtures):
    f = fixtures["n500"]
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    path = str(tmp_path / "n500.cnf")
    dmm.write_cnf(form, path)
    for args in (["-w", "3", "-l", "0"], ["-P", "fp32", "-l", "4"], ["-w", "4", "-P", "fp32"]):
        out = parse(run_cli(["-i", path] + args))
        assert out["sat"] and out["verified"]
        assign = np.array([1 if l > 0 else -1 for l in out["v"]], np.int8)
        assert len(assign) == f["n"]


def test_cli_reports_unknown_at_step_cap(tmp_path, fixtures):
    f = fixtures["n1000"]
    path = str(tmp_path / "n1000.cnf")
    dmm.write_cnf(dmm.from_arrays(f["lits"], f["off"], f["n"]), path)
    out = run_cli(["-i", path, "-l", "1", "-z", "5"])
    assert "s [0] UNKNOWN" in out
    assert not os.path.exists(path + ".solution.txt")


def test_cli_rejects_long_clause(tmp_path):
    path = tmp_path / "long.cnf"
    path.write_text("p cnf 30 1\n" + " ".join(str(i) for i in range(1, 27)) + " 0\n")
    r = subprocess.run([_lib.CLI_PATH, "-i", str(path)], capture_output=True, text=True)
    assert r.returncode != 0
    assert "MORE THAN 25 LITERALS" in r.stdout


def test_cli_alpha_heuristic_matches_reference(tmp_path, known_answers):
    """-p 1: the reference's alpha heuristic every 10^4 steps.  On a formula that needs more
    than 10^4 steps, the printed heuristic counts and median, the step count, T and the
    assignment equal the reference CLI's (the heuristic moves the solve from step 12164 to
    13672 there)."""
    import hashlib
    ka = known_answers["cli_heuristics"]
    f = ka["formula"]
    form, _ = dmm.generate_planted(f["n"], f["m"], f["p0"], f["p1"], seed=f["seed"])
    path = str(tmp_path / "heuristics.cnf")
    dmm.write_cnf(form, path)
    text = run_cli(["-i", path, "-p", "1"], timeout=600)
    heur = [[int(a), int(b), int(c), d] for a, b, c, d in re.findall(
        r"alpha heuristic changed (\d+) up, (\d+) down, (\d+) max reached \(median = ([0-9.]+)\)",
        text)]
    assert heur == ka["heuristics"]
    out = parse(text)
    assert out["sat"] and out["verified"]
    assert out["steps"] == ka["steps"]
    assert out["T"] == pytest.approx(ka["T"], abs=1e-9)
    assert hashlib.sha256(np.array(out["v"], dtype="<i4").tobytes()).hexdigest() == ka["v_sha256"]


def test_cli_state_checkpoint_save_and_resume(tmp_path, fixtures):
    """-S 1 writes the final state and its t to <cnf>.assignment.txt; -L 1 resumes every
    replica from it at that t (the reference's load_assignment, dynex.cc:2521-2532, values
    read through a float).  The resumed CLI run equals the library resumed from the file."""
    f = fixtures["n1000"]
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    n, m = f["n"], f["m"]
    path = str(tmp_path / "n1000.cnf")
    dmm.write_cnf(form, path)
    out = run_cli(["-i", path, "-l", "1", "-z", "40", "-S", "1"])
    assert "s [0] UNKNOWN" in out
    t_cap = float(re.search(r"STEPS = 40 \(T = ([0-9.]+)\)", out).group(1))
    x_file, t_file = dmm.read_state(path + ".assignment.txt", n, m)
    assert t_file == pytest.approx(t_cap, abs=1e-5)
    # the library's own state after the same 40 steps, printed as the file holds it
    x0, _ = dmm.initial_state_reference(form, 1, 0)
    with dmm.Instance(form, precision="fp64") as inst:  # the CLI's default arithmetic
        inst.set_state(x0)
        inst.step(40)
        x_lib, t_lib = inst.get_state()
    assert np.array_equal(x_file, [float("%.15f" % v) for v in x_lib])
    assert t_file == float("%.15f" % t_lib)
    # resume: the CLI from the file against the library from the same (float-read) values
    out2 = run_cli(["-i", path, "-l", "1", "-z", "25", "-L", "1"])
    assert "LOADED, WILL START AT t=" in out2
    steps2 = int(re.search(r"STEPS = (\d+)", out2).group(1))
    t2 = float(re.search(r"STEPS = \d+ \(T = ([0-9.]+)\)", out2).group(1))
    xr, tr = dmm.read_state(path + ".assignment.txt", n, m, reference_rounding=True)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_state_at(xr, tr, 0)
        r = inst.solve(max_steps=25)
    assert steps2 == (r.solved_step if r.solved else r.steps)
    assert t2 == pytest.approx(r.solved_t if r.solved else r.t, abs=1e-5)
    assert t2 > tr


def _tune(path, *args):
    return run_cli(["-i", path, "-t", "1", "-q", "1"] + list(args))


def test_cli_tuner_is_deterministic_and_scores_with_the_batch(tmp_path, fixtures):
    """-t 1: the reference's simulated-annealing tuner with one Metropolis chain per replica.
    Its random draws come from one mt19937 seeded with -l, so a run repeats exactly; iteration
    0 runs every replica with its original parameters, so its scores are the lowest loc of
    each replica run alone to the step cap; the tuning file holds one line per new global."""
    f = fixtures["n1000"]
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    path = str(tmp_path / "n1000.cnf")
    dmm.write_cnf(form, path)
    args = ["-s", "4", "-z", "30", "-w", "3", "-l", "1"]
    out = _tune(path, *args)
    assert out == _tune(path, *args)
    assert out.count("c [TUNE] ITERATION") == 4 and "c [TUNE] FINISHED." in out
    decisions = re.findall(r"c \[TUNE\] \[(\d)\] (?:\d+ CANDIDATES ACCEPTED|CANDIDATE REJECTED) "
                           r"\(E=(\d+)", out)
    assert len(decisions) == 4 * 3
    # iteration 0 against the library: replica r from its reference state, alpha / r
    e0 = {int(r): int(e) for r, e in decisions[:3]}
    for r in range(3):
        x0, div = dmm.initial_state_reference(form, 1, r)
        p = dmm.default_params()
        p.alpha = p.alpha / div
        b = dmm.Batch.for_formulas([form], precision="fp64")
        try:
            b.add(form, x0, params=p, max_steps=30)
            b.run()
            res, _ = b.result(0)
        finally:
            b.close()
        assert e0[r] == res.best_loc
    assert float(out.strip().splitlines()[-1]) == min(int(e) for _, e in decisions)
    lines = open(path + ".tuning.txt").read().splitlines()
    assert lines[0].startswith("ITERATION;INSTANCE;PARAM_01") and len(lines) >= 2


def test_cli_tuner_stops_on_a_solution(tmp_path, fixtures):
    f = fixtures["n100"]
    path = str(tmp_path / "n100.cnf")
    dmm.write_cnf(dmm.from_arrays(f["lits"], f["off"], f["n"]), path)
    out = _tune(path, "-s", "50", "-z", "5000", "-w", "2", "-l", "0")
    assert "c [TUNE] SOLUTION FOUND." in out and out.rstrip().endswith("0")


def test_cli_alpha_heuristic_with_replicas(tmp_path, known_answers):
    """-p 1 -w 2: each replica runs the heuristic on its own state and clause alphas (floor:
    the replica's alpha).  Replica 0 runs first and unchanged, so its heuristic lines are the
    reference's one-replica lines; replica 1 runs at most to replica 0's solving step, and
    the reported solve is the earlier one."""
    ka = known_answers["cli_heuristics"]
    f = ka["formula"]
    form, _ = dmm.generate_planted(f["n"], f["m"], f["p0"], f["p1"], seed=f["seed"])
    path = str(tmp_path / "heuristics.cnf")
    dmm.write_cnf(form, path)
    text = run_cli(["-i", path, "-p", "1", "-w", "2"], timeout=600)
    lines = re.findall(r"c \[(\d)\] alpha heuristic changed (\d+) up, (\d+) down, (\d+) max "
                       r"reached \(median = ([0-9.]+)\)", text)
    r0 = [[int(a), int(b), int(c), d] for k, a, b, c, d in lines if k == "0"]
    assert r0 == ka["heuristics"]
    assert all(k in "01" for k, *_ in lines)
    out = parse(text)
    assert out["sat"] and out["verified"]
    winner = int(re.search(r"s \[(\d)\] SATISFIABLE", text).group(1))
    if winner == 0:
        assert out["steps"] == ka["steps"] and out["T"] == pytest.approx(ka["T"], abs=1e-9)
    else:
        assert out["steps"] < ka["steps"]


@pytest.mark.parametrize("case", ["n200_seed0", "n200_seed1", "n500_seed0", "n500_seed1"])
def test_replica_portfolio_matches_oracle_and_reference(tmp_path, fixtures, known_answers, case):
    """-w 3 (dynex.cc:2643-2700): three replicas, replica i from the reference's initial state
    for the seed with alpha / i, run together as one FP64 batch.  Every replica's trajectory
    equals the oracle's for that replica bit for bit (solve step, T, final state); every
    replica the reference CLI saw solve has the reference's step count and T; and the
    `dynex -w 3` report names the replica that solves in the fewest steps with its answer."""
    from oracle.oracle import DEFAULT_PARAMS, Oracle

    name, seed = case.split("_seed")
    seed = int(seed)
    f = fixtures[name]
    form = formula_of(f)
    b = dmm.Batch.for_formulas([form] * 3, precision="fp64")
    want = []
    try:
        for i in range(3):
            x0, div = dmm.initial_state_reference(form, seed, i)
            b.add(form, x0, params=_lib.default_params(alpha=2.5 / div), max_steps=2000)
            o = Oracle(f["n"], f["m"], f["lits"], f["off"], params=(2.5 / div,) + DEFAULT_PARAMS[1:])
            want.append(o.run(x0, 2000, dump_every=1))
        b.run()
        for i in range(3):
            got, _ = b.result(i)
            ref = want[i]
            assert got.solved == ref["solved"]
            assert got.solved_step == ref["solve_step"] and got.solved_t == ref["solve_t"]
            assert np.array_equal(b.state(i)[0], ref["dump"][ref["steps"]])
    finally:
        b.close()
    for rid, ka in known_answers["cli_replicas"][case].items():
        ref = want[int(rid)]
        assert ref["solve_step"] == ka["steps"]
        assert round(ref["solve_t"], 2) == pytest.approx(ka["T"], abs=1e-9)
    path = str(tmp_path / f"{name}.cnf")
    dmm.write_cnf(form, path)
    text = run_cli(["-i", path, "-l", str(seed), "-w", "3"])
    out = parse(text)
    best = min(range(3), key=lambda i: (want[i]["solve_step"], i))
    assert re.search(rf"c \[{best}\] T=[0-9.]+ SOLUTION FOUND", text)
    assert out["steps"] == want[best]["solve_step"]
    assert out["T"] == pytest.approx(round(want[best]["solve_t"], 2), abs=1e-9)


@pytest.mark.parametrize("case", ["n1000_seed1_w3", "n500_seed2_w2"])
def test_cli_tuner_initial_objective_matches_reference(tmp_path, fixtures, known_answers, case):
    """`dynex -t 1`: the tuner's initial objective of every replica (the `c [TUNE] E:` line)
    equals the reference tuner's, which takes one Euler step through odeint
    (dynex.cc:1711-1722); its later iterations run to a wall-clock limit in the reference,
    so only this objective is compared."""
    name, seed, reps = case.split("_")
    f = fixtures[name]
    path = str(tmp_path / f"{name}.cnf")
    dmm.write_cnf(formula_of(f), path)
    text = run_cli(["-i", path, "-l", seed[4:], "-w", reps[1:], "-t", "1", "-s", "1", "-z", "20"])
    m = re.search(r"c \[TUNE\] E: ((?:\[[0-9.]+\])+)", text)
    got = [float(v) for v in re.findall(r"\[([0-9.]+)\]", m.group(1))]
    assert got == known_answers["cli_tuner"][case]["initial_objective"]
