"""GPU parity at the benchmarked sizes.

The small fixtures pin the arithmetic; these tests pin the kernels' tiling, grid split and
long per-variable lists, which only appear at the benchmarked sizes:

* n = 100,000, m = 800,000 (the bench formula): FP64 states equal the reference harness's
  (SHA-256, every 25 steps) until it solves, with the same solve step, T and assignments;
* n = 100,000 with the fixtures' literal split, which does not solve within 1000 steps:
  FP64 equal to the reference for 1000 steps and FP32 equal to the oracle's FP32
  restatement for 1000 steps (hashes every 50 steps) -- the required tolerance is 1e-12
  relative over the first 1000 steps, and the states are bit-identical;
* n = 1,000,000, m = 8,000,000: the first 8 steps of both precisions (a hash per step);
* the reference's n = 10000 fixture through the `dynex` command line: its known answer.

The hashes come from tests/golden/make_golden.py (the reference harness for FP64, the
oracle for FP32) on formulas and initial states of the library's seeded generator.
"""
import hashlib
import os
import re
import subprocess

import numpy as np
import pytest

import dmm_b200 as dmm
from dmm_b200 import _lib

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def state_hash(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<f8").tobytes()).hexdigest()


def sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


_forms = {}


def case_formula(ka):
    key = (ka["n"], ka["m"], ka["p0"], ka["p1"], ka["seed"], ka["init_seed"])
    if key not in _forms:
        _forms.clear()  # keep at most one large formula on the host
        f, _ = dmm.generate_planted(ka["n"], ka["m"], ka["p0"], ka["p1"], seed=ka["seed"])
        _forms[key] = (f, dmm.initial_state_uniform(f, ka["init_seed"]))
    return _forms[key]


def check_hashes(ka, precision, expect_form=None):
    f, x0 = case_formula(ka)
    marks = sorted(int(s) for s in ka["hashes"])
    with dmm.Instance(f, precision=precision) as inst:
        if expect_form is not None:
            assert inst.launch_form == expect_form
        inst.set_state(x0)
        done = 0
        for s in marks:
            if s > done:
                r = inst.step(s - done)
                done = s
                if s <= ka["steps"]:
                    assert r.steps == s, f"stopped at {r.steps} before step {s}"
            x, _ = inst.get_state()
            assert state_hash(x) == ka["hashes"][str(s)], f"{precision} state differs at step {s}"
        rep = inst.step(ka["max_steps"] - done) if done < ka["max_steps"] else inst.report()
        assert rep.steps == ka["steps"]
        assert rep.solved == ka["solved"]
        if ka["solved"]:
            assert rep.solved_step == ka["solve_step"]
            assert rep.solved_t == ka["solve_t"]
            pre, post = inst.assignment()
            assert sha(pre, "<i1") == ka["pre_sha256"]
            assert sha(post, "<i1") == ka["post_sha256"]
            assert dmm.check_assignment(f, pre) == 0
        else:
            assert rep.t == ka["t"]


def test_bench_formula_fp64_matches_reference_until_solved(known_answers):
    check_hashes(known_answers["large"]["c2_bench_fp64"], "fp64")


def test_balanced_formula_fp64_matches_reference_1000_steps(known_answers):
    ka = known_answers["large"]["c2_balanced_fp64"]
    assert not ka["solved"] and ka["steps"] == 1000
    check_hashes(ka, "fp64")


def test_balanced_formula_fp32_matches_oracle_1000_steps(known_answers):
    ka = known_answers["large"]["c2_balanced_fp32"]
    assert not ka["solved"] and ka["steps"] == 1000
    check_hashes(ka, "fp32", expect_form="staged")


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_million_variables_first_steps(known_answers, precision):
    check_hashes(known_answers["large"][f"c4_{precision}"], precision,
                 expect_form="staged-multi" if precision == "fp32" else None)


def test_cli_n10000_fixture_known_answer(tmp_path, known_answers):
    z = np.load(os.path.join(GOLDEN, "fixture_n10000.npz"))
    form = dmm.from_arrays(z["lits"].astype(np.int32), z["off"].astype(np.int64), 10000)
    assert dmm.check_assignment(form, z["planted"]) == 0
    path = str(tmp_path / "n10000.cnf")
    dmm.write_cnf(form, path)
    r = subprocess.run([_lib.CLI_PATH, "-i", path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    ka = known_answers["cli"]["n10000_seed0"]
    m = re.search(r"c \[0\] T=([0-9.]+) SOLUTION FOUND", out)
    assert m and float(m.group(1)) == pytest.approx(ka["T"], abs=1e-9)
    assert int(re.search(r"STEPS = (\d+)", out).group(1)) == ka["steps"]
    v = []
    for line in out.splitlines():
        if line.startswith("v "):
            v += [int(t) for t in line[2:].split()]
    assert v[-1] == 0
    assert sha(np.array(v[:-1]), "<i4") == ka["v_sha256"]
    assert "SAT (VERIFIED)" in out
