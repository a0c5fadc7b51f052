"""GPU parity: the CUDA path through the C ABI against the oracle and the reference's
golden answers.  FP64 mode is compared bit for bit (the required tolerance is 1e-12
relative per step; the implementation reproduces the reference's arithmetic exactly).
FP32 mode is compared bit for bit against the oracle's FP32 restatement, and against FP64
within stated per-horizon bounds."""
import hashlib

import numpy as np
import pytest

import dmm_b200 as dmm
from conftest import uniform_init
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FIXTURES = ["n100", "n200", "n500", "n1000"]


def formula(f):
    return dmm.from_arrays(f["lits"], f["off"], f["n"])


def state_hash(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<f8").tobytes()).hexdigest()


def run_steps(inst, x0, nsteps):
    """States after each accepted step (row 0 = x0) until solved or nsteps."""
    inst.set_state(x0)
    rows = [inst.get_state()[0]]
    for _ in range(nsteps):
        r = inst.step(1)
        rows.append(inst.get_state()[0])
        if r.status != dmm.RUNNING:
            break
    return np.array(rows), inst.report()


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_fp64_solve_matches_reference_cli(fixtures, known_answers, name, seed):
    f = fixtures[name]
    form = formula(f)
    ka = known_answers["cli"][f"{name}_seed{seed}"]
    with dmm.Instance(form, precision="fp64") as inst:
        x0, _ = dmm.initial_state_reference(form, seed)
        inst.set_state(x0)
        r = inst.solve(max_steps=5000)
        assert r.solved
        assert r.solved_step == ka["steps"]
        assert round(r.solved_t, 2) == pytest.approx(ka["T"], abs=1e-9)
        pre, post = inst.assignment()
        assert dmm.check_assignment(form, pre) == 0
        v = [(i + 1) if a > 0 else -(i + 1) for i, a in enumerate(post)]
        assert v == ka["v"]


@pytest.mark.parametrize("name", FIXTURES)
def test_fp64_per_step_matches_reference_harness(fixtures, known_answers, name):
    """SHA-256 of the reference's own FP64 states at selected steps."""
    f = fixtures[name]
    ka = known_answers["harness"][f"{name}_uniform"]
    x0 = uniform_init(f["n"], f["m"], ka["init_seed"])
    with dmm.Instance(formula(f), precision="fp64") as inst:
        rows, rep = run_steps(inst, x0, ka["max_steps"])
    assert rep.steps == ka["steps"]
    assert rep.solved_step == ka["solve_step"]
    for s, h in ka["hashes"].items():
        assert state_hash(rows[int(s)]) == h, f"step {s}"


@pytest.mark.parametrize("name,seed", [("n100", 21), ("n200", 22), ("n500", 23), ("n1000", 24)])
def test_fp64_per_step_bitexact_vs_oracle_1000_steps(fixtures, name, seed):
    """Every state of the first 1000 steps (or until solved) equals the oracle's."""
    f = fixtures[name]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    x0 = uniform_init(f["n"], f["m"], seed)
    ref = o.run(x0, 1000, dump_every=1)
    with dmm.Instance(formula(f), precision="fp64") as inst:
        rows, rep = run_steps(inst, x0, 1000)
    assert rep.steps == ref["steps"]
    assert np.array_equal(rows, ref["dump"][: ref["steps"] + 1])
    if ref["solved"]:
        assert rep.solved_step == ref["solve_step"] and rep.solved_t == ref["solve_t"]
    assert rep.loc == ref["loc"][-1]
    assert rep.energy == pytest.approx(ref["energy"][-1], rel=1e-12, abs=1e-12)


def test_fp64_rhs_and_dostep_match_oracle(fixtures):
    """dmm_generate_dxdt / dmm_dostep mirrors, bit for bit."""
    f = fixtures["n500"]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    ref = o.run(uniform_init(f["n"], f["m"], 5), 30, dump_every=1)
    with dmm.Instance(formula(f), precision="fp64") as inst:
        for s in (0, 3, 17, 29):
            x = ref["dump"][s]
            d_gpu, loc_gpu, e_gpu = inst.generate_dxdt(x)
            d_cpu, loc_cpu, e_cpu = o.rhs(x)
            assert np.array_equal(d_gpu, d_cpu)
            assert loc_gpu == loc_cpu
            assert e_gpu == pytest.approx(e_cpu, rel=1e-12)
            for h in (0.125, 0.0625, 0.015625):
                assert np.array_equal(inst.dostep(x, d_cpu, h), o.dostep(x, d_cpu, h))


def test_fp64_general_ksat_bitexact():
    """Unit, 2-, 3- and long clauses (up to 25 literals), repeated variables."""
    rng = np.random.default_rng(7)
    n = 60
    lits, off = [], [0]
    for c in range(400):
        k = int(rng.choice([1, 2, 3, 3, 3, 4, 5, 7, 12, 25])) if c % 50 else 1
        vs = rng.integers(1, n + 1, size=k)
        sg = rng.choice([-1, 1], size=k)
        lits += list(vs * sg)
        off.append(len(lits))
    lits = np.array(lits, np.int32)
    off = np.array(off, np.int64)
    o = Oracle(n, len(off) - 1, lits, off)
    form = dmm.from_arrays(lits, off, n)
    x0, _ = dmm.initial_state_reference(form, 5)
    ref = o.run(x0, 300, dump_every=1)
    with dmm.Instance(form, precision="fp64") as inst:
        rows, rep = run_steps(inst, x0, 300)
        d_gpu, _, _ = inst.generate_dxdt(ref["dump"][9])
    assert np.array_equal(rows, ref["dump"][: ref["steps"] + 1])
    assert np.array_equal(d_gpu, o.rhs(ref["dump"][9])[0])


@pytest.mark.parametrize("name,seed", [("n200", 31), ("n1000", 32)])
def test_fp32_per_step_bitexact_vs_oracle_fp32(fixtures, name, seed):
    f = fixtures[name]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"], precision="fp32")
    x0 = uniform_init(f["n"], f["m"], seed)
    ref = o.run(x0, 400, dump_every=1)
    with dmm.Instance(formula(f), precision="fp32") as inst:
        assert inst.launch_form == "staged"
        rows, rep = run_steps(inst, x0, 400)
    assert rep.steps == ref["steps"]
    assert np.array_equal(rows, ref["dump"][: ref["steps"] + 1])


def test_fp32_launch_shape_does_not_change_results(fixtures):
    f = fixtures["n1000"]
    x0 = uniform_init(f["n"], f["m"], 41)
    outs = []
    shapes = [dict(var_group=g, steps_per_graph=s, clause_tile=ct, var_tile=vt, launch_mode=lm)
              for g, s, ct, vt, lm in [(1, 16, 1024, 256, 0), (2, 7, 2048, 512, 1),
                                       (4, 32, 0, 0, 0), (8, 64, 4096, 1024, 1),
                                       (16, 3, 256, 32, 0), (32, 256, 8192, 256, 1),
                                       (4, 5, 260, 96, 2), (8, 9, 0, 0, 3), (1, 40, 0, 0, 3)]]
    forms = set()
    for kw in shapes:
        with dmm.Instance(formula(f), precision="fp32") as inst:
            inst.set_tuning(**kw)
            forms.add(inst.launch_form)
            inst.set_state(x0)
            inst.step(150)
            outs.append((inst.get_state()[0], inst.report().steps))
    assert forms == {"staged", "cooperative-single", "two-kernel", "one-block-per-formula"}
    for x, s in outs[1:]:
        assert s == outs[0][1]
        assert np.array_equal(x, outs[0][0])


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_contribution_layout_does_not_change_results(fixtures, prec):
    """Slot-major (gathered through the CSR) and variable-major (scattered through the slot
    positions) storage of the per-literal contributions give identical states."""
    f = fixtures["n500"]
    x0 = uniform_init(f["n"], f["m"], 71)
    outs = []
    for lay, mode in ((0, 0), (1, 0), (2, 0), (1, 1), (2, 1), (2, 3), (1, 3)):
        if prec == "fp64" and mode == 3:
            continue
        with dmm.Instance(formula(f), precision=prec) as inst:
            inst.set_tuning(u_layout=lay, launch_mode=mode)
            if mode == 0:  # the staged kernel is the FP32 default layout's
                want = "staged" if prec == "fp32" and lay == 0 else "cooperative-single"
                assert inst.launch_form == want
            inst.set_state(x0)
            inst.step(120)
            d, loc, _ = inst.generate_dxdt(inst.get_state()[0])
            outs.append((inst.get_state()[0], d, loc))
    for x, d, loc in outs[1:]:
        assert np.array_equal(x, outs[0][0])
        assert np.array_equal(d, outs[0][1]) and loc == outs[0][2]


def test_fp32_error_vs_fp64_per_horizon(fixtures):
    """Max |dV| and |dXl| of FP32 against FP64 from the same state, at steps 10 and 100
    (chaotic dynamics: the bound loosens with the horizon)."""
    f = fixtures["n1000"]
    n, m = f["n"], f["m"]
    x0 = uniform_init(n, m, 51)
    states = {}
    for prec in ("fp32", "fp64"):
        with dmm.Instance(formula(f), precision=prec) as inst:
            inst.set_state(x0)
            inst.step(10)
            s10 = inst.get_state()[0]
            inst.step(90)
            states[prec] = (s10, inst.get_state()[0])
    dv10 = np.max(np.abs(states["fp32"][0][:n] - states["fp64"][0][:n]))
    dxl10 = np.max(np.abs(states["fp32"][0][n + m:] - states["fp64"][0][n + m:]))
    assert dv10 < 1e-4 and dxl10 < 1e-4


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_solution_is_verified(fixtures, prec):
    f = fixtures["n500"]
    form = formula(f)
    with dmm.Instance(form, precision=prec) as inst:
        inst.set_state(dmm.initial_state_uniform(form, 9))
        r = inst.solve(max_steps=20000)
        assert r.solved
        pre, post = inst.assignment()
        assert dmm.check_assignment(form, pre) == 0
        assert r.loc == 0


def test_step_limit_and_resume(fixtures):
    f = fixtures["n1000"]
    form = formula(f)
    with dmm.Instance(form, precision="fp32") as inst:
        inst.set_state(dmm.initial_state_uniform(form, 1))
        r = inst.solve(max_steps=5)
        assert r.status in (dmm.STEP_LIMIT, dmm.SOLVED) and r.steps <= 5
        inst.set_state(dmm.initial_state_uniform(form, 1))
        r1 = inst.step(3)
        r2 = inst.step(4)
        assert r1.steps == 3 and r2.steps == 7 and r2.status == dmm.RUNNING


def test_edge_formulas():
    # empty formula: loc = 0 at step 0 (reference: loc = m = 0, verification passes)
    form = dmm.from_arrays(np.zeros(0, np.int32), np.zeros(1, np.int64), 5)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_state(np.zeros(5))
        r = inst.solve(max_steps=10)
        assert r.solved and r.solved_step == 0 and r.steps == 1
    # unused variables and a repeated variable inside a clause
    lits = np.array([1, 1, -3, 3, 4, -1, -4, 3, 1], np.int32)
    off = np.array([0, 3, 6, 9], np.int64)
    form = dmm.from_arrays(lits, off, 8)
    o = Oracle(8, 3, lits, off)
    x0 = uniform_init(8, 3, 2)
    ref = o.run(x0, 50, dump_every=1)
    with dmm.Instance(form, precision="fp64") as inst:
        rows, _ = run_steps(inst, x0, 50)
    assert np.array_equal(rows, ref["dump"][: ref["steps"] + 1])


def test_lists_longer_than_the_device_sorter():
    """A variable in 3000 clauses: its occurrence list is longer than the device sorter takes
    (1024), so it is sorted on the host before the first step, for a lone instance and for
    two formulas added to one batch (both recorded before one commit).  FP64 states equal
    the oracle's bit for bit."""
    rng = np.random.default_rng(11)
    n, m = 50, 3000
    rows = []
    for c in range(m):
        vs = np.concatenate([[1], rng.choice(np.arange(2, n + 1), size=2, replace=False)])
        rows.append(vs * rng.choice([-1, 1], size=3))
    lits = np.array(rows, np.int32).reshape(-1)
    off = np.arange(0, 3 * m + 1, 3, dtype=np.int64)
    form = dmm.from_arrays(lits, off, n)
    assert form.max_occurrence == m
    o = Oracle(n, m, lits, off)
    x0, _ = dmm.initial_state_reference(form, 3)
    ref = o.run(x0, 40, dump_every=1)
    with dmm.Instance(form, precision="fp64") as inst:
        got, _ = run_steps(inst, x0, 40)
    assert np.array_equal(got, ref["dump"][: ref["steps"] + 1])
    b = dmm.Batch(3, 3 * n, 3 * m, 9 * m, precision="fp64")
    try:
        b.add(form, x0, max_steps=40)
        b.add(form, x0, max_steps=40)
        b.run()
        for k in range(2):
            res, _ = b.result(k)
            assert res.steps == ref["steps"]
            assert np.array_equal(b.state(k)[0], ref["dump"][ref["steps"]])
    finally:
        b.close()


def test_fp64_many_variable_tiles_per_block():
    """FP64 with 32-variable tiles at n = 6,000 (188 tiles, more than one per block, the
    sorted sums' group counter restarting for each): bit-exact against the oracle."""
    form, _ = dmm.generate_planted(6_000, 25_200, 0.08, 0.46, seed=12)
    o = Oracle(form.n, form.m, form.lits, form.clause_off)
    x0 = uniform_init(form.n, form.m, 4)
    ref = o.run(x0, 30, dump_every=10)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_tuning(var_tile=32, clause_tile=256)
        inst.set_state(x0)
        for r in range(1, 4):
            inst.step(10)
            assert np.array_equal(inst.get_state()[0], ref["dump"][r])


def skewed_formula(n, m, a, seed):
    """3-SAT with variable i drawn with weight (i+1)^-a: occurrence lists from a few entries
    to hundreds, so one step takes every path of the FP64 sorted sum."""
    rng = np.random.default_rng(seed)
    w = 1.0 / np.arange(1, n + 1) ** a
    w /= w.sum()
    rows = np.empty((m, 3), np.int64)
    for c in range(m):
        rows[c] = rng.choice(np.arange(1, n + 1), size=3, replace=False, p=w)
    lits = (rows * rng.choice([-1, 1], size=(m, 3))).astype(np.int32).reshape(-1)
    return lits, np.arange(0, 3 * m + 1, 3, dtype=np.int64)


@pytest.mark.parametrize("tuning", [{}, {"var_tile": 64, "clause_tile": 512}])
def test_fp64_sorted_sum_every_list_length(tuning):
    """FP64 sums by list length: at most 32 entries (one thread), 33-64 (queued, an 8-lane
    segment), 65-256 (warp-wide network) and longer (warp-wide selection), on one formula
    whose lists span all four; per-step states equal the oracle's bit for bit."""
    n, m = 400, 8000
    lits, off = skewed_formula(n, m, 0.9, 5)
    form = dmm.from_arrays(lits, off, n)
    occ = np.bincount(np.abs(lits), minlength=n + 1)[1:]
    assert occ.max() > 256 and ((occ > 64) & (occ <= 256)).any()
    assert ((occ > 32) & (occ <= 64)).any() and (occ <= 32).any()
    o = Oracle(n, m, lits, off)
    x0 = uniform_init(n, m, 6)
    ref = o.run(x0, 25, dump_every=1)
    with dmm.Instance(form, precision="fp64") as inst:
        if tuning:
            inst.set_tuning(**tuning)
        got, _ = run_steps(inst, x0, 25)
    assert np.array_equal(got, ref["dump"][: ref["steps"] + 1])


def test_fp64_long_list_queue_overflow():
    """A variable tile with more lists longer than 32 than the block's queue holds (512):
    the ones past its end are summed in the first pass.  Bit-exact against the oracle."""
    form, _ = dmm.generate_planted(6_000, 84_000, 0.08, 0.46, seed=21)  # mean list 42
    occ = np.bincount(np.abs(form.lits), minlength=form.n + 1)[1:]
    assert (occ[:4096] > 32).sum() > 600
    o = Oracle(form.n, form.m, form.lits, form.clause_off)
    x0 = uniform_init(form.n, form.m, 8)
    ref = o.run(x0, 12, dump_every=4)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_tuning(var_tile=4096)
        inst.set_state(x0)
        for r in range(1, 4):
            inst.step(4)
            assert np.array_equal(inst.get_state()[0], ref["dump"][r])
