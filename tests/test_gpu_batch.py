"""Batched and served paths: every instance's result is identical alone and in the mix;
plus full-size (n = 100,000, m = 800,000) checks of the production FP32 path."""
import numpy as np
import pytest

import dmm_b200 as dmm
from conftest import uniform_init
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def formula(f):
    return dmm.from_arrays(f["lits"], f["off"], f["n"])


def alone(form, x0, prec, max_steps):
    with dmm.Instance(form, precision=prec) as inst:
        inst.set_state(x0)
        r = inst.solve(max_steps=max_steps)
        _, post = inst.assignment(pre=False)
        return r, post, inst.get_state()[0]


def mix(fixtures):
    items = []
    for i, name in enumerate(["n100", "n200", "n500", "n1000", "n200", "n100", "n1000", "n500"]):
        f = fixtures[name]
        form = formula(f)
        items.append((form, uniform_init(f["n"], f["m"], 100 + i)))
    return items


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("mode", [0, 3])
def test_batch_results_equal_alone(fixtures, prec, mode):
    if prec == "fp64" and mode == 3:
        pytest.skip("one block per formula is the FP32 production path")
    items = mix(fixtures)
    b = dmm.Batch.for_formulas([f for f, _ in items], precision=prec)
    b.set_tuning(launch_mode=mode)
    for form, x0 in items:
        b.add(form, x0, max_steps=300)
    stats = b.run()
    assert stats["solved"] + stats["unsolved"] == len(items)
    for k, (form, x0) in enumerate(items):
        r_b, post_b = b.result(k)
        x_b, _ = b.state(k)
        r_a, post_a, x_a = alone(form, x0, prec, 300)
        assert (r_b.status, r_b.steps, r_b.solved_step, r_b.t, r_b.loc) == (
            r_a.status, r_a.steps, r_a.solved_step, r_a.t, r_a.loc)
        assert np.array_equal(post_b, post_a)
        assert np.array_equal(x_b, x_a)


def test_batch_tuning_does_not_change_results(fixtures):
    items = mix(fixtures)
    finals = []
    for kw in (dict(var_group=1, steps_per_graph=8, launch_mode=0),
               dict(var_group=32, steps_per_graph=64, clause_tile=2048, var_tile=512,
                    launch_mode=1),
               dict(var_group=4, steps_per_graph=5, clause_tile=256, var_tile=32,
                    launch_mode=2),
               dict(var_group=8, steps_per_graph=7, launch_mode=3),
               dict(var_group=2, steps_per_graph=300, launch_mode=3)):
        b = dmm.Batch.for_formulas([f for f, _ in items], precision="fp32")
        b.set_tuning(**kw)
        for form, x0 in items:
            b.add(form, x0, max_steps=120)
        b.run()
        finals.append([b.state(k)[0] for k in range(len(items))])
    for other in finals[1:]:
        for a, c in zip(finals[0], other):
            assert np.array_equal(a, c)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_server_results_equal_alone(fixtures, prec):
    """Requests arriving while others run; a formula may run alone for a while (the
    single-formula form) and with others (the multi-formula form): every result equals
    the formula's run alone."""
    items = mix(fixtures) + mix(fixtures)[:4]
    srv = dmm.Server(budget_bytes=8 << 20, max_slots=5, steps_per_launch=16, precision=prec)
    tickets = {}
    pending = list(enumerate(items))
    done = {}
    rounds = 0
    while pending or len(done) < len(items):
        # arrivals interleaved with work on the device
        for _ in range(2):
            if pending:
                k, (form, x0) = pending.pop(0)
                tickets[srv.submit(form, x0=x0, max_steps=250)] = k
        srv.pump()
        for res in srv.take():
            done[tickets[res["ticket"]]] = res
        rounds += 1
        assert rounds < 10000
    for k, (form, x0) in enumerate(items):
        r_a, post_a, _ = alone(form, x0, prec, 250)
        r_s = done[k]["result"]
        assert (r_s.status, r_s.steps, r_s.solved_step, r_s.t) == (
            r_a.status, r_a.steps, r_a.solved_step, r_a.t)
        assert np.array_equal(done[k]["assignment"], post_a)
        assert done[k]["finish_s"] >= done[k]["admit_s"] >= done[k]["submit_s"]


def test_server_budget_beyond_free_memory_is_refused():
    """The server reserves its budget when it is created, so a budget larger than the
    device's free memory is refused up front with DMM_ERR_BUDGET (nothing is allocated)."""
    import torch

    free, total = torch.cuda.mem_get_info()
    with pytest.raises(dmm.DmmError) as e:
        dmm.Server(int(total) + (1 << 30), max_slots=4, precision="fp32")
    assert e.value.name == "DMM_ERR_BUDGET"


def test_server_budget_admission(fixtures):
    f = fixtures["n1000"]
    form = formula(f)
    srv = dmm.Server(budget_bytes=1 << 18, max_slots=4, steps_per_launch=8)
    with pytest.raises(dmm.DmmError) as e:
        srv.submit(form, seed=1)
    assert e.value.name == "DMM_ERR_BUDGET"
    small = formula(fixtures["n100"])
    tickets = [srv.submit(small, seed=s, max_steps=40) for s in range(6)]
    resident, queued = srv.pump()
    assert resident + queued <= 6 and resident <= 4
    got = []
    for _ in range(200):
        srv.pump()
        got += srv.take()
        if len(got) == len(tickets):
            break
    assert sorted(r["ticket"] for r in got) == sorted(tickets)


@pytest.fixture(scope="module")
def big():
    form, planted = dmm.generate_planted(100_000, 800_000, p0=0.08, p1=0.46, seed=2024)
    return form, planted


def test_full_size_fp32_bitexact_vs_oracle_first_steps(big):
    """n = 100,000, m = 800,000: the first 12 steps equal the oracle's FP32 restatement."""
    form, _ = big
    x0 = dmm.initial_state_uniform(form, 77)
    o = Oracle(form.n, form.m, form.lits, form.clause_off, precision="fp32")
    ref = o.run(x0, 12, dump_every=4)
    with dmm.Instance(form, precision="fp32") as inst:
        assert inst.launch_form == "staged"  # the production kernel at this size
        inst.set_state(x0)
        for r in range(1, 4):
            inst.step(4)
            assert np.array_equal(inst.get_state()[0], ref["dump"][r])


def test_full_size_fp64_bitexact_vs_oracle_first_steps(big):
    """n = 100,000, m = 800,000 in the reference's FP64 arithmetic (sorted per-variable sums,
    warps taking variable groups dynamically): the first 6 steps equal the oracle's."""
    form, _ = big
    x0 = dmm.initial_state_uniform(form, 79)
    o = Oracle(form.n, form.m, form.lits, form.clause_off, precision="fp64")
    ref = o.run(x0, 6, dump_every=3)
    with dmm.Instance(form, precision="fp64") as inst:
        assert inst.launch_form == "cooperative-single"
        inst.set_state(x0)
        for r in range(1, 3):
            inst.step(3)
            assert np.array_equal(inst.get_state()[0], ref["dump"][r])


def test_full_size_fp32_properties(big):
    """Determinism, state bounds and the unsatisfied count against a host recount."""
    form, planted = big
    n, m = form.n, form.m
    x0 = dmm.initial_state_uniform(form, 78)
    finals = []
    for _ in range(2):
        with dmm.Instance(form, precision="fp32") as inst:
            inst.set_state(x0)
            rep = inst.step(60)
            finals.append((inst.get_state()[0], rep))
    (x, rep), (x2, rep2) = finals
    assert np.array_equal(x, x2) and rep.t == rep2.t and rep.loc == rep2.loc
    assert np.all(np.abs(x[:n]) <= 1)
    assert np.all((x[n:n + m] >= 0) & (x[n:n + m] <= 1)) and np.all(x[n + m:] >= 1)
    # loc of the right-hand side at the final state, recounted on the host in FP32
    with dmm.Instance(form, precision="fp32") as inst:
        _, loc, _ = inst.generate_dxdt(x)
    v = np.clip(x[:n].astype(np.float32), -1, 1)
    lits = form.lits.reshape(-1, 3)
    q = np.sign(lits).astype(np.float32)
    a = (np.float32(1) - q * v[np.abs(lits) - 1]).min(axis=1) * np.float32(0.5)
    assert loc == int((a >= 0.5).sum())
    assert dmm.check_assignment(form, planted) == 0


def test_many_small_formulas_auto_mode_equal_alone(fixtures):
    """More small formulas than SMs: the automatic launch runs one block per formula; every
    formula's result equals its run alone."""
    f = fixtures["n100"]
    form = formula(f)
    count = 300
    x0s = [uniform_init(f["n"], f["m"], 500 + k) for k in range(count)]
    b = dmm.Batch(count, count * f["n"], count * f["m"], count * 3 * f["m"], precision="fp32")
    for x0 in x0s:
        b.add(form, x0, max_steps=400)
    stats = b.run()
    assert stats["solved"] + stats["unsolved"] == count
    for k in (0, 1, 77, 150, 299):
        r_b, post_b = b.result(k)
        r_a, post_a, x_a = alone(form, x0s[k], "fp32", 400)
        assert (r_b.status, r_b.steps, r_b.solved_step, r_b.t, r_b.loc) == (
            r_a.status, r_a.steps, r_a.solved_step, r_a.t, r_a.loc)
        assert np.array_equal(b.state(k)[0], x_a)
        assert np.array_equal(post_b, post_a)


@pytest.mark.parametrize("n,m,form_want", [(200_000, 840_000, "staged"),
                                           (300_000, 1_260_000, "staged-multi"),
                                           (300_007, 2_400_013, "staged-multi"),
                                           (1_000_003, 8_000_009, "staged-multi")])
def test_staged_kernel_limits(n, m, form_want):
    """The staged kernel runs one clause tile and one variable tile per block while those
    fit (16-bit indices, shared memory) and several of each per block beyond that (ragged
    last tiles in the odd sizes; more than one bitmap range of variables when building the
    tables above 262,144 variables).  Either way the states equal the plain kernel's bit for
    bit."""
    form, _ = dmm.generate_planted(n, m, p0=0.08, p1=0.46, seed=n)
    x0 = dmm.initial_state_uniform(form, 5)
    outs = []
    for lay in (0, 1):
        with dmm.Instance(form, precision="fp32") as inst:
            inst.set_tuning(u_layout=lay)
            assert inst.launch_form == (form_want if lay == 0 else "cooperative-single")
            inst.set_state(x0)
            rep = inst.step(10)
            outs.append((inst.get_state()[0], rep.t, rep.loc, rep.energy))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1:] == outs[1][1:]


def test_batch_resume_from_checkpoint_equals_instance(tmp_path, fixtures):
    """A state checkpoint written after 40 steps and read back resumes a batch member exactly
    as it resumes a lone instance (FP64: same steps, time, best loc and final state)."""
    f = fixtures["n500"]
    form = formula(f)
    x0, _ = dmm.initial_state_reference(form, 2, 0)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_state(x0)
        inst.step(40)
        x, t = inst.get_state()
    path = str(tmp_path / "n500.cnf.assignment.txt")
    dmm.write_state(path, x, form.n, form.m, t)
    xr, tr = dmm.read_state(path, form.n, form.m)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_state_at(xr, tr, 0)
        want = inst.solve(max_steps=60)
        want_x = inst.get_state()[0]
    b = dmm.Batch.for_formulas([form], precision="fp64")
    try:
        b.add(form, x0, max_steps=60)
        b.set_state_at(0, xr, tr, 0)
        b.run()
        got, _ = b.result(0)
        got_x = b.state(0)[0]
    finally:
        b.close()
    assert (got.status, got.steps, got.t, got.best_loc) == (want.status, want.steps, want.t,
                                                             want.best_loc)
    assert np.array_equal(got_x, want_x)


@pytest.mark.parametrize("m", [976_211, 976_797])
def test_staged_clause_rounds_with_ragged_tiles(m):
    """The staged kernel's clause rounds: 4-clause groups per thread, then a remainder of at
    most 2 x 1024 clauses as pairs (m = 976,211: the last tile has an odd remainder, one
    clause alone) or, above that, as groups again (m = 976,797: 6,600-clause tiles and a last
    tile of 6,597, whose remainder ends with one clause alone).  First 4 steps bit-exact
    against the oracle's FP32 restatement."""
    n = m // 8
    form, _ = dmm.generate_planted(n, m, p0=0.08, p1=0.46, seed=m)
    x0 = dmm.initial_state_uniform(form, 5)
    o = Oracle(form.n, form.m, form.lits, form.clause_off, precision="fp32")
    ref = o.run(x0, 4, dump_every=2)
    with dmm.Instance(form, precision="fp32") as inst:
        assert inst.launch_form == "staged"
        inst.set_state(x0)
        for r in range(1, 3):
            inst.step(2)
            assert np.array_equal(inst.get_state()[0], ref["dump"][r])


def test_cooperative_batch_with_formulas_finishing_at_different_steps():
    """Many formulas on the cooperative multi-formula kernel, solving at different steps: the
    tiles of formulas that already finished are skipped while the others keep stepping
    (the pattern that once let a block's warps fall out of step).  Every formula's result
    and final state equal its run alone."""
    forms = [dmm.generate_planted(10_000, 80_000, 0.08, 0.46, seed=500 + k)[0] for k in range(48)]
    x0s = [dmm.initial_state_uniform(f, 900 + k) for k, f in enumerate(forms)]
    b = dmm.Batch.for_formulas(forms, precision="fp32")
    try:
        b.set_tuning(launch_mode=2)
        for f, x0 in zip(forms, x0s):
            b.add(f, x0, max_steps=400)
        b.run()
        steps = set()
        for k, (f, x0) in enumerate(zip(forms, x0s)):
            got, post_b = b.result(k)
            want, post_a, x_a = alone(f, x0, "fp32", 400)
            assert (got.status, got.steps, got.solved_step, got.t, got.loc) == (
                want.status, want.steps, want.solved_step, want.t, want.loc), k
            assert np.array_equal(b.state(k)[0], x_a), k
            assert np.array_equal(post_b, post_a), k
            steps.add(got.steps)
        assert len(steps) > 10  # the formulas finish at many different steps
    finally:
        b.close()


def test_fp64_energy_same_alone_and_in_a_batch_with_the_same_tiles(fixtures):
    """FP64 energies are sums of per-tile partials: with the same clause and variable tiles,
    a formula alone (single-formula cooperative form) and in a batch of two (multi-formula
    form) report the same energy, bit for bit, and the same state."""
    f, g = fixtures["n500"], fixtures["n1000"]
    form, other = formula(f), formula(g)
    x0, x1 = uniform_init(f["n"], f["m"], 41), uniform_init(g["n"], g["m"], 42)
    tiles = dict(clause_tile=512, var_tile=64)
    with dmm.Instance(form, precision="fp64") as inst:
        inst.set_tuning(**tiles)
        assert inst.launch_form == "cooperative-single"
        inst.set_state(x0)
        r_a = inst.step(30)
        x_a = inst.get_state()[0]
    b = dmm.Batch.for_formulas([form, other], precision="fp64")
    try:
        b.set_tuning(**tiles)
        b.add(form, x0, max_steps=30)
        b.add(other, x1, max_steps=30)
        b.run()
        r_b, _ = b.result(0)
        assert (r_b.steps, r_b.t, r_b.loc) == (r_a.steps, r_a.t, r_a.loc)
        assert r_b.energy == r_a.energy
        assert np.array_equal(b.state(0)[0], x_a)
    finally:
        b.close()


def test_one_block_per_formula_with_contributions_in_global_memory():
    """One block per formula (launch mode 3) for formulas whose contributions do not fit in
    the block's shared memory (more than 32,256 literal slots: in global memory) and for ones
    that do, mixed in one batch: every formula's state and report equal its run alone."""
    sizes = [(5000, 40000), (8000, 20000), (1000, 8000), (4000, 10753), (4096, 10752)]
    forms = [dmm.generate_planted(n, m, 0.08, 0.46, seed=60 + k)[0] for k, (n, m) in enumerate(sizes)]
    x0s = [dmm.initial_state_uniform(f, 70 + k) for k, f in enumerate(forms)]
    b = dmm.Batch.for_formulas(forms, precision="fp32")
    try:
        b.set_tuning(launch_mode=3)
        for f, x0 in zip(forms, x0s):
            b.add(f, x0, max_steps=150)
        b.run()
        for k, (f, x0) in enumerate(zip(forms, x0s)):
            r_b, post_b = b.result(k)
            r_a, post_a, x_a = alone(f, x0, "fp32", 150)
            assert (r_b.status, r_b.steps, r_b.solved_step, r_b.t, r_b.loc) == (
                r_a.status, r_a.steps, r_a.solved_step, r_a.t, r_a.loc)
            assert np.array_equal(b.state(k)[0], x_a)
            assert np.array_equal(post_b, post_a)
    finally:
        b.close()
