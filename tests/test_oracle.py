"""The oracle (CPU restatement) pinned against the reference: the golden known answers of
the unmodified reference CLI and, where the reference harness is built, per-step states."""
import hashlib

import numpy as np
import pytest

from conftest import uniform_init
from oracle.oracle import DEFAULT_PARAMS, Oracle, Reference, reference_available

FIXTURES = ["n100", "n200", "n500", "n1000"]


def state_hash(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<f8").tobytes()).hexdigest()


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_reference_cli(fixtures, known_answers, name, seed):
    """Steps, T and the reported `v` assignment of `dynex -i fixture -l seed`."""
    f = fixtures[name]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    x0 = o.init_state(seed)
    ka = known_answers["cli"][f"{name}_seed{seed}"]
    r = o.run(x0, 2000)
    assert r["solved"]
    assert r["solve_step"] == ka["steps"]
    assert round(r["solve_t"], 2) == pytest.approx(ka["T"], abs=1e-9)
    v = [(i + 1) if a > 0 else -(i + 1) for i, a in enumerate(r["post"])]
    assert v == ka["v"]
    assert o.check(r["pre"]) == 0


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_reference_harness_hashes(fixtures, known_answers, name):
    """FP64 state after selected steps from a seeded uniform initial state (SHA-256 of the
    reference's own per-step states)."""
    f = fixtures[name]
    ka = known_answers["harness"][f"{name}_uniform"]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    x0 = uniform_init(f["n"], f["m"], ka["init_seed"])
    r = o.run(x0, ka["max_steps"], dump_every=1)
    assert r["steps"] == ka["steps"]
    assert r["solved"] == ka["solved"]
    assert r["solve_step"] == ka["solve_step"]
    assert r["solve_t"] == ka["solve_t"]
    for s, h in ka["hashes"].items():
        assert state_hash(r["dump"][int(s)]) == h, f"step {s}"
    assert r["loc"][: len(ka["loc"])].tolist() == ka["loc"]


def test_oracle_n10000_known_answer(known_answers):
    """The reference CLI's answer on its largest fixture (n = 10000, seed 0): step count, T
    and the reported assignment (SHA-256 of the `v` list)."""
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "fixture_n10000.npz"))
    lits, off = z["lits"].astype(np.int32), z["off"].astype(np.int64)
    o = Oracle(10000, len(off) - 1, lits, off)
    assert o.check(z["planted"]) == 0
    ka = known_answers["cli"]["n10000_seed0"]
    r = o.run(o.init_state(0), 400)
    assert r["solved"] and r["solve_step"] == ka["steps"]
    assert round(r["solve_t"], 2) == pytest.approx(ka["T"], abs=1e-9)
    v = np.array([(i + 1) if a > 0 else -(i + 1) for i, a in enumerate(r["post"])], dtype="<i4")
    assert hashlib.sha256(v.tobytes()).hexdigest() == ka["v_sha256"]


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("p1,seed,init_seed", [(0.46, 1, 1001), (0.58, 2, 1002), (0.5, 9, None)])
def test_harness_generator_equals_library_generator(p1, seed, init_seed):
    """The reference harness builds the bench formulas without the library
    (oracle/instance_gen.h); both must give the same arrays for the same arguments."""
    import dmm_b200 as dmm
    from oracle.oracle import planted_instance

    for n, m in ((100, 800), (5000, 21500), (100_000, 800_000)):
        lits, off, sigma, x0 = planted_instance(n, m, 0.08, p1, seed, init_seed)
        f, pl = dmm.generate_planted(n, m, 0.08, p1, seed=seed)
        assert np.array_equal(lits, f.lits) and np.array_equal(off, f.clause_off)
        assert np.array_equal(sigma, pl)
        if init_seed is not None:
            assert np.array_equal(x0, dmm.initial_state_uniform(f, init_seed))


@pytest.mark.parametrize("case", ["n200_seed0", "n200_seed1", "n500_seed0", "n500_seed1"])
def test_oracle_replicas_match_reference_cli(fixtures, known_answers, case):
    """Replica portfolio (-w 3): every replica the reference CLI saw solve, with its initial
    state and alpha / i (dynex.cc:2643-2700), solves at the same step and T in the oracle."""
    name, seed = case.split("_seed")
    f = fixtures[name]
    for rid, ka in known_answers["cli_replicas"][case].items():
        i = int(rid)
        o = Oracle(f["n"], f["m"], f["lits"], f["off"],
                   params=(2.5 / max(i, 1),) + DEFAULT_PARAMS[1:])
        r = o.run(o.init_state(int(seed), i), 2000)
        assert r["solved"] and r["solve_step"] == ka["steps"]
        assert round(r["solve_t"], 2) == pytest.approx(ka["T"], abs=1e-9)


@pytest.mark.parametrize("case", ["n1000_seed1_w3", "n500_seed2_w2"])
def test_oracle_tuner_initial_objective_matches_reference(fixtures, known_answers, case):
    """The reference tuner's initial objective (`-t 1`, one Euler step through odeint,
    dynex.cc:1711-1722) of every replica is the unsatisfied count of its initial state."""
    name, seed, reps = case.split("_")
    f = fixtures[name]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    want = known_answers["cli_tuner"][case]["initial_objective"]
    got = [float(o.rhs(o.init_state(int(seed[4:]), i))[1]) for i in range(int(reps[1:]))]
    assert got == want


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("name", ["n100", "n200"])
def test_oracle_bitexact_vs_reference_per_step(fixtures, name):
    f = fixtures[name]
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    ref = Reference(f["n"], f["m"], f["lits"], f["off"])
    for seed in (3, 4):
        x0 = uniform_init(f["n"], f["m"], seed)
        a = o.run(x0, 150, dump_every=1)
        b = ref.run(x0, 150, dump_every=1)
        assert np.array_equal(a["dump"], b["dump"])
        assert np.array_equal(a["loc"], b["loc"])
        assert np.array_equal(a["energy"], b["energy"])


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
def test_oracle_general_ksat_vs_reference():
    """Mixed clause sizes (unit, 2-, 3-, k-literal up to 25, repeated variables)."""
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
    ref = Reference(n, len(off) - 1, lits, off)
    x0 = o.init_state(5)
    a = o.run(x0, 120, dump_every=1)
    b = ref.run(x0, 120, dump_every=1)
    assert np.array_equal(a["dump"], b["dump"])
    d1, l1, e1 = o.rhs(a["dump"][7])
    d2, l2, e2 = ref.rhs(a["dump"][7])
    assert np.array_equal(d1, d2) and l1 == l2 and e1 == e2


def test_oracle_fp32_mode_tracks_fp64(fixtures):
    """FP32 production mode stays close to FP64 over a short horizon."""
    f = fixtures["n200"]
    o64 = Oracle(f["n"], f["m"], f["lits"], f["off"])
    o32 = Oracle(f["n"], f["m"], f["lits"], f["off"], precision="fp32")
    x0 = uniform_init(f["n"], f["m"], 11)
    a = o64.run(x0, 10, dump_every=1)
    b = o32.run(x0, 10, dump_every=1)
    n = f["n"]
    assert np.max(np.abs(a["dump"][10][:n] - b["dump"][10][:n])) < 1e-3


def test_oracle_planted_fixtures_verify(fixtures):
    for name in ("n200", "n500", "n1000"):
        f = fixtures[name]
        o = Oracle(f["n"], f["m"], f["lits"], f["off"])
        assert o.check(f["planted"]) == 0


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
def test_oracle_long_occurrence_list_vs_reference():
    """A variable in every one of 3000 clauses (its sorted sum runs over 3000 entries)."""
    rng = np.random.default_rng(11)
    n, m = 50, 3000
    rows = [np.concatenate([[1], rng.choice(np.arange(2, n + 1), size=2, replace=False)])
            * rng.choice([-1, 1], size=3) for _ in range(m)]
    lits = np.array(rows, np.int32).reshape(-1)
    off = np.arange(0, 3 * m + 1, 3, dtype=np.int64)
    o = Oracle(n, m, lits, off)
    ref = Reference(n, m, lits, off)
    x0 = o.init_state(3)
    a = o.run(x0, 40, dump_every=1)
    b = ref.run(x0, 40, dump_every=1)
    assert np.array_equal(a["dump"], b["dump"])
    assert np.array_equal(a["loc"], b["loc"])


def test_gpu_prior_art_harness_is_built():
    """The reference's GPU code (dynex.cu) compiled for sm_100a with its timing driver: the
    library loads and exports the driver's entry points (it runs only on a GPU)."""
    import ctypes
    import os

    from oracle.oracle import REF_GPU_SO

    if not os.path.exists(REF_GPU_SO):
        pytest.skip("reference sources absent and no prebuilt library")
    lib = ctypes.CDLL(REF_GPU_SO)
    for name in ("refgpu_setup", "refgpu_run", "refgpu_teardown"):
        assert hasattr(lib, name)
