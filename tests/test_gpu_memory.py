"""Instances take their device buffers from a process-wide cache (a destroyed instance's
buffers are reused by the next one).  A reused buffer holds the previous owner's data, so
these tests check that results never depend on where an instance's memory came from."""
import numpy as np
import pytest

import dmm_b200 as dmm
from dmm_b200._lib import lib

pytestmark = pytest.mark.gpu


def run(form, x0, prec, steps):
    with dmm.Instance(form, precision=prec) as inst:
        inst.set_state(x0)
        r = inst.step(steps)
        x, t = inst.get_state()
        _, post = inst.assignment(pre=False)
        return (r.status, r.steps, r.t, r.loc, r.energy), x, post


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_results_do_not_depend_on_reused_memory(prec):
    form, _ = dmm.generate_planted(20_000, 80_000, 0.08, 0.46, seed=7)
    other, _ = dmm.generate_planted(20_000, 84_000, 0.08, 0.46, seed=8)
    x0 = dmm.initial_state_uniform(form, 11)
    x_other = dmm.initial_state_uniform(other, 12)
    lib().dmm_release_cached_memory()
    fresh = run(form, x0, prec, 40)  # buffers straight from the driver
    for _ in range(2):  # fill the cache with another formula's data, then reuse it
        run(other, x_other, prec, 40)
        again = run(form, x0, prec, 40)
        assert again[0] == fresh[0]
        assert np.array_equal(again[1], fresh[1])
        assert np.array_equal(again[2], fresh[2])


def test_release_between_instances():
    form, _ = dmm.generate_planted(5_000, 21_000, 0.08, 0.46, seed=3)
    x0 = dmm.initial_state_uniform(form, 4)
    a = run(form, x0, "fp32", 25)
    lib().dmm_release_cached_memory()
    b = run(form, x0, "fp32", 25)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])


def test_instance_rejects_bad_formulas():
    """Creation rejects bad literals and clause lengths with DMM_ERR_LITERAL, _CLAUSE_LEN and
    _ARG, and the library keeps working after the rejections."""
    def make(lits, off, n):
        return dmm.Formula(n, len(off) - 1, np.asarray(lits, np.int32),
                           np.asarray(off, np.int64), 1)
    big, _ = dmm.generate_planted(100_000, 420_000, 0.08, 0.46, seed=5)
    big_lits = big.lits.copy()
    big_lits[1_000_001] = -100_001  # one bad literal deep inside a large formula
    cases = [(make([1, -2, 5], [0, 3], 3), "DMM_ERR_LITERAL"),
             (make([1, 0, 2], [0, 3], 3), "DMM_ERR_LITERAL"),
             (make([7, 1, 2, 3], [0, 1, 4], 3), "DMM_ERR_LITERAL"),  # in a unit clause
             (dmm.Formula(big.n, big.m, big_lits, big.clause_off, big.max_occurrence),
              "DMM_ERR_LITERAL"),
             (make(list(range(1, 27)), [0, 26], 30), "DMM_ERR_CLAUSE_LEN"),
             (make([1, 2, 3], [0, 3, 2], 3), "DMM_ERR_ARG")]
    for form, name in cases:
        for prec in ("fp32", "fp64"):
            with pytest.raises(dmm.DmmError) as e:
                dmm.Instance(form, precision=prec)
            assert e.value.name == name
            if form.n == big.n:  # the literal checked on the device is named as on the host
                assert "literal -100001 at position 1000001" in str(e.value)
    ok, _ = dmm.generate_planted(1_000, 4_200, 0.08, 0.46, seed=5)
    with dmm.Instance(ok, precision="fp32") as inst:
        inst.set_state(dmm.initial_state_uniform(ok, 6))
        assert inst.step(3).steps == 3
