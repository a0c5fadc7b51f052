"""Failure path of the cooperative step kernels: a grid-barrier wait that never completes
ends after its bounded wait, the library reports DMM_ERR_CUDA, and the device context and
the instance stay usable.  The failure is made on the host (the test hook asks the first
barrier for one arrival more than the grid has); nothing faults or hangs."""
import numpy as np
import pytest

import dmm_b200 as dmm
from dmm_b200._lib import check, lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,layout,form_want", [("fp32", 0, "staged"),
                                                    ("fp32", 1, "cooperative-single"),
                                                    ("fp64", 0, "cooperative-single")])
def test_barrier_wait_gives_up_and_instance_recovers(prec, layout, form_want):
    form, _ = dmm.generate_planted(3_000, 12_600, 0.08, 0.46, seed=31)
    x0 = dmm.initial_state_uniform(form, 32)
    with dmm.Instance(form, precision=prec) as ref:
        ref.set_tuning(u_layout=layout)
        ref.set_state(x0)
        want = ref.step(10)
        want_x = ref.get_state()[0]
    with dmm.Instance(form, precision=prec) as inst:
        inst.set_tuning(u_layout=layout)
        assert inst.launch_form == form_want
        inst.set_state(x0)
        with pytest.raises(dmm.DmmError) as e:
            check(lib().dmm_instance_test_barrier_timeout(inst._h))
        assert e.value.name == "DMM_ERR_CUDA"
        assert "gave up" in str(e.value)
        # the error is reported once; the same instance then integrates normally
        inst.set_state(x0)
        got = inst.step(10)
        assert (got.status, got.steps, got.t, got.loc) == (want.status, want.steps, want.t,
                                                           want.loc)
        assert np.array_equal(inst.get_state()[0], want_x)
