"""The allocation-free right-hand side, dmm_rhs3_f32_noalloc.

Some callers cannot allocate device memory themselves (a host framework whose allocator
owns the GPU, a plug-in limited to the buffers it is handed, work issued while a stream is
being captured).  They call an entry point whose intermediates live in a fixed __device__
array.  This test owns its device buffers (torch tensors), calls that entry point through
the C ABI twice in a row, and checks each output against the allocating entry point
dmm_instance_rhs on an FP32 instance: the tolerance is bit-exact, as for every FP32
comparison against the same arithmetic in these tests.  It lives in its own file, collected
last, and works alone in a fresh process or after the other tests.
"""
import ctypes

import numpy as np
import pytest

import dmm_b200 as dmm
from conftest import uniform_init
from dmm_b200 import _lib

pytestmark = pytest.mark.gpu


def _noalloc(lits_d, n, m, x_d, dxdt_d, loc_d):
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    st = _lib.lib().dmm_rhs3_f32_noalloc(
        ctypes.c_void_p(lits_d.data_ptr()), int(n), int(m), ctypes.c_void_p(x_d.data_ptr()), None,
        ctypes.c_void_p(dxdt_d.data_ptr()), ctypes.c_void_p(loc_d.data_ptr()),
        ctypes.c_void_p(stream))
    _lib.check(st)
    torch.cuda.synchronize()


def _reference(f, x):
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    with dmm.Instance(form, precision="fp32") as inst:
        dxdt, loc, _ = inst.generate_dxdt(x)
    return dxdt, loc


def test_noalloc_rhs_equals_instance_rhs_on_consecutive_calls(fixtures):
    import torch

    # larger formula first, then a smaller one: the shared scratch keeps the last call's
    # contents, and each call must clear what it accumulates
    for name, seed in (("n1000", 61), ("n100", 62), ("n1000", 63)):
        f = fixtures[name]
        n, m = f["n"], f["m"]
        # a state that is exact in FP32, so both entry points see the same input
        x = uniform_init(n, m, seed).astype(np.float32).astype(np.float64)
        ref, ref_loc = _reference(f, x)
        lits_d = torch.from_numpy(f["lits"]).to("cuda")
        x_d = torch.from_numpy(x.astype(np.float32)).to("cuda")
        outs = []
        for _ in range(2):
            dxdt_d = torch.full((n + 2 * m,), float("nan"), dtype=torch.float32, device="cuda")
            loc_d = torch.full((1,), -1, dtype=torch.int32, device="cuda")
            _noalloc(lits_d, n, m, x_d, dxdt_d, loc_d)
            out = dxdt_d.cpu().numpy().astype(np.float64)
            assert np.array_equal(out, ref), name
            assert int(loc_d.item()) == ref_loc
            outs.append(out)
        assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_formulas_beyond_its_scratch():
    import torch

    lits_d = torch.ones(3, dtype=torch.int32, device="cuda")
    x_d = torch.zeros(8, dtype=torch.float32, device="cuda")
    out_d = torch.zeros(8, dtype=torch.float32, device="cuda")
    loc_d = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(dmm.DmmError) as e:
        _noalloc(lits_d, 1 << 15, (1 << 16) + 1, x_d, out_d, loc_d)
    assert e.value.name == "DMM_ERR_ARG"
    with pytest.raises(dmm.DmmError) as e:
        _noalloc(lits_d, (1 << 15) + 1, 1, x_d, out_d, loc_d)
    assert e.value.name == "DMM_ERR_ARG"
