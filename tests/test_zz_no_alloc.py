"""The allocation-free right-hand side, dmm_rhs3_f32_noalloc.

Some callers cannot allocate device memory themselves (a host framework whose caching
allocator owns the GPU, a plug-in limited to the buffers it is handed).  They call an entry
point whose intermediates live in a fixed __device__ array.  This test owns its device
buffers (torch tensors), calls that entry point through the C ABI twice in a row, and checks
each output against the allocating entry point dmm_instance_rhs on an FP32 instance and
against the oracle's FP32 right-hand side: the tolerance is bit-exact, as for every FP32
comparison against the same arithmetic in these tests.  It also checks that a call rejected
part-way (a bad literal, an over-long variable list) leaves the shared array fit for the
next call.  It lives in its own file, collected last, and works alone in a fresh process or
after the other tests.
"""
import ctypes

import numpy as np
import pytest

import dmm_b200 as dmm
from conftest import uniform_init
from dmm_b200 import _lib
from oracle.oracle import Oracle

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
    o = Oracle(f["n"], f["m"], f["lits"], f["off"], precision="fp32")
    odxdt, oloc, _ = o.rhs(x)
    assert np.array_equal(dxdt, odxdt) and loc == oloc
    return dxdt, loc


def _run_valid(f, seed):
    """One valid call on fixture f, twice; both outputs must equal the references."""
    import torch

    n, m = f["n"], f["m"]
    # a state that is exact in FP32, so every path sees the same input
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
        assert np.array_equal(out, ref)
        assert int(loc_d.item()) == ref_loc
        outs.append(out)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rhs_equals_instance_rhs_on_consecutive_calls(fixtures):
    # larger formula first, then a smaller one: the shared scratch keeps the last call's
    # contents, and each call must clear what it accumulates
    for name, seed in (("n1000", 61), ("n100", 62), ("n1000", 63)):
        _run_valid(fixtures[name], seed)


def test_noalloc_rejected_calls_leave_the_scratch_usable(fixtures):
    import torch

    n, m = 100, 1025
    # variable 1 in all 1025 clauses: one list longer than the 1024 slots the call sorts
    rng = np.random.default_rng(5)
    lits = np.empty(3 * m, dtype=np.int32)
    for c in range(m):
        a, b = rng.choice(np.arange(2, n + 1), size=2, replace=False)
        lits[3 * c:3 * c + 3] = (1, -int(a), int(b))
    x_d = torch.zeros(n + 2 * m, dtype=torch.float32, device="cuda")
    out_d = torch.zeros(n + 2 * m, dtype=torch.float32, device="cuda")
    loc_d = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(dmm.DmmError) as e:
        _noalloc(torch.from_numpy(lits).to("cuda"), n, m, x_d, out_d, loc_d)
    assert e.value.name == "DMM_ERR_ARG"
    _run_valid(fixtures["n100"], 71)
    # a zero literal and one beyond n: rejected before any indexing by them
    for bad in (0, n + 1, -(n + 1)):
        lb = lits.copy()
        lb[7] = bad
        with pytest.raises(dmm.DmmError) as e:
            _noalloc(torch.from_numpy(lb).to("cuda"), n, m, x_d, out_d, loc_d)
        assert e.value.name == "DMM_ERR_LITERAL"
        _run_valid(fixtures["n1000"], 72)


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
