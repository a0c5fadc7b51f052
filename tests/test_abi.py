"""The C ABI library without a GPU: it loads, exports every entry point of include/dmm.h,
and its host-side functions (DIMACS, generator, checker, initial states) are correct."""
import ctypes
import os
import re

import numpy as np
import pytest

import dmm_b200 as dmm
from dmm_b200 import _lib
from conftest import ROOT
from oracle.oracle import Oracle


def header_functions():
    text = open(os.path.join(ROOT, "include", "dmm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dmm_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the ctypes binding covers the whole header
    assert sorted(_lib.SIGNATURES) == names


def test_abi_version_and_strings():
    L = _lib.lib()
    assert L.dmm_abi_version() == 1
    assert L.dmm_status_string(0) == b"ok"
    p = dmm.default_params()
    assert (p.alpha, p.beta, p.gamma, p.delta, p.epsilon, p.zeta, p.xl_max) == (
        2.5, 20.0, 0.25, 0.05, 0.1, 0.1, 10000)


def test_struct_sizes():
    assert ctypes.sizeof(_lib.Params) == 56
    assert ctypes.sizeof(_lib.Report) == 56
    assert ctypes.sizeof(_lib.Tuning) == 32
    assert ctypes.sizeof(_lib.Cnf) == 40


@pytest.mark.skipif(_lib.lib().dmm_device_count() > 0, reason="a GPU is present")
def test_no_device_is_an_error_not_a_fallback(fixtures):
    f = fixtures["n100"]
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    with pytest.raises(dmm.DmmError) as e:
        dmm.Instance(form)
    assert e.value.name == "DMM_ERR_NO_DEVICE"


def test_read_fixture_roundtrip(tmp_path, fixtures):
    f = fixtures["n200"]
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    p = str(tmp_path / "x.cnf")
    dmm.write_cnf(form, p, planted=f["planted"])
    g = dmm.read_cnf(p)
    assert g.n == f["n"] and g.m == f["m"]
    assert np.array_equal(g.lits, f["lits"]) and np.array_equal(g.clause_off, f["off"])
    assert g.max_occurrence == np.bincount(np.abs(f["lits"])).max()
    assert dmm.check_assignment(g, f["planted"]) == 0


def test_dimacs_parser_edge_cases(tmp_path):
    p = tmp_path / "a.cnf"
    p.write_text("c comment line\nc key=101\np cnf 4 3\n1 -2 0\nc inline comment 5 6\n3 0\n"
                 "-4 2 1 3 0\n")
    g = dmm.read_cnf(str(p))
    assert (g.n, g.m) == (4, 3)
    assert g.lits.tolist() == [1, -2, 3, -4, 2, 1, 3]
    assert g.clause_off.tolist() == [0, 2, 3, 7]
    # clause longer than 25 literals (dynex.cc:2388-2391)
    p.write_text("p cnf 30 1\n" + " ".join(str(i) for i in range(1, 27)) + " 0\n")
    with pytest.raises(dmm.DmmError) as e:
        dmm.read_cnf(str(p))
    assert e.value.name == "DMM_ERR_CLAUSE_LEN"
    p.write_text("p cnf 3 1\n1 5 0\n")
    with pytest.raises(dmm.DmmError) as e:
        dmm.read_cnf(str(p))
    assert e.value.name == "DMM_ERR_LITERAL"
    p.write_text("p cnf 3 2\n1 2 0\n")
    with pytest.raises(dmm.DmmError) as e:
        dmm.read_cnf(str(p))
    assert e.value.name == "DMM_ERR_PARSE"
    with pytest.raises(dmm.DmmError) as e:
        dmm.read_cnf(str(tmp_path / "missing.cnf"))
    assert e.value.name == "DMM_ERR_IO"


def test_planted_generator_statistics():
    f, planted = dmm.generate_planted(2000, 16000, p0=0.08, p1=0.46, seed=3)
    assert f.m == 16000 and f.nlits == 48000
    assert dmm.check_assignment(f, planted) == 0
    lits = f.lits.reshape(-1, 3)
    v = np.abs(lits) - 1
    assert np.all(v[:, 0] != v[:, 1]) and np.all(v[:, 1] != v[:, 2]) and np.all(v[:, 0] != v[:, 2])
    agree = (np.sign(lits) == planted[v]).sum(axis=1)
    frac = np.bincount(agree, minlength=4)[1:] / f.m
    assert abs(frac[0] - 0.46) < 0.02 and abs(frac[1] - 0.46) < 0.02 and abs(frac[2] - 0.08) < 0.01
    g, p2 = dmm.generate_planted(2000, 16000, p0=0.08, p1=0.46, seed=3)
    assert np.array_equal(f.lits, g.lits) and np.array_equal(planted, p2)


def test_initial_states(fixtures):
    f = fixtures["n100"]
    form = dmm.from_arrays(f["lits"], f["off"], f["n"])
    o = Oracle(f["n"], f["m"], f["lits"], f["off"])
    for seed in (0, 1, 2, 7, -1, -2):
        for rep in (0, 1, 3):
            x, div = dmm.initial_state_reference(form, seed, rep)
            assert np.array_equal(x, o.init_state(seed, rep))
            assert div == (rep if rep > 0 else 1)
    x = dmm.initial_state_uniform(form, 5)
    n, m = f["n"], f["m"]
    assert np.all(np.abs(x[:n]) <= 1) and np.all((x[n:n + m] >= 0) & (x[n:n + m] < 1))
    assert np.all(x[n + m:] == 1)
    assert np.array_equal(x, dmm.initial_state_uniform(form, 5))


def test_checker_counts_strict_signs():
    form = dmm.from_arrays([1, -2, 2, 3, -1], [0, 2, 4, 5], 3)
    assert dmm.check_assignment(form, [1, 1, 1]) == 1      # clause 3 (-1) fails
    assert dmm.check_assignment(form, [0, 0, 0]) == 3      # V == 0 satisfies nothing
    assert dmm.check_assignment(form, [-1, -1, 1]) == 0


def test_formula_validation():
    with pytest.raises(dmm.DmmError):
        dmm.from_arrays([1, 0, 2], [0, 3], 2)
    with pytest.raises(dmm.DmmError):
        dmm.from_arrays([1, 2], [0, 2], 0)


def test_state_checkpoint_file_format(tmp_path):
    """`<cnf>.assignment.txt` as the reference writes it (dynex.cc:2131-2135) and reads it
    (dynex.cc:2521-2532, each value through a float)."""
    n, m = 5, 3
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-1, 1, n), rng.uniform(0, 1, m), rng.uniform(1, 900, m)])
    x[0], x[1] = -0.0, 1.0
    t = 1234.56789012345678
    path = str(tmp_path / "f.cnf.assignment.txt")
    dmm.write_state(path, x, n, m, t)
    want = "".join("%.15f, " % v for v in x) + "%.15f " % t
    assert open(path).read() == want
    xd, td = dmm.read_state(path, n, m)
    assert np.array_equal(xd, [float("%.15f" % v) for v in x]) and td == float("%.15f" % t)
    xf, tf = dmm.read_state(path, n, m, reference_rounding=True)
    assert np.array_equal(xf, np.float32(["%.15f" % v for v in x]).astype(np.float64))
    assert tf == float(np.float32("%.15f" % t))
    # separators as the reference's fscanf("%f, ") accepts them; trailing text is ignored
    loose = tmp_path / "loose.txt"
    loose.write_text("\n".join("%.6f ," % v for v in x) + "\n%.3f trailing" % t)
    xl, tl = dmm.read_state(str(loose), n, m)
    assert np.array_equal(xl, [float("%.6f" % v) for v in x]) and tl == float("%.3f" % t)
    short = tmp_path / "short.txt"
    short.write_text("".join("%.15f, " % v for v in x[:-1]))
    with pytest.raises(dmm.DmmError) as e:
        dmm.read_state(str(short), n, m)
    assert e.value.name == "DMM_ERR_PARSE"
    with pytest.raises(dmm.DmmError) as e:
        dmm.read_state(str(tmp_path / "missing.txt"), n, m)
    assert e.value.name == "DMM_ERR_IO"


def test_validation_of_large_formulas_split_over_threads():
    """The host checks of large formulas run on several threads; an error anywhere, in the
    last chunk too, is still found and named."""
    f, _ = dmm.generate_planted(200_000, 800_000, 0.08, 0.46, seed=9)
    assert dmm.from_arrays(f.lits, f.clause_off, f.n).m == f.m
    for pos in (5, len(f.lits) // 2 + 1, len(f.lits) - 1):
        bad = f.lits.copy()
        bad[pos] = f.n + 1
        with pytest.raises(dmm.DmmError) as e:
            dmm.from_arrays(bad, f.clause_off, f.n)
        assert e.value.name == "DMM_ERR_LITERAL"
        assert f"literal {f.n + 1} at position {pos}" in str(e.value)
    off = f.clause_off.copy()
    off[-2] = off[-3] - 1  # offsets decrease near the end
    with pytest.raises(dmm.DmmError) as e:
        dmm.from_arrays(f.lits, off, f.n)
    assert e.value.name == "DMM_ERR_ARG"
