import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dynex-neuromorphic-chip_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_sessionstart(session):
    # Build the oracle and the library once (both are quick no-ops when up to date).
    from oracle.oracle import build as build_oracle

    import importlib.util

    build_oracle()
    spec = importlib.util.spec_from_file_location("dmm_pkg_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()


@pytest.fixture(scope="session")
def fixtures():
    """Reference CNF fixtures (cnf/*.cnf, n = 100 .. 1000) as arrays."""
    z = np.load(os.path.join(GOLDEN, "fixtures.npz"))
    out = {}
    for key in z.files:
        name, kind = key.split("_", 1)
        out.setdefault(name, {})[kind] = z[key]
    for name, d in out.items():
        d["n"] = int(name[1:])
        d["lits"] = d["lits"].astype(np.int32)
        d["off"] = d["off"].astype(np.int64)
        d["m"] = len(d["off"]) - 1
    return out


@pytest.fixture(scope="session")
def known_answers():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def uniform_init(n, m, seed):
    """The seeded uniform initial state used by the golden harness runs."""
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.uniform(-1, 1, n), rng.uniform(0, 1, m), np.ones(m)])
