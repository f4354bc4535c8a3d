"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
TESTS = ROOT / "tests"
GOLDEN = TESTS / "golden"
for p in (str(ROOT), str(TESTS)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Native libraries of the package and the oracle port, built in-tree."""
    from spatialjoincountovershells_b200 import build as b
    out = b.build()
    from oracle import oracle
    oracle.lib()
    return out


@pytest.fixture(scope="session")
def manifest():
    return json.loads((GOLDEN / "manifest.json").read_text())


def golden_counts(name: str):
    z = np.load(GOLDEN / f"{name}.npz")
    return z["ids"], z["counts"], z["totals"]


@pytest.fixture(scope="session")
def case_dirs(tmp_path_factory, built):
    """Materialised inputs of every golden case (generated once per session)."""
    from golden import cases
    base = tmp_path_factory.mktemp("golden_inputs")
    out = {}
    for name in cases.CASES:
        d = base / name
        out[name] = (d, cases.materialize(name, d))
    return out


@pytest.fixture(scope="session")
def ctx(built):
    from spatialjoincountovershells_b200 import Context
    c = Context(0)
    yield c
    c.close()
