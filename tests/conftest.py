"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    return load


def load_golden_system(tag):
    """(wfn, basis, density, golden npz) of a committed small fixture."""
    from fastesp_b200 import Basis, read_molden
    wfn = read_molden(GOLDEN / f"{tag}.molden")
    basis = Basis(wfn)
    return wfn, basis, basis.density_matrix_cartesian(), np.load(GOLDEN / f"{tag}.npz")


@pytest.fixture(scope="session")
def small_system():
    return load_golden_system("small")


@pytest.fixture(scope="session")
def tz6_system():
    return load_golden_system("tz6")


@pytest.fixture(scope="session")
def frag54():
    """The 54-atom l<=3 synthetic system (molecule seed 0): wfn, basis, density."""
    from fastesp_b200 import synth
    wfn, basis, P, _ = synth.load_workload("frag54", 10, seed=0)
    return wfn, basis, P
