"""Shared fixtures: the gpu marker, fixture loading and temp .xyz files."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def golden_cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def golden_xyz(case, tmpdir):
    """Write the fixture's geometry to an .xyz file; returns (gbs path, xyz path)."""
    from gtfock_b200 import molecules as mol
    g = load_golden(case) if isinstance(case, str) else case
    atoms = [(str(s),) + tuple(float(v) for v in x) for s, x in zip(g["atoms_sym"], g["atoms_xyz"])]
    name = case if isinstance(case, str) else "mol"
    xyz = mol.write_xyz(atoms, os.path.join(str(tmpdir), name + ".xyz"), name)
    return mol.basis_file(str(g["basis"])), xyz


@pytest.fixture
def tmpxyz(tmp_path):
    return tmp_path
