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


def large_density(n, seed):
    """Seeded symmetric density-like matrix of the large-molecule fixtures
    (tests/golden/make_large.py): diagonal 0.3, off-diagonal N(0, 0.05^2)
    damped by exp(-|i-j|/20), symmetrised.  numpy's PCG64 stream is the same
    on every machine, so the fixtures store the seed, not the matrix."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) * 0.05
    idx = np.arange(n)
    A *= np.exp(-np.abs(idx[:, None] - idx[None, :]) / 20.0)
    return 0.5 * (A + A.T) + np.eye(n) * 0.3


def unpack_upper(v, n):
    """Symmetric n x n matrix from its row-major upper triangle."""
    F = np.zeros((n, n))
    iu = np.triu_indices(n)
    F[iu] = v
    F.T[iu] = v
    return F


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
