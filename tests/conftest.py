import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__ as entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def entry_oracle():
    return entry.load_oracle()


@pytest.fixture(scope="session")
def oracle():
    return entry.load_oracle()


@pytest.fixture(scope="session")
def pkg():
    return entry.load_package()


@pytest.fixture(scope="session")
def golden():
    d = np.load(os.path.join(ROOT, "tests", "golden", "lu_cases.npz"))
    cases = {}
    for name in d["names"]:
        name = str(name)
        key = f"{name}/A" if f"{name}/A" in d else f"{str(d[name + '/same_as'])}/A"
        cases[name] = dict(A=d[key], ipiv=d[f"{name}/ipiv"], bs=int(d[f"{name}/bs"]),
                           info=int(d[f"{name}/info"]), lu_fro=float(d[f"{name}/lu_fro"]),
                           lu=d[f"{name}/lu"] if f"{name}/lu" in d else None)
    return cases


def bwd(E, A):
    """Normwise backward error in units of eps (test/lapack/lapack_dense.jl:4)."""
    return np.linalg.norm(E) / (max(np.linalg.norm(A), np.finfo(float).tiny) * max(1, *A.shape)
                                * np.finfo(A.dtype).eps)


def split_lu(F, m, n):
    q = min(m, n)
    L = np.tril(F[:, :q], -1) + np.eye(m, q)
    U = np.triu(F[:q, :])
    return L, U
