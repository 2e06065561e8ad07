import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


SMALL_CASES = ["c0_norb8_4e4e_s0", "norb6_3e3e_s1", "norb5_3e2e_s12", "norb6_4e2e_s1",
               "norb4_2e2e_s2", "norb4_4e4e_s0", "norb5_1e0e_s12", "norb7_4e3e_s32"]


@pytest.fixture(params=SMALL_CASES)
def golden_case(request):
    g = load_golden(request.param)
    g["name"] = request.param
    return g


def seeded_integrals(norb, rank, seed=0):
    """The synthetic integrals of the benchmark configurations (seeded h1
    symmetric N(0,0.3) off-diagonal, diagonal linspace(-2,0.5); eri = 1/2
    sum_x L_x (x) L_x with L (rank, norb^2) ~ N(0,0.2) symmetrised)."""
    rng = np.random.default_rng(seed)
    h1 = rng.normal(0.0, 0.3, (norb, norb))
    h1 = 0.5 * (h1 + h1.T)
    np.fill_diagonal(h1, np.linspace(-2.0, 0.5, norb))
    L = rng.normal(0.0, 0.2, (rank, norb * norb)).reshape(rank, norb, norb)
    L = 0.5 * (L + L.transpose(0, 2, 1))
    eri = 0.5 * np.einsum("xpq,xrs->pqrs", L, L)
    return h1, eri
