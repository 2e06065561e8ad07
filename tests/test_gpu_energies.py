"""GPU: solver energies for every spin multiplicity of one system against
the dense CSF-basis Hamiltonian, with and without davidson_only (the
structure of the reference's test_csf.py:60-114: brute-force H from
contract_2e on unit vectors, transformed to CSFs)."""
import numpy as np
import pytest

import gasref
import restate as R
from conftest import seeded_integrals

pytestmark = pytest.mark.gpu


def _dense_csf_energies(h1, eri, norb, nelec, smult, k):
    h2e = R.absorb_h1e(h1, eri, norb, nelec, 0.5)
    na, nb = R.num_strings(norb, nelec[0]), R.num_strings(norb, nelec[1])
    H = np.empty((na * nb, na * nb))
    for i in range(na * nb):
        e = np.zeros(na * nb)
        e[i] = 1.0
        H[:, i] = gasref.contract_2e(h2e, e.reshape(na, nb), norb, nelec).ravel()
    ncsf = R.count_all_csfs(norb, nelec[0], nelec[1], smult)
    U = R.transform_det2csf(np.eye(ncsf), norb, nelec[0], nelec[1], smult, reverse=True)
    return np.linalg.eigvalsh(U @ H @ U.T)[:k]


@pytest.mark.parametrize("nelec,smults", [((3, 3), (1, 3, 5, 7)), ((4, 3), (2, 4, 6))])
@pytest.mark.parametrize("davidson_only", [False, True])
def test_energies_every_multiplicity(nelec, smults, davidson_only):
    if not gasref.available():
        pytest.skip("reference library not built")
    import pyscf_forge_b200 as P
    norb = 6
    h1, eri = seeded_integrals(norb, 12, seed=21)
    for smult in smults:
        sol = P.csf_solver(None, smult=smult)
        sol.davidson_only = davidson_only
        sol.conv_tol = 1e-12
        sol.max_cycle = 300
        nroots = min(2, R.count_all_csfs(norb, nelec[0], nelec[1], smult))
        sol.nroots = nroots
        e, ci = sol.kernel(h1, eri, norb, nelec)
        ref = _dense_csf_energies(h1, eri, norb, nelec, smult, nroots)
        np.testing.assert_allclose(np.atleast_1d(e), ref, atol=1e-9)     # energy tolerance 1e-9 Eh
        cs = ci if isinstance(ci, list) else [ci]
        for c in cs:
            ss, mult = sol.spin_square(c, norb, nelec)
            assert abs(mult - smult) < 1e-6
