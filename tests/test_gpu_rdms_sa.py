"""GPU: spin-resolved RDMs against the reference's make_rdm12s (GAS library
in oracle/_ref) and the state-averaged solver wrapper."""
import numpy as np
import pytest

import gasref
from conftest import load_golden, SMALL_CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", SMALL_CASES)
def test_rdm12s_against_reference(tag):
    """make_rdm12s and trans_rdm12s within 1e-12 of fci_rdm_gas_plan_make_rdm12s."""
    if not gasref.available():
        pytest.skip("reference library not built")
    from pyscf_forge_b200.fci import direct_spin1 as D
    g = load_golden(tag)
    norb, nelec = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"]))
    rng = np.random.default_rng(3)
    ket = g["ci_rand"]
    bra = rng.normal(size=ket.size)
    (r1a, r1b), (r2aa, r2ab, r2bb) = gasref.make_rdm12s(ket, ket, norb, nelec)
    (d1a, d1b), (d2aa, d2ab, d2bb) = D.make_rdm12s(ket, norb, nelec)
    for x, y in ((d1a, r1a), (d1b, r1b), (d2aa, r2aa), (d2ab, r2ab), (d2bb, r2bb)):
        np.testing.assert_allclose(x, y, atol=1e-12)
    (t1a, t1b), (t2aa, t2ab, t2bb) = gasref.make_rdm12s(bra, ket, norb, nelec)
    (e1a, e1b), (e2aa, e2ab, e2bb) = D.trans_rdm12s(bra, ket, norb, nelec)
    for x, y in ((e1a, t1a), (e1b, t1b), (e2aa, t2aa), (e2ab, t2ab), (e2bb, t2bb)):
        np.testing.assert_allclose(x, y, atol=1e-12)
    a, b = D.make_rdm1s(ket, norb, nelec)
    np.testing.assert_allclose(a, r1a, atol=1e-12)
    np.testing.assert_allclose(b, r1b, atol=1e-12)


def test_state_average_wrapper():
    """2-root triplet: weighted energy and root energies against the
    reference solver's, averaged RDMs against the weighted reference
    make_rdm12/make_rdm12s of the solved vectors, weighted <S^2> = 2."""
    import pyscf_forge_b200 as P
    from pyscf_forge_b200.state_average import state_average
    g = load_golden("norb6_3e3e_s1")
    norb, nelec = 6, (3, 3)
    w = np.array([0.7, 0.3])
    sol = P.csf_solver(None, smult=3)
    sol.conv_tol = 1e-12
    sa = state_average(sol, w)
    e, ci = sa.kernel(g["h1"], g["eri"], norb, nelec)
    np.testing.assert_allclose(sa.e_states, g["energies"], atol=1e-9)
    assert abs(e - float(np.dot(w, g["energies"]))) < 1e-9
    d1, d2 = sa.make_rdm12(ci, norb, nelec)
    r1 = sum(wk * gasref.make_rdm12(c, c, norb, nelec)[0] for wk, c in zip(w, ci))
    r2 = sum(wk * gasref.make_rdm12(c, c, norb, nelec)[1] for wk, c in zip(w, ci))
    np.testing.assert_allclose(d1, r1, atol=1e-10)
    np.testing.assert_allclose(d2, r2, atol=1e-10)
    (a, b), (aa, ab, bb) = sa.make_rdm12s(ci, norb, nelec)
    np.testing.assert_allclose(a + b, d1, atol=1e-10)
    np.testing.assert_allclose(aa + bb + ab + ab.transpose(2, 3, 0, 1), d2, atol=1e-10)
    ss, mult = sa.spin_square(ci, norb, nelec)
    assert abs(ss - 2.0) < 1e-8 and abs(mult - 3.0) < 1e-8
    assert sa.undo_state_average() is sol
