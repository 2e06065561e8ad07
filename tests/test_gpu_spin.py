"""GPU: spin ladder operators and <S^2> against the reference's
csf_fci/spin_op.py (fixtures generated by running it, tests/golden)."""
import numpy as np
import pytest

from conftest import load_golden, SMALL_CASES

pytestmark = pytest.mark.gpu


def test_ladder_operators_match_reference():
    from pyscf_forge_b200.csf_fci import spin_op as S
    g = load_golden("spin_ladder_norb6")
    np.testing.assert_allclose(S.contract_sup(g["x_33"], 6, (3, 3)), g["sup_x"], atol=1e-13)
    np.testing.assert_allclose(S.contract_sdown(g["x_33"], 6, (3, 3)), g["sdown_x"], atol=1e-13)
    np.testing.assert_allclose(S.contract_sup(g["y_42_n7"], 7, (4, 2)), g["sup_y"], atol=1e-13)
    np.testing.assert_allclose(S.contract_sdown(g["y_42_n7"], 7, (4, 2)), g["sdown_y"], atol=1e-13)
    assert S.contract_sup(np.zeros((1, 6)), 6, (6, 1)).shape == (0, 0)  # S+ on all-alpha-occupied


def test_mdown_mup_match_reference():
    from pyscf_forge_b200.csf_fci import spin_op as S
    g = load_golden("spin_ladder_norb6")
    c = g["ci_high"]
    d33 = S.mdown(c, 6, (3, 3), 3)
    np.testing.assert_allclose(d33, g["mdown_33"], atol=1e-12)
    np.testing.assert_allclose(S.mdown(c, 6, (2, 4), 3), g["mdown_24"], atol=1e-12)
    np.testing.assert_allclose(S.mup(d33, 6, (3, 3), 3), g["mup_from_33"], atol=1e-12)
    np.testing.assert_allclose(S.mup(d33, 6, (3, 3), 3), c, atol=1e-10)   # round trip
    assert abs(np.linalg.norm(d33) - 1.0) < 1e-10


@pytest.mark.parametrize("tag", [t for t in SMALL_CASES])
def test_spin_square_of_solutions(tag):
    """<S^2> of the reference's converged CI vectors is S(S+1) and the
    multiplicity is smult."""
    import pyscf_forge_b200 as P
    g = load_golden(tag)
    if "ci_roots" not in g:
        pytest.skip("no solved vectors in this fixture")
    norb, nelec, smult = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"])), int(g["smult"])
    sol = P.csf_solver(None, smult=smult)
    s = 0.5 * (smult - 1)
    for c in g["ci_roots"]:
        ss, mult = sol.spin_square(c, norb, nelec)
        assert abs(ss - s * (s + 1)) < 1e-8 and abs(mult - smult) < 1e-8, (tag, ss, mult)


def _cc_chc_smult(h2e, c, norb, nelec):
    from pyscf_forge_b200.fci import direct_spin1 as D
    from pyscf_forge_b200.csf_fci.spin_op import spin_square
    cc = float(np.dot(c.ravel(), c.ravel()))
    chc = float(np.dot(c.ravel(), np.asarray(D.contract_2e(h2e, c, norb, nelec)).ravel()))
    ss, mult = spin_square(c, norb, nelec)
    return cc, chc, mult


@pytest.mark.parametrize("norb,ntot", [(6, 6), (6, 7), (7, 6), (7, 7)])
def test_ladder_preserves_norm_energy_and_spin(norb, ntot):
    """Walking a maximal-M_S vector down to M_S = -S with normalised S- and
    back up with S+ keeps the norm, <H> and <S^2> (the checks of the
    reference's test_spin_op.py test_ladder, with symmetric seeded
    integrals); S+ on M_S = S and S- on M_S = -S give empty arrays."""
    from pyscf_forge_b200.csf_fci.spin_op import contract_sdown, contract_sup, norm_sdown, norm_sup
    from pyscf_forge_b200.fci import direct_spin1 as D
    from conftest import seeded_integrals
    from math import comb
    h1, eri = seeded_integrals(norb, 2 * norb, seed=norb + ntot)
    nelec = (min(norb, ntot), ntot - min(norb, ntot))
    smult = nelec[0] - nelec[1] + 1
    rng = np.random.default_rng(norb * 10 + ntot)
    ci = rng.random((comb(norb, nelec[0]), comb(norb, nelec[1])))
    ci /= np.linalg.norm(ci)
    h2e = {}

    def h(ne):
        if ne not in h2e:
            h2e[ne] = D.absorb_h1e(h1, eri, norb, ne, 0.5)
        return h2e[ne]

    cc0, chc0, m0 = _cc_chc_smult(h(nelec), ci, norb, nelec)
    assert abs(cc0 - 1) < 1e-9 and abs(m0 - smult) < 1e-9
    assert contract_sup(ci, norb, nelec).size == 0
    s = (smult - 1) / 2
    for _ in np.arange(s, -s, -1):
        ci = contract_sdown(ci, norb, nelec) / norm_sdown(smult, nelec)
        nelec = (nelec[0] - 1, nelec[1] + 1)
        cc, chc, m = _cc_chc_smult(h(nelec), ci, norb, nelec)
        assert abs(cc - 1) < 1e-9 and abs(m - smult) < 1e-9 and abs(chc - chc0) < 1e-9
    assert contract_sdown(ci, norb, nelec).size == 0
    for _ in np.arange(-s, s, 1):
        ci = contract_sup(ci, norb, nelec) / norm_sup(smult, nelec)
        nelec = (nelec[0] + 1, nelec[1] - 1)
        cc, chc, m = _cc_chc_smult(h(nelec), ci, norb, nelec)
        assert abs(cc - 1) < 1e-9 and abs(m - smult) < 1e-9 and abs(chc - chc0) < 1e-9


def test_mup_mdown_round_trip_input_forms():
    """mup(mdown(c)) = c for an array, a list and a stacked array, at every
    M_S (test_spin_op.py test_mdown_mup)."""
    from pyscf_forge_b200.csf_fci.spin_op import mdown, mup
    from math import comb
    # 7 electrons in 6 orbitals with M_S = 5/2 = S_max: every vector is spin-pure
    norb, nelec = 6, (6, 1)
    smult = nelec[0] - nelec[1] + 1
    ci = np.random.default_rng(4).random((comb(norb, 6), comb(norb, 1)))
    ci /= np.linalg.norm(ci)
    s = (smult - 1) / 2
    for ci0 in (ci, [ci], ci[None, :, :]):
        nelec1 = nelec
        for _ in np.arange(s, -s, -1):
            ci1 = mup(mdown(ci0, norb, nelec1, smult), norb, nelec1, smult)
            assert abs(float(np.ravel(ci0).dot(np.ravel(ci1))) - 1.0) < 1e-9
            nelec1 = (nelec1[0] - 1, nelec1[1] + 1)


def test_csf_phase_convention_across_ms():
    """The same CSF coefficients, transformed to determinants at any M_S and
    raised to M_S = S with mup, give the M_S = S vector (overlap +1): the
    CSF phase convention of the transforms agrees with the ladder operators
    (test_spin_op.py test_csf_sign)."""
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    from pyscf_forge_b200.csf_fci.spin_op import mup
    from itertools import product
    rng = np.random.default_rng(8)
    for smult, ndocc, nvirt in product(range(1, 8), range(3), range(3)):
        if smult == 1 and ndocc == 0:
            continue
        nelec = ((smult - 1) + ndocc, ndocc)
        norb = (smult - 1) + ndocc + nvirt
        t0 = CSFTransformer(norb, nelec[0], nelec[1], smult)
        x = 2 * rng.random(t0.ncsf) - 1
        x /= np.linalg.norm(x)
        ci0 = t0.vec_csf2det(x)
        ntot = sum(nelec)
        for spin in range(1 - smult, smult - 1, 2):
            ne = ((ntot + spin) // 2, (ntot - spin) // 2)
            t1 = CSFTransformer(norb, ne[0], ne[1], smult)
            ci1 = mup(np.asarray(t1.vec_csf2det(x)).reshape(t1.ndeta, t1.ndetb), norb, ne, smult)
            ov = float(np.ravel(ci1).dot(np.ravel(ci0)))
            assert abs(ov - 1.0) < 1e-8, (smult, ndocc, nvirt, spin, ov)
