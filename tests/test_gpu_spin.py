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
