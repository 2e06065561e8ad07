"""GPU: the point-group-symmetric solver (csf_symm) against fixtures made by
the reference's own csf_symm.FCISolver and symmetric CSFTransformer
(tests/golden/make_golden.py, symm_* cases)."""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

SYMM_CASES = ["symm_norb8_4e4e_s0_w2", "symm_norb7_4e3e_s12_w1", "symm_norb6_3e3e_s1_w3"]


def _transformer(g):
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    return CSFTransformer(int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"]),
                          orbsym=g["orbsym"], wfnsym=int(g["wfnsym"]))


@pytest.mark.parametrize("tag", SYMM_CASES)
def test_confsym_and_packing_bit_exact(tag):
    g = load_golden(tag)
    t = _transformer(g)
    np.testing.assert_array_equal(t.confsym.cpu().numpy(), g["confsym"])
    np.testing.assert_array_equal(t.idx_sym.cpu().numpy(), g["idx_sym"])
    assert t.ncsf == int(np.count_nonzero(g["idx_sym"]))


@pytest.mark.parametrize("tag", SYMM_CASES)
def test_packed_transforms(tag):
    """Packed det->CSF and CSF->det (only the configurations of the irrep are
    formed) against the reference's vec_det2csf / vec_csf2det; pack/unpack
    round trips."""
    g = load_golden(tag)
    t = _transformer(g)
    y = t.vec_det2csf(g["ci_rand"], normalize=False)
    np.testing.assert_allclose(y, g["det2csf_sym"], atol=1e-12)
    d = t.vec_csf2det(g["csf_sym_rand"], normalize=False)
    np.testing.assert_allclose(d, g["csf2det_sym"], atol=1e-12)
    full = t.unpack_csf(g["csf_sym_rand"])
    assert full.size == g["idx_sym"].size and np.all(full[~g["idx_sym"]] == 0)
    np.testing.assert_array_equal(t.pack_csf(full), g["csf_sym_rand"])


@pytest.mark.parametrize("tag", SYMM_CASES)
def test_symmetric_pspace(tag):
    import pyscf_forge_b200.csf_fci.csf_symm as S
    g = load_golden(tag)
    norb, nelec = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"]))
    sol = S.FCISolver(None, smult=int(g["smult"]), orbsym=g["orbsym"], wfnsym=int(g["wfnsym"]))
    sol.norb, sol.nelec = norb, nelec
    sol.check_transformer_cache()
    npsp = min(60, sol.transformer.ncsf)
    addr, h0 = sol.pspace(g["h1"], g["eri"], norb, nelec, npsp=npsp)
    order = np.argsort(addr)
    np.testing.assert_array_equal(np.asarray(addr)[order], g["pspace_addr"])
    np.testing.assert_allclose(np.asarray(h0)[np.ix_(order, order)], g["pspace_h0"], atol=1e-11)


@pytest.mark.parametrize("tag", SYMM_CASES)
def test_symmetric_solver_energies(tag):
    """Energies of irrep wfnsym within 1e-9 Eh of the reference's
    csf_symm.FCISolver; CI vectors equal up to phase."""
    import pyscf_forge_b200 as P
    import pyscf_forge_b200.csf_fci.csf_symm as S
    g = load_golden(tag)
    norb, nelec = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"]))
    nroots = int(g["nroots"])
    sol = P.csf_solver(None, smult=int(g["smult"]), symm=True)
    assert isinstance(sol, S.FCISolver)
    sol.nroots = nroots
    sol.conv_tol = 1e-12
    e, c = sol.kernel(g["h1"], g["eri"], norb, nelec, orbsym=g["orbsym"], wfnsym=int(g["wfnsym"]))
    np.testing.assert_allclose(np.atleast_1d(e), g["energies"], atol=1e-9)
    cs = [c] if nroots == 1 else c
    for k, ck in enumerate(cs):
        ov = abs(float(np.dot(np.asarray(ck).ravel(), g["ci_roots"][k])))
        assert abs(ov - 1.0) < 1e-6, (k, ov)


def test_symmetric_roots_are_in_the_full_spectrum():
    """For every irrep, the symmetric solver's lowest root is an eigenvalue
    of the unrestricted CSF solver on the same symmetry-adapted integrals,
    and the lowest over all irreps is the unrestricted ground state."""
    import pyscf_forge_b200 as P
    import pyscf_forge_b200.csf_fci.csf_symm as S
    g = load_golden("symm_norb6_3e3e_s1_w3")
    norb, nelec, smult = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"])), int(g["smult"])
    full = P.csf_solver(None, smult=smult)
    from pyscf_forge_b200.csf_fci.csfstring import count_all_csfs
    full.nroots = count_all_csfs(norb, nelec[0], nelec[1], smult)
    ef, _ = full.kernel(g["h1"], g["eri"], norb, nelec)
    ef = np.atleast_1d(ef)
    lows = []
    for w in range(4):
        sol = S.FCISolver(None, smult=smult, orbsym=g["orbsym"], wfnsym=w)
        try:
            e, _ = sol.kernel(g["h1"], g["eri"], norb, nelec)
        except AssertionError:
            continue  # no CSF of this irrep
        e = float(np.atleast_1d(e)[0])
        assert np.min(np.abs(ef - e)) < 1e-9, (w, e)
        lows.append(e)
    assert abs(min(lows) - ef[0]) < 1e-9
