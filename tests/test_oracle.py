"""CPU: the numpy restatement (oracle/restate.py) against the golden
fixtures generated from the reference itself, and against the reference's
own C built into oracle/_ref."""
import numpy as np
import pytest

import restate as R
import gasref
from conftest import load_golden, seeded_integrals

needs_ref = pytest.mark.skipif(not gasref.available(), reason="oracle/_ref not built")


def test_masks_and_links(golden_case):
    g = golden_case
    n, na, nb, sm = int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"])
    csd = R.make_csd_mask(n, na, nb)
    assert np.array_equal(csd, g["csd_mask"])
    assert np.array_equal(R.make_econf_det_mask(n, na, nb, csd), g["econf_det_mask"])
    assert np.array_equal(R.make_econf_csf_mask(n, na, nb, sm), g["econf_csf_mask"])
    assert np.array_equal(R.link_table(n, na), g["link_a"])
    assert np.array_equal(R.link_table(n, nb), g["link_b"])


def test_transforms_and_diagonals(golden_case):
    g = golden_case
    n, na, nb, sm = int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"])
    h1, eri = g["h1"], g["eri"]
    np.testing.assert_allclose(R.make_hdiag(h1, eri, n, (na, nb)), g["hdiag_det"], atol=1e-12)
    np.testing.assert_allclose(R.make_hdiag_csf(h1, eri, n, (na, nb), sm), g["hdiag_csf"], atol=1e-12)
    np.testing.assert_allclose(R.absorb_h1e(h1, eri, n, (na, nb), 0.5), g["h2e"], atol=1e-13)
    np.testing.assert_allclose(R.transform_det2csf(g["ci_rand"], n, na, nb, sm)[0], g["det2csf_rand"],
                               atol=1e-13)
    np.testing.assert_allclose(R.transform_det2csf(g["csf_rand"], n, na, nb, sm, reverse=True)[0],
                               g["csf2det_rand"], atol=1e-13)
    for key in g:
        if key.startswith("umat_"):
            nspin = int(key.split("_")[1])
            assert np.array_equal(R.get_spin_evecs(nspin, na, nb, sm), g[key])


def test_sigma_and_rdms(golden_case):
    g = golden_case
    n, na, nb = int(g["norb"]), int(g["neleca"]), int(g["nelecb"])
    sig = R.contract_2e(g["h2e"], g["ci_rand"], n, (na, nb))
    np.testing.assert_allclose(sig, g["sigma_rand"], atol=1e-11)
    if "rdm1" in g:
        c = g["ci_roots"][0]
        d1, d2 = R.make_rdm12(c, c, n, (na, nb))
        np.testing.assert_allclose(d1, g["rdm1"], atol=1e-12)
        np.testing.assert_allclose(d2, g["rdm2"], atol=1e-12)


def test_pspace_and_energy(golden_case):
    g = golden_case
    n, na, nb, sm = int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"])
    if g["hdiag_det"].size > 1300:
        pytest.skip("dense check is sized for the small cases")
    h2e = g["h2e"]
    nd = g["hdiag_det"].size
    H = np.array([R.contract_2e(h2e, np.eye(nd)[i], n, (na, nb)) for i in range(nd)])
    Hc = R.transform_det2csf(H, n, na, nb, sm)
    Hc = R.transform_det2csf(Hc.T, n, na, nb, sm)
    addr = g["pspace_addr"]
    np.testing.assert_allclose(g["pspace_h0"], Hc[np.ix_(addr, addr)], atol=1e-11)
    if "energies" in g:
        w = np.linalg.eigvalsh(Hc)
        np.testing.assert_allclose(g["energies"], w[:len(g["energies"])], atol=1e-9)


@needs_ref
@pytest.mark.parametrize("norb,nelec", [(6, (3, 3)), (7, (4, 2)), (8, (3, 5))])
def test_restatement_vs_reference_c(norb, nelec):
    h1, eri = seeded_integrals(norb, 10, seed=3)
    h2e = R.absorb_h1e(h1, eri, norb, nelec, 0.5)
    rng = np.random.default_rng(4)
    ci = rng.normal(size=R.num_strings(norb, nelec[0]) * R.num_strings(norb, nelec[1]))
    np.testing.assert_allclose(R.contract_2e(h2e, ci, norb, nelec), gasref.contract_2e(h2e, ci, norb, nelec),
                               atol=1e-11)
    np.testing.assert_allclose(R.make_hdiag(h1, eri, norb, nelec), gasref.make_hdiag(h1, eri, norb, nelec),
                               atol=1e-12)
    ket = rng.normal(size=ci.size)
    d1, d2 = R.make_rdm12(ci, ket, norb, nelec)
    e1, e2 = gasref.make_rdm12(ci, ket, norb, nelec)
    np.testing.assert_allclose(d1, e1, atol=1e-11)
    np.testing.assert_allclose(d2, e2, atol=1e-11)
    sp = gasref.CASSpace(norb, nelec)
    la = sp.raw_link_table(0)
    sp.close()
    assert np.array_equal(la, R.link_table(norb, nelec[0])) or np.array_equal(la, R.link_table(norb, nelec[1]))


@needs_ref
def test_umat_vs_libcsf():
    for nspin in range(0, 11):
        for twoms in range(-(nspin % 2 + 0), nspin + 1, 2):
            if twoms < 0 or (nspin - twoms) % 2:
                continue
            na = (nspin + twoms) // 2
            nb = nspin - na
            for smult in range(twoms + 1, nspin + 2, 2):
                u = R.get_spin_evecs(nspin, na, nb, smult)
                det = R.addrs2str(nspin, na, np.arange(u.shape[0]))
                coup = R.gen_addrs2str(nspin, smult, np.arange(u.shape[1]))
                ref = gasref.makecsf(det, coup, nspin, smult - 1, na - nb)
                assert np.array_equal(u, ref)


def test_c1_fixture_integer_maps():
    import hashlib
    g = load_golden("c1_norb12_6e6e_s0")
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()
    csd = R.make_csd_mask(12, 6, 6)
    assert sha(csd) == str(g["sha_csd_mask"])
    assert np.array_equal(R.link_table(12, 6), g["link_a"])


SYMM_CASES = ["symm_norb8_4e4e_s0_w2", "symm_norb7_4e3e_s12_w1", "symm_norb6_3e3e_s1_w3"]


@pytest.mark.parametrize("tag", SYMM_CASES)
def test_confsym_restatement_matches_reference(tag):
    """Configuration irreps: the numpy restatement equals the reference's
    make_confsym (csfstring.py:278-290) bit for bit."""
    g = load_golden(tag)
    norb, na, nb = int(g["norb"]), int(g["neleca"]), int(g["nelecb"])
    csd = R.make_csd_mask(norb, na, nb)
    econf = R.make_econf_det_mask(norb, na, nb, csd)
    cs = R.make_confsym(norb, na, nb, econf, g["orbsym"])
    np.testing.assert_array_equal(cs, g["confsym"])
    ecsf = R.make_econf_csf_mask(norb, na, nb, int(g["smult"]))
    np.testing.assert_array_equal(cs[ecsf] == int(g["wfnsym"]), g["idx_sym"])


@pytest.mark.parametrize("tag", SYMM_CASES)
def test_symmetric_energies_against_dense_csf_hamiltonian(tag):
    """Pins the reference's symmetric-solver energies independently: the
    dense CSF-basis Hamiltonian restricted to the CSFs of irrep wfnsym
    (built from the reference GAS sigma on unit vectors and the restated
    transforms) has the same lowest eigenvalues (1e-9 Eh)."""
    if not gasref.available():
        pytest.skip("reference library not built")
    g = load_golden(tag)
    norb, na, nb, smult = int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"])
    if R.num_strings(norb, na) * R.num_strings(norb, nb) > 2000:
        pytest.skip("dense check only for the small cases")
    h2e = R.absorb_h1e(g["h1"], g["eri"], norb, (na, nb), 0.5)
    ndet = R.num_strings(norb, na) * R.num_strings(norb, nb)
    H = np.empty((ndet, ndet))
    for i in range(ndet):
        e = np.zeros(ndet)
        e[i] = 1.0
        H[:, i] = gasref.contract_2e(h2e, e.reshape(R.num_strings(norb, na), -1), norb, (na, nb)).ravel()
    idx = np.asarray(g["idx_sym"], dtype=bool)
    U = R.transform_det2csf(np.eye(idx.size), norb, na, nb, smult, reverse=True)  # (ncsf, ndet)
    Us = U[idx]
    w = np.linalg.eigvalsh(Us @ H @ Us.T)
    e = np.atleast_1d(g["energies"])
    np.testing.assert_allclose(w[:e.size], e, atol=1e-9)


GAS_CASES = ["gas_ras_norb6_3e3e", "gas_cumocc_norb7_4e3e", "gas_supergroup_norb6_3e3e", "gas_spinsg_norb6_2e2e"]


@pytest.mark.parametrize("tag", GAS_CASES)
def test_gas_membership_restatement_matches_reference(tag):
    """The determinants of the reference's GAS space (fci_gas.gas2fci of its
    canonical blocks) equal the restated membership rule bit for bit, and
    form whole configurations (the spin-complete sets the CSF solver
    takes)."""
    g = load_golden(tag)
    norb, na, nb = int(g["norb"]), int(g["neleca"]), int(g["nelecb"])
    allowed = R.gas_allowed_dets(norb, na, nb, g["kernel_gas_orbs"].tolist(), g["blocks"])
    np.testing.assert_array_equal(allowed, g["allowed_dets"])
    econf = R.make_econf_det_mask(norb, na, nb, R.make_csd_mask(norb, na, nb))
    R.make_confgas(econf, allowed)


@pytest.mark.parametrize("tag", GAS_CASES)
def test_gas_energies_against_dense_csf_hamiltonian(tag):
    """The CSF solver's GAS restriction is a filter on configurations: the
    dense CSF-basis Hamiltonian restricted to the CSFs of the allowed
    configurations (reference GAS sigma on unit vectors, restated
    transforms) has, for each spin, the lowest eigenvalues that the
    reference's GAS determinant Hamiltonian gives that spin (1e-9 Eh)."""
    if not gasref.available():
        pytest.skip("reference library not built")
    g = load_golden(tag)
    norb, na, nb = int(g["norb"]), int(g["neleca"]), int(g["nelecb"])
    h2e = R.absorb_h1e(g["h1"], g["eri"], norb, (na, nb), 0.5)
    nsa, nsb = R.num_strings(norb, na), R.num_strings(norb, nb)
    ndet = nsa * nsb
    H = np.empty((ndet, ndet))
    for i in range(ndet):
        e = np.zeros(ndet)
        e[i] = 1.0
        H[:, i] = gasref.contract_2e(h2e, e.reshape(nsa, nsb), norb, (na, nb)).ravel()
    econf = R.make_econf_det_mask(norb, na, nb, R.make_csd_mask(norb, na, nb))
    confok = R.make_confgas(econf, g["allowed_dets"])
    for sm in g["smults"].tolist():
        idx = confok[R.make_econf_csf_mask(norb, na, nb, sm)]
        U = R.transform_det2csf(np.eye(idx.size), norb, na, nb, sm, reverse=True)
        Us = U[idx]
        w = np.linalg.eigvalsh(Us @ H @ Us.T)
        e = g["energies_s%d" % sm]
        np.testing.assert_allclose(w[:e.size], e, atol=1e-9)


def test_davidson1_restatement_matches_eigh():
    """The restatement of lib.davidson1 (oracle/davidson_np.py) finds the
    lowest roots of a symmetric matrix, with the diagonal and the p-space
    Olsen preconditioners, to 1e-10."""
    import davidson_np as Dv
    rng = np.random.default_rng(3)
    n = 400
    A = rng.normal(size=(n, n)) * 0.3
    A = A + A.T + np.diag(np.linspace(0.0, 40.0, n))
    w = np.linalg.eigvalsh(A)
    hd = np.diag(A).copy()
    addr = np.argsort(hd)[:30]
    pw, pv = np.linalg.eigh(A[np.ix_(addr, addr)])
    for pre in (Dv.make_diag_precond(hd, 1e-3), Dv.make_pspace_precond(hd, pw, pv, addr, 1e-3)):
        for nroots in (1, 3):
            x0 = [np.eye(n)[i] for i in np.argsort(hd)[:nroots]]
            conv, e, x = Dv.davidson1(lambda v: A @ v, x0, pre, tol=1e-12, nroots=nroots, max_cycle=300)
            assert all(conv)
            np.testing.assert_allclose(e, w[:nroots], atol=1e-10)
