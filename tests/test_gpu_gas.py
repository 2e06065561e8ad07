"""GPU: GAS-restricted CSF spaces against the reference's GAS determinant
solver (pyscf/mcscf/fci_gas.py and its C kernels; fixtures from
tests/golden/make_golden.py, gas_* cases): the configuration filter
(csffci_gas_conf_mask) bit for bit against the reference's GAS determinant
set, and the solver's energies for each spin within 1e-9 Eh of the spectrum
of the reference's GAS Hamiltonian restricted to that spin."""
import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

GAS_CASES = ["gas_ras_norb6_3e3e", "gas_cumocc_norb7_4e3e", "gas_supergroup_norb6_3e3e", "gas_spinsg_norb6_2e2e"]


def _spec(g):
    t = str(g["gas_restr_type"])
    if t == "ras":
        restr = {"max_holes": int(g["ras_max_holes"]), "max_particles": int(g["ras_max_particles"])}
    else:
        restr = g["gas_restr"].tolist()
    return tuple(g["gas_orbs"].tolist()), restr, t


@pytest.mark.parametrize("tag", GAS_CASES)
def test_allowed_determinants_bit_exact(tag):
    import pyscf_forge_b200.csf_fci.gas as G
    from pyscf_forge_b200.csf_fci.csfstring import CSFTransformer
    g = load_golden(tag)
    norb, na, nb = int(g["norb"]), int(g["neleca"]), int(g["nelecb"])
    orbs, restr, t = _spec(g)
    spec = G.spin_free_supergroups(orbs, (na, nb), restr, t)
    T = CSFTransformer(norb, na, nb, int(g["smults"][0]), gas=spec)
    allowed = T._idx_sym_det().cpu().numpy().reshape(g["allowed_dets"].shape)
    np.testing.assert_array_equal(allowed, g["allowed_dets"])


@pytest.mark.parametrize("tag", GAS_CASES)
def test_gas_energies_per_spin(tag):
    import pyscf_forge_b200 as P
    from pyscf_forge_b200.csf_fci.spin_op import spin_square
    g = load_golden(tag)
    norb, nelec = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"]))
    orbs, restr, t = _spec(g)
    outside = ~np.asarray(g["allowed_dets"]).ravel()
    for sm in g["smults"].tolist():
        ref = g["energies_s%d" % sm]
        sol = P.csf_solver(None, smult=sm, gas_orbs=orbs, gas_restr=restr, gas_restr_type=t)
        sol.nroots = ref.size
        sol.conv_tol = 1e-12
        e, c = sol.kernel(g["h1"], g["eri"], norb, nelec)
        np.testing.assert_allclose(np.atleast_1d(e), ref, atol=1e-9)
        cs = c if isinstance(c, list) else [c]
        for ck in cs:
            v = np.asarray(ck).ravel()
            assert np.max(np.abs(v[outside])) < 1e-12  # no weight outside the GAS space
            ss, _ = spin_square(ck, norb, nelec)
            assert abs(ss - 0.25 * (sm - 1) * (sm + 1)) < 1e-8


def test_single_space_is_full_cas():
    """gas_orbs=(norb,) with no restriction is the whole CAS space."""
    import pyscf_forge_b200 as P
    g = load_golden("norb6_3e3e_s1")
    norb, nelec = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"]))
    full = P.csf_solver(None, smult=int(g["smult"]))
    full.nroots = 2
    ef, _ = full.kernel(g["h1"], g["eri"], norb, nelec)
    one = P.csf_solver(None, smult=int(g["smult"]), gas_orbs=(norb,))
    one.nroots = 2
    eg, _ = one.kernel(g["h1"], g["eri"], norb, nelec)
    np.testing.assert_allclose(eg, ef, atol=1e-10)


def test_gas_with_point_group_symmetry():
    """GAS and irrep restrictions together select the intersection of the
    two configuration sets: energies against the dense CSF Hamiltonian of
    the oracle restricted to those CSFs."""
    import pyscf_forge_b200 as P
    import pyscf_forge_b200.csf_fci.gas as G
    import restate as R
    import gasref
    if not gasref.available():
        pytest.skip("reference library not built")
    g = load_golden("symm_norb6_3e3e_s1_w3")
    norb, na, nb, smult = int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"])
    orbs, restr, t = (3, 3), [[4, 2], [3, 3], [5, 1]], "supergroup"
    sol = P.csf_solver(None, smult=smult, symm=True, gas_orbs=orbs, gas_restr=restr, gas_restr_type=t)
    sol.conv_tol = 1e-12
    e, c = sol.kernel(g["h1"], g["eri"], norb, (na, nb), orbsym=g["orbsym"], wfnsym=int(g["wfnsym"]))
    # dense oracle
    korbs, blocks = G.normalize_gas_spec(orbs, (na, nb), restr, t)
    allowed = R.gas_allowed_dets(norb, na, nb, korbs, blocks)
    econf = R.make_econf_det_mask(norb, na, nb, R.make_csd_mask(norb, na, nb))
    confok = R.make_confgas(econf, allowed) & (R.make_confsym(norb, na, nb, econf, g["orbsym"]) ==
                                                int(g["wfnsym"]))
    idx = confok[R.make_econf_csf_mask(norb, na, nb, smult)]
    h2e = R.absorb_h1e(g["h1"], g["eri"], norb, (na, nb), 0.5)
    nsa, nsb = R.num_strings(norb, na), R.num_strings(norb, nb)
    H = np.empty((nsa * nsb, nsa * nsb))
    for i in range(nsa * nsb):
        u = np.zeros(nsa * nsb)
        u[i] = 1.0
        H[:, i] = gasref.contract_2e(h2e, u.reshape(nsa, nsb), norb, (na, nb)).ravel()
    U = R.transform_det2csf(np.eye(idx.size), norb, na, nb, smult, reverse=True)[idx]
    w = np.linalg.eigvalsh(U @ H @ U.T)
    assert sol.transformer.ncsf == int(idx.sum())
    np.testing.assert_allclose(np.atleast_1d(e)[0], w[0], atol=1e-9)


def test_gas_transformer_reset_between_problems():
    """A solver reused without a GAS restriction forms the full space again."""
    import pyscf_forge_b200 as P
    from pyscf_forge_b200.csf_fci.csfstring import count_all_csfs
    g = load_golden("gas_supergroup_norb6_3e3e")
    norb, nelec = int(g["norb"]), (int(g["neleca"]), int(g["nelecb"]))
    sol = P.csf_solver(None, smult=1, gas_orbs=(3, 3), gas_restr=g["gas_restr"].tolist(),
                       gas_restr_type="supergroup")
    e1, _ = sol.kernel(g["h1"], g["eri"], norb, nelec)
    n_gas = sol.transformer.ncsf
    sol.gas_orbs = None
    e0, _ = sol.kernel(g["h1"], g["eri"], norb, nelec)
    assert sol.transformer.ncsf == count_all_csfs(norb, nelec[0], nelec[1], 1) > n_gas
    assert e0 <= e1 + 1e-12
