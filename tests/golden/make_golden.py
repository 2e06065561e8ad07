"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's unmodified pyscf/csf_fci/{csf,csfstring,csdstring}.py
(read from the reference checkout) on the PySCF stand-in under
oracle/shim, whose numerical routines are the reference's own C
(oracle/_ref: libcsf.so, libfci_gas.so) or the numpy restatement in
oracle/restate.py.  Only this container can run it (it needs the reference
checkout); the fixtures it writes travel with the repository.

    PYTHONPATH=oracle/shim:oracle python tests/golden/make_golden.py [--c1]
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path[:0] = [os.path.join(ROOT, "oracle", "shim"), os.path.join(ROOT, "oracle")]

import gasref  # noqa: E402
import restate as R  # noqa: E402
from pyscf.csf_fci import csf_solver  # noqa: E402
from pyscf.csf_fci.csfstring import CSFTransformer, get_spin_evecs  # noqa: E402


def seeded_integrals(norb, rank, seed=0):
    """The synthetic integrals of the benchmark configurations: h1 symmetric
    N(0,0.3) off-diagonal with diagonal linspace(-2,0.5); eri = 1/2 sum_x
    L_x (x) L_x with L (rank, norb^2) ~ N(0,0.2) symmetrised over (p,q)."""
    rng = np.random.default_rng(seed)
    h1 = rng.normal(0.0, 0.3, (norb, norb))
    h1 = 0.5 * (h1 + h1.T)
    np.fill_diagonal(h1, np.linspace(-2.0, 0.5, norb))
    L = rng.normal(0.0, 0.2, (rank, norb * norb)).reshape(rank, norb, norb)
    L = 0.5 * (L + L.transpose(0, 2, 1))
    eri = 0.5 * np.einsum("xpq,xrs->pqrs", L, L)
    return h1, eri


def fp(a):
    a = np.asarray(a, dtype=np.float64).ravel()
    return float(np.dot(np.cos(np.arange(a.size)), a))


def sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def small_case(tag, norb, nelec, smult, rank, nroots=1, full=True):
    t0 = time.time()
    na, nb = nelec
    h1, eri = seeded_integrals(norb, rank)
    sol = csf_solver(None, smult=smult)
    sol.nroots = nroots
    T = CSFTransformer(norb, na, nb, smult)
    out = dict(norb=norb, neleca=na, nelecb=nb, smult=smult, nroots=nroots, h1=h1, eri=eri)
    out["csd_mask"] = T.csd_mask.astype(np.uint32)
    out["econf_det_mask"] = T.econf_det_mask.astype(np.uint32)
    out["econf_csf_mask"] = T.econf_csf_mask.astype(np.uint32)
    sp = gasref.CASSpace(norb, nelec)
    out["link_a"] = R.link_table(norb, na)
    out["link_b"] = R.link_table(norb, nb)
    sp.close()
    hdiag = sol.make_hdiag(h1, eri, norb, nelec)
    out["hdiag_det"] = hdiag
    out["hdiag_csf"] = sol.make_hdiag_csf(h1, eri, norb, nelec, hdiag_det=hdiag)
    h2e = sol.absorb_h1e(h1, eri, norb, nelec, 0.5)
    out["h2e"] = np.asarray(h2e)
    ndet = hdiag.size
    rng = np.random.default_rng(1)
    ci = rng.normal(size=ndet)
    ci /= np.linalg.norm(ci)
    out["ci_rand"] = ci
    out["sigma_rand"] = np.asarray(sol.contract_2e(h2e, ci.reshape(R.num_strings(norb, na), -1),
                                                   norb, nelec)).ravel()
    out["det2csf_rand"] = T.vec_det2csf(ci, normalize=False)
    x = rng.normal(size=T.ncsf)
    out["csf_rand"] = x
    out["csf2det_rand"] = T.vec_csf2det(x, normalize=False)
    npsp = min(200, T.ncsf)
    addr, h0 = sol.pspace(h1, eri, norb, nelec, npsp=npsp)
    order = np.argsort(addr)
    out["pspace_addr"] = np.asarray(addr)[order]
    out["pspace_h0"] = np.asarray(h0)[np.ix_(order, order)]
    if full:
        e, c = sol.kernel(h1, eri, norb, nelec)
        e = np.atleast_1d(e)
        cs = [c] if nroots == 1 else list(c)
        out["energies"] = e
        out["ci_roots"] = np.array([np.asarray(ci_).ravel() for ci_ in cs])
        dm1, dm2 = gasref.make_rdm12(cs[0], cs[0], norb, nelec)
        out["rdm1"] = dm1
        out["rdm2"] = dm2
    # spin eigenvector blocks straight from libcsf (csfstring.c:86-141)
    for npair in range(max(0, na + nb - norb), min(na, nb) + 1):
        nspin = na + nb - 2 * npair
        if smult - 1 <= nspin:
            out["umat_%d" % nspin] = get_spin_evecs(nspin, na, nb, smult)
    path = os.path.join(HERE, "%s.npz" % tag)
    np.savez_compressed(path, **out)
    print("%s: ndet=%d ncsf=%d  %.1fs -> %s" % (tag, ndet, T.ncsf, time.time() - t0, path))


def symmetric_integrals(norb, rank, orbsym, seed=0):
    """The seeded integrals with every element that breaks the point group
    of orbsym zeroed: h1[p,q] = 0 unless irrep(p) = irrep(q); (pq|rs) = 0
    unless irrep(p)^irrep(q)^irrep(r)^irrep(s) = 0 (D2h subgroup ids)."""
    h1, eri = seeded_integrals(norb, rank, seed)
    o = np.asarray(orbsym)
    h1 = h1 * (o[:, None] == o[None, :])
    eri = eri * ((o[:, None, None, None] ^ o[None, :, None, None] ^ o[None, None, :, None]
                  ^ o[None, None, None, :]) == 0)
    return h1, eri


def symm_case(tag, norb, nelec, smult, rank, orbsym, wfnsym, nroots=1):
    """The reference's point-group-symmetric solver (csf_symm.FCISolver) and
    symmetric transformer on symmetry-adapted integrals: configuration
    irreps, packed det<->CSF transforms, the symmetric p-space and the
    energies of irrep wfnsym."""
    from pyscf.csf_fci import csf_symm
    t0 = time.time()
    na, nb = nelec
    h1, eri = symmetric_integrals(norb, rank, orbsym)
    out = dict(norb=norb, neleca=na, nelecb=nb, smult=smult, nroots=nroots, h1=h1, eri=eri,
               orbsym=np.asarray(orbsym), wfnsym=wfnsym)
    T = CSFTransformer(norb, na, nb, smult, orbsym=np.asarray(orbsym), wfnsym=wfnsym)
    out["confsym"] = np.asarray(T.confsym)
    idx_sym = T.confsym[T.econf_csf_mask] == wfnsym
    out["idx_sym"] = idx_sym
    rng = np.random.default_rng(2)
    ci = rng.normal(size=T.ndet)
    out["ci_rand"] = ci
    out["det2csf_sym"] = T.vec_det2csf(ci, normalize=False)
    x = rng.normal(size=T.ncsf)
    out["csf_sym_rand"] = x
    out["csf2det_sym"] = T.vec_csf2det(x, normalize=False)
    sol = csf_symm.FCISolver(None, smult=smult)
    sol.nroots = nroots
    sol.orbsym = np.asarray(orbsym)
    sol.wfnsym = wfnsym
    sol.norb, sol.nelec = norb, nelec
    sol.check_transformer_cache()
    npsp = min(60, T.ncsf)
    addr, h0 = sol.pspace(h1, eri, norb, nelec, npsp=npsp)
    order = np.argsort(addr)
    out["pspace_addr"] = np.asarray(addr)[order]
    out["pspace_h0"] = np.asarray(h0)[np.ix_(order, order)]
    sol.conv_tol = 1e-12
    e, c = sol.kernel(h1, eri, norb, nelec, orbsym=np.asarray(orbsym), wfnsym=wfnsym)
    out["energies"] = np.atleast_1d(e)
    cs = [c] if nroots == 1 else list(c)
    out["ci_roots"] = np.array([np.asarray(ci_).ravel() for ci_ in cs])
    path = os.path.join(HERE, "%s.npz" % tag)
    np.savez_compressed(path, **out)
    print("%s: ndet=%d ncsf_sym=%d  %.1fs -> %s  E=%s" % (tag, T.ndet, T.ncsf, time.time() - t0, path, e))


def spin_case():
    """The reference's spin ladder operators (csf_fci/spin_op.py) on the
    triplet solution of norb6_4e2e_s1 (M_S = 1): mdown to M_S = 0 and -1,
    mup back, and S+/S- of a random M_S = 0 vector."""
    from pyscf.csf_fci import spin_op
    g = np.load(os.path.join(HERE, "norb6_4e2e_s1.npz"))
    norb, smult = 6, 3
    c = g["ci_roots"][0].reshape(R.num_strings(6, 4), R.num_strings(6, 2))
    out = dict(norb=norb, smult=smult, ci_high=c)
    out["mdown_33"] = spin_op.mdown(c, norb, (3, 3), smult)
    out["mdown_24"] = spin_op.mdown(c, norb, (2, 4), smult)
    out["mup_from_33"] = spin_op.mup(out["mdown_33"], norb, (3, 3), smult)
    # the lowered vector is an eigenvector of H with the same energy
    h2e = R.absorb_h1e(g["h1"], g["eri"], norb, (3, 3), 0.5)
    v = out["mdown_33"]
    hv = gasref.contract_2e(h2e, v, norb, (3, 3))
    e = float(g["energies"][0])
    assert np.linalg.norm(hv - e * v) < 1e-8, np.linalg.norm(hv - e * v)
    rng = np.random.default_rng(5)
    x = rng.normal(size=(R.num_strings(6, 3), R.num_strings(6, 3)))
    out["x_33"] = x
    out["sup_x"] = spin_op.contract_sup(x, norb, (3, 3))
    out["sdown_x"] = spin_op.contract_sdown(x, norb, (3, 3))
    y = rng.normal(size=(R.num_strings(7, 4), R.num_strings(7, 2)))
    out["y_42_n7"] = y
    out["sup_y"] = spin_op.contract_sup(y, 7, (4, 2))
    out["sdown_y"] = spin_op.contract_sdown(y, 7, (4, 2))
    path = os.path.join(HERE, "spin_ladder_norb6.npz")
    np.savez_compressed(path, **out)
    print("spin ladder -> %s" % path)


def c1_case():
    """norb=12 (6,6) singlet, 3 roots: bit-exact hashes of the integer maps
    and fingerprints of the floating results (the full vectors are too big
    to commit)."""
    t0 = time.time()
    norb, nelec, smult, rank = 12, (6, 6), 1, 24
    h1, eri = seeded_integrals(norb, rank)
    sol = csf_solver(None, smult=smult)
    sol.nroots = 3
    T = CSFTransformer(norb, 6, 6, smult)
    out = dict(norb=norb, neleca=6, nelecb=6, smult=smult, nroots=3)
    out["sha_csd_mask"] = sha(T.csd_mask, "<u4")
    out["sha_econf_det_mask"] = sha(T.econf_det_mask, "<u4")
    out["sha_econf_csf_mask"] = sha(T.econf_csf_mask, "<u4")
    sp = gasref.CASSpace(norb, nelec)
    out["link_a"] = sp.raw_link_table(0)
    sp.close()
    hdiag = sol.make_hdiag(h1, eri, norb, nelec)
    out["fp_hdiag_det"] = fp(hdiag)
    hcsf = sol.make_hdiag_csf(h1, eri, norb, nelec, hdiag_det=hdiag)
    out["fp_hdiag_csf"] = fp(hcsf)
    out["hdiag_csf_head"] = hcsf[:64]
    h2e = sol.absorb_h1e(h1, eri, norb, nelec, 0.5)
    rng = np.random.default_rng(1)
    ci = rng.normal(size=hdiag.size)
    ci /= np.linalg.norm(ci)
    sig = np.asarray(sol.contract_2e(h2e, ci.reshape(924, 924), norb, nelec)).ravel()
    out["fp_sigma_rand"] = fp(sig)
    out["sigma_rand_head"] = sig[:64]
    out["fp_det2csf_rand"] = fp(T.vec_det2csf(ci, normalize=False))
    print("C1 pieces %.1fs" % (time.time() - t0))
    e, c = sol.kernel(h1, eri, norb, nelec)
    out["energies"] = np.asarray(e)
    dm1, dm2 = gasref.make_rdm12(c[0], c[0], norb, nelec)
    out["rdm1_root0"] = dm1
    out["fp_rdm2_root0"] = fp(dm2)
    path = os.path.join(HERE, "c1_norb12_6e6e_s0.npz")
    np.savez_compressed(path, **out)
    print("C1: %.1fs -> %s  E=%s" % (time.time() - t0, path, e))


def gas_case(tag, norb, nelec, gas_orbs, gas_restr, gas_restr_type, rank, smults, nroots=2):
    """The reference's GAS determinant solver (pyscf/mcscf/fci_gas.py and its
    C kernels) on the stand-in: the canonical spin-supergroups of the
    restriction (addons_gas.normalize_gas_spec), the allowed determinants in
    full-CAS order (fci_gas.gas2fci), and the spectrum of the GAS Hamiltonian
    (the reference's GAS sigma applied to unit vectors) with <S^2> of every
    eigenvector (the reference's GAS spin_square).  The golden energies of a
    spin multiplicity are the lowest eigenvalues whose <S^2> is S(S+1)."""
    from pyscf.mcscf import addons_gas, fci_gas
    t0 = time.time()
    h1, eri = seeded_integrals(norb, rank)
    kernel_orbs, blocks = addons_gas.normalize_gas_spec(gas_orbs, nelec, gas_restr, gas_restr_type)
    solver = fci_gas.FCISolver(gas_orbs=gas_orbs, gas_restr=gas_restr, gas_restr_type=gas_restr_type)
    h2e = fci_gas.absorb_h1e(h1, eri, norb, nelec, fac=0.5)
    with solver.make_space(norb, nelec, compress_links=True) as gas:
        ndet = gas.ndet
        allowed = fci_gas.gas2fci(np.ones(ndet), gas) != 0
        with fci_gas.GasContractPlan(gas, h2e) as plan:
            H = np.empty((ndet, ndet))
            unit = np.zeros(ndet)
            for i in range(ndet):
                unit[i] = 1.0
                H[:, i] = plan.contract(unit)
                unit[i] = 0.0
    e, v = np.linalg.eigh(0.5 * (H + H.T))
    s2 = np.array([solver.spin_square(v[:, k], norb, nelec)[0] for k in range(ndet)])
    out = dict(norb=norb, neleca=nelec[0], nelecb=nelec[1], h1=h1, eri=eri,
               gas_orbs=np.asarray(gas_orbs), kernel_gas_orbs=np.asarray(kernel_orbs),
               blocks=np.asarray(blocks), allowed_dets=allowed, spectrum=e, spectrum_s2=s2,
               smults=np.asarray(smults), nroots=nroots, gas_restr_type=gas_restr_type)
    if isinstance(gas_restr, dict):
        out["ras_max_holes"] = gas_restr["max_holes"]
        out["ras_max_particles"] = gas_restr["max_particles"]
    else:
        out["gas_restr"] = np.asarray(gas_restr)
    for sm in smults:
        ss = 0.25 * (sm - 1) * (sm + 1)
        sel = np.nonzero(np.abs(s2 - ss) < 1e-6)[0][:nroots]
        out["energies_s%d" % sm] = e[sel]
    path = os.path.join(HERE, "%s.npz" % tag)
    np.savez_compressed(path, **out)
    print("%s: ndet_gas=%d nblock=%d  %.1fs -> %s  E=%s" % (
        tag, ndet, len(blocks), time.time() - t0, path,
        {sm: out["energies_s%d" % sm] for sm in smults}))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--c1", action="store_true")
    args = ap.parse_args()
    small_case("c0_norb8_4e4e_s0", 8, (4, 4), 1, 16)
    small_case("norb6_3e3e_s1", 6, (3, 3), 3, 8, nroots=2)
    small_case("norb5_3e2e_s12", 5, (3, 2), 2, 8)
    small_case("norb6_4e2e_s1", 6, (4, 2), 3, 8)
    small_case("norb4_2e2e_s2", 4, (2, 2), 5, 6)
    small_case("norb4_4e4e_s0", 4, (4, 4), 1, 6, full=False)
    small_case("norb5_1e0e_s12", 5, (1, 0), 2, 6, full=False)
    small_case("norb7_4e3e_s32", 7, (4, 3), 4, 10, nroots=2)
    symm_case("symm_norb8_4e4e_s0_w2", 8, (4, 4), 1, 16, [0, 2, 0, 3, 1, 0, 2, 3], 2, nroots=2)
    symm_case("symm_norb7_4e3e_s12_w1", 7, (4, 3), 2, 12, [0, 1, 0, 1, 3, 2, 0], 1, nroots=2)
    symm_case("symm_norb6_3e3e_s1_w3", 6, (3, 3), 3, 10, [0, 1, 2, 3, 0, 1], 3, nroots=1)
    spin_case()
    gas_case("gas_ras_norb6_3e3e", 6, (3, 3), (2, 2, 2), {"max_holes": 1, "max_particles": 1}, "ras", 8, (1, 3))
    gas_case("gas_cumocc_norb7_4e3e", 7, (4, 3), (3, 2, 2), [[4, 6], [6, 7], [7, 7]], "cumulative-occ", 10,
             (2, 4))
    gas_case("gas_supergroup_norb6_3e3e", 6, (3, 3), (3, 3), [[4, 2], [3, 3], [5, 1]], "supergroup", 8, (1, 3))
    gas_case("gas_spinsg_norb6_2e2e", 6, (2, 2), (2, 4),
             [[1, 1, 1, 1], [2, 0, 0, 2], [0, 2, 2, 0], [1, 1, 0, 2], [0, 2, 1, 1]], "spin-supergroup", 8, (1, 3))
    if args.c1:
        c1_case()
