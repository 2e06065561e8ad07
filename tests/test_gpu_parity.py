"""GPU parity: every kernel of the CSF-FCI path against the golden fixtures
(generated from the reference) and the oracle (reference C in oracle/_ref
and the numpy restatement).  Integer maps must be bit-exact; floating-point
results use the tolerances stated next to each assertion."""
import hashlib

import numpy as np
import pytest
import torch

import gasref
import restate as R
from conftest import load_golden, seeded_integrals

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not gasref.available(), reason="oracle/_ref not built")


def _mods():
    import pyscf_forge_b200 as P
    from pyscf_forge_b200.fci import direct_spin1 as D
    from pyscf_forge_b200.csf_fci import csfstring as C
    return P, D, C


def _case(g):
    return int(g["norb"]), int(g["neleca"]), int(g["nelecb"]), int(g["smult"])


def test_link_tables_bit_exact(golden_case):
    P, D, C = _mods()
    n, na, nb, sm = _case(golden_case)
    assert np.array_equal(D.decode_link_table(D.dev_link_table(n, na))[:, :golden_case["link_a"].shape[1]],
                          golden_case["link_a"])
    assert np.array_equal(D.decode_link_table(D.dev_link_table(n, nb))[:, :golden_case["link_b"].shape[1]],
                          golden_case["link_b"])


@needs_ref
@pytest.mark.parametrize("norb,nelec", [(12, 6), (16, 8), (14, 5), (9, 1)])
def test_link_tables_vs_reference_c(norb, nelec):
    _, D, _ = _mods()
    sp = gasref.CASSpace(norb, (nelec, nelec))
    ref = sp.raw_link_table(0)
    sp.close()
    assert np.array_equal(D.decode_link_table(D.dev_link_table(norb, nelec)), ref)


def test_masks_bit_exact(golden_case):
    _, _, C = _mods()
    n, na, nb, sm = _case(golden_case)
    t = C.CSFTransformer(n, na, nb, sm)
    assert np.array_equal(t.csd_mask.cpu().numpy().view(np.uint32), golden_case["csd_mask"])
    assert np.array_equal(t.econf_det_mask.cpu().numpy().view(np.uint32), golden_case["econf_det_mask"])
    assert np.array_equal(t.econf_csf_mask.cpu().numpy().view(np.uint32), golden_case["econf_csf_mask"])


def _sha(t):
    return hashlib.sha256(np.ascontiguousarray(t.cpu().numpy().view(np.uint32)).tobytes()).hexdigest()


def test_masks_c1_bit_exact():
    _, _, C = _mods()
    g = load_golden("c1_norb12_6e6e_s0")
    t = C.CSFTransformer(12, 6, 6, 1)
    assert _sha(t.csd_mask) == str(g["sha_csd_mask"])
    assert _sha(t.econf_det_mask) == str(g["sha_econf_det_mask"])
    assert _sha(t.econf_csf_mask) == str(g["sha_econf_csf_mask"])


def test_masks_permutation_large():
    """norb=16 (8,8): csd_mask is a permutation and econf_det_mask inverts it
    blockwise (size-independent properties at the full size)."""
    _, _, C = _mods()
    t = C.CSFTransformer(16, 8, 8, 1)
    m = t.csd_mask.long()
    n = m.numel()
    assert n == 165636900
    seen = torch.zeros(n, dtype=torch.int8, device=m.device)
    seen[m] = 1
    assert int(seen.sum()) == n
    assert t.ncsf == 34763300
    del seen


@needs_ref
def test_spin_evecs_bit_exact():
    _, _, C = _mods()
    for nspin in range(0, 13):
        for na in range(0, nspin + 1):
            nb = nspin - na
            for smult in range(abs(na - nb) + 1, nspin + 2, 2):
                u = C.get_spin_evecs(nspin, na, nb, smult).cpu().numpy()
                det = R.addrs2str(nspin, na, np.arange(u.shape[0]))
                coup = R.gen_addrs2str(nspin, smult, np.arange(u.shape[1]))
                ref = gasref.makecsf(det, coup, nspin, smult - 1, na - nb)
                assert np.array_equal(u, ref), (nspin, na, nb, smult)


@needs_ref
@pytest.mark.parametrize("nspin", [13, 14, 15, 16])
def test_spin_evecs_bit_exact_large(nspin):
    """The large spin-coupling blocks (up to 16 unpaired electrons, the
    12870 x 1430 singlet block every CAS(16,16) transform multiplies by)
    against FCICSFmakecsf (csfstring.c:86-141), bit for bit, at the smallest
    |2MS| and every spin multiplicity."""
    _, _, C = _mods()
    na = (nspin + 1) // 2
    nb = nspin - na
    det = R.addrs2str(nspin, na, np.arange(R.num_strings(nspin, na)))
    for smult in range(abs(na - nb) + 1, nspin + 2, 2):
        u = C.get_spin_evecs(nspin, na, nb, smult).cpu().numpy()
        coup = R.gen_addrs2str(nspin, smult, np.arange(u.shape[1]))
        ref = gasref.makecsf(det, coup, nspin, smult - 1, na - nb)
        assert np.array_equal(u, ref), (nspin, na, nb, smult)
        del u, ref


def test_spin_evecs_fixture(golden_case):
    _, _, C = _mods()
    n, na, nb, sm = _case(golden_case)
    for key in golden_case:
        if key.startswith("umat_"):
            nspin = int(key.split("_")[1])
            assert np.array_equal(C.get_spin_evecs(nspin, na, nb, sm).cpu().numpy(), golden_case[key])


def test_spin_evecs_orthonormal_s2():
    """test_csfstring.py:7-37: umat orthonormal and diagonalises S^2 (from
    FCICSFmakeS2mat) with eigenvalue S(S+1); tolerance 1e-8 as there."""
    if not gasref.available():
        pytest.skip("oracle/_ref not built")
    _, _, C = _mods()
    for nspin in range(1, 11):
        for twoms in range(nspin % 2, nspin + 1, 2):
            na = (nspin + twoms) // 2
            nb = nspin - na
            det = R.addrs2str(nspin, na, np.arange(R.num_strings(nspin, na)))
            s2 = gasref.makeS2mat(det, nspin, twoms)
            for smult in range(twoms + 1, nspin + 2, 2):
                u = C.get_spin_evecs(nspin, na, nb, smult).cpu().numpy()
                s = (smult - 1) / 2
                assert np.linalg.norm(u.T @ u - np.eye(u.shape[1])) < 1e-8
                assert np.linalg.norm(u.T @ s2 @ u - s * (s + 1) * np.eye(u.shape[1])) < 1e-8


def test_transforms(golden_case):
    _, _, C = _mods()
    n, na, nb, sm = _case(golden_case)
    t = C.CSFTransformer(n, na, nb, sm)
    # tolerance 1e-13: same sums as the reference in a different order
    np.testing.assert_allclose(t.vec_det2csf(golden_case["ci_rand"], normalize=False),
                               golden_case["det2csf_rand"], atol=1e-13)
    np.testing.assert_allclose(t.vec_csf2det(golden_case["csf_rand"], normalize=False),
                               golden_case["csf2det_rand"], atol=1e-13)
    # batched, list and column layouts follow the reference shapes
    xs = [golden_case["ci_rand"], 2.0 * golden_case["ci_rand"]]
    out = t.vec_det2csf(xs, normalize=False)
    assert isinstance(out, list) and len(out) == 2
    np.testing.assert_allclose(out[1], 2.0 * golden_case["det2csf_rand"], atol=1e-12)
    cols = t.vec_det2csf(np.stack(xs, axis=1), order='F', normalize=False)
    np.testing.assert_allclose(cols[:, 0], golden_case["det2csf_rand"], atol=1e-13)


def test_round_trip_c1():
    """det -> csf -> det is a projector: csf2det(det2csf(x)) applied twice is
    idempotent, and csf -> det -> csf is the identity (full size C1)."""
    _, _, C = _mods()
    t = C.CSFTransformer(12, 6, 6, 1)
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.randn(2, t.ncsf, generator=g, dtype=torch.float64).cuda()
    y = t.dev_det2csf(t.dev_csf2det(x))
    torch.testing.assert_close(y, x, atol=1e-12, rtol=0)


def test_diagonals_and_absorb(golden_case):
    P, D, C = _mods()
    n, na, nb, sm = _case(golden_case)
    h1, eri = golden_case["h1"], golden_case["eri"]
    sol = P.csf_solver(None, smult=sm)
    hd = sol.make_hdiag(h1, eri, n, (na, nb))
    np.testing.assert_allclose(hd, golden_case["hdiag_det"], atol=1e-12)
    hc = sol.make_hdiag_csf(h1, eri, n, (na, nb))
    np.testing.assert_allclose(hc, golden_case["hdiag_csf"], atol=1e-12)
    h2e = D.absorb_h1e(h1, eri, n, (na, nb), 0.5)
    np.testing.assert_allclose(h2e, golden_case["h2e"], atol=1e-13)


def test_sigma_golden(golden_case):
    P, D, C = _mods()
    n, na, nb, sm = _case(golden_case)
    # 1e-11: the reference's own GAS-vs-direct_spin1 tolerance (test_gasci.py:285-290)
    sig = D.contract_2e(golden_case["h2e"], golden_case["ci_rand"], n, (na, nb))
    np.testing.assert_allclose(sig, golden_case["sigma_rand"], atol=1e-11)


@needs_ref
@pytest.mark.parametrize("norb,nelec,rank", [(10, (5, 4), 12), (11, (3, 6), 10), (12, (6, 6), 24),
                                             (9, (9, 2), 8), (13, (2, 2), 8)])
def test_sigma_vs_reference_c(norb, nelec, rank):
    _, D, _ = _mods()
    h1, eri = seeded_integrals(norb, rank, seed=5)
    h2e = R.absorb_h1e(h1, eri, norb, nelec, 0.5)
    rng = np.random.default_rng(6)
    ci = rng.normal(size=R.num_strings(norb, nelec[0]) * R.num_strings(norb, nelec[1]))
    ci /= np.linalg.norm(ci)
    ref = gasref.contract_2e(h2e, ci, norb, nelec)
    got = D.contract_2e(h2e, ci, norb, nelec)
    np.testing.assert_allclose(got, ref, atol=1e-10)  # sigma tolerance 1e-9 of the target, tighter here


def test_sigma_c1_fixture():
    _, D, _ = _mods()
    g = load_golden("c1_norb12_6e6e_s0")
    h1, eri = seeded_integrals(12, 24)
    h2e = R.absorb_h1e(h1, eri, 12, (6, 6), 0.5)
    rng = np.random.default_rng(1)
    ci = rng.normal(size=924 * 924)
    ci /= np.linalg.norm(ci)
    sig = D.contract_2e(h2e, ci, 12, (6, 6))
    np.testing.assert_allclose(sig[:64], g["sigma_rand_head"], atol=1e-11)
    fp = float(np.dot(np.cos(np.arange(sig.size)), sig))
    assert abs(fp - float(g["fp_sigma_rand"])) < 1e-8


@pytest.mark.parametrize("norb,nelec,smult", [(8, (4, 4), 1), (8, (4, 4), 3), (10, (5, 5), 1),
                                              (9, (3, 3), 5)])
def test_sigma_spin_symmetric_mode(norb, nelec, smult):
    """The row-local kernel + transpose-add equals the general kernel for
    vectors built from CSFs (c = eta c^T)."""
    _, D, C = _mods()
    t = C.CSFTransformer(norb, nelec[0], nelec[1], smult)
    h1, eri = seeded_integrals(norb, 8, seed=2)
    h2e = D.dev_absorb_h1e(h1, R.restore4(eri, norb), norb, nelec, 0.5)
    g = torch.Generator(device="cpu").manual_seed(1)
    x = torch.randn(t.ncsf, generator=g, dtype=torch.float64).cuda()
    c = t.dev_csf2det(x)[0]
    eta = t.spin_parity
    assert eta in (1, -1)
    ref = D.dev_contract_2e(h2e, c, norb, nelec)
    got = D.dev_contract_2e(h2e, c, norb, nelec, eta=eta)
    torch.testing.assert_close(got, ref, atol=1e-11, rtol=0)


def test_contract_1e():
    _, D, _ = _mods()
    norb, nelec = 7, (4, 2)
    rng = np.random.default_rng(3)
    ha = rng.normal(size=(norb, norb))
    hb = rng.normal(size=(norb, norb))
    ci = rng.normal(size=R.num_strings(norb, 4) * R.num_strings(norb, 2))
    got = D.contract_1e(np.array([ha, hb]), ci, norb, nelec)
    ref = R.contract_1e_ab(ha, hb, ci, norb, nelec)
    np.testing.assert_allclose(got, ref, atol=1e-12)


def test_rdms_golden(golden_case):
    P, D, C = _mods()
    if "rdm1" not in golden_case:
        pytest.skip("no solve in this fixture")
    n, na, nb, sm = _case(golden_case)
    c = golden_case["ci_roots"][0]
    dm1, dm2 = D.make_rdm12(c, n, (na, nb))
    # 1e-12 as test_gasci.py:765-786 (RDM target 1e-8)
    np.testing.assert_allclose(dm1, golden_case["rdm1"], atol=1e-12)
    np.testing.assert_allclose(dm2, golden_case["rdm2"], atol=1e-12)


@needs_ref
@pytest.mark.parametrize("norb,nelec", [(6, (3, 3)), (8, (5, 3)), (10, (4, 4))])
def test_trans_rdm_vs_reference_c(norb, nelec):
    _, D, _ = _mods()
    rng = np.random.default_rng(8)
    nd = R.num_strings(norb, nelec[0]) * R.num_strings(norb, nelec[1])
    bra = rng.normal(size=nd)
    ket = rng.normal(size=nd)
    bra /= np.linalg.norm(bra)
    ket /= np.linalg.norm(ket)
    d1, d2 = D.trans_rdm12(bra, ket, norb, nelec)
    e1, e2 = gasref.make_rdm12(bra, ket, norb, nelec)
    np.testing.assert_allclose(d1, e1, atol=1e-12)
    np.testing.assert_allclose(d2, e2, atol=1e-12)


def _dense_csf_columns(g, addr):
    """<csf_i|H|csf_j> for j in addr through the reference C sigma."""
    n, na, nb, sm = _case(g)
    plan = gasref.SigmaPlan(n, (na, nb), g["h2e"])
    ncsf = g["hdiag_csf"].size
    cols = []
    for j in addr:
        x = np.zeros(ncsf)
        x[j] = 1.0
        d = R.transform_det2csf(x, n, na, nb, sm, csd_mask=g["csd_mask"], reverse=True)[0]
        cols.append(R.transform_det2csf(plan(d), n, na, nb, sm, csd_mask=g["csd_mask"])[0])
    plan.close()
    return np.array(cols).T


@needs_ref
def test_pspace(golden_case):
    P, _, _ = _mods()
    n, na, nb, sm = _case(golden_case)
    sol = P.csf_solver(None, smult=sm)
    addr, h0 = sol.pspace(golden_case["h1"], golden_case["eri"], n, (na, nb), npsp=200)
    assert len(set(addr.tolist())) == len(addr)
    H = _dense_csf_columns(golden_case, addr)
    np.testing.assert_allclose(h0, H[addr], atol=1e-11)
    if np.array_equal(np.sort(addr), golden_case["pspace_addr"]):
        o = np.argsort(addr)
        np.testing.assert_allclose(h0[np.ix_(o, o)], golden_case["pspace_h0"], atol=1e-11)


def test_kernel_energies(golden_case):
    P, _, _ = _mods()
    if "energies" not in golden_case:
        pytest.skip("no solve in this fixture")
    n, na, nb, sm = _case(golden_case)
    nroots = int(golden_case["nroots"])
    for davidson_only in (False, True):
        sol = P.csf_solver(None, smult=sm)
        sol.nroots = nroots
        sol.davidson_only = davidson_only
        e, ci = sol.kernel(golden_case["h1"], golden_case["eri"], n, (na, nb))
        e = np.atleast_1d(e)
        # energies within 1e-9 Eh of the reference CPU CSFFCISolver
        np.testing.assert_allclose(e, golden_case["energies"], atol=1e-9)
        cis = ci if isinstance(ci, list) else [ci]
        for k, c in enumerate(cis):
            ref = golden_case["ci_roots"][k]
            ov = abs(float(np.dot(c.ravel(), ref)))
            assert ov > 1 - 1e-7
            ss, m = R.spin_square(c, n, (na, nb))
            assert abs(m - sm) < 1e-6


@pytest.mark.parametrize("device_resident", [False, True])
def test_kernel_c1_three_roots(device_resident):
    """C1 (norb 12 (6,6), 3 roots) against the reference's own solver:
    energies within 1e-9 Eh on both paths.  The host-driven Davidson (the
    reference's p-space Olsen preconditioner) gives the reference's root-0
    1-RDM within 1e-8; the device-resident one (diagonal Olsen
    preconditioner, another iteration path to the same conv_tol, residual
    1e-5) within 1e-7, the spread of two vectors converged to that residual."""
    P, _, _ = _mods()
    g = load_golden("c1_norb12_6e6e_s0")
    h1, eri = seeded_integrals(12, 24)
    sol = P.csf_solver(None, smult=1)
    sol.nroots = 3
    sol.device_resident = device_resident
    e, ci = sol.kernel(h1, eri, 12, (6, 6))
    np.testing.assert_allclose(e, g["energies"], atol=1e-9)
    dm1, dm2 = sol.make_rdm12(ci[0], 12, (6, 6))
    np.testing.assert_allclose(dm1, g["rdm1_root0"], atol=1e-7 if device_resident else 1e-8)
    fp = float(np.dot(np.cos(np.arange(dm2.size)), dm2.ravel()))
    assert abs(fp - float(g["fp_rdm2_root0"])) < (1e-5 if device_resident else 1e-6)


def test_errors_are_raised():
    P, D, C = _mods()
    from pyscf_forge_b200 import _capi
    with pytest.raises(C.ImpossibleSpinError):
        C.CSFTransformer(6, 3, 1, 1)
    with pytest.raises(_capi.CSFFCIError):
        _capi.call("csffci_sigma", 40, 2, 2, None, None, None, None, None, 0, 1, None, 0, None)
    with pytest.raises(MemoryError):
        _capi.call("csffci_hdiag_det", 6, 3, 3, None, None, None, None, None, 16, None)
    t = C.CSFTransformer(6, 3, 3, 1)
    with pytest.raises(C.ImpossibleCIvecError):
        t.vec_det2csf(np.zeros(17))
    # the p-space memory guard of csf.py:294-303, driven by a memory budget
    # (max_memory in MB): here 20 CSFs need about 0.07 MB
    from conftest import seeded_integrals
    h1, eri = seeded_integrals(6, 12, seed=2)
    sol = P.csf_solver(None, smult=1)
    with pytest.raises(MemoryError):
        sol.pspace(h1, eri, 6, (3, 3), npsp=20, max_memory=0.01)
    sol.pspace(h1, eri, 6, (3, 3), npsp=20, max_memory=1.0)
    sol.max_memory = 0.01
    sol.device_resident = False
    with pytest.raises(MemoryError):
        sol.kernel(h1, eri, 6, (3, 3))


@pytest.mark.parametrize("norb,nelec,smult", [(8, (4, 4), 1), (10, (5, 5), 3), (12, (6, 6), 1),
                                              (11, (6, 5), 2), (9, (6, 2), 5), (14, (5, 5), 1)])
def test_sigma_kernels_agree(norb, nelec, smult):
    """The register-resident kernel (general and spin-symmetric modes)
    against the simple shared-memory kernel and, where small enough, the
    reference C."""
    _, D, C = _mods()
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200._runtime import ptr, stream, workspace
    h1, eri = seeded_integrals(norb, 10, seed=4)
    h2e = D.dev_absorb_h1e(h1, R.restore4(eri, norb), norb, nelec, 0.5)
    t = C.CSFTransformer(norb, nelec[0], nelec[1], smult)
    g = torch.Generator(device="cpu").manual_seed(3)
    c = t.dev_csf2det(torch.randn(t.ncsf, generator=g, dtype=torch.float64).cuda())[0]
    la, lb = D.dev_link_table(norb, nelec[0]), D.dev_link_table(norb, nelec[1])
    ref = torch.empty_like(c)
    _capi.call("csffci_sigma", norb, nelec[0], nelec[1], ptr(h2e), ptr(la), ptr(lb), ptr(c), ptr(ref),
               _capi.SIGMA_REFERENCE_KERNEL, 1, None, 0, stream())
    got = D.dev_contract_2e(h2e, c, norb, nelec)
    torch.testing.assert_close(got, ref, atol=1e-11, rtol=0)
    if t.spin_parity is not None:
        got2 = D.dev_contract_2e(h2e, c, norb, nelec, eta=t.spin_parity)
        torch.testing.assert_close(got2, ref, atol=1e-11, rtol=0)
    if gasref.available() and c.numel() < 2e6:
        h2e_np = h2e.cpu().numpy()
        np.testing.assert_allclose(got.cpu().numpy(), gasref.contract_2e(h2e_np, c.cpu().numpy(), norb, nelec),
                                   atol=1e-10)


@needs_ref
def test_solver_contract_2e_out_buffers():
    """FCISolver.contract_2e: numpy in/out, pinned host in with the result
    in pinned host memory, out= into a reused pinned host buffer and into a
    device buffer -- all equal to the reference C sigma; a wrong out is a
    ValueError."""
    import pyscf_forge_b200 as P
    norb, nelec = 8, (4, 4)
    h1, eri = seeded_integrals(norb, 12, seed=7)
    sol = P.csf_solver(None, smult=1)
    h2eff = sol.absorb_h1e(h1, eri, norb, nelec, 0.5)
    rng = np.random.default_rng(8)
    n = R.num_strings(norb, nelec[0])
    c = rng.normal(size=(n, n))
    c = (c + c.T) / np.linalg.norm(c + c.T)  # singlet-symmetric: the row-local singlet kernel runs
    ref = gasref.contract_2e(R.absorb_h1e(h1, eri, norb, nelec, 0.5), c, norb, nelec).ravel()
    got = sol.contract_2e(h2eff, c, norb, nelec)
    np.testing.assert_allclose(np.asarray(got).ravel(), ref, atol=1e-10)
    ch = torch.from_numpy(c.ravel().copy()).pin_memory()
    r1 = sol.contract_2e(h2eff, ch, norb, nelec)
    assert r1.device.type == "cpu" and r1.is_pinned()
    np.testing.assert_allclose(r1.numpy(), ref, atol=1e-10)
    buf = torch.empty(n * n, dtype=torch.float64).pin_memory()
    assert sol.contract_2e(h2eff, ch, norb, nelec, out=buf) is buf
    np.testing.assert_allclose(buf.numpy(), ref, atol=1e-10)
    dbuf = torch.empty(n * n, dtype=torch.float64, device="cuda")
    assert sol.contract_2e(h2eff, ch, norb, nelec, out=dbuf) is dbuf
    np.testing.assert_allclose(dbuf.cpu().numpy(), ref, atol=1e-10)
    with pytest.raises(ValueError):
        sol.contract_2e(h2eff, ch, norb, nelec, out=torch.empty(n * n - 1, dtype=torch.float64))


@needs_ref
@pytest.mark.parametrize("norb,nelec,rank", [(14, (3, 3), 10), (14, (3, 2), 10), (15, (4, 3), 10),
                                             (16, (2, 2), 8), (13, (3, 3), 8), (16, (3, 3), 8),
                                             (16, (3, 2), 8)])
def test_warp_specialised_sigma(norb, nelec, rank, monkeypatch):
    """The warp-specialised sigma kernels (tile variant 4 from 13 orbitals,
    variant 5 -- registers re-split between the roles -- and variant 6 --
    the same with the alpha rows moved by the bulk-copy engine -- at 16;
    variant 6 also from a vector 8 bytes off 16-byte alignment, which it
    copies element by element instead): against the
    reference C (1e-10) and against the phase-serial kernel (1e-12), in the
    general mode and, for na == nb, the spin-symmetric mode with a symmetric
    (eta = +1) and an antisymmetric (eta = -1) vector."""
    import torch
    _, D, _ = _mods()
    from math import comb
    h1, eri = seeded_integrals(norb, rank, seed=11)
    h2e_np = R.absorb_h1e(h1, eri, norb, nelec, 0.5)
    h2e = torch.as_tensor(h2e_np, device="cuda")
    na, nb = comb(norb, nelec[0]), comb(norb, nelec[1])
    rng = np.random.default_rng(12)
    c0 = rng.normal(size=(na, nb))
    cases = [(c0, (None,))]
    if na == nb:
        cases = [(c0 + c0.T, (None, 1)), (c0 - c0.T, (-1,))]
    variants = (4, 5, 6) if norb == 16 else (4,)
    for c, etas in cases:
        c = c / np.linalg.norm(c)
        ref = gasref.contract_2e(h2e_np, c, norb, nelec).ravel()
        cd = torch.as_tensor(c.ravel(), device="cuda")
        for eta in etas:
            monkeypatch.setenv("CSFFCI_SIGMA_VARIANT", "1")
            rr = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta).cpu().numpy()
            for v in variants:
                monkeypatch.setenv("CSFFCI_SIGMA_VARIANT", str(v))
                ws = D.dev_contract_2e(h2e, cd, norb, nelec, eta=eta).cpu().numpy()
                np.testing.assert_allclose(ws, ref, atol=1e-10)
                np.testing.assert_allclose(ws, rr, atol=1e-12)
                if v == 6:
                    buf = torch.empty(cd.numel() + 1, dtype=torch.float64, device="cuda")
                    buf[1:] = cd
                    ws = D.dev_contract_2e(h2e, buf[1:], norb, nelec, eta=eta).cpu().numpy()
                    np.testing.assert_allclose(ws, rr, atol=1e-12)
    monkeypatch.delenv("CSFFCI_SIGMA_VARIANT")


@pytest.mark.parametrize("norb,nelec,smult", [(8, (4, 4), 1), (12, (6, 6), 3), (11, (6, 5), 2),
                                              (16, (3, 3), 1)])
def test_sigma_plan_c_abi(norb, nelec, smult):
    """csffci_sigma_plan_create/bind/execute/destroy through the C ABI gives
    the same sigma as the stateless csffci_sigma (general, spin-symmetric
    and accumulating modes; 1e-12, the scatters' atomic additions may land
    in another order), and refuses the spin-symmetric mode when created
    without it."""
    import ctypes
    _, D, C = _mods()
    from pyscf_forge_b200 import _capi
    from pyscf_forge_b200._runtime import ptr, stream
    h1, eri = seeded_integrals(norb, 10, seed=21)
    h2e = D.dev_absorb_h1e(h1, R.restore4(eri, norb), norb, nelec, 0.5)
    t = C.CSFTransformer(norb, nelec[0], nelec[1], smult)
    g = torch.Generator(device="cpu").manual_seed(22)
    c = t.dev_csf2det(torch.randn(t.ncsf, generator=g, dtype=torch.float64).cuda())[0]
    la, lb = D.dev_link_table(norb, nelec[0]), D.dev_link_table(norb, nelec[1])
    lib = _capi.load()
    modes = [(0, 1)]
    if t.spin_parity is not None:
        modes.append((_capi.SIGMA_SPIN_SYMMETRIC, t.spin_parity))
    for flags, eta in modes:
        nbytes = _capi.query("csffci_sigma_workspace", norb, nelec[0], nelec[1], flags)
        ws = torch.empty(max(nbytes, 8), dtype=torch.uint8, device="cuda")
        ref = torch.empty_like(c)
        _capi.call("csffci_sigma", norb, nelec[0], nelec[1], ptr(h2e), ptr(la), ptr(lb), ptr(c), ptr(ref),
                   flags, eta, ptr(ws), nbytes, stream())
        plan = ctypes.c_void_p()
        need = ctypes.c_size_t()
        _capi.call("csffci_sigma_plan_create", norb, nelec[0], nelec[1], ptr(h2e), ptr(la), ptr(lb), flags,
                   ctypes.byref(plan), ctypes.byref(need))
        try:
            assert need.value == nbytes
            pws = torch.empty(max(need.value, 8), dtype=torch.uint8, device="cuda")
            _capi.call("csffci_sigma_plan_bind", plan, ptr(pws), need.value)
            got = torch.full_like(c, float("nan"))
            _capi.call("csffci_sigma_plan_execute", plan, ptr(c), ptr(got), eta, flags, stream())
            torch.cuda.synchronize()
            torch.testing.assert_close(got, ref, atol=1e-12, rtol=0)
            _capi.call("csffci_sigma_plan_execute", plan, ptr(c), ptr(got), eta,
                       flags | _capi.SIGMA_ACCUMULATE, stream())
            torch.cuda.synchronize()
            torch.testing.assert_close(got, 2 * ref, atol=1e-12, rtol=0)
            if flags == 0 and t.spin_parity is not None:
                st = lib.csffci_sigma_plan_execute(plan, ptr(c), ptr(got), 1, _capi.SIGMA_SPIN_SYMMETRIC,
                                                   stream())
                assert st == _capi.CSFFCI_ERR_INVALID
        finally:
            lib.csffci_sigma_plan_destroy(plan)


@pytest.mark.parametrize("nx,ny,n", [(48, 1, 1000003), (40, 4, 300001), (3, 40, 200003), (64, 4, 70001),
                                     (1, 1, 17), (2, 3, 5000), (7, 9, 100000), (33, 2, 65536)])
def test_gram_and_combine_vs_torch(nx, ny, n):
    """csffci_gram (the skinny kernel for up to 4 vectors on one side, the
    tiled split-K kernel otherwise) and csffci_combine against a plain torch
    fp64 reference (x y^T and beta*y + coef x) at 1e-12 relative; the Gram
    is bit-reproducible from one call to the next."""
    from pyscf_forge_b200.fci.davidson import combine, gram
    g = torch.Generator(device="cpu").manual_seed(nx * 1000 + ny)
    x = torch.randn(nx, n, generator=g, dtype=torch.float64).cuda()
    y = torch.randn(ny, n, generator=g, dtype=torch.float64).cuda()
    ref = x @ y.T
    got = gram(x, y)
    scale = float(ref.abs().max()) + 1.0
    assert float((got - ref).abs().max()) < 1e-12 * scale * max(1.0, n / 1e4)
    assert torch.equal(got, gram(x, y))
    coef = np.random.default_rng(nx + ny).normal(size=(ny, nx))
    y0 = y.clone()
    combine(y, x, coef, beta=0.5)
    ref2 = 0.5 * y0 + torch.as_tensor(coef, device="cuda") @ x
    assert float((y - ref2).abs().max()) < 1e-12 * (float(ref2.abs().max()) + 1.0) * max(1.0, nx / 8)
